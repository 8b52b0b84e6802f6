"""The GNU introsort restatement (kgraph_b200/csrc/kg_sort.h) must order
records exactly as libstdc++ std::sort does, ties included: the reference
sorts the search seed pool and the reversed adjacency lists with it
(kgraph.cpp:476, 697) and the tie order decides which node the walk expands
first.  The same header is compiled here for the host and compared."""
import ctypes as C
import os
import subprocess

import numpy as np

from conftest import ROOT

HARNESS = r"""
#include "kg_sort.h"
#include <algorithm>
#include <vector>
struct Rec { float d; unsigned id; };
struct Acc { Rec *v; float key(int i) const { return v[i].d; } void swap(int i, int j) { std::swap(v[i], v[j]); }
  Rec get(int i) const { return v[i]; } void put(int i, Rec r) { v[i] = r; } float rkey(Rec r) const { return r.d; } };
extern "C" int check(const float *d, int n, int heap) {
  std::vector<Rec> a(n), b;
  for (int i = 0; i < n; ++i) a[i] = Rec{d[i], (unsigned)i};
  b = a;
  auto lt = [](const Rec &x, const Rec &y) { return x.d < y.d; };
  Acc acc{b.data()};
  if (heap) { std::partial_sort(a.begin(), a.end(), a.end(), lt); kgb::gs_heapsort(acc, 0, n); }
  else { std::sort(a.begin(), a.end(), lt); kgb::gnu_sort(acc, 0, n); }
  for (int i = 0; i < n; ++i) if (a[i].id != b[i].id) return i + 1;
  return 0;
}
"""


def test_gnu_sort_matches_std_sort(tmp_path):
    src = tmp_path / "h.cpp"
    so = tmp_path / "h.so"
    src.write_text(HARNESS)
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I",
                           os.path.join(ROOT, "kgraph_b200", "csrc"), str(src), "-o", str(so)])
    lib = C.CDLL(str(so))
    lib.check.argtypes = [np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"), C.c_int, C.c_int]
    rng = np.random.default_rng(0)
    for t in range(3000):
        n = int(rng.integers(0, 2500))
        vals = int(rng.integers(1, 40)) if t % 3 else 1 << 30
        a = rng.integers(0, vals, n).astype(np.float32)
        if t % 5 == 0:
            a = np.sort(a)[::-1].copy()
        assert lib.check(a, n, 0) == 0
        assert lib.check(a, min(n, 400), 1) == 0
