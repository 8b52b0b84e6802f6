"""The `found` rule of the deferred join, modelled in Python and checked
against the reference's serial inserts on the CPU.

`found` (kgraph.cpp:808-810) marks a node whose pair offered y to x and
UpdateKnnList returned a position below K.  That depends on the order the
offers reach x's pool, not only on the final list, so offer_merge_kernel
(kgraph_b200/csrc/kg_build.cu) replays each pool's offers in arrival order
against a copy of the list's first K entries, 32 offers at a time:

* an offer can land below K only while the copy is short or its distance is
  below the copy's K-th entry;
* it is a duplicate when the copy holds its (id, distance) before its
  position, or an earlier offer of the chunk with the same (id, distance)
  landed (kgraph.cpp:187-193);
* a non-duplicate lands below K iff (copy entries <= d) + (earlier landing
  candidates of the chunk with distance <= d) < K: an earlier offer that does
  not land is no closer than one that does;
* a duplicate returns the list's length + 1 (kgraph.cpp:193), below K while the
  list is short, which also sets `found`;
* the landed offers enter the copy together, after entries of equal distance,
  and the copy keeps its first K.

This file is that model; the GPU test of the kernel (tests/test_join_merge_gpu.py)
checks the kernel on fewer cases.  Here the model's `found` sets must equal
the ones the oracle's serial inserts give in arrival order, pool by pool, on
many random pools with ties, duplicates, short lists and full lists.
"""
import numpy as np
import pytest

from oracle import kgoracle as ko
from test_join_merge_gpu import UU, _case

FMAX = float(np.finfo(np.float32).max)
CHUNK = 32


def model_found(pool_d, pool_i, Lc, L, K, cand, dist, src):
    """Sources the chunked replay marks found, for one pool's offers in arrival order."""
    Kc = min(K, L)
    kd = [float(x) for x in pool_d[:min(Lc, Kc)]]
    ki = [int(x) & 0x7FFFFFFF for x in pool_i[:min(Lc, Kc)]]
    found = set()
    for c0 in range(0, len(cand), CHUNK):
        cc = [int(x) for x in cand[c0:c0 + CHUNK]]
        dd = [float(x) for x in dist[c0:c0 + CHUNK]]
        ss = [int(x) for x in src[c0:c0 + CHUNK]]
        n, kc = len(cc), len(kd)
        kth = kd[Kc - 1] if kc == Kc else FMAX
        possible = [kc < Kc or d < kth for d in dd]
        base = [sum(1 for e in kd if e <= d) for d in dd]
        dup_listed = [possible[i] and any(kd[j] == dd[i] and ki[j] == cc[i] for j in range(base[i]))
                      for i in range(n)]
        first = []
        for i in range(n):
            f = i
            for j in range(i):
                if possible[j] and possible[i] and dd[j] == dd[i] and cc[j] == cc[i]:
                    f = j
                    break
            first.append(f)
        cand_ok = [possible[i] and not dup_listed[i] and first[i] == i for i in range(n)]
        landed = [cand_ok[i] and base[i] + sum(1 for j in range(i) if cand_ok[j] and dd[j] <= dd[i]) < Kc
                  for i in range(n)]
        for i in range(n):
            if not ss[i] & UU:
                continue
            if landed[i]:
                found.add(ss[i] & 0x7FFFFFFF)
            dup = possible[i] and (dup_listed[i] or (first[i] != i and landed[first[i]]))
            if dup and kc + sum(landed[:i]) + 1 < K:
                found.add(ss[i] & 0x7FFFFFFF)
        for i in range(n):
            if landed[i]:
                r = sum(1 for e in kd if e <= dd[i])
                kd.insert(r, dd[i])
                ki.insert(r, cc[i])
        kd, ki = kd[:Kc], ki[:Kc]
    return found


CASES = [(1, 64, 16, 8, 120), (2, 48, 100, 50, 300), (3, 40, 12, 12, 60), (4, 32, 100, 10, 300),
         (7, 40, 8, 8, 90), (8, 40, 24, 3, 150), (9, 30, 40, 40, 200), (10, 40, 6, 1, 70),
         (11, 24, 60, 30, 400)]


@pytest.mark.parametrize("seed,n,L,K,max_off", CASES)
def test_chunked_found_replay_equals_serial_inserts(seed, n, L, K, max_off):
    pool_d, pool_i, nodeL, radius, tg, cd, ds, sr = _case(seed, n, L, max_off)
    for x in range(n):
        arr = np.nonzero(tg == x)[0]     # arrival order: the input order
        _, _, _, _, r = ko.serial_inserts(pool_d[x], pool_i[x], nodeL[x], radius[x], cd[arr], ds[arr])
        want = {int(sr[k]) & 0x7FFFFFFF for k, rk in zip(arr, r) if (sr[k] & UU) and rk < K}
        got = model_found(pool_d[x], pool_i[x], int(nodeL[x]), L, K, cd[arr], ds[arr], sr[arr])
        assert got == want, (seed, x, len(arr))
