"""ctypes wrappers over the CPU checkers -- TEST INFRASTRUCTURE ONLY.

* ``Oracle``: the project's own restatement (oracle/libkgoracle.so, see
  oracle/kgoracle.h for the per-function reference citations).
* ``load_reference_module()`` / ``RefLib``: the reference itself, compiled from
  its sources into oracle/_ref by oracle/Makefile (Python module ``kgraph`` and
  the C++ MatrixOracle driver ``libkgref.so``).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm import this module.  The product (kgraph_b200) never does.
"""
import ctypes as C
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
METRICS = {"euclidean": 0, "angular": 1, "l2sqr": 2}

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


def _metric(m):
    return METRICS[m] if isinstance(m, str) else int(m)


def _lib():
    path = os.path.join(HERE, "libkgoracle.so")
    if not os.path.exists(path):
        raise RuntimeError("oracle/libkgoracle.so is not built (run make -C oracle oracle)")
    lib = C.CDLL(path)
    u, f, i = C.c_uint, C.c_float, C.c_int
    lib.kgo_dot.restype = f
    lib.kgo_norm2.restype = f
    lib.kgo_l2sqr.restype = f
    lib.kgo_pair.restype = f
    lib.kgo_query_norm.restype = f
    lib.kgo_norms.argtypes = [_f32p, u, u, i, _f32p]
    lib.kgo_bruteforce.restype = u
    lib.kgo_bruteforce.argtypes = [_f32p, _f32p, u, u, i, _f32p, u, f, _u32p, _f32p]
    lib.kgo_linear_search.argtypes = [_f32p, _f32p, u, u, i, u, u, _u32p, _f32p]
    lib.kgo_genrandom.argtypes = [u, u, u, u, _u32p]
    lib.kgo_search.restype = u
    lib.kgo_search.argtypes = [_f32p, _f32p, u, u, i, _u64p, _u32p, _u32p, _f32p,
                               u, u, u, u, u, f, u, u, _u32p, _f32p, C.POINTER(C.c_float)]
    lib.kgo_build.restype = i
    lib.kgo_build.argtypes = [_f32p, _f32p, u, u, i, u, u, u, u, u, u, u, f, f, u, i, u,
                              C.POINTER(C.c_uint64), _f32p, _f32p, u]
    lib.kgo_build_result.argtypes = [_u64p, _u32p, _f32p, _u32p]
    lib.kgo_reverse.restype = C.c_uint64
    lib.kgo_reverse.argtypes = [u, _u64p, _u32p, _f32p, _u32p, i]
    lib.kgo_prune.restype = C.c_uint64
    lib.kgo_prune.argtypes = [u, _u64p, _u32p, _f32p, _u32p, u]
    lib.kgo_std_sort_pairs.argtypes = [_f32p, _u32p, u]
    lib.kgo_serial_inserts.argtypes = [u, _f32p, _u32p, C.POINTER(C.c_uint), C.POINTER(C.c_float), u, _u32p, _f32p,
                                       _u32p]
    lib.kgo_last_error.restype = C.c_char_p
    return lib


class Graph:
    """CSR k-NN graph: offsets[n+1] (u64), ids[E] (u32), dists[E] (f32), M[n] (u32)."""

    def __init__(self, offsets, ids, dists, M):
        self.offsets = np.ascontiguousarray(offsets, np.uint64)
        self.ids = np.ascontiguousarray(ids, np.uint32)
        self.dists = np.ascontiguousarray(dists, np.float32)
        self.M = np.ascontiguousarray(M, np.uint32)

    @property
    def n(self):
        return len(self.M)

    def row(self, i):
        a, b = int(self.offsets[i]), int(self.offsets[i + 1])
        return self.ids[a:b], self.dists[a:b]


class Oracle:
    """The project's restatement over one dense dataset X (n x d float32)."""

    def __init__(self, X, metric="euclidean"):
        self.lib = _lib()
        self.X = np.ascontiguousarray(X, np.float32)
        self.n, self.d = self.X.shape
        self.metric = _metric(metric)
        self.norms = np.zeros(self.n, np.float32)
        self.lib.kgo_norms(self.X, self.n, self.d, self.metric, self.norms)

    def pair(self, i, j):
        return self.lib.kgo_pair(self.X.ctypes.data_as(C.POINTER(C.c_float)),
                                 self.norms.ctypes.data_as(C.POINTER(C.c_float)),
                                 self.d, self.metric, int(i), int(j))

    def bruteforce(self, Q, K, epsilon=1e30):
        Q = np.ascontiguousarray(Q, np.float32)
        nq = Q.shape[0]
        ids = np.zeros((nq, K), np.uint32)
        dists = np.zeros((nq, K), np.float32)
        cnt = np.zeros(nq, np.uint32)
        for q in range(nq):
            i1 = np.zeros(K, np.uint32)
            d1 = np.zeros(K, np.float32)
            cnt[q] = self.lib.kgo_bruteforce(self.X, self.norms, self.n, self.d, self.metric,
                                             np.ascontiguousarray(Q[q]), K, epsilon, i1, d1)
            ids[q], dists[q] = i1, d1
        return ids, dists, cnt

    def linear_search(self, i, K):
        ids = np.zeros(K, np.uint32)
        dists = np.zeros(K, np.float32)
        self.lib.kgo_linear_search(self.X, self.norms, self.n, self.d, self.metric, int(i), K, ids, dists)
        return ids, dists

    def search(self, graph, Q, K=25, P=100, M=0, S=10, T=1, epsilon=1e30, seed=1998, init=0,
               init_ids=None):
        Q = np.ascontiguousarray(Q, np.float32)
        nq = Q.shape[0]
        ids = np.zeros((nq, K), np.uint32)
        dists = np.zeros((nq, K), np.float32)
        cnt = np.zeros(nq, np.uint32)
        cost = np.zeros(nq, np.float32)
        for q in range(nq):
            i1 = np.zeros(max(K, 1), np.uint32)
            if init_ids is not None:
                i1[:init] = init_ids[q][:init]
            d1 = np.zeros(max(K, 1), np.float32)
            c = C.c_float(0)
            r = self.lib.kgo_search(self.X, self.norms, self.n, self.d, self.metric,
                                    graph.offsets, graph.ids, graph.M, np.ascontiguousarray(Q[q]),
                                    K, P, M, S, T, epsilon, seed, init, i1, d1, C.byref(c))
            if r == 0xFFFFFFFF:
                raise RuntimeError(self.lib.kgo_last_error().decode())
            ids[q], dists[q], cnt[q], cost[q] = i1[:K], d1[:K], r, c.value
        return ids, dists, cnt, cost

    def _result(self, E):
        off = np.zeros(self.n + 1, np.uint64)
        ids = np.zeros(max(E, 1), np.uint32)
        dists = np.zeros(max(E, 1), np.float32)
        M = np.zeros(self.n, np.uint32)
        self.lib.kgo_build_result(off, ids, dists, M)
        return Graph(off, ids[:E], dists[:E], M)

    def build(self, iterations=30, L=100, K=25, S=10, R=100, controls=100, seed=1998,
              delta=0.002, recall=0.99, prune=0, reverse=0, rand_seed=1):
        E = C.c_uint64(0)
        info = np.zeros(7, np.float32)
        log = np.zeros((max(iterations, 1) if iterations else 1000, 9), np.float32)
        r = self.lib.kgo_build(self.X, self.norms, self.n, self.d, self.metric, iterations, L, K, S,
                               R, controls, seed, delta, recall, prune, reverse, rand_seed,
                               C.byref(E), info, log, log.shape[0])
        if r != 0:
            raise RuntimeError(self.lib.kgo_last_error().decode())
        return self._result(E.value), info, log[: int(info[1])]

    def reverse(self, g, rev_k=-1):
        E = self.lib.kgo_reverse(g.n, g.offsets, g.ids, g.dists, g.M, rev_k)
        return self._result(E)

    def prune(self, g, level):
        E = self.lib.kgo_prune(g.n, g.offsets, g.ids, g.dists, g.M, level)
        return self._result(E)


def genrandom(seed, size, N, calls=0):
    out = np.zeros(max(size, 1), np.uint32)
    _lib().kgo_genrandom(seed, size, N, calls, out)
    return out[:size]


def serial_inserts(pool_d, pool_i, L, radius, cand, dist):
    """Nhood::parallel_try_insert of the offers (cand[k], dist[k]) in order into
    one pool (Lp = len(pool_d) entries, ids with the new-flag in bit 31).
    Returns (pool_d, pool_i, L, radius, r)."""
    pd = np.ascontiguousarray(pool_d, np.float32).copy()
    pi = np.ascontiguousarray(pool_i, np.uint32).copy()
    c = np.ascontiguousarray(cand, np.uint32)
    d = np.ascontiguousarray(dist, np.float32)
    r = np.zeros(len(c), np.uint32)
    Lv, rv = C.c_uint(int(L)), C.c_float(float(radius))
    _lib().kgo_serial_inserts(len(pd), pd, pi, C.byref(Lv), C.byref(rv), len(c), c, d, r)
    return pd, pi, Lv.value, rv.value, r


def std_sort_pairs(dists, ids):
    d = np.ascontiguousarray(dists, np.float32).copy()
    i = np.ascontiguousarray(ids, np.uint32).copy()
    _lib().kgo_std_sort_pairs(d, i, len(d))
    return d, i


# ---------------------------------------------------------------- reference
def host_isa():
    """'v4' when the host CPU has the AVX-512 subset x86-64-v4 needs, else 'v3'."""
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return "v3"
    need = ("avx512f", "avx512bw", "avx512dq", "avx512vl")
    return "v4" if all(f in flags for f in need) else "v3"


def reference_dir(isa=None):
    return os.path.join(HERE, "_ref", isa or host_isa())


def reference_available(isa=None):
    d = reference_dir(isa)
    return os.path.isdir(d) and any(f.startswith("kgraph") and f.endswith(".so") for f in os.listdir(d))


def load_reference_module(isa=None):
    """Imports the reference's own Python module (python-api.cpp) from oracle/_ref."""
    d = reference_dir(isa)
    for f in os.listdir(d) if os.path.isdir(d) else []:
        if f.startswith("kgraph.") and f.endswith(".so"):
            spec = importlib.util.spec_from_file_location("kgraph", os.path.join(d, f))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            return mod
    raise RuntimeError("reference module not built under %s" % d)


class RefLib:
    """The reference's C++ API (KGraph + MatrixOracle<l2sqr>) via oracle/ref_driver.cpp."""

    def __init__(self, isa=None):
        self.lib = C.CDLL(os.path.join(reference_dir(isa), "libkgref.so"))
        u, f, i = C.c_uint, C.c_float, C.c_int
        self.lib.kgref_build_l2sqr.restype = i
        self.lib.kgref_build_l2sqr.argtypes = [_f32p, u, u, u, u, u, u, u, u, u, f, f, u, i,
                                               C.c_char_p, _f32p]
        self.lib.kgref_search_l2sqr.restype = i
        self.lib.kgref_search_l2sqr.argtypes = [_f32p, u, u, C.c_char_p, _f32p, u, u, u, u, u, u,
                                                f, u, u, _u32p, _f32p, _u32p, _f32p, i]
        self.lib.kgref_last_error.restype = C.c_char_p
        self.lib.kgref_set_verbosity.argtypes = [u]
        self.lib.kgref_set_threads.argtypes = [i]
        self.lib.kgref_resave.restype = i
        self.lib.kgref_save_lshkit.restype = i
        self.lib.kgref_save_lshkit.argtypes = [_f32p, u, u, C.c_char_p]
        self.lib.kgref_load_lshkit.restype = i
        self.lib.kgref_load_lshkit.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(u), C.POINTER(u)]
        self.lib.kgref_resave.argtypes = [C.c_char_p, C.c_char_p, i]

    def set_verbosity(self, v):
        self.lib.kgref_set_verbosity(v)

    def set_threads(self, t):
        self.lib.kgref_set_threads(t)

    def save_lshkit(self, X, path):
        """The reference's Matrix<float>::save_lshkit of X."""
        X = np.ascontiguousarray(X, np.float32)
        if self.lib.kgref_save_lshkit(X, X.shape[0], X.shape[1], path.encode()):
            raise RuntimeError(self.lib.kgref_last_error().decode())

    def load_lshkit(self, path):
        """The reference's Matrix<float>::load_lshkit; returns an n x d float32 array."""
        n, d = C.c_uint(), C.c_uint()
        if self.lib.kgref_load_lshkit(path.encode(), None, C.byref(n), C.byref(d)):
            raise RuntimeError(self.lib.kgref_last_error().decode())
        out = np.zeros((n.value, d.value), np.float32)
        if self.lib.kgref_load_lshkit(path.encode(), out.ctypes.data_as(C.c_void_p), C.byref(n), C.byref(d)):
            raise RuntimeError(self.lib.kgref_last_error().decode())
        return out

    def resave(self, in_path, out_path, fmt):
        """The reference loads in_path and saves it to out_path in format fmt (0, 1 no-dist, 128 text)."""
        if self.lib.kgref_resave(in_path.encode(), out_path.encode(), fmt):
            raise RuntimeError(self.lib.kgref_last_error().decode())

    def build_l2sqr(self, X, path, iterations=30, L=100, K=25, S=10, R=100, controls=100,
                    seed=1998, delta=0.002, recall=0.99, prune=0, reverse=0):
        X = np.ascontiguousarray(X, np.float32)
        info = np.zeros(7, np.float32)
        r = self.lib.kgref_build_l2sqr(X, X.shape[0], X.shape[1], iterations, L, K, S, R, controls,
                                       seed, delta, recall, prune, reverse, path.encode(), info)
        if r:
            raise RuntimeError(self.lib.kgref_last_error().decode())
        return info

    def search_l2sqr(self, X, path, Q, K=25, P=100, M=0, S=10, T=1, epsilon=1e30, seed=1998,
                     init=0, init_ids=None, threads=0):
        X = np.ascontiguousarray(X, np.float32)
        Q = np.ascontiguousarray(Q, np.float32)
        nq = Q.shape[0]
        ids = np.zeros((nq, K), np.uint32)
        if init_ids is not None:
            ids[:, :init] = init_ids[:, :init]
        dists = np.zeros((nq, K), np.float32)
        cnt = np.zeros(nq, np.uint32)
        cost = np.zeros(nq, np.float32)
        r = self.lib.kgref_search_l2sqr(X, X.shape[0], X.shape[1], path.encode(), Q, nq, K, P, M, S,
                                        T, epsilon, seed, init, ids, dists, cnt, cost, threads)
        if r:
            raise RuntimeError(self.lib.kgref_last_error().decode())
        return ids, dists, cnt, cost


def read_index(path_or_bytes):
    """Parses the reference's binary index file (kgraph.cpp:291-331) into a Graph."""
    if isinstance(path_or_bytes, (bytes, bytearray, np.ndarray)):
        raw = bytes(path_or_bytes)
    else:
        raw = open(path_or_bytes, "rb").read()
    if raw[:8] != b"KNNGRAPH":
        raise ValueError("bad magic")
    version, cap, n = np.frombuffer(raw, np.uint32, 3, 8)
    if version != 2:
        raise ValueError("data version not supported.")
    no_dist = bool(cap & 1)
    pos = 20
    offsets = np.zeros(n + 1, np.uint64)
    M = np.zeros(n, np.uint32)
    ids_l, d_l = [], []
    e = 0
    rec = np.dtype([("id", "<u4"), ("dist", "<f4"), ("flag", "u1"), ("pad", "u1", 3)])
    for i in range(n):
        m, k = np.frombuffer(raw, np.uint32, 2, pos)
        pos += 8
        M[i] = m
        if no_dist:
            ids_l.append(np.frombuffer(raw, np.uint32, k, pos))
            d_l.append(np.zeros(k, np.float32))
            pos += 4 * k
        else:
            r = np.frombuffer(raw, rec, k, pos)
            ids_l.append(r["id"].copy())
            d_l.append(r["dist"].copy())
            pos += 12 * k
        e += k
        offsets[i + 1] = e
    ids = np.concatenate(ids_l) if ids_l else np.zeros(0, np.uint32)
    dists = np.concatenate(d_l) if d_l else np.zeros(0, np.float32)
    return Graph(offsets, ids, dists, M)
