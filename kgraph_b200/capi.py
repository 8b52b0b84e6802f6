"""ctypes binding of the C-ABI (include/kgraph_b200.h).

This is the binding a foreign caller would write; the tests and bench.py use
it to drive the library exactly through its C entry points.  Loading fails
loudly when the library has not been built: there is no fallback.
"""
import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libkgraph_b200.so")

METRIC = {"euclidean": 0, "angular": 1, "l2sqr": 2}

# Every entry point include/kgraph_b200.h declares.
SYMBOLS = [
    "kg_index_params_default", "kg_search_params_default", "kg_ctx_create", "kg_ctx_destroy",
    "kg_last_error", "kg_version", "kg_set_verbosity", "kg_set_data", "kg_build", "kg_graph_size",
    "kg_graph_export", "kg_graph_import", "kg_search_batch", "kg_reverse", "kg_prune", "kg_last_timing",
    "kg_last_search_work", "kg_search_batch_noalloc", "kg_noalloc_scratch_bytes",
    "kg_router_params_default", "kg_router_train", "kg_router_seeds", "kg_router_gradients", "kg_last_router_timing",
    "kg_set_join_precision", "kg_set_join_inserts", "kg_set_join_offer_capacity", "kg_join_merge_check", "kg_last_join_stats", "kg_last_build_graphs", "kg_search_autotune",
    "kg_set_search_tuning", "kg_get_search_tuning", "kg_last_search_shape", "kg_set_search_precision",
    "kg_last_search_filter",
    "kg_filter_bounds", "kg_router_search", "kg_tc_gemm_check", "kg_tc_assign_check", "kg_last_build_work",
    "kg_last_build_iterations", "kg_set_bruteforce_mode", "kg_last_bruteforce_stats",
]

JOIN = {"auto": 0, "fp32": 1, "bf16": 2, "bf16_always": 3, "fp8": 4, "fp8_always": 5}


class IndexParams(C.Structure):
    _fields_ = [("iterations", C.c_uint), ("L", C.c_uint), ("K", C.c_uint), ("S", C.c_uint), ("R", C.c_uint),
                ("controls", C.c_uint), ("seed", C.c_uint), ("delta", C.c_float), ("recall", C.c_float),
                ("prune", C.c_uint), ("reverse", C.c_int)]


class IndexInfo(C.Structure):
    _fields_ = [("stop_condition", C.c_int), ("iterations", C.c_uint), ("cost", C.c_float), ("recall", C.c_float),
                ("accuracy", C.c_float), ("delta", C.c_float), ("M", C.c_float)]


class RouterParams(C.Structure):
    _fields_ = [("clusters", C.c_uint), ("hidden", C.c_uint), ("kmeans_iters", C.c_uint), ("label_P", C.c_uint),
                ("epochs", C.c_uint), ("batch", C.c_uint), ("lr", C.c_float), ("seed", C.c_uint),
                ("entries", C.c_uint), ("probe", C.c_uint), ("refine", C.c_uint), ("refine_P", C.c_uint)]


class RouterInfo(C.Structure):
    _fields_ = [("steps", C.c_uint), ("final_loss", C.c_float), ("train_accuracy", C.c_float),
                ("empty_clusters", C.c_uint), ("entries", C.c_uint), ("component_entries", C.c_uint),
                ("relabelled", C.c_uint), ("label_s", C.c_float), ("cluster_s", C.c_float), ("mlp_s", C.c_float),
                ("refine_s", C.c_float)]


class JoinStats(C.Structure):
    _fields_ = [("mode", C.c_int), ("pairs", C.c_ulonglong), ("rechecked", C.c_ulonglong),
                ("sampled", C.c_ulonglong), ("violations", C.c_ulonglong), ("max_abs_err", C.c_double),
                ("mean_abs_err", C.c_double), ("max_rel_err", C.c_double), ("mean_rel_err", C.c_double),
                ("max_err_over_margin", C.c_double), ("mean_err_over_margin", C.c_double),
                ("tc_iterations", C.c_uint)]


class SearchTuning(C.Structure):
    _fields_ = [("split", C.c_uint), ("warps_per_block", C.c_uint), ("prefetch", C.c_uint), ("ms", C.c_float),
                ("default_ms", C.c_float), ("variants", C.c_uint), ("regs", C.c_uint), ("compact", C.c_uint)]


class FilterStats(C.Structure):
    _fields_ = [("mode", C.c_int), ("approx", C.c_ulonglong), ("skipped", C.c_ulonglong),
                ("max_rel_row_error", C.c_double), ("mean_rel_row_error", C.c_double)]


SEARCH_PRECISION = {"fp32": 0, "bf16": 1, "fp8": 2}


class BuildIteration(C.Structure):
    _fields_ = [("pairs", C.c_ulonglong), ("list_entries", C.c_ulonglong), ("insert_attempts", C.c_ulonglong),
                ("inserts_landed", C.c_ulonglong), ("ms", C.c_float), ("tensor_core", C.c_uint)]


class BruteforceStats(C.Structure):
    _fields_ = [("tensor", C.c_int), ("candidates", C.c_ulonglong), ("full_scans", C.c_ulonglong)]


BRUTEFORCE = {"auto": 0, "scan": 1, "tensor": 2}
INSERTS = {"auto": 0, "locked": 1, "deferred": 2}


class SearchParams(C.Structure):
    _fields_ = [("K", C.c_uint), ("M", C.c_uint), ("P", C.c_uint), ("S", C.c_uint), ("T", C.c_uint),
                ("epsilon", C.c_float), ("seed", C.c_uint), ("init", C.c_uint)]


_lib = None


def lib():
    """Loads libkgraph_b200.so (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libkgraph_b200.so is not built; run python -m kgraph_b200.build")
        L = C.CDLL(LIB_PATH)
        vp, sz = C.c_void_p, C.c_size_t
        L.kg_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
        L.kg_ctx_destroy.argtypes = [vp]
        L.kg_last_error.argtypes = [vp]
        L.kg_last_error.restype = C.c_char_p
        L.kg_version.restype = C.c_char_p
        L.kg_set_verbosity.argtypes = [C.c_uint]
        L.kg_set_data.argtypes = [vp, vp, sz, sz, sz, C.c_int]
        L.kg_build.argtypes = [vp, C.POINTER(IndexParams), C.POINTER(IndexInfo)]
        L.kg_graph_size.argtypes = [vp, C.POINTER(sz), C.POINTER(sz)]
        L.kg_graph_export.argtypes = [vp, vp, vp, vp, vp]
        L.kg_graph_import.argtypes = [vp, sz, vp, vp, vp, vp]
        L.kg_search_batch.argtypes = [vp, vp, sz, sz, C.POINTER(SearchParams), vp, vp, sz, vp, vp, vp, vp]
        L.kg_reverse.argtypes = [vp, C.c_int]
        L.kg_prune.argtypes = [vp, C.c_uint]
        L.kg_last_timing.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.kg_last_search_work.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.kg_search_batch_noalloc.argtypes = [vp, vp, sz, sz, C.POINTER(SearchParams), sz, vp, vp, vp, vp]
        L.kg_noalloc_scratch_bytes.restype = sz
        L.kg_router_params_default.argtypes = [C.POINTER(RouterParams)]
        L.kg_last_router_timing.argtypes = [vp, C.POINTER(C.c_float)]
        L.kg_router_train.argtypes = [vp, C.POINTER(RouterParams), vp, sz, sz, C.POINTER(RouterInfo)]
        L.kg_router_seeds.argtypes = [vp, vp, sz, sz, C.c_uint, vp, sz]
        L.kg_router_gradients.argtypes = [vp, C.c_uint, C.c_uint, C.c_uint, vp, vp, vp, C.c_uint,
                                          C.POINTER(C.c_float), vp]
        L.kg_set_join_precision.argtypes = [vp, C.c_int]
        L.kg_set_join_inserts.argtypes = [vp, C.c_int]
        L.kg_set_join_offer_capacity.argtypes = [vp, sz]
        L.kg_join_merge_check.argtypes = [vp, C.c_uint, C.c_uint, C.c_uint, vp, vp, vp, vp, sz, vp, vp, vp, vp, vp]
        L.kg_last_join_stats.argtypes = [vp, C.POINTER(JoinStats)]
        L.kg_last_build_graphs.argtypes = [vp, C.POINTER(C.c_uint)]
        L.kg_search_autotune.argtypes = [vp, vp, sz, sz, C.POINTER(SearchParams), vp, vp, vp, sz,
                                         C.POINTER(SearchTuning)]
        L.kg_set_search_tuning.argtypes = [vp, C.POINTER(SearchTuning)]
        L.kg_get_search_tuning.argtypes = [vp, C.POINTER(SearchTuning)]
        L.kg_last_search_shape.argtypes = [vp, C.POINTER(SearchTuning)]
        L.kg_set_search_precision.argtypes = [vp, C.c_int]
        L.kg_last_search_filter.argtypes = [vp, C.POINTER(FilterStats)]
        L.kg_filter_bounds.argtypes = [vp, vp, sz, sz, vp, sz, vp, vp]
        L.kg_router_search.argtypes = [vp, vp, sz, sz, C.POINTER(SearchParams), sz, vp, vp, vp, vp]
        L.kg_tc_gemm_check.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, C.c_int, C.c_int,
                                       vp, C.c_int, C.c_float, vp, C.c_int]
        L.kg_tc_assign_check.argtypes = [vp, vp, C.c_int, C.c_int, vp, C.c_int, vp, vp, vp]
        L.kg_last_build_work.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint)]
        L.kg_last_build_iterations.argtypes = [vp, C.POINTER(BuildIteration), C.c_uint, C.POINTER(C.c_uint)]
        L.kg_set_bruteforce_mode.argtypes = [vp, C.c_int]
        L.kg_last_bruteforce_stats.argtypes = [vp, C.POINTER(BruteforceStats)]
        L.kg_index_params_default.argtypes = [C.POINTER(IndexParams)]
        L.kg_search_params_default.argtypes = [C.POINTER(SearchParams)]
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):   # torch tensor (device-resident buffers)
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def _set_fields(p, kw):
    """Keyword arguments onto a parameter struct; a name that is not one of its
    fields raises TypeError (ctypes would keep it as a plain attribute and the
    library would never see it)."""
    names = {f for f, _ in type(p)._fields_}
    for k, v in kw.items():
        if k not in names:
            raise TypeError("%s has no parameter %r (fields: %s)" % (type(p).__name__, k, ", ".join(sorted(names))))
        setattr(p, k, v)
    return p


class KGError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class Context:
    """One kg_ctx: a dataset, a graph and a stream on one GPU."""

    def __init__(self, device=0):
        self.L = lib()
        h = C.c_void_p()
        r = self.L.kg_ctx_create(device, C.byref(h))
        if r != 0:
            raise KGError(r, "kg_ctx_create failed (no CUDA device?)")
        self.h = h
        self._keep = []

    def close(self):
        if self.h:
            self.L.kg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, r):
        if r != 0:
            raise KGError(r, self.L.kg_last_error(self.h).decode())

    def set_data(self, X, metric="euclidean"):
        m = METRIC[metric] if isinstance(metric, str) else int(metric)
        if hasattr(X, "data_ptr"):
            n, d = X.shape
            stride = X.stride(0) * X.element_size()
        else:
            X = np.ascontiguousarray(X, np.float32)
            n, d = X.shape
            stride = X.strides[0]
        self._check(self.L.kg_set_data(self.h, _ptr(X), n, d, stride, m))
        self.n, self.d = n, d

    def build(self, **kw):
        p = IndexParams()
        self.L.kg_index_params_default(C.byref(p))
        _set_fields(p, kw)
        info = IndexInfo()
        self._check(self.L.kg_build(self.h, C.byref(p), C.byref(info)))
        return {f: getattr(info, f) for f, _ in IndexInfo._fields_}

    def graph(self):
        n, E = C.c_size_t(), C.c_size_t()
        self._check(self.L.kg_graph_size(self.h, C.byref(n), C.byref(E)))
        off = np.zeros(n.value + 1, np.uint64)
        ids = np.zeros(max(E.value, 1), np.uint32)
        dists = np.zeros(max(E.value, 1), np.float32)
        M = np.zeros(n.value, np.uint32)
        self._check(self.L.kg_graph_export(self.h, _ptr(off), _ptr(ids), _ptr(dists), _ptr(M)))
        return off, ids[: E.value], dists[: E.value], M

    def set_graph(self, offsets, ids, dists, M):
        offsets = np.ascontiguousarray(offsets, np.uint64)
        ids = np.ascontiguousarray(ids, np.uint32)
        M = np.ascontiguousarray(M, np.uint32)
        dists = None if dists is None else np.ascontiguousarray(dists, np.float32)
        self._check(self.L.kg_graph_import(self.h, len(M), _ptr(offsets), _ptr(ids), _ptr(dists), _ptr(M)))

    def search(self, Q, K=25, P=100, M=0, S=10, T=1, epsilon=1e30, seed=1998, init=0, init_ids=None,
               K_per_q=None, P_per_q=None, out_ld=None, with_cost=True):
        """Returns (ids, dists, counts, costs) as numpy arrays (host path)."""
        Q = np.ascontiguousarray(Q, np.float32)
        nq = Q.shape[0]
        p = SearchParams(K, M, P, S, T, epsilon, seed, init)
        kmax = int(np.max(K_per_q)) if K_per_q is not None else K
        ld = out_ld or max(kmax, 1)
        ids = np.zeros((nq, ld), np.uint32)
        if init_ids is not None:
            ids[:, :init] = np.asarray(init_ids)[:, :init]
        dists = np.zeros((nq, ld), np.float32)
        counts = np.zeros(nq, np.uint32)
        costs = np.zeros(nq, np.float32) if with_cost else None
        kq = None if K_per_q is None else np.ascontiguousarray(K_per_q, np.uint32)
        pq = None if P_per_q is None else np.ascontiguousarray(P_per_q, np.uint32)
        self._check(self.L.kg_search_batch(self.h, _ptr(Q), nq, Q.strides[0], C.byref(p), _ptr(kq), _ptr(pq), ld,
                                           _ptr(ids), _ptr(dists), _ptr(counts), _ptr(costs)))
        return ids, dists, counts, costs

    def search_raw(self, q_ptr, nq, q_stride, params, kq_ptr, pq_ptr, out_ld, ids_ptr, d_ptr, c_ptr, cost_ptr):
        """kg_search_batch on raw (device or host) pointers."""
        self._check(self.L.kg_search_batch(self.h, q_ptr, nq, q_stride, C.byref(params), kq_ptr, pq_ptr, out_ld,
                                           ids_ptr, d_ptr, c_ptr, cost_ptr))

    def search_noalloc(self, q_ptr, nq, q_stride, params, out_ld, ids_ptr, d_ptr, c_ptr, cost_ptr):
        """kg_search_batch_noalloc on device pointers (no device allocation)."""
        self._check(self.L.kg_search_batch_noalloc(self.h, q_ptr, nq, q_stride, C.byref(params), out_ld, ids_ptr,
                                                   d_ptr, c_ptr, cost_ptr))

    def router_train(self, Qtrain, **kw):
        Qtrain = np.ascontiguousarray(Qtrain, np.float32)
        p = RouterParams()
        self.L.kg_router_params_default(C.byref(p))
        _set_fields(p, kw)
        info = RouterInfo()
        self._check(self.L.kg_router_train(self.h, C.byref(p), _ptr(Qtrain), Qtrain.shape[0], Qtrain.strides[0],
                                           C.byref(info)))
        return {f: getattr(info, f) for f, _ in RouterInfo._fields_}

    def router_seeds(self, Q, m, out_ld=None):
        Q = np.ascontiguousarray(Q, np.float32)
        ld = out_ld or m
        seeds = np.zeros((Q.shape[0], ld), np.uint32)
        self._check(self.L.kg_router_seeds(self.h, _ptr(Q), Q.shape[0], Q.strides[0], m, _ptr(seeds), ld))
        return seeds

    def router_search(self, Q, K=10, P=10, seeds=3, S=10, epsilon=1e30, out_ld=None, with_cost=True):
        """Router seeds + seeded walk in one call; returns (ids, dists, counts, costs)."""
        Q = np.ascontiguousarray(Q, np.float32)
        nq = Q.shape[0]
        ld = out_ld or K
        p = SearchParams(K, 0, P, S, 1, epsilon, 1998, seeds)
        ids = np.zeros((nq, ld), np.uint32)
        dists = np.zeros((nq, ld), np.float32)
        counts = np.zeros(nq, np.uint32)
        costs = np.zeros(nq, np.float32) if with_cost else None
        self._check(self.L.kg_router_search(self.h, _ptr(Q), nq, Q.strides[0], C.byref(p), ld, _ptr(ids), _ptr(dists),
                                            _ptr(counts), _ptr(costs)))
        return ids, dists, counts, costs

    def router_search_raw(self, q_ptr, nq, q_stride, params, out_ld, ids_ptr, d_ptr, c_ptr, cost_ptr):
        """kg_router_search on raw (device or host) pointers."""
        self._check(self.L.kg_router_search(self.h, q_ptr, nq, q_stride, C.byref(params), out_ld, ids_ptr, d_ptr,
                                            c_ptr, cost_ptr))

    def router_seeds_raw(self, q_ptr, nq, q_stride, m, seeds_ptr, out_ld):
        """kg_router_seeds on raw (device or host) pointers; returns its device milliseconds."""
        self._check(self.L.kg_router_seeds(self.h, q_ptr, nq, q_stride, m, seeds_ptr, out_ld))
        ms = C.c_float()
        self._check(self.L.kg_last_router_timing(self.h, C.byref(ms)))
        return ms.value

    def router_gradients(self, d, hidden, clusters, weights, x, labels):
        x = np.ascontiguousarray(x, np.float32)
        labels = np.ascontiguousarray(labels, np.int32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        nparam = d * hidden + hidden + hidden * hidden + hidden + hidden * clusters + clusters
        grads = np.zeros(nparam, np.float32)
        loss = C.c_float()
        self._check(self.L.kg_router_gradients(self.h, d, hidden, clusters, _ptr(w), _ptr(x), _ptr(labels),
                                               x.shape[0], C.byref(loss), _ptr(grads)))
        return loss.value, grads

    def tc_gemm_check(self, A, B, ta=False, tb=False, bias=None, relu=False, beta=0.0, C_in=None):
        """kg_tc_gemm_check: op(A) @ op(B) (+ beta C_in) (+ bias) (ReLU) on the tensor cores.
        A and B are uint16 arrays of BF16 bit patterns."""
        A = np.ascontiguousarray(A, np.uint16)
        B = np.ascontiguousarray(B, np.uint16)
        M, K = (A.shape[1], A.shape[0]) if ta else A.shape
        N = B.shape[0] if tb else B.shape[1]
        out = np.zeros((M, N), np.float32) if C_in is None else np.ascontiguousarray(C_in, np.float32).copy()
        b = None if bias is None else np.ascontiguousarray(bias, np.float32)
        self._check(self.L.kg_tc_gemm_check(self.h, M, N, K, _ptr(A), A.shape[1], int(ta), _ptr(B), B.shape[1],
                                            int(tb), _ptr(b), int(relu), beta, _ptr(out), N))
        return out

    def tc_assign_check(self, F, cent, cn):
        """kg_tc_assign_check: argmin_c cn[c] - 2 F.cent[c] per row (BF16 bit patterns in)."""
        F = np.ascontiguousarray(F, np.uint16)
        cent = np.ascontiguousarray(cent, np.uint16)
        cn = np.ascontiguousarray(cn, np.float32)
        lab = np.zeros(F.shape[0], np.int32)
        best = np.zeros(F.shape[0], np.float32)
        self._check(self.L.kg_tc_assign_check(self.h, _ptr(F), F.shape[0], F.shape[1], _ptr(cent), cent.shape[0],
                                              _ptr(cn), _ptr(lab), _ptr(best)))
        return lab, best

    def reverse(self, k):
        self._check(self.L.kg_reverse(self.h, k))

    def prune(self, level):
        self._check(self.L.kg_prune(self.h, level))

    def build_work(self):
        """kg_last_build_work: (join pairs, join list entries, iterations) of the last build."""
        p, e, it = C.c_uint64(), C.c_uint64(), C.c_uint()
        self._check(self.L.kg_last_build_work(self.h, C.byref(p), C.byref(e), C.byref(it)))
        return p.value, e.value, it.value

    def build_iterations(self):
        """kg_last_build_iterations: per-iteration counters and device milliseconds of the last build."""
        n = C.c_uint()
        self._check(self.L.kg_last_build_iterations(self.h, None, 0, C.byref(n)))
        arr = (BuildIteration * max(1, n.value))()
        self._check(self.L.kg_last_build_iterations(self.h, arr, n.value, C.byref(n)))
        return [{f: getattr(arr[i], f) for f, _ in BuildIteration._fields_} for i in range(n.value)]

    def set_bruteforce_mode(self, mode):
        """kg_set_bruteforce_mode: 'auto', 'scan' (CUDA cores) or 'tensor'."""
        self._check(self.L.kg_set_bruteforce_mode(self.h, BRUTEFORCE[mode]))

    def bruteforce_stats(self):
        st = BruteforceStats()
        self._check(self.L.kg_last_bruteforce_stats(self.h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in BruteforceStats._fields_}

    def search_work(self):
        ev, adj = C.c_uint64(), C.c_uint64()
        self._check(self.L.kg_last_search_work(self.h, C.byref(ev), C.byref(adj)))
        return ev.value, adj.value

    def timing(self):
        b, s = C.c_float(), C.c_float()
        self._check(self.L.kg_last_timing(self.h, C.byref(b), C.byref(s)))
        return b.value, s.value

    def set_join_precision(self, mode):
        """'auto' (BF16 tensor-core join for d >= 64), 'fp32', 'bf16' or 'bf16_always'."""
        self._check(self.L.kg_set_join_precision(self.h, JOIN[mode] if isinstance(mode, str) else int(mode)))

    def join_merge_check(self, L, K, pool_d, pool_i, nodeL, radius, target, cand, dist, src):
        """kg_join_merge_check: the deferred-insert merge on caller pools (n x (L+1)) and offers.
        Returns (pool_d, pool_i, nodeL, radius, found)."""
        pd = np.ascontiguousarray(pool_d, np.float32).copy()
        pi = np.ascontiguousarray(pool_i, np.uint32).copy()
        nl = np.ascontiguousarray(nodeL, np.uint32).copy()
        rd = np.ascontiguousarray(radius, np.float32).copy()
        n = pd.shape[0]
        t = np.ascontiguousarray(target, np.uint32)
        c = np.ascontiguousarray(cand, np.uint32)
        d = np.ascontiguousarray(dist, np.float32)
        s_ = np.ascontiguousarray(src, np.uint32)
        found = np.zeros(n, np.uint32)
        self._check(self.L.kg_join_merge_check(self.h, n, L, K, _ptr(pd), _ptr(pi), _ptr(nl), _ptr(rd), len(t),
                                               _ptr(t), _ptr(c), _ptr(d), _ptr(s_), _ptr(found)))
        return pd, pi, nl, rd, found

    def set_join_offer_capacity(self, offers):
        """kg_set_join_offer_capacity: bound the deferred inserts' record buffers (0 = automatic)."""
        self._check(self.L.kg_set_join_offer_capacity(self.h, int(offers)))

    def set_join_inserts(self, mode):
        """kg_set_join_inserts: 'auto', 'locked' or 'deferred'."""
        self._check(self.L.kg_set_join_inserts(self.h, INSERTS[mode] if isinstance(mode, str) else int(mode)))

    def join_stats(self):
        st = JoinStats()
        self._check(self.L.kg_last_join_stats(self.h, C.byref(st)))
        out = {f: getattr(st, f) for f, _ in JoinStats._fields_}
        out["mode"] = {1: "fp32", 2: "bf16", 4: "fp8"}.get(st.mode, "none")
        return out

    def search_autotune(self, Q, K=10, P=100, M=0, S=10, T=1, epsilon=1e30, seed=1998, K_per_q=None, P_per_q=None,
                        init=0, init_ids=None):
        """Times every search shape on Q, checks they agree bit for bit, keeps the fastest."""
        Q = np.ascontiguousarray(Q, np.float32)
        p = SearchParams(K, M, P, S, T, epsilon, seed, init)
        kq = None if K_per_q is None else np.ascontiguousarray(K_per_q, np.uint32)
        pq = None if P_per_q is None else np.ascontiguousarray(P_per_q, np.uint32)
        ii = None if init_ids is None else np.ascontiguousarray(init_ids, np.uint32)
        t = SearchTuning()
        self._check(self.L.kg_search_autotune(self.h, _ptr(Q), Q.shape[0], Q.strides[0], C.byref(p), _ptr(kq),
                                              _ptr(pq), _ptr(ii), 0 if ii is None else ii.shape[1], C.byref(t)))
        return {f: getattr(t, f) for f, _ in SearchTuning._fields_}

    def set_search_tuning(self, split=4, warps_per_block=0, prefetch=2, regs=64, compact=1):
        t = SearchTuning(split, warps_per_block, prefetch, 0.0, 0.0, 0, regs, compact)
        self._check(self.L.kg_set_search_tuning(self.h, C.byref(t)))

    def search_tuning(self):
        t = SearchTuning()
        self._check(self.L.kg_get_search_tuning(self.h, C.byref(t)))
        return {"split": t.split, "warps_per_block": t.warps_per_block, "prefetch": t.prefetch, "regs": t.regs,
                "compact": t.compact}

    def last_search_shape(self):
        """kg_last_search_shape: the shape the last search launched (compact = 1 if the compact pool ran)."""
        t = SearchTuning()
        self._check(self.L.kg_last_search_shape(self.h, C.byref(t)))
        return {"split": t.split, "warps_per_block": t.warps_per_block, "prefetch": t.prefetch, "regs": t.regs,
                "compact": t.compact, "ms": t.ms}

    def set_search_precision(self, mode):
        """'fp32' (default), 'bf16' or 'fp8': compressed rows that filter the walk's candidates."""
        self._check(self.L.kg_set_search_precision(self.h, SEARCH_PRECISION[mode] if isinstance(mode, str)
                                                    else int(mode)))

    def search_filter_stats(self):
        st = FilterStats()
        self._check(self.L.kg_last_search_filter(self.h, C.byref(st)))
        out = {f: getattr(st, f) for f, _ in FilterStats._fields_}
        out["mode"] = {0: "fp32", 1: "bf16", 2: "fp8"}[st.mode]
        return out

    def filter_bounds(self, Q, ids):
        """(lower bound, canonical distance) of every (query, ids[q, j]) pair."""
        Q = np.ascontiguousarray(Q, np.float32)
        ids = np.ascontiguousarray(ids, np.uint32)
        lb = np.zeros(ids.shape, np.float32)
        dist = np.zeros(ids.shape, np.float32)
        self._check(self.L.kg_filter_bounds(self.h, _ptr(Q), Q.shape[0], Q.strides[0], _ptr(ids), ids.shape[1],
                                            _ptr(lb), _ptr(dist)))
        return lb, dist

    def build_graph_launches(self):
        """CUDA graph launches of the last build's iterations."""
        v = C.c_uint()
        self._check(self.L.kg_last_build_graphs(self.h, C.byref(v)))
        return v.value


def version():
    return lib().kg_version().decode()


def set_verbosity(v):
    lib().kg_set_verbosity(v)
