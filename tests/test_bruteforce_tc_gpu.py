"""The brute-force path on the tensor cores (kg_bruteforce.cu), through the C-ABI.

SearchOracle::search (kgraph.cpp:231-252): the K rows with the smallest
canonical FP32 distance, ties by id, within epsilon.  The tensor cores only
pick candidates (BF16 products, a rigorous error margin); every returned id
and distance comes from the canonical FP32 evaluation, so the results must
equal, bit for bit, both the CUDA-core scan (the reference's loop) and the
reference's own brute-force output in the golden fixtures.
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, WIDE_GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def run(ctx, Q, K, mode, epsilon=1e30):
    ctx.set_bruteforce_mode(mode)
    try:
        r = ctx.search(Q, K=K, epsilon=epsilon)   # no graph: every query is a brute-force query
        st = ctx.bruteforce_stats()
    finally:
        ctx.set_bruteforce_mode("auto")
    return r, st


def same(a, b):
    (i1, d1, c1, k1), (i2, d2, c2, k2) = a, b
    assert (c1 == c2).all()
    for q in range(len(c1)):
        c = int(c1[q])
        assert (i1[q, :c] == i2[q, :c]).all(), q
        assert (bits(d1[q, :c]) == bits(d2[q, :c])).all(), q
    assert (bits(k1) == bits(k2)).all()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_tensor_bruteforce_matches_reference_fixture(name):
    from kgraph_b200 import capi
    g = load_golden(name)
    ctx = capi.Context(0)
    try:
        ctx.set_data(g["X"], g["metric"])
        (ids, d, cnt, cost), st = run(ctx, g["Q"], 10, "tensor")
        assert st["tensor"] == 1
        assert (cnt == 10).all() and (cost == 1.0).all()
        assert (ids == g["bf_ids"]).all()
        assert (bits(d) == bits(g["bf_dists"])).all()
    finally:
        ctx.close()


@pytest.mark.parametrize("name", WIDE_GOLDEN_CASES)
def test_rows_too_wide_for_the_tiles_take_the_scan(name):
    """Rows wider than 256 floats: the tensor mode falls back to the warp scan
    (the tile path stages at most 256 columns), with the reference's results."""
    from kgraph_b200 import capi
    g = load_golden(name)
    ctx = capi.Context(0)
    try:
        ctx.set_data(g["X"], g["metric"])
        (ids, d, cnt, cost), st = run(ctx, g["Q"], 10, "tensor")
        assert st["tensor"] == 0
        assert (cnt == 10).all() and (cost == 1.0).all()
        assert (ids == g["bf_ids"]).all()
        assert (bits(d) == bits(g["bf_dists"])).all()
    finally:
        ctx.close()


def dataset(kind, n, d, rng):
    if kind == "uniform":
        return rng.random((n, d), dtype=np.float32)
    if kind == "mixture":   # integers: BF16 holds them exactly, many exact ties
        c = rng.uniform(0, 128, (32, d))
        return np.round(np.maximum(c[rng.integers(0, 32, n)] + rng.normal(0, 20, (n, d)), 0)).astype(np.float32)
    if kind == "sphere":
        x = rng.standard_normal((n, d)).astype(np.float32)
        return x / np.linalg.norm(x, axis=1, keepdims=True)
    if kind == "far":       # far from the origin: centring matters
        return (1000.0 + rng.standard_normal((n, d))).astype(np.float32)
    if kind == "near":      # clusters of near-duplicates: BF16 error large against the gaps
        base = rng.standard_normal((40, d)).astype(np.float32) * 10
        return (base[rng.integers(0, 40, n)] + rng.standard_normal((n, d)).astype(np.float32) * 1e-3).astype(np.float32)
    raise ValueError(kind)


CASES = [("uniform", 20000, 100, "euclidean", 10), ("mixture", 30000, 128, "euclidean", 100),
         ("sphere", 20000, 96, "angular", 10), ("uniform", 15000, 24, "l2sqr", 1),
         ("far", 12000, 48, "euclidean", 16), ("near", 10000, 64, "l2sqr", 10),
         ("mixture", 9000, 33, "l2sqr", 128), ("sphere", 5000, 256, "angular", 20)]


@pytest.mark.parametrize("kind,n,d,metric,K", CASES)
def test_tensor_bruteforce_equals_scan(kind, n, d, metric, K):
    from kgraph_b200 import capi
    rng = np.random.default_rng(n + d + K)
    X = dataset(kind, n, d, rng)
    Q = dataset(kind, 333, d, np.random.default_rng(d))   # not a multiple of the 128-query tile
    ctx = capi.Context(0)
    try:
        ctx.set_data(X, metric)
        ref, st0 = run(ctx, Q, K, "scan")
        assert st0["tensor"] == 0
        got, st = run(ctx, Q, K, "tensor")
        assert st["tensor"] == 1
        same(ref, got)
        # the candidates stay few where the BF16 error is small against the distance gaps
        if kind in ("mixture", "uniform", "sphere"):
            assert st["full_scans"] == 0 and st["candidates"] < 40 * K * len(Q), st
        # epsilon cuts some lists short
        eps = float(np.median(ref[1][:, K // 2]))
        same(run(ctx, Q, K, "scan", eps)[0], run(ctx, Q, K, "tensor", eps)[0])
    finally:
        ctx.close()


def test_tensor_bruteforce_all_ties_falls_back_to_full_scan():
    """Every row identical: all distances tie, every row is a candidate, the
    per-query capacity overflows and the query is scanned in full -- still
    the reference's list (the K smallest ids)."""
    from kgraph_b200 import capi
    X = np.ones((5000, 32), np.float32)
    Q = np.ones((7, 32), np.float32) * 2
    ctx = capi.Context(0)
    try:
        ctx.set_data(X, "euclidean")
        ref, _ = run(ctx, Q, 10, "scan")
        got, st = run(ctx, Q, 10, "tensor")
        same(ref, got)
        assert st["full_scans"] == len(Q)
        assert (got[0] == np.arange(10, dtype=np.uint32)[None, :]).all()
    finally:
        ctx.close()


def test_python_blas_flag_uses_the_same_exact_path():
    import kgraph_b200 as kgraph
    g = load_golden("u16")
    index = kgraph.KGraph(g["X"], g["metric"])
    ids, d = index.search(g["Q"], K=10, blas=True, withDistance=True)
    assert (ids == g["bf_ids"]).all() and (bits(d) == bits(g["bf_dists"])).all()
