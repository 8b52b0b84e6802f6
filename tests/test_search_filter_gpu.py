"""The search's distance filter on compressed rows (BF16, FP8 E4M3 with
per-row scales), through the C-ABI.

The filter may only skip candidates the reference would drop into the
pool's spare slot, so every result must equal the FP32 walk's -- and the
reference's fixtures -- bit for bit, and it must actually skip candidates.
Its lower bound is checked directly against the canonical FP32 distance on
many pairs, including near-duplicate rows where the quantisation error is
large against the distances.
"""
import numpy as np
import pytest

from conftest import load_golden
from oracle import kgoracle as ko

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def same(r1, r2):
    (i1, d1, c1, k1), (i2, d2, c2, k2) = r1, r2
    assert (c1 == c2).all() and (bits(k1) == bits(k2)).all()
    for q in range(len(c1)):
        c = int(c1[q])
        assert (i1[q, :c] == i2[q, :c]).all(), q
        assert (bits(d1[q, :c]) == bits(d2[q, :c])).all(), q


def dataset(kind, n, d, rng):
    if kind == "mixture":   # integer values with exact ties (BF16 holds them exactly)
        c = rng.uniform(0, 128, (16, d))
        return np.round(np.maximum(c[rng.integers(0, 16, n)] + rng.normal(0, 20, (n, d)), 0)).astype(np.float32)
    if kind == "sphere":
        x = rng.standard_normal((n, d)).astype(np.float32)
        return x / np.linalg.norm(x, axis=1, keepdims=True)
    if kind == "near":      # near-duplicates: quantisation error large against the distances
        base = rng.standard_normal((64, d)).astype(np.float32) * 10
        return (base[rng.integers(0, 64, n)] + rng.standard_normal((n, d)).astype(np.float32) * 0.01).astype(np.float32)
    return rng.random((n, d), dtype=np.float32)


CASES = [("mixture", 128, "euclidean"), ("sphere", 96, "angular"), ("uniform", 20, "l2sqr"),
         ("near", 48, "euclidean"), ("uniform", 16, "euclidean")]


@pytest.mark.parametrize("kind,d,metric", CASES)
@pytest.mark.parametrize("prec", ["bf16", "fp8"])
def test_filtered_walk_equals_fp32_walk(gpu_ctx, kind, d, metric, prec):
    rng = np.random.default_rng(d)
    n = 8000
    X = dataset(kind, n, d, rng)
    Q = dataset(kind, 200, d, np.random.default_rng(d + 1))
    gpu_ctx.set_search_precision("fp32")
    gpu_ctx.set_data(X, metric)
    gpu_ctx.build(K=16, L=32, S=8, reverse=-1)
    try:
        for s in [dict(K=10, P=20), dict(K=10, P=60, S=5), dict(K=5, P=30, T=2)]:
            ref = gpu_ctx.search(Q, **s)
            gpu_ctx.set_search_precision(prec)
            got = gpu_ctx.search(Q, **s)
            st = gpu_ctx.search_filter_stats()
            gpu_ctx.set_search_precision("fp32")
            same(ref, got)
            assert st["mode"] == prec and st["approx"] > 0
            if kind != "near":
                assert st["skipped"] > 0, st
    finally:
        gpu_ctx.set_search_precision("fp32")


@pytest.mark.parametrize("prec", ["bf16", "fp8"])
def test_filtered_walk_matches_reference_fixture(gpu_ctx, prec):
    g = load_golden("mix32")
    G = ko.read_index(g["index_bytes"])
    gpu_ctx.set_data(g["X"], g["metric"])
    gpu_ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    gpu_ctx.set_search_precision(prec)
    try:
        for i, s in enumerate(g["searches"]):
            init_ids = g.get("s%d_init" % i)
            ids, d, cnt, cost = gpu_ctx.search(g["Q"], init_ids=init_ids, **s)
            if "s%d_counts" % i in g:
                assert (cnt == g["s%d_counts" % i]).all() and (cost == g["s%d_costs" % i]).all()
                for q in range(len(cnt)):
                    c = int(cnt[q])
                    assert (ids[q, :c] == g["s%d_ids" % i][q, :c]).all()
                    assert (bits(d[q, :c]) == bits(g["s%d_dists" % i][q, :c])).all()
            else:
                assert (ids == g["s%d_ids" % i]).all() and (bits(d) == bits(g["s%d_dists" % i])).all()
    finally:
        gpu_ctx.set_search_precision("fp32")


@pytest.mark.parametrize("kind,d,metric", CASES + [("uniform", 256, "angular"), ("mixture", 33, "l2sqr")])
@pytest.mark.parametrize("prec", ["bf16", "fp8"])
def test_lower_bound_never_exceeds_canonical_distance(gpu_ctx, kind, d, metric, prec):
    rng = np.random.default_rng(7 * d)
    n = 20000
    X = dataset(kind, n, d, rng)
    Q = dataset(kind, 256, d, np.random.default_rng(d + 3))
    gpu_ctx.set_data(X, metric)
    gpu_ctx.set_search_precision(prec)
    try:
        ids = rng.integers(0, n, (len(Q), 512)).astype(np.uint32)
        lb, dist = gpu_ctx.filter_bounds(Q, ids)
        assert (lb <= dist).all(), float(np.max(lb - dist))
        st = gpu_ctx.search_filter_stats()
        limit = 2 ** -8 if prec == "bf16" else 0.07
        assert 0 <= st["mean_rel_row_error"] <= st["max_rel_row_error"] <= limit
        if prec == "bf16":   # the bound is informative: its slack is small against the spread of distances
            spread = np.percentile(dist, 90) - np.percentile(dist, 10)
            assert np.median(dist - lb) < 0.5 * spread
    finally:
        gpu_ctx.set_search_precision("fp32")


@pytest.mark.parametrize("metric", ["euclidean", "angular", "l2sqr"])
@pytest.mark.parametrize("prec", ["bf16", "fp8"])
def test_filter_ignores_junk_in_device_query_padding(gpu_ctx, metric, prec):
    """Device queries used in place carry padding columns [d, ld) that may hold
    anything (the C-ABI asks for d floats per row); NaN or huge values there
    must not reach the filter's bound: results equal the FP32 walk's on clean
    host queries."""
    import torch
    from kgraph_b200 import capi
    d, ld, n, nq = 20, 32, 8000, 200
    rng = np.random.default_rng(41)
    X = dataset("sphere" if metric == "angular" else "uniform", n, d, rng)
    Q = dataset("sphere" if metric == "angular" else "uniform", nq, d, np.random.default_rng(42))
    gpu_ctx.set_search_precision("fp32")
    gpu_ctx.set_data(X, metric)
    gpu_ctx.build(K=16, L=32, S=8, reverse=-1)
    ref = gpu_ctx.search(Q, K=10, P=40)
    params = capi.SearchParams(10, 0, 40, 10, 1, 1e30, 1998, 0)
    try:
        gpu_ctx.set_search_precision(prec)
        for pad in (float("nan"), 1e30, -3.0e38):
            qd = torch.full((nq, ld), pad, dtype=torch.float32, device="cuda")
            qd[:, :d] = torch.as_tensor(Q, device="cuda")
            ids = np.zeros((nq, 10), np.uint32)
            dist = np.zeros((nq, 10), np.float32)
            cnt = np.zeros(nq, np.uint32)
            cost = np.zeros(nq, np.float32)
            gpu_ctx.search_raw(capi._ptr(qd), nq, ld * 4, params, None, None, 10, capi._ptr(ids), capi._ptr(dist),
                               capi._ptr(cnt), capi._ptr(cost))
            same(ref, (ids, dist, cnt, cost))
            assert gpu_ctx.search_filter_stats()["skipped"] > 0
    finally:
        gpu_ctx.set_search_precision("fp32")
