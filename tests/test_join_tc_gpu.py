"""Tensor-core local join (tcgen05, BF16 or FP8 E4M3 tiles + FP32 recheck), through the C-ABI.

The BF16 Gram block only decides which pairs can be skipped; every pair that
may pass the reference's radius test is recomputed with the canonical FP32
distance and inserted exactly as the FP32 join does.  So the graph must keep
the reference's quality (recall within 0.005 of the reference's own build),
every stored distance must be the canonical FP32 distance of its pair, and
the FP64 tile-error report must show the margin was never exceeded.
"""
import numpy as np
import pytest

from oracle import kgoracle as ko
from test_build_gpu import bits, data, exact_knn, graph_recall

pytestmark = pytest.mark.gpu

CASES = [("mixture", 12000, 64, "euclidean", dict(K=20, L=40, S=10)),
         ("mixture", 10000, 128, "euclidean", dict(K=25, L=50, S=10)),
         ("sphere", 10000, 96, "angular", dict(K=15, L=40, S=8)),
         ("uniform", 8000, 80, "l2sqr", dict(K=10, L=30, S=8)),
         # long lists: new lists above 128 entries take two column tiles
         ("mixture", 6000, 64, "euclidean", dict(K=20, L=80, S=40)),
         # the tile also runs (forced) at small d
         ("uniform", 8000, 16, "euclidean", dict(K=25, L=50, S=10))]


FP8_CASES = [("mixture", 12000, 64, "euclidean", dict(K=20, L=40, S=10)),
             ("mixture", 10000, 128, "euclidean", dict(K=25, L=50, S=10)),
             ("sphere", 10000, 96, "angular", dict(K=15, L=40, S=8)),
             ("uniform", 8000, 32, "l2sqr", dict(K=10, L=30, S=8))]


@pytest.mark.parametrize("prec,kind,n,d,metric,bp", [("bf16",) + c for c in CASES] + [("fp8",) + c for c in FP8_CASES])
def test_tc_join_matches_reference_quality(gpu_ctx, prec, kind, n, d, metric, bp):
    """BF16 tiles, and FP8 E4M3 tiles with a scale per row: the tile only
    filters, so the graph keeps the reference's quality and every stored
    distance is canonical; the FP64 check of sampled tile errors never
    exceeds the margin."""
    from kgraph_b200 import capi
    X = data(kind, n, d, 7 * n + d)
    gpu_ctx.set_data(X, metric)
    gpu_ctx.set_join_precision(prec + "_always")   # the tensor-core filter in every iteration
    try:
        info = gpu_ctx.build(iterations=30, reverse=0, **bp)
        st = gpu_ctx.join_stats()
    finally:
        gpu_ctx.set_join_precision("auto")
    off, ids, dists, M = gpu_ctx.graph()
    G = ko.Graph(off, ids, dists, M)
    K = bp["K"]
    c2 = capi.Context(0)
    c2.set_data(X, metric)
    ex_i, ex_d = exact_knn(c2, X, K)
    c2.close()
    R, rinfo, _ = ko.Oracle(X, metric).build(iterations=30, reverse=0, **bp)
    r_gpu, r_ref = graph_recall(G, ex_d, K), graph_recall(R, ex_d, K)
    assert abs(r_gpu - r_ref) <= 0.005, (r_gpu, r_ref, info, rinfo, st)
    # the report: the join that ran, its pair count, and a safe margin
    assert st["mode"] == prec and st["tc_iterations"] == info["iterations"]
    total = n * (n - 1) / 2
    assert abs(st["pairs"] - info["cost"] * total) <= 1e-4 * st["pairs"] + 1
    assert 0 < st["rechecked"] <= st["pairs"]
    assert st["sampled"] > 0
    assert st["violations"] == 0, st
    assert st["max_err_over_margin"] < 1.0, st
    # every stored distance is the canonical FP32 distance; rows sorted, no duplicates
    o = ko.Oracle(X, metric)
    rng = np.random.default_rng(1)
    for r in rng.choice(n, 200, replace=False):
        a, b = int(off[r]), int(off[r + 1])
        row_i, row_d = ids[a:b], dists[a:b]
        assert (np.diff(row_d) >= 0).all()
        assert len(set(row_i.tolist())) == len(row_i)
        for j in range(0, len(row_i), 5):
            assert bits(np.float32(o.pair(r, row_i[j]))) == bits(row_d[j])


def test_join_precision_modes(gpu_ctx):
    X = data("mixture", 6000, 64, 3)
    gpu_ctx.set_data(X, "euclidean")
    gpu_ctx.set_join_precision("fp32")
    info32 = gpu_ctx.build(K=10, L=30, S=8, iterations=5)
    st32 = gpu_ctx.join_stats()
    gpu_ctx.set_join_precision("bf16")   # the tensor-core filter once pools fill
    info_a = gpu_ctx.build(K=10, L=30, S=8, iterations=5)
    st_a = gpu_ctx.join_stats()
    gpu_ctx.set_join_precision("auto")
    assert st32["mode"] == "fp32" and st32["rechecked"] == st32["pairs"] and st32["sampled"] == 0
    assert st_a["mode"] == "bf16" and 1 <= st_a["tc_iterations"] <= 5 and st_a["rechecked"] < st_a["pairs"]
    total = 6000 * 5999 / 2
    assert abs(st32["pairs"] - info32["cost"] * total) <= 1e-4 * st32["pairs"] + 1
    assert abs(st_a["pairs"] - info_a["cost"] * total) <= 1e-4 * st_a["pairs"] + 1
    # auto runs the CUDA-core join
    gpu_ctx.build(K=10, L=30, S=8, iterations=2)
    assert gpu_ctx.join_stats()["mode"] == "fp32"


def test_fp8_join_needs_d_padded_to_32(gpu_ctx):
    from kgraph_b200 import capi
    X = data("uniform", 3000, 80, 5)   # rows padded to 80 floats: not a multiple of 32
    gpu_ctx.set_data(X, "euclidean")
    gpu_ctx.set_join_precision("fp8_always")
    try:
        with pytest.raises(capi.KGError, match="multiple of 32"):
            gpu_ctx.build(K=10, L=30, S=8, iterations=2)
    finally:
        gpu_ctx.set_join_precision("auto")
