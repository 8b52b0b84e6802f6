"""Search launch shapes and the autotuner, through the C-ABI.

Every shape of the search kernel -- D-split (lanes per distance), query tile
(warps per block), L2 prefetch depth, register budget and pool entry (the
12-byte entry or the compact 8-byte one) -- must return the reference's
results bit for bit: the reference's fixtures and the oracle on random
graphs with tails (D % 16 != 0), per-query K/P and T > 1.  The autotuner
must time every shape, find them all identical and keep the fastest.
"""
import numpy as np
import pytest

from conftest import load_golden
from oracle import kgoracle as ko

pytestmark = pytest.mark.gpu

SHAPES = [(s, w, p, r, c) for s in (2, 4, 8) for w in (1, 2, 8) for p in (0, 2) for r in (56, 64, 80) for c in (0, 1)]


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def random_graph(rng, n, dmin, dmax):
    deg = rng.integers(dmin, dmax + 1, n)
    off = np.zeros(n + 1, np.uint64)
    off[1:] = np.cumsum(deg)
    ids = rng.integers(0, n, int(off[-1])).astype(np.uint32)
    M = np.minimum(deg, rng.integers(1, dmax + 1, n)).astype(np.uint32)
    return ko.Graph(off, ids, np.zeros(len(ids), np.float32), M)


@pytest.mark.parametrize("split,wpb,pf,regs,compact", SHAPES)
def test_every_shape_matches_reference_fixture(gpu_ctx, split, wpb, pf, regs, compact):
    g = load_golden("mix32")
    G = ko.read_index(g["index_bytes"])
    gpu_ctx.set_data(g["X"], g["metric"])
    gpu_ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    gpu_ctx.set_search_tuning(split, wpb, pf, regs, compact)
    try:
        for i, s in enumerate(g["searches"]):
            init_ids = g.get("s%d_init" % i)
            ids, d, cnt, cost = gpu_ctx.search(g["Q"], init_ids=init_ids, **s)
            ran = gpu_ctx.last_search_shape()
            if s.get("P", 100) < len(g["X"]) and s.get("S", 10) >= 1:
                assert ran["compact"] == compact, (s, ran)   # the fixture graphs allow the compact entry
            if "s%d_counts" % i in g:
                ref_c = g["s%d_counts" % i]
                assert (cnt == ref_c).all() and (cost == g["s%d_costs" % i]).all()
                for q in range(len(cnt)):
                    c = int(cnt[q])
                    assert (ids[q, :c] == g["s%d_ids" % i][q, :c]).all()
                    assert (bits(d[q, :c]) == bits(g["s%d_dists" % i][q, :c])).all()
            else:
                assert (ids == g["s%d_ids" % i]).all()
                assert (bits(d) == bits(g["s%d_dists" % i])).all()
    finally:
        gpu_ctx.set_search_tuning(4, 0, 2)


@pytest.mark.parametrize("metric,d", [("euclidean", 40), ("angular", 96), ("l2sqr", 27)])
def test_every_split_matches_oracle_with_tails(gpu_ctx, metric, d):
    rng = np.random.default_rng(d + 1)
    n = 4000
    X = rng.integers(0, 9, (n, d)).astype(np.float32)   # integer values: many exact ties
    Q = rng.integers(0, 9, (40, d)).astype(np.float32)
    G = random_graph(rng, n, 4, 60)
    gpu_ctx.set_data(X, metric)
    gpu_ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    o = ko.Oracle(X, metric)
    Kq = rng.choice([1, 10, 30], len(Q)).astype(np.uint32)
    Pq = rng.choice([20, 60, 5000], len(Q)).astype(np.uint32)   # 5000 >= n: brute-force rows
    ref = [o.search(G, Q[q:q + 1], K=int(Kq[q]), P=int(Pq[q])) for q in range(len(Q))]
    try:
        for split, compact in ((2, 0), (4, 0), (8, 0), (2, 1), (4, 1), (8, 1)):
            gpu_ctx.set_search_tuning(split, 0, 2, 64, compact)
            ids, dd, cnt, cost = gpu_ctx.search(Q, K_per_q=Kq, P_per_q=Pq)
            assert gpu_ctx.last_search_shape()["compact"] == compact
            for q, (oi, od, oc, ocost) in enumerate(ref):
                c = int(oc[0])
                assert cnt[q] == c and cost[q] == ocost[0], (split, q)
                assert (ids[q, :c] == oi[0, :c]).all(), (split, q)
                assert (bits(dd[q, :c]) == bits(od[0, :c])).all(), (split, q)
            ids3, d3, c3, k3 = gpu_ctx.search(Q, K=5, P=30, T=3)
            oi, od, oc, ocost = o.search(G, Q, K=5, P=30, T=3)
            assert (c3 == oc).all() and (k3 == ocost).all()
            for q in range(len(Q)):
                assert (ids3[q, :c3[q]] == oi[q, :c3[q]]).all()
                assert (bits(d3[q, :c3[q]]) == bits(od[q, :c3[q]])).all()
    finally:
        gpu_ctx.set_search_tuning(4, 0, 2)


def test_autotune_keeps_fastest_identical_shape(gpu_ctx):
    from kgraph_b200 import capi
    rng = np.random.default_rng(11)
    n, d = 20000, 64
    X = rng.random((n, d), dtype=np.float32)
    Q = rng.random((512, d), dtype=np.float32)
    G = random_graph(rng, n, 10, 40)
    gpu_ctx.set_data(X, "euclidean")
    gpu_ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    before = gpu_ctx.search(Q, K=10, P=64)
    best = gpu_ctx.search_autotune(Q, K=10, P=64)
    # the default shape, then 2 register budgets x 3 splits x 3 tiles x 2 prefetch depths, each with
    # the 12-byte and the compact pool entry
    assert best["variants"] == 109 and best["ms"] <= best["default_ms"]
    assert gpu_ctx.search_tuning() == {k: best[k] for k in ("split", "warps_per_block", "prefetch", "regs",
                                                             "compact")}
    after = gpu_ctx.search(Q, K=10, P=64)
    for a, b in zip(before, after):
        assert (np.asarray(a).view(np.uint32) == np.asarray(b).view(np.uint32)).all()
    with pytest.raises(capi.KGError, match="split must be"):
        gpu_ctx.set_search_tuning(3, 0, 2)
    gpu_ctx.set_search_tuning(4, 0, 2)


def test_compact_pool_on_hub_nodes_and_its_fallback(gpu_ctx):
    """Node 0 gets degree and M 200 (a hub, as reverse=-1 makes them): with S = 1 its
    expansion is 200 batches, which the compact word holds (3,000 nodes: 12 id bits,
    19 progress bits), and the walk matches the oracle.  The compressed-row filter
    has no compact variant: asked for it, the BF16-filtered walk runs the 12-byte
    entry, with the same results."""
    rng = np.random.default_rng(5)
    n, d = 3000, 24
    X = rng.integers(0, 9, (n, d)).astype(np.float32)
    Q = rng.integers(0, 9, (30, d)).astype(np.float32)
    G = random_graph(rng, n, 4, 40)
    deg0 = int(G.offsets[1])
    extra = rng.integers(0, n, 200 - deg0).astype(np.uint32)
    ids = np.concatenate([G.ids[:deg0], extra, G.ids[deg0:]]).astype(np.uint32)
    off = G.offsets.astype(np.int64).copy()
    off[1:] += len(extra)
    M = G.M.copy()
    M[0] = 200
    G2 = ko.Graph(off.astype(np.uint64), ids, np.zeros(len(ids), np.float32), M)
    gpu_ctx.set_data(X, "euclidean")
    gpu_ctx.set_graph(G2.offsets, G2.ids, G2.dists, G2.M)
    o = ko.Oracle(X, "euclidean")
    try:
        gpu_ctx.set_search_tuning(4, 0, 2, 64, 1)
        for S in (1, 3, 10):
            gi, gd, gc, gk = gpu_ctx.search(Q, K=10, P=40, S=S)
            assert gpu_ctx.last_search_shape()["compact"] == 1, S
            oi, od, oc, ok = o.search(G2, Q, K=10, P=40, S=S)
            assert (gc == oc).all() and (gk == ok).all()
            for q in range(len(Q)):
                assert (gi[q, :gc[q]] == oi[q, :gc[q]]).all()
                assert (bits(gd[q, :gc[q]]) == bits(od[q, :gc[q]])).all()
        gpu_ctx.set_search_precision("bf16")
        fi, fd, fc, fk = gpu_ctx.search(Q, K=10, P=40, S=3)
        assert gpu_ctx.last_search_shape()["compact"] == 0
        oi, od, oc, ok = o.search(G2, Q, K=10, P=40, S=3)
        assert (fc == oc).all() and (fk == ok).all()
        for q in range(len(Q)):
            assert (fi[q, :fc[q]] == oi[q, :fc[q]]).all()
    finally:
        gpu_ctx.set_search_precision("fp32")
        gpu_ctx.set_search_tuning(4, 0, 2)
