"""Search parity on the GPU, through the C-ABI.

The CUDA walk must return the reference's results bit for bit: ids,
distances, result counts and SearchInfo.cost, on the reference's own index
files (committed fixtures), and the oracle's on random graphs, per-query K/P
batches, T > 1, init seeds, epsilon and the P >= N brute-force path.
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, WIDE_GOLDEN_CASES, load_golden
from oracle import kgoracle as ko

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def assert_rows_equal(ids, d, cnt, rids, rd, rcnt):
    assert (cnt == rcnt).all()
    for q in range(len(cnt)):
        c = int(cnt[q])
        assert (ids[q, :c] == rids[q, :c]).all(), q
        assert (bits(d[q, :c]) == bits(rd[q, :c])).all(), q


@pytest.mark.parametrize("name", GOLDEN_CASES + WIDE_GOLDEN_CASES)
def test_search_matches_reference_fixtures(gpu_ctx, name):
    g = load_golden(name)
    G = ko.read_index(g["index_bytes"])
    gpu_ctx.set_data(g["X"], g["metric"])
    gpu_ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    o = ko.Oracle(g["X"], g["metric"])
    for i, s in enumerate(g["searches"]):
        init_ids = g.get("s%d_init" % i)
        ids, d, cnt, cost = gpu_ctx.search(g["Q"], init_ids=init_ids, **s)
        oi, od, oc, ocost = o.search(G, g["Q"], init_ids=init_ids, **s)
        assert_rows_equal(ids, d, cnt, oi, od, oc)
        assert (cost == ocost).all()
        if "s%d_counts" % i in g:
            assert_rows_equal(ids, d, cnt, g["s%d_ids" % i], g["s%d_dists" % i], g["s%d_counts" % i])
            assert (cost == g["s%d_costs" % i]).all()
        else:
            K = s["K"]
            assert (cnt == K).all()
            assert (ids == g["s%d_ids" % i]).all()
            assert (bits(d) == bits(g["s%d_dists" % i])).all()


@pytest.mark.parametrize("name", GOLDEN_CASES + WIDE_GOLDEN_CASES)
def test_bruteforce_matches_reference_fixtures(name):
    from kgraph_b200 import capi
    g = load_golden(name)
    c = capi.Context(0)
    c.set_data(g["X"], g["metric"])     # no graph: every query is brute force
    ids, d, cnt, cost = c.search(g["Q"], K=10)
    assert (cnt == 10).all()
    assert (ids == g["bf_ids"]).all()
    assert (bits(d) == bits(g["bf_dists"])).all()
    assert (cost == 1.0).all()
    c.close()


def random_graph(rng, n, dmin, dmax):
    deg = rng.integers(dmin, dmax + 1, n)
    off = np.zeros(n + 1, np.uint64)
    off[1:] = np.cumsum(deg)
    ids = rng.integers(0, n, int(off[-1])).astype(np.uint32)   # duplicates and self loops included
    M = np.minimum(deg, rng.integers(1, dmax + 1, n)).astype(np.uint32)
    return ko.Graph(off, ids, np.zeros(len(ids), np.float32), M)


@pytest.mark.parametrize("metric,d", [("euclidean", 128), ("angular", 96), ("l2sqr", 24), ("euclidean", 16)])
def test_search_random_graph_matches_oracle(gpu_ctx, metric, d):
    rng = np.random.default_rng(d)
    n = 6000
    X = rng.integers(0, 16, (n, d)).astype(np.float32)   # integer values: many exact ties
    Q = rng.integers(0, 16, (48, d)).astype(np.float32)
    G = random_graph(rng, n, 4, 40)
    gpu_ctx.set_data(X, metric)
    gpu_ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    o = ko.Oracle(X, metric)
    for s in [dict(K=10, P=50), dict(K=25, P=200, S=7, M=12), dict(K=5, P=40, T=3), dict(K=10, P=30, epsilon=float(d))]:
        ids, dd, cnt, cost = gpu_ctx.search(Q, **s)
        oi, od, oc, ocost = o.search(G, Q, **s)
        assert_rows_equal(ids, dd, cnt, oi, od, oc)
        assert (cost == ocost).all()


def test_search_uneven_K_P_in_one_launch(gpu_ctx):
    rng = np.random.default_rng(5)
    n, d = 5000, 32
    X = rng.random((n, d), dtype=np.float32)
    Q = rng.random((96, d), dtype=np.float32)
    G = random_graph(rng, n, 8, 30)
    gpu_ctx.set_data(X, "euclidean")
    gpu_ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    Kq = rng.choice([1, 10, 100], 96).astype(np.uint32)
    Pq = rng.choice([50, 100, 200, 6000], 96).astype(np.uint32)   # 6000 >= n: brute force rows
    ids, dd, cnt, cost = gpu_ctx.search(Q, K_per_q=Kq, P_per_q=Pq)
    o = ko.Oracle(X, "euclidean")
    for q in range(96):
        oi, od, oc, ocost = o.search(G, Q[q:q + 1], K=int(Kq[q]), P=int(Pq[q]))
        c = int(oc[0])
        assert cnt[q] == c and cost[q] == ocost[0]
        assert (ids[q, :c] == oi[0, :c]).all()
        assert (bits(dd[q, :c]) == bits(od[0, :c])).all()


def test_search_init_seeds_and_errors(gpu_ctx):
    from kgraph_b200 import capi
    rng = np.random.default_rng(9)
    n, d = 3000, 20
    X = rng.random((n, d), dtype=np.float32)
    Q = rng.random((32, d), dtype=np.float32)
    G = random_graph(rng, n, 5, 25)
    gpu_ctx.set_data(X, "l2sqr")
    gpu_ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    init = rng.integers(0, n, (32, 7)).astype(np.uint32)
    ids, dd, cnt, cost = gpu_ctx.search(Q, K=10, P=40, init=7, init_ids=init)
    oi, od, oc, ocost = ko.Oracle(X, "l2sqr").search(G, Q, K=10, P=40, init=7, init_ids=init)
    assert_rows_equal(ids, dd, cnt, oi, od, oc)
    with pytest.raises(capi.KGError, match="L < params.K"):
        gpu_ctx.search(Q, K=5, P=40, init=7, init_ids=init, out_ld=10)
    with pytest.raises(capi.KGError, match="T must be 1"):
        gpu_ctx.search(Q, K=10, P=40, T=2, init=3, init_ids=init)


def test_python_module_load_search_save_roundtrip(tmp_path):
    import kgraph_b200 as kgraph
    g = load_golden("u16")
    p = tmp_path / "ref.idx"
    p.write_bytes(g["index_bytes"].tobytes())
    k = kgraph.KGraph(g["X"], "euclidean")
    k.load(str(p))
    s = g["searches"][0]
    ids, d = k.search(g["Q"], withDistance=True, **s)
    assert (ids == g["s0_ids"]).all()
    assert (bits(d) == bits(g["s0_dists"])).all()
    only = k.search(g["Q"], **s)
    assert (only == ids).all()
    out = tmp_path / "again.idx"
    k.save(str(out))
    # Same header, node records, ids and distances; the reference leaves each
    # record's flag and padding bytes uninitialised (kgraph.cpp:67-74, 370),
    # this library writes zeros there.
    a, b = ko.read_index(str(out)), ko.read_index(g["index_bytes"])
    assert out.read_bytes()[:20] == g["index_bytes"].tobytes()[:20]
    assert (a.offsets == b.offsets).all() and (a.ids == b.ids).all() and (a.M == b.M).all()
    assert (bits(a.dists) == bits(b.dists)).all()
    bf = kgraph.KGraph(g["X"], "euclidean").search(g["Q"], K=10, withDistance=True)
    assert (bf[0] == g["bf_ids"]).all()


def test_empty_query_batch(gpu_ctx, tmp_path):
    """A batch of zero queries returns empty results and launches nothing,
    through the C-ABI and the Python module (python-api.cpp:266-273 sizes the
    result from the query count: 0 x K)."""
    import kgraph_b200 as kgraph
    g = load_golden("u16")
    G = ko.read_index(g["index_bytes"])
    gpu_ctx.set_data(g["X"], g["metric"])
    gpu_ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    Q0 = np.zeros((0, g["X"].shape[1]), np.float32)
    ids, d, cnt, cost = gpu_ctx.search(Q0, K=10, P=40)
    assert ids.shape == (0, 10) and d.shape == (0, 10) and cnt.shape == (0,) and cost.shape == (0,)
    p = tmp_path / "ref.idx"
    p.write_bytes(g["index_bytes"].tobytes())
    k = kgraph.KGraph(g["X"], "euclidean")
    k.load(str(p))
    r, rd = k.search(Q0, K=10, withDistance=True)
    assert r.shape == (0, 10) and rd.shape == (0, 10)
    # and the index still answers a real batch afterwards
    ids, d, cnt, cost = gpu_ctx.search(g["Q"], **g["searches"][0])
    assert (ids == g["s0_ids"]).all()
