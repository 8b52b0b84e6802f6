"""Pins the oracle (oracle/kgoracle.cpp) to the reference.

Always: against the committed fixtures made by the reference itself
(tests/golden/make_golden.py) -- search ids/dists (and counts/costs where the
reference reports them), brute force, and the single-thread build graph bit
for bit.  When the reference is compiled here (oracle/_ref), also live on
fresh random inputs.
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, WIDE_GOLDEN_CASES, load_golden
from oracle import kgoracle as ko


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("name", GOLDEN_CASES + WIDE_GOLDEN_CASES)
def test_oracle_search_matches_reference_fixtures(name):
    g = load_golden(name)
    G = ko.read_index(g["index_bytes"])
    o = ko.Oracle(g["X"], g["metric"])
    for i, s in enumerate(g["searches"]):
        init_ids = g.get("s%d_init" % i)
        ids, d, cnt, cost = o.search(G, g["Q"], init_ids=init_ids, **s)
        if "s%d_counts" % i in g:
            assert (cnt == g["s%d_counts" % i]).all()
            assert (cost == g["s%d_costs" % i]).all()
            for q in range(len(cnt)):
                c = cnt[q]
                assert (ids[q, :c] == g["s%d_ids" % i][q, :c]).all()
                assert (bits(d[q, :c]) == bits(g["s%d_dists" % i][q, :c])).all()
        else:
            assert (ids == g["s%d_ids" % i]).all(), (name, s)
            assert (bits(d) == bits(g["s%d_dists" % i])).all(), (name, s)


@pytest.mark.parametrize("name", GOLDEN_CASES + WIDE_GOLDEN_CASES)
def test_oracle_bruteforce_matches_reference_fixtures(name):
    g = load_golden(name)
    o = ko.Oracle(g["X"], g["metric"])
    ids, d, cnt = o.bruteforce(g["Q"], 10)
    assert (ids == g["bf_ids"]).all()
    assert (bits(d) == bits(g["bf_dists"])).all()


@pytest.mark.parametrize("name", GOLDEN_CASES + WIDE_GOLDEN_CASES)
def test_oracle_single_thread_build_is_the_reference_graph(name):
    g = load_golden(name)
    ref = ko.read_index(g["index_bytes"])
    o = ko.Oracle(g["X"], g["metric"])
    G, info, log = o.build(rand_seed=1, **g["build"])
    assert (G.offsets == ref.offsets).all()
    assert (G.ids == ref.ids).all()
    assert (bits(G.dists) == bits(ref.dists)).all()
    assert (G.M == ref.M).all()


def test_oracle_rejects_what_the_reference_rejects():
    X = np.random.default_rng(0).random((50, 4), dtype=np.float32)
    o = ko.Oracle(X, "euclidean")
    with pytest.raises(RuntimeError, match="prune level not supported"):
        o.build(K=5, L=10, S=4, prune=3)
    with pytest.raises(RuntimeError, match="K larger than dataset size"):
        o.build(K=50, L=60, S=4)


def test_genrandom_distinct_and_in_range():
    for N, size in [(10, 10), (100, 7), (1000, 999), (5, 0)]:
        s = ko.genrandom(1998, size, N)
        assert len(set(s.tolist())) == size
        assert (s < N).all()


needs_ref = pytest.mark.skipif(not ko.reference_available("v4") or ko.host_isa() != "v4",
                               reason="reference not compiled here (oracle/_ref/v4)")


@needs_ref
@pytest.mark.parametrize("metric,d", [("euclidean", 16), ("euclidean", 20), ("angular", 24), ("euclidean", 29),
                                      ("angular", 31), ("euclidean", 37), ("euclidean", 40), ("angular", 96),
                                      ("euclidean", 128), ("angular", 7), ("euclidean", 9)])
def test_oracle_distances_live_against_reference(metric, d):
    kg = ko.load_reference_module("v4")
    rng = np.random.default_rng(d)
    X = rng.standard_normal((1500, d)).astype(np.float32)
    Q = rng.standard_normal((20, d)).astype(np.float32)
    ri, rd = kg.KGraph(X, metric).search(Q, K=15, withDistance=True)
    oi, od, _ = ko.Oracle(X, metric).bruteforce(Q, 15)
    assert (ri == oi).all()
    assert (bits(rd) == bits(od)).all()


REF_BUILD = r"""
import sys, numpy as np
sys.path.insert(0, %(root)r)
from oracle import kgoracle as ko
kg = ko.load_reference_module('v4')
X = np.load(sys.argv[1])
g = kg.KGraph(X, sys.argv[3])
g.build(K=8, L=20, S=6, reverse=int(sys.argv[4]), prune=int(sys.argv[5]))
g.save(sys.argv[2])
"""


@needs_ref
@pytest.mark.parametrize("metric,reverse,prune", [("euclidean", 5, 0), ("euclidean", -1, 1), ("angular", 0, 2),
                                                  ("euclidean", -1, 2)])
def test_oracle_build_reverse_prune_live_against_reference(tmp_path, metric, reverse, prune):
    import os
    import subprocess
    import sys
    from conftest import ROOT
    rng = np.random.default_rng(7 + reverse + prune)
    X = rng.random((1200, 12), dtype=np.float32)
    xp, ip, wp = str(tmp_path / "X.npy"), str(tmp_path / "g.idx"), str(tmp_path / "w.py")
    np.save(xp, X)
    open(wp, "w").write(REF_BUILD % dict(root=ROOT))
    r = subprocess.run([sys.executable, wp, xp, ip, metric, str(reverse), str(prune)], capture_output=True,
                       text=True, env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert r.returncode == 0, r.stderr
    ref = ko.read_index(ip)
    G, _, _ = ko.Oracle(X, metric).build(rand_seed=1, K=8, L=20, S=6, reverse=reverse, prune=prune)
    assert (G.offsets == ref.offsets).all()
    assert (G.ids == ref.ids).all()
    assert (G.M == ref.M).all()
