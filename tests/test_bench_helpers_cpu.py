"""bench.py's host-side helpers, without a GPU: the index writer it hands the
reference's CPU search, the synthetic workload generators, the tie-aware
recall ground truth and the roofline peak lookup."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT
from oracle import kgoracle as ko

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def random_csr(rng, n, dmax):
    deg = rng.integers(1, dmax + 1, n)
    off = np.zeros(n + 1, np.uint64)
    off[1:] = np.cumsum(deg)
    ids = rng.integers(0, n, int(off[-1])).astype(np.uint32)
    dists = rng.random(int(off[-1])).astype(np.float32)
    M = np.minimum(deg, rng.integers(1, dmax + 1, n)).astype(np.uint32)
    return off, ids, dists, M


def test_index_writer_round_trips_and_the_reference_reads_it(tmp_path):
    rng = np.random.default_rng(0)
    n, d = 500, 16
    off, ids, dists, M = random_csr(rng, n, 12)
    p = str(tmp_path / "g.idx")
    bench.ctx_save(p, off, ids, dists, M)
    G = ko.read_index(p)
    assert (G.offsets == off).all() and (G.ids == ids).all() and (G.M == M).all()
    assert (G.dists.view(np.uint32) == dists.view(np.uint32)).all()
    if not ko.reference_available():
        pytest.skip("reference not compiled")
    kg = ko.load_reference_module()
    X = rng.random((n, d), dtype=np.float32)
    g = kg.KGraph(X, "euclidean")
    g.load(p)                                 # the reference's own loader (kgraph.cpp:291-331)
    out = g.search(X[:5], K=3, P=10)
    assert np.asarray(out).shape == (5, 3)


@pytest.mark.parametrize("name", ["c1", "c3", "c4", "c5"])
def test_workload_generators(name):
    w = dict(bench.WORKLOADS[name], n=2000, nq=50)
    if "router_train" in w:
        w["router_train"] = 100
    X, Q, T = bench.make_workload_data(w)
    assert X.shape == (2000, w["d"]) and Q.shape == (50, w["d"]) and X.dtype == np.float32
    assert (T is None) == ("router_train" not in w)
    if w["kind"] == "sphere":
        assert np.allclose(np.linalg.norm(X, axis=1), 1, atol=1e-5)
    if w["kind"] == "mixture":
        assert (X >= 0).all() and (X == np.round(X)).all()
    X2, _, _ = bench.make_workload_data(w)
    assert (X2 == X).all()   # seeded


def test_recall_ground_truth_is_tie_aware():
    import torch
    rng = np.random.default_rng(1)
    X = np.round(rng.random((400, 8)) * 3).astype(np.float32)   # many exact ties
    Q = np.round(rng.random((20, 8)) * 3).astype(np.float32)
    Xt = torch.as_tensor(X, dtype=torch.float64)
    Qt = torch.as_tensor(Q, dtype=torch.float64)
    gd, gi = bench.exact_topk_fp64(Xt, Qt, 10, torch)
    ids = gi.numpy().astype(np.uint32)
    assert bench.recall_at(ids, Xt, Qt, gd, 10, torch) == 1.0
    # any other id at a tied K-th distance counts too; a far id does not
    d = ((X[None, :, :] - Q[:, None, :]) ** 2).sum(2)
    swapped = ids.copy()
    q = 0
    tied = np.nonzero(d[q] == d[q, ids[q, 9]])[0]
    other = [t for t in tied if t not in ids[q]]
    if other:
        swapped[q, 9] = other[0]
        assert bench.recall_at(swapped, Xt, Qt, gd, 10, torch) == 1.0
    far = int(np.argmax(d[q]))
    swapped[q, 9] = far
    assert bench.recall_at(swapped, Xt, Qt, gd, 10, torch) < 1.0


def test_roofline_peak_source():
    v, src = bench.hbm_peak()
    if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        assert src.startswith("measured") and v > 1000
    else:
        assert src.startswith("fallback") and v == 6650.0
