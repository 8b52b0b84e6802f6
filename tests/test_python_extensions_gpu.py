"""The Python module's extensions beyond the reference's interface, on the GPU:
search(..., router=m) with a trained router, the distance filter and the
search autotuner, each leaving the reference-exact results unchanged where it
must."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mixture(rng, n, d, centres, spread):
    c = rng.uniform(0, 100, (centres, d))
    return np.round(np.maximum(c[rng.integers(0, centres, n)] + rng.normal(0, spread, (n, d)), 0)).astype(np.float32)


def test_router_filter_and_autotune_through_the_python_module():
    import kgraph_b200 as kgraph
    rng = np.random.default_rng(3)
    allx = mixture(rng, 30000 + 20000 + 400, 32, 64, 6.0)
    X, Qtrain, Q = allx[:30000], allx[30000:50000], allx[50000:]
    index = kgraph.KGraph(X, "euclidean")
    with pytest.raises(RuntimeError, match="no index"):
        index.train_router(Qtrain)
    index.build(K=20, L=40, S=10, reverse=-1)
    # exact neighbours for recall
    Xd, Qd = X.astype(np.float64), Q.astype(np.float64)
    dd = (Xd ** 2).sum(1)[None, :] - 2 * Qd @ Xd.T
    kth = np.sort(dd, 1)[:, 9]

    def recall(ids):
        return np.mean([(dd[q, ids[q, :10]] <= kth[q] + 1e-6).sum() / 10 for q in range(len(Q))])

    plain, pd = index.search(Q, K=10, P=20, withDistance=True)
    info = index.train_router(Qtrain, clusters=128, hidden=64, epochs=3, label_P=300, batch=512)
    assert info["steps"] > 0
    routed = index.search(Q, K=10, P=20, router=3)
    assert recall(routed) > recall(plain) and recall(routed) >= 0.9
    with pytest.raises(ValueError):
        index.search(Q, K=3, P=20, router=3)   # the reference requires init < K
    # the distance filter and the autotuner change no result
    for mode in ("bf16", "fp8"):
        index.set_search_precision(mode)
        ids, d = index.search(Q, K=10, P=20, withDistance=True)
        assert (ids == plain).all() and (d.view(np.uint32) == pd.view(np.uint32)).all()
    index.set_search_precision("fp32")
    t = index.autotune(Q, K=10, P=20)
    assert t["ms"] <= t["default_ms"] and t["split"] in (2, 4, 8)
    ids, d = index.search(Q, K=10, P=20, withDistance=True)
    assert (ids == plain).all() and (d.view(np.uint32) == pd.view(np.uint32)).all()
    with pytest.raises(ValueError):
        index.set_search_precision("fp16")
