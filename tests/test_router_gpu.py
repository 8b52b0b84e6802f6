"""Learned entry router: its training kernels against an independent FP64
implementation, and what the trained router gains over plain seeding."""
import numpy as np
import pytest

from oracle.router_oracle import mlp_fp64

pytestmark = pytest.mark.gpu


def test_router_gradients_match_fp64():
    from kgraph_b200 import capi
    d, h, c, n = 16, 32, 48, 96
    rng = np.random.default_rng(0)
    nparam = d * h + h + h * h + h + h * c + c
    W = (rng.standard_normal(nparam) * 0.3).astype(np.float32)
    x = rng.standard_normal((n, d)).astype(np.float32)
    y = rng.integers(0, c, n).astype(np.int32)
    ctx = capi.Context(0)
    loss, g = ctx.router_gradients(d, h, c, W, x, y)
    rloss, rg = mlp_fp64(W, x, y, d, h, c)
    assert abs(loss - rloss) < 1e-3 * max(1.0, abs(rloss))
    o = 0
    for ref in rg:
        got = g[o:o + ref.size].reshape(ref.shape)
        o += ref.size
        rel = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-12)
        assert rel < 1e-2, rel
    ctx.close()


def mixture(rng, n, d, centres, spread):
    c = rng.uniform(0, 100, (centres, d))
    lab = rng.integers(0, centres, n)
    return np.round(np.maximum(c[lab] + rng.normal(0, spread, (n, d)), 0)).astype(np.float32)


def test_router_beats_plain_seeding_at_equal_P():
    from kgraph_b200 import capi
    rng = np.random.default_rng(1)
    d, centres = 32, 64
    allx = mixture(rng, 30000 + 20000 + 500, d, centres, 6.0)
    X, Qtrain, Q = allx[:30000], allx[30000:50000], allx[50000:]
    ctx = capi.Context(0)
    capi.set_verbosity(0)
    ctx.set_data(X, "euclidean")
    ctx.build(K=20, L=40, S=10, reverse=-1)
    info = ctx.router_train(Qtrain, clusters=128, hidden=64, epochs=3, label_P=300, batch=512)
    assert info["train_accuracy"] > 0.5, info
    # exact neighbours (FP64) for recall
    Xd, Qd = X.astype(np.float64), Q.astype(np.float64)
    dd = (Xd ** 2).sum(1)[None, :] - 2 * Qd @ Xd.T
    kth = np.sort(dd, 1)[:, 9]

    def recall(ids):
        return np.mean([(dd[q, ids[q, :10]] <= kth[q] + 1e-6).sum() / 10 for q in range(len(Q))])

    P = 20
    plain, _, _, _ = ctx.search(Q, K=10, P=P)
    seeds = ctx.router_seeds(Q, 3, out_ld=10)
    routed, _, cnt, _ = ctx.search(Q, K=10, P=P, init=3, init_ids=seeds)
    r_plain, r_router = recall(plain), recall(routed)
    assert r_router > r_plain and r_router >= 0.9, (r_plain, r_router)
    # the fused call: same seeds, same walk, same results
    fi, fd, fc, fk = ctx.router_search(Q, K=10, P=P, seeds=3)
    _, rd, _, rk = ctx.search(Q, K=10, P=P, init=3, init_ids=seeds)
    assert (fc == cnt).all() and (fk.view(np.uint32) == rk.view(np.uint32)).all()
    for q in range(len(Q)):
        c = int(cnt[q])
        assert (fi[q, :c] == routed[q, :c]).all()
        assert (fd[q, :c].view(np.uint32) == rd[q, :c].view(np.uint32)).all()
    with pytest.raises(capi.KGError, match="L < params.K"):
        ctx.router_search(Q, K=3, P=P, seeds=3)
    ctx.close()
