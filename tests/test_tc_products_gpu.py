"""The router's tensor-core products at the shapes the router trains on.

tcgen05 BF16 x BF16 -> FP32 GEMM (kg_gemm.cu tc_gemm_kernel) and the fused
k-means assignment (tc_assign_kernel), called through their C-ABI check entry
points and compared with an FP64 evaluation of the same BF16 operands.  The
shapes are the MLP's (4096-row batches, 128 -> 256 -> 256 -> 1024) forward
and backward products, K that is not a multiple of the 64-wide K chunk, M and N
that are not multiples of the 128-wide tile, products split along K, both the
TMA-fed path (16-byte aligned row pitches) and the register-staged fallback,
and the assignment of 10k rows to 8,192 centroids at D = 128 and D = 96.

Tolerance: products of BF16 values are exact in FP32; the K-long FP32
accumulation is bounded by K * 2^-22 * sum_k |a_k b_k| (twice the unit
roundoff, allowing truncating adds), written per element below.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def to_bf16(x):
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)


def from_bf16(u):
    return (np.asarray(u, np.uint16).astype(np.uint32) << 16).view(np.float32)


def _mm64(a, b):
    import torch
    if torch.cuda.is_available():
        ta = torch.as_tensor(a, dtype=torch.float64, device="cuda")
        tb = torch.as_tensor(b, dtype=torch.float64, device="cuda")
        return (ta @ tb).cpu().numpy()
    return a.astype(np.float64) @ b.astype(np.float64)


def _check_gemm(ctx, M, N, K, ta, tb, seed, bias=False, relu=False, beta=0.0):
    rng = np.random.default_rng(seed)
    A = to_bf16(rng.standard_normal((K, M) if ta else (M, K)))
    B = to_bf16(rng.standard_normal((N, K) if tb else (K, N)))
    a = from_bf16(A).astype(np.float64)
    b = from_bf16(B).astype(np.float64)
    opa = a.T if ta else a
    opb = b.T if tb else b
    bv = rng.standard_normal(N).astype(np.float32) if bias else None
    C0 = rng.standard_normal((M, N)).astype(np.float32) if beta else None
    got = ctx.tc_gemm_check(A, B, ta=ta, tb=tb, bias=bv, relu=relu, beta=beta, C_in=C0)
    ref = _mm64(opa, opb)
    mag = _mm64(np.abs(opa), np.abs(opb))
    if beta:
        ref = ref + beta * C0
        mag = mag + abs(beta) * np.abs(C0)
    if bias:
        ref = ref + bv
        mag = mag + np.abs(bv)
    if relu:
        ref = np.maximum(ref, 0)
    tol = (K + 4) * 2.0 ** -22 * mag + 1e-30
    err = np.abs(got - ref)
    assert (err <= tol).all(), (M, N, K, ta, tb, float((err / tol).max()))
    return float((err / np.maximum(mag, 1e-30)).max())


@pytest.mark.parametrize("M,N,K,ta,tb,extra", [
    (4096, 256, 128, False, False, dict(bias=True, relu=True)),      # layer 1 forward
    (4096, 256, 256, False, False, dict(bias=True, relu=True)),      # layer 2 forward
    (4096, 1024, 256, False, False, dict(bias=True)),                # logits
    (256, 1024, 4096, True, False, {}),                              # dW3 = H^T dY
    (4096, 256, 1024, False, True, {}),                              # dH = dY W3^T
    (128, 256, 4096, True, False, {}),                               # dW1 = X^T dH1
    (256, 256, 4096, True, False, {}),                               # dW2 = H1^T dH2 (split along K)
    (4096, 256, 256, False, True, {}),                               # dH1 = dH2 W2^T
    # TMA path (16-byte aligned pitches) at ragged shapes: partial tiles, K not a multiple of 64, splits
    (1000, 200, 104, False, False, dict(beta=0.5, bias=True)),
    (136, 264, 72, True, True, dict(relu=True)),
    (200, 136, 4000, True, True, dict(bias=True)),
    (72, 1000, 3000, True, False, dict(beta=-1.0)),
    (300, 40, 8, False, True, {}),
    # register-staged fallback (pitches that TMA cannot address)
    (1000, 200, 100, False, False, dict(beta=0.5, bias=True)),       # ragged M, N; K not a multiple of 64
    (130, 257, 65, True, True, dict(relu=True)),                     # ragged, both transposed
    (1, 1, 1, False, False, {}),
])
def test_tc_gemm_matches_fp64(gpu_ctx, M, N, K, ta, tb, extra):
    _check_gemm(gpu_ctx, M, N, K, ta, tb, seed=M * 7 + N * 3 + K, **extra)


@pytest.mark.parametrize("n,C,D", [(10_000, 8192, 128), (10_000, 8192, 96), (3000, 1000, 100), (129, 1, 16),
                                   (5000, 300, 64), (1000, 129, 256), (777, 4100, 40)])
def test_tc_assign_matches_fp64_argmin(gpu_ctx, n, C, D):
    rng = np.random.default_rng(n + C + D)
    cent_f = rng.standard_normal((C, D)).astype(np.float32)
    lab_true = rng.integers(0, C, n)
    F = to_bf16(cent_f[lab_true] + 0.7 * rng.standard_normal((n, D)))
    cent = to_bf16(cent_f)
    f = from_bf16(F).astype(np.float64)
    c = from_bf16(cent).astype(np.float64)
    cn = (c * c).sum(1).astype(np.float32)
    lab, best = gpu_ctx.tc_assign_check(F, cent, cn)
    assert lab.min() >= 0 and lab.max() < C
    fnorm = np.sqrt((f * f).sum(1))
    cmax = np.sqrt((c * c).sum(1)).max()
    worst = 0.0
    for a in range(0, n, 2000):
        val = cn[None, :].astype(np.float64) - 2.0 * _mm64(f[a:a + 2000], c.T)
        opt = val.min(1)
        chosen = val[np.arange(val.shape[0]), lab[a:a + 2000]]
        # two FP32 dot products of length D, each within D * 2^-22 * ||f|| ||c||, plus cn's own rounding
        tol = 4.0 * (D + 4) * 2.0 ** -22 * fnorm[a:a + 2000] * cmax + 2.0 ** -20 * np.abs(cn).max()
        assert (chosen - opt <= tol).all(), float(((chosen - opt) / tol).max())
        assert (np.abs(best[a:a + 2000] - chosen) <= tol).all()
        worst = max(worst, float(((chosen - opt) / tol).max()))
    # the assignment is exact for all but near-ties: at most 0.1% of rows off the FP64 argmin
    exact = 0
    for a in range(0, n, 2000):
        val = cn[None, :].astype(np.float64) - 2.0 * _mm64(f[a:a + 2000], c.T)
        exact += int((val.argmin(1) == lab[a:a + 2000]).sum())
    assert exact >= n - max(1, n // 1000), (exact, n)
