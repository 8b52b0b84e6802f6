"""The search filter's lower bound, restated on the CPU in FP64 and checked
against the oracle's canonical FP32 distance.

This checks the derivation behind kg_search.cu's filter_lb -- the
reconstruction error e >= ||x - y||, the rounding allowance of the
approximate sum (gamma_{ld+8}) and of the canonical distance
(gamma_{d/16+24}) -- independently of the kernel: for rows reconstructed
from BF16 and from FP8 E4M3 with a per-row scale, the bound never exceeds
the canonical distance.  (The kernel's own arithmetic is checked on the GPU
by test_search_filter_gpu.py.)
"""
import numpy as np
import pytest

from oracle import kgoracle as ko

U = 2.0 ** -24


def bf16(x):
    """Round-to-nearest-even to BF16, back in float32."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return b.astype(np.uint32).view(np.float32)


def e4m3(v):
    """Round-to-nearest-even to FP8 E4M3 with saturation at 448 (float64 in, float64 out)."""
    a = np.abs(v)
    e = np.floor(np.log2(np.maximum(a, 2.0 ** -20)))
    e = np.maximum(e, -6)                 # subnormals: quantum 2^-9
    q = 2.0 ** (e - 3)
    r = np.round(a / q) * q               # numpy rounds halves to even
    return np.sign(v) * np.minimum(r, 448.0)


def reconstruct(x, prec):
    if prec == "bf16":
        return bf16(x)
    scale = np.float32(np.max(np.abs(x)) / np.float32(448.0)) if np.any(x) else np.float32(1.0)
    q = e4m3(x.astype(np.float64) / np.float64(scale))
    return (q.astype(np.float32) * scale).astype(np.float32)


def lower_bound(metric, raw, e, nq, nx, d, ld):
    """filter_lb in FP64 (kg_search.cu)."""
    ga = (ld + 8) * U * 1.01
    gc = (d // 16 + 24) * U * 1.01
    if metric == "angular":
        qn, xn = nq * (1 + 2 * gc), nx * (1 + 2 * gc)
        B = qn * (e + ga * (xn + e) + gc * xn)
        den = np.float32(np.float32(nx) * np.float32(nq) + np.float32(np.finfo(np.float32).eps))
        return (-raw - B) / float(den)
    r = np.sqrt(max(raw * (1 - ga), 0.0))
    t2 = max(r - e, 0.0) ** 2
    if metric == "l2sqr":
        return t2 * (1 - 2 * gc)
    return 0.5 * t2 - 2.2 * gc * (nq + nx)


def dataset(kind, n, d, rng):
    if kind == "mixture":
        c = rng.uniform(0, 128, (8, d))
        return np.round(np.maximum(c[rng.integers(0, 8, n)] + rng.normal(0, 20, (n, d)), 0)).astype(np.float32)
    if kind == "sphere":
        x = rng.standard_normal((n, d)).astype(np.float32)
        return x / np.linalg.norm(x, axis=1, keepdims=True)
    if kind == "near":
        base = rng.standard_normal((4, d)).astype(np.float32) * 10
        return (base[rng.integers(0, 4, n)] + rng.standard_normal((n, d)).astype(np.float32) * 0.01).astype(np.float32)
    return rng.random((n, d), dtype=np.float32)


@pytest.mark.parametrize("kind,d,metric", [("mixture", 128, "euclidean"), ("sphere", 96, "angular"),
                                            ("uniform", 20, "l2sqr"), ("near", 48, "euclidean"),
                                            ("uniform", 33, "angular"), ("near", 16, "l2sqr")])
@pytest.mark.parametrize("prec", ["bf16", "fp8"])
def test_bound_is_below_the_canonical_distance(kind, d, metric, prec):
    rng = np.random.default_rng(d * 7 + len(kind))
    n = 300
    X = dataset(kind, n, d, rng)
    o = ko.Oracle(X, metric)
    ld = (d + 15) // 16 * 16
    Y = np.stack([reconstruct(X[j], prec) for j in range(n)])
    err = np.sqrt(((X.astype(np.float64) - Y.astype(np.float64)) ** 2).sum(1))
    err = np.nextafter(err.astype(np.float32), np.float32(np.inf))   # rounded up, as the copy stores it
    slack = []
    for _ in range(2000):
        i, j = rng.integers(0, n, 2)
        q, y = X[i], Y[j]
        if metric == "angular":
            raw = float(np.sum((q * y).astype(np.float32), dtype=np.float32))
        else:
            df = (q - y).astype(np.float32)
            raw = float(np.sum((df * df).astype(np.float32), dtype=np.float32))
        lb = lower_bound(metric, raw, float(err[j]), float(o.norms[i]), float(o.norms[j]), d, ld)
        dist = float(o.pair(i, j))
        assert lb <= dist, (i, j, lb, dist)
        slack.append(dist - lb)
    # the bound is not vacuous: for BF16 its slack is small against the spread of distances
    if prec == "bf16" and kind != "near":
        dists = [float(o.pair(i, j)) for i, j in rng.integers(0, n, (500, 2))]
        assert np.median(slack) < 0.5 * (np.percentile(dists, 90) - np.percentile(dists, 10))
