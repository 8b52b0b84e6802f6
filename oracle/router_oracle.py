"""FP64 restatement of the router MLP's training step -- TEST INFRASTRUCTURE ONLY.

The GPU trains the router with its own kernels (kgraph_b200/csrc/kg_router.cu);
this module is the independent implementation the tests compare their loss
and gradients with.  `rounding=True` applies the BF16 roundings the kernels
apply (weights, inputs, activations fed to the next GEMM, output gradients
fed to the backward GEMMs); `rounding=False` is the exact FP64 network, whose
gradients tests/test_router_oracle_cpu.py checks by finite differences.
"""
import numpy as np


def _bf16_exact(a):
    return np.asarray(a, np.float64)


def bf16(a):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def mlp_fp64(W, x, y, d, h, c, rounding=True):
    """Forward + backward of d -> h -> h -> c (ReLU, softmax CE, mean loss) in FP64,
    with the same BF16 roundings of weights, inputs, activations and output
    gradients the GPU kernels apply."""
    r = bf16 if rounding else _bf16_exact
    shapes = [(d, h), (h,), (h, h), (h,), (h, c), (c,)]
    ps, o = [], 0
    for s in shapes:
        n = int(np.prod(s))
        ps.append(W[o:o + n].reshape(s).astype(np.float64))
        o += n
    W1, b1, W2, b2, W3, b3 = ps
    W1b, W2b, W3b = r(W1), r(W2), r(W3)
    xb = r(x)
    B = x.shape[0]
    H1 = np.maximum(xb @ W1b + b1, 0)
    H1b = r(H1)
    H2 = np.maximum(H1b @ W2b + b2, 0)
    H2b = r(H2)
    Z = H2b @ W3b + b3
    Zs = Z - Z.max(1, keepdims=True)
    P = np.exp(Zs) / np.exp(Zs).sum(1, keepdims=True)
    loss = -np.log(P[np.arange(B), y]).mean()
    dZ = P.copy()
    dZ[np.arange(B), y] -= 1
    dZ /= B
    dZb = r(dZ)
    gW3 = H2b.T @ dZb
    gb3 = dZ.sum(0)
    dH2 = (dZb @ W3b.T) * (H2 > 0)
    dH2b = r(dH2)
    gW2 = H1b.T @ dH2b
    gb2 = dH2.sum(0)
    dH1 = (dH2b @ W2b.T) * (H1 > 0)
    dH1b = r(dH1)
    gW1 = xb.T @ dH1b
    gb1 = dH1.sum(0)
    return loss, [gW1, gb1, gW2, gb2, gW3, gb3]


