"""kg_search_batch_noalloc: the search entry point that allocates no device
memory, for callers that may not call cudaMalloc while serving (a thread
that must never block on the allocator, an application that owns all GPU
memory through its own pool).  Its scratch is a static device array of the
library.

Checked through the C-ABI against kg_search_batch on the same inputs, on two
calls in a row (the shared scratch keeps the previous call's contents, so the
second call proves the entry point clears what must start at zero).  The
results of both entry points are exact (bit-identical), so the tolerance is
zero.  The file is named to be collected last; it passes alone in a fresh
process (the first call then performs the one-time scratch address lookup)
and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden
from oracle import kgoracle as ko

pytestmark = pytest.mark.gpu


def _device_rows(torch, X, ld):
    t = torch.zeros((X.shape[0], ld), dtype=torch.float32, device="cuda")
    t[:, : X.shape[1]] = torch.as_tensor(X, device="cuda")
    return t


def _run_noalloc(torch, ctx, capi, qd, params, K):
    nq = qd.shape[0]
    ids = torch.zeros((nq, K), dtype=torch.int32, device="cuda")
    d = torch.zeros((nq, K), dtype=torch.float32, device="cuda")
    cnt = torch.zeros((nq,), dtype=torch.int32, device="cuda")
    cost = torch.zeros((nq,), dtype=torch.float32, device="cuda")
    ctx.search_noalloc(capi._ptr(qd), nq, qd.stride(0) * 4, params, K, capi._ptr(ids), capi._ptr(d), capi._ptr(cnt),
                       capi._ptr(cost))
    torch.cuda.synchronize()
    return (ids.cpu().numpy().view(np.uint32), d.cpu().numpy(), cnt.cpu().numpy().view(np.uint32),
            cost.cpu().numpy())


@pytest.mark.parametrize("name,K,P,T", [("u16", 10, 50, 1), ("mix32", 20, 60, 2), ("ang20", 8, 20, 1)])
def test_noalloc_matches_search_batch_twice(name, K, P, T):
    import torch
    from kgraph_b200 import capi
    g = load_golden(name)
    G = ko.read_index(g["index_bytes"])
    ctx = capi.Context(0)
    ctx.set_data(g["X"], g["metric"])
    ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    ref_i, ref_d, ref_c, ref_cost = ctx.search(g["Q"], K=K, P=P, T=T)
    ld = (g["X"].shape[1] + 15) // 16 * 16
    qd = _device_rows(torch, g["Q"], ld)
    params = capi.SearchParams(K, 0, P, 10, T, 1e30, 1998, 0)
    for _ in range(2):
        ids, d, cnt, cost = _run_noalloc(torch, ctx, capi, qd, params, K)
        assert (cnt == ref_c).all()
        assert (ids == ref_i).all()
        assert (d.view(np.uint32) == ref_d.view(np.uint32)).all()
        assert (cost == ref_cost).all()
    ctx.close()


def test_noalloc_bruteforce_without_graph_and_limits():
    import torch
    from kgraph_b200 import capi
    g = load_golden("l2sq24")
    ctx = capi.Context(0)
    ctx.set_data(g["X"], g["metric"])           # no graph: brute force
    ref_i, ref_d, ref_c, _ = ctx.search(g["Q"], K=10)
    qd = _device_rows(torch, g["Q"], 32)
    params = capi.SearchParams(10, 0, 100, 10, 1, 1e30, 1998, 0)
    for _ in range(2):
        ids, d, cnt, cost = _run_noalloc(torch, ctx, capi, qd, params, 10)
        assert (cnt == ref_c).all() and (ids == ref_i).all()
        assert (d.view(np.uint32) == ref_d.view(np.uint32)).all()
    assert capi.lib().kg_noalloc_scratch_bytes() == 64 << 20
    # host buffers and oversized requests are refused with a clear error
    G = ko.read_index(g["index_bytes"])
    ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    hi = np.zeros((qd.shape[0], 10), np.uint32)
    with pytest.raises(capi.KGError, match="device buffers"):
        ctx.search_noalloc(capi._ptr(qd), qd.shape[0], qd.stride(0) * 4, params, 10, hi.ctypes.data_as(C.c_void_p),
                           None, hi.ctypes.data_as(C.c_void_p), None)
    ctx.close()
    # a seed table beyond the stated maximum (P <= 4096) is refused
    rng = np.random.default_rng(3)
    n = 6000
    X = rng.random((n, 16), dtype=np.float32)
    off = np.arange(0, 10 * (n + 1), 10, dtype=np.uint64)
    nbr = rng.integers(0, n, 10 * n).astype(np.uint32)
    c2 = capi.Context(0)
    c2.set_data(X, "euclidean")
    c2.set_graph(off, nbr, None, np.full(n, 10, np.uint32))
    q = _device_rows(torch, X[:4], 16)
    ids = torch.zeros((4, 10), dtype=torch.int32, device="cuda")
    cnt = torch.zeros((4,), dtype=torch.int32, device="cuda")
    big = capi.SearchParams(10, 0, 4097, 10, 1, 1e30, 1998, 0)
    with pytest.raises(capi.KGError, match="P <= 4096"):
        c2.search_noalloc(capi._ptr(q), 4, 64, big, 10, capi._ptr(ids), None, capi._ptr(cnt), None)
    c2.close()


def test_noalloc_allocates_nothing_and_takes_init_seeds():
    """On a fresh context, before any kg_search_batch, the device's free memory
    is the same before and after two calls; then results (plain and with
    init > 0 starting points, which ride in the caller's ids buffer) equal
    kg_search_batch's."""
    import torch
    from kgraph_b200 import capi
    g = load_golden("u16")
    G = ko.read_index(g["index_bytes"])
    ctx = capi.Context(0)
    ctx.set_data(g["X"], g["metric"])
    ctx.set_graph(G.offsets, G.ids, G.dists, G.M)
    K, P, m = 10, 50, 5
    ld = (g["X"].shape[1] + 15) // 16 * 16
    qd = _device_rows(torch, g["Q"], ld)
    nq = qd.shape[0]
    ids = torch.zeros((nq, K), dtype=torch.int32, device="cuda")
    d = torch.zeros((nq, K), dtype=torch.float32, device="cuda")
    cnt = torch.zeros((nq,), dtype=torch.int32, device="cuda")
    cost = torch.zeros((nq,), dtype=torch.float32, device="cuda")
    params = capi.SearchParams(K, 0, P, 10, 1, 1e30, 1998, 0)

    def call(p):
        ctx.search_noalloc(capi._ptr(qd), nq, ld * 4, p, K, capi._ptr(ids), capi._ptr(d), capi._ptr(cnt),
                           capi._ptr(cost))

    call(params)   # first call: the context's address lookup and the kernel's first load
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        call(params)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    got = ids.cpu().numpy().view(np.uint32).copy(), d.cpu().numpy().copy(), cnt.cpu().numpy().view(np.uint32).copy()
    ref_i, ref_d, ref_c, _ = ctx.search(g["Q"], K=K, P=P)
    assert (got[2] == ref_c).all() and (got[0] == ref_i).all()
    assert (got[1].view(np.uint32) == ref_d.view(np.uint32)).all()
    # init > 0: starting points in the first m columns of the ids buffer
    init = np.random.default_rng(5).integers(0, g["X"].shape[0], (nq, m)).astype(np.uint32)
    ref_i, ref_d, ref_c, ref_cost = ctx.search(g["Q"], K=K, P=P, init=m, init_ids=init)
    params_i = capi.SearchParams(K, 0, P, 10, 1, 1e30, 1998, m)
    for _ in range(2):
        ids.zero_()
        ids[:, :m] = torch.as_tensor(init.view(np.int32), device="cuda")
        call(params_i)
        torch.cuda.synchronize()
        assert (cnt.cpu().numpy().view(np.uint32) == ref_c).all()
        assert (ids.cpu().numpy().view(np.uint32) == ref_i).all()
        assert (d.cpu().numpy().view(np.uint32) == ref_d.view(np.uint32)).all()
        assert (cost.cpu().numpy() == ref_cost).all()
    ctx.close()
