"""The N>1 path of bench.py on CPU: world_size-2 gloo ranks.  Search shards
by query (replicas, no collective on the data path); the only collective is
the max-over-ranks of the timed region, and the whole-job value counts every
rank's queries over the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    per_rank_ms = [100.0, 250.0][rank]     # rank 1 is the slow one
    value, slowest = bench.replica_throughput(per_rank_ms, 10_000, 5, dist, world, "cpu")
    X, Q = bench.make_data(n=1000, nq=8, rank=rank)
    q.put((rank, value, slowest, float(Q[0, 0]), float(X[0, 0])))
    dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    (r0, v0, s0, q0, x0), (r1, v1, s1, q1, x1) = res
    assert s0 == s1 == 250.0                       # max over ranks
    assert v0 == v1 == pytest.approx(10_000 * 2 * 5 / 0.25)
    assert x0 == x1                                # same dataset replica on every rank
    assert q0 != q1                                # each rank searches its own queries
