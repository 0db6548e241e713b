"""Multi-GPU is replicas only: the bench's rank helpers (max/sum over ranks, per-rank id
ranges) checked with two gloo ranks on the CPU."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    mx = bench.max_over_ranks(dist, 10.0 * (rank + 1))
    sm = bench.sum_over_ranks(dist, rank + 1)
    first, count = bench.replica_range(rank, 1000)
    bench.barrier(dist)
    out.put((rank, mx, sm, first, count))
    dist.destroy_process_group()


def test_rank_helpers_with_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in results] == [20.0, 20.0]       # max over ranks
    assert [r[2] for r in results] == [3.0, 3.0]         # sum over ranks
    (r0, _, _, f0, c0), (r1, _, _, f1, c1) = results
    assert (f0, c0, f1, c1) == (0, 1000, 1000, 1000)     # disjoint, contiguous id ranges
