"""Multi-rank host logic of bench.py on CPU with the gloo backend
(world size 2): every target is owned by exactly one rank, and the reported
step time is the maximum and the check count the sum over ranks."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import workloads


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lo, hi = workloads.shard_bounds(n, rank, world)
    owned = torch.zeros(n, dtype=torch.int64)
    owned[lo:hi] = 1
    dist.all_reduce(owned)
    t = torch.tensor([float(10 + rank)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(hi - lo)], dtype=torch.float64)
    dist.all_reduce(c)
    if rank == 0:
        out.put((owned.tolist(), t.item(), c.item()))
    dist.barrier()
    dist.destroy_process_group()


def test_shards_cover_targets_once_gloo():
    world, n = 2, 1001
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    owned, tmax, count = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert owned == [1] * n
    assert tmax == 11.0 and count == float(n)


def test_shard_bounds_partition():
    for n in (0, 1, 7, 9818041):
        for world in (1, 2, 3, 8):
            bounds = [workloads.shard_bounds(n, r, world) for r in range(world)]
            assert bounds[0][0] == 0 and bounds[-1][1] == n
            assert all(bounds[i][1] == bounds[i + 1][0] for i in range(world - 1))
            sizes = np.diff([0] + [b[1] for b in bounds])
            assert sizes.max() - sizes.min() <= 1
