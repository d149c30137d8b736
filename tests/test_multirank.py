"""Multi-rank host logic of bench.py on CPU with the gloo backend
(world size 2): every target is owned by exactly one rank, and the reported
step time is the maximum and the check count the sum over ranks.  On a GPU:
two shards of an enumeration give together the rules of the whole."""
import os
import socket

import numpy as np
import pytest
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


@pytest.mark.gpu
def test_range_shards_union_equals_whole(tmp_path):
    """Sharding the enumeration by first instruction (the reference's
    --first-op-start/--first-op-end split across processes or GPUs,
    README.md:216-221): two ranks, run as two concurrent z80opt processes on
    the same device, each search its shard_bounds part of [1000, 1040); the
    union of their rule sets equals the rule set of one process over the
    whole range."""
    import json
    import subprocess

    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "z80-optimizer_b200", "_build",
                       "z80opt")
    lo, hi, world = 1000, 1040, 2

    def cmd(a, b, out):
        return [exe, "enumerate", "--max-target", "2", "--first-op-start", str(a), "--first-op-end", str(b),
                "--output", str(out)]

    procs, outs = [], []
    for rank in range(world):
        a, b = workloads.shard_bounds(hi - lo, rank, world)
        out = tmp_path / f"shard{rank}.json"
        outs.append(out)
        procs.append(subprocess.Popen(cmd(lo + a, lo + b, out), stdout=subprocess.DEVNULL, stderr=subprocess.PIPE))
    for p in procs:
        assert p.wait(timeout=600) == 0, p.stderr.read()
    whole = tmp_path / "whole.json"
    assert subprocess.run(cmd(lo, hi, whole), capture_output=True, timeout=600).returncode == 0
    key = lambda x: (x["source_asm"], x["replacement_asm"], x["bytes_saved"], x["cycles_saved"])  # noqa: E731
    union = sorted(key(x) for o in outs for x in json.load(open(o)))
    assert union == sorted(key(x) for x in json.load(open(whole)))
    assert len(union) > 100
