"""Multi-process (gloo, world size 2, CPU) checks of the replica plumbing used by
bench.py --gpus N: barrier, max / sum reductions, whole-job throughput, per-rank seeds and
the set partition of ensembles."""
import os
import socket

import numpy as np
import pytest

from gpudelaunaytriangulation_b200.replicas import ReplicaGroup, replica_seed, shard_sets
from gpudelaunaytriangulation_b200 import workloads as W

torch = pytest.importorskip("torch")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    g = ReplicaGroup(world, rank, "cpu")
    g.barrier()
    ms = 10.0 + rank * 5.0
    value, mx = g.throughput(1000 * (rank + 1), ms)
    sizes = W.ensemble_sizes(37, 1000, 65536, seed=7)
    mine = shard_sets(sizes, world, rank).tolist()
    out.put((rank, value, mx, replica_seed(2026, rank), mine))
    g.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_replicas():
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, v0, m0, s0, sets0), (r1, v1, m1, s1, sets1) = res
    assert m0 == m1 == 15.0                      # max over ranks
    assert abs(v0 - 3000 / 0.015 / 1e6) < 1e-9 and v0 == v1   # all points / slowest rank
    assert s0 != s1
    assert sorted(sets0 + sets1) == list(range(37)) and not set(sets0) & set(sets1)


def test_shard_balance_single_process():
    sizes = W.ensemble_sizes(256, 1000, 65536, seed=7)
    loads = [int(sizes[shard_sets(sizes, 8, r)].sum()) for r in range(8)]
    assert sum(loads) == int(sizes.sum())
    assert max(loads) - min(loads) <= int(sizes.max())
