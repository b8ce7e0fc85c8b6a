"""CPU, two ranks over gloo: the multi-GPU host logic (replicas only).

Each rank takes its share of a batch of independent runs (LPT by cost), the
timing reduction is a max over ranks, and the per-run series are gathered on
every rank -- the same calls bench.py makes under torchrun, with gloo standing
in for NCCL."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from hv_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, costs, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        info = replicas.rank_info()
        mine = replicas.assign_runs(costs, info.world)[info.rank]
        # each rank "runs" its runs: the series is a deterministic function of the run
        series = {i: [float(i), float(i) * 0.5] for i in mine}
        t = replicas.max_over_ranks(1.0 + rank, info.world)
        merged = replicas.gather_series(series, info.world)
        dist.barrier()
        q.put((rank, mine, t, sorted(merged)))
    finally:
        dist.destroy_process_group()


def test_two_rank_batch_partition_timing_and_gather():
    costs = [replicas.run_cost(p, g) for p, g in
             [(4000, 32 ** 3), (104000, 64 ** 3), (8000, 48 ** 3), (30000, 96 ** 3), (16000, 32 ** 3),
              (200000, 96 ** 3), (3200, 32 ** 3), (50000, 64 ** 3), (9000, 40 ** 3)]]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    parts = [r[1] for r in res]
    assert sorted(parts[0] + parts[1]) == list(range(len(costs)))
    assert not set(parts[0]) & set(parts[1])
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= sum(costs) / world + max(costs)  # LPT bound
    assert all(r[2] == 2.0 for r in res)  # max over ranks
    assert all(r[3] == list(range(len(costs))) for r in res)


@pytest.mark.parametrize("world", [1, 3, 8])
def test_assignment_covers_every_run_once(world):
    costs = [float((7 * i) % 11 + 1) for i in range(20)]
    parts = replicas.assign_runs(costs, world)
    assert sorted(sum(parts, [])) == list(range(20))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
