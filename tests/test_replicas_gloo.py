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


def _batch_runs():
    """Small instances of the batched workload (grids up to 48^3, 20 test
    particles per nucleon) for CPU ranks."""
    from dataclasses import replace

    from hv_b200.workloads import batch_workloads
    return [replace(w, ppn=20) for w in batch_workloads(64, seed=0) if w.n <= 48][:6]


def _oracle_dipole(w, steps):
    """D(t) of one run from the C oracle (the CPU stand-in for a rank's device
    compute), from the seeded inputs the library's generator gives."""
    import numpy as np

    from hv_oracle import Oracle, RunSpec, workload_inputs
    o = Oracle(np.float64)
    o.set_threads(1)
    A, B, C, gm = w.skyrme()
    run = RunSpec(z=w.Z, n=w.N, part_per_nucleon=w.ppn, sigma_r=w.sigma_r, dt=w.dt, t_exc=w.t_exc, eta_exc=w.eta,
                  A=A, B=B, C=C, gamma=gm, sor_omega=w.sor_omega, sor_tol=w.sor_tol,
                  sor_criterion=w.sor_criterion, sor_max_iter=w.sor_max_iter)
    parts = workload_inputs(o.lib, w, np.float64)
    obs, _ = o.simulate(w.world_tuple(), run, w.protons, w.neutrons, *parts, steps)
    return [float(v) for v in obs["dipole"]]


def _batch_worker(rank, world, port, steps, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        runs = _batch_runs()
        mine = replicas.assign_runs([replicas.run_cost(w.particles, w.G) for w in runs], world)[rank]
        series = {i: _oracle_dipole(runs[i], steps) for i in mine}
        merged = replicas.gather_series(series, world)
        q.put((rank, mine, merged))
    finally:
        dist.destroy_process_group()


def test_two_ranks_share_a_batch_and_gather_its_dipole_series():
    """Two gloo ranks take their LPT shares of six instances of the batched
    workload, compute each run's D(t) (the C oracle standing in for the
    device), and gather the series: every rank ends with all six, equal bit
    for bit to one process computing them all."""
    steps = 3
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, world, port, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(world)], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    runs = _batch_runs()
    assert sorted(res[0][1] + res[1][1]) == list(range(len(runs)))
    single = {i: _oracle_dipole(w, steps) for i, w in enumerate(runs)}
    for _, _, merged in res:
        assert sorted(merged) == list(range(len(runs)))
        assert all(merged[i] == single[i] for i in single)
