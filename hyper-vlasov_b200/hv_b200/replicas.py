"""Host-side logic of multi-GPU runs: one process per GPU, replicas only.

A single run of the step fits one B200 many times over and sharding its
particles would need an all-reduce of the 2G density grid every step, so the
path does not shard: N GPUs run N independent replicas (or, for a batch of
independent runs, disjoint subsets of the batch).  The only cross-rank
traffic is a barrier and a max over ranks of the timed region, plus, for a
batch, gathering the per-run D(t) series at the end.
"""
from __future__ import annotations

import heapq
import os
from dataclasses import dataclass


@dataclass
class RankInfo:
    world: int
    rank: int
    local: int


def rank_info() -> RankInfo:
    return RankInfo(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                    int(os.environ.get("LOCAL_RANK", "0")))


def run_cost(particles: int, grid_nodes: int, sor_iterations: float = 500.0) -> float:
    """Relative cost of one step: 48 B per particle plus 4 G (24 + 3 n_sor) B
    of grid traffic (the algorithmic bytes of the step)."""
    return 48.0 * particles + 4.0 * grid_nodes * (24.0 + 3.0 * sor_iterations)


def assign_runs(costs, world: int):
    """Longest-processing-time-first assignment of independent runs to ranks:
    runs sorted by decreasing cost, each given to the least-loaded rank (ties
    to the lowest rank).  Returns a list of run indices per rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for r in range(world):
        out[r].sort()
    return out


def max_over_ranks(value: float, world: int) -> float:
    """Max of a per-rank float over the default process group (any backend)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_series(series, world: int):
    """All ranks' per-run series (lists of floats keyed by run index) merged
    into one dict on every rank."""
    if world <= 1:
        return dict(series)
    import torch.distributed as dist
    objs = [None] * world
    dist.all_gather_object(objs, dict(series))
    merged = {}
    for o in objs:
        merged.update(o)
    return merged
