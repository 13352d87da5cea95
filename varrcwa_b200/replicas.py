"""Multi-GPU form of the batched solve: independent replicas.

Cells are independent solves, so N GPUs run N replicas, one process per GPU,
each on its own disjoint set of seeded cells; nothing is exchanged on the
data path.  The only collective is the max over ranks of the per-rank device
and wall times, so that the job's throughput is the cells of all ranks over
the slowest rank's time.
"""
from __future__ import annotations

from typing import List, Sequence

RANK_STRIDE = 100000  # seeds of rank r start at base + r * RANK_STRIDE


def cell_seeds(workload: str, batch: int, rank: int, step_seed: int = 0) -> List[int]:
    """Seeds of this rank's cells: seed = 1000 * config + instance, offset by
    rank so that replicas never solve the same cell."""
    if batch > RANK_STRIDE:
        raise ValueError("batch per rank exceeds the seed stride")
    base = 1000 * {"c1": 1, "c2": 2, "c3": 3, "c4": 4, "c5": 5}[workload] + RANK_STRIDE * rank + step_seed
    return [base + i for i in range(batch)]


def make_cells(workload: str, batch: int, rank: int, npix: int, step_seed: int = 0, orders: int = 9):
    import numpy as np

    from . import structures as st
    seeds = cell_seeds(workload, batch, rank, step_seed)
    if workload == "c1":  # the config-1 taper at seeded wavelengths around 1.55 um
        return [st.taper_2d(lam=float(np.random.default_rng(s).uniform(1.50, 1.60))) for s in seeds]
    if workload == "c2":
        return [st.pillar_config2(seed=s, npix=npix) for s in seeds]
    if workload == "c4":  # freeform metagrating stacks (npix is the 256 raster of c2/c3; c4 keeps 64x64)
        return [st.metagrating_c4(seed=s, norders=orders) for s in seeds]
    if workload == "c5":  # PML mode converters (orders: harmonics per axis, 21 = config 5)
        return [st.converter_c5(s, norders=orders) for s in seeds]
    return [st.pillar_config3(seed=s, npix=npix) for s in seeds]


def cell_cost(desc: dict) -> float:
    """Relative cost of one solve: n^3 (eigensolver and GEMMs per sample)
    times the expected number of segments, which grows with the structure's
    length in wavelengths (a pillar cell's 600 nm at ~550 nm is about one)."""
    n = 2 * int(desc["nx"]) * int(desc["ny"])
    if "layers" in desc:  # z-uniform stacks: one eigen-solve per layer
        return float(n) ** 3 * len(desc["layers"])
    length = abs(float(desc.get("z1", 0.0)) - float(desc.get("z0", 0.0)))
    return float(n) ** 3 * max(1.0, length / float(desc["lam"]))


def shard_by_cost(costs: Sequence[float], world: int) -> List[List[int]]:
    """Partition cell indices over `world` ranks so that the per-rank cost
    sums are balanced: longest first onto the least loaded rank (Graham's
    LPT rule, whose makespan is within 4/3 of the optimum).  Each rank's
    indices come back in queue order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        shards[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in shards]


def make_queue(workload: str, total: int, npix: int, orders: int = 9):
    """The job's whole cell queue (seeds independent of the rank count)."""
    return make_cells(workload, total, 0, npix, 0, orders)


def rank_queue(workload: str, total: int, rank: int, world: int, npix: int, orders: int = 9):
    """This rank's cost-balanced share of the job queue."""
    q = make_queue(workload, total, npix, orders)
    return [q[i] for i in shard_by_cost([cell_cost(d) for d in q], world)[rank]]


def max_over_ranks(values: Sequence[float], device=None) -> List[float]:
    """Elementwise max of per-rank values over the default process group
    (identity without one).  device: where the reduction tensor lives (a CUDA
    device for NCCL, None for gloo on the CPU)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def job_throughput(cells_per_rank: int, steps: int, world: int, seconds: float) -> float:
    """Whole-job throughput: all ranks' cells over the (max-over-ranks) time."""
    return cells_per_rank * world * steps / seconds
