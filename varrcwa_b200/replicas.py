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
    base = 1000 * {"c1": 1, "c2": 2, "c3": 3, "c4": 4}[workload] + RANK_STRIDE * rank + step_seed
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
    return [st.pillar_config3(seed=s, npix=npix) for s in seeds]


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
