"""Multi-GPU form of the batched solve (independent replicas), checked with
two gloo ranks on the CPU: the ranks' cell sets are disjoint, the timing
reduction is the max over ranks, and the job throughput counts every rank's
cells."""
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

    from varrcwa_b200 import replicas

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = replicas.cell_seeds("c2", 64, rank)
        gathered = [None] * world
        dist.all_gather_object(gathered, seeds)
        # per-rank "device" and wall times; rank 1 is the slow one in both
        dev_ms, wall = replicas.max_over_ranks([100.0 + 50.0 * rank, 2.0 + rank])
        cells = replicas.make_cells("c2", 2, rank, 16)
        out.put((rank, gathered, dev_ms, wall, [c["seed"] if "seed" in c else None for c in cells]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_disjoint_cells_and_max_timing():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, dev_ms, wall, _ in res:
        s0, s1 = set(gathered[0]), set(gathered[1])
        assert len(s0) == 64 and len(s1) == 64 and not (s0 & s1)
        assert dev_ms == 150.0 and wall == 3.0  # max over ranks, seen by every rank
    from varrcwa_b200.replicas import job_throughput
    assert job_throughput(64, 3, 2, 3.0) == pytest.approx(128.0)


def test_single_process_reduction_is_identity():
    from varrcwa_b200 import replicas

    assert replicas.max_over_ranks([1.0, 2.5]) == [1.0, 2.5]
    with pytest.raises(ValueError):
        replicas.cell_seeds("c2", replicas.RANK_STRIDE + 1, 0)
