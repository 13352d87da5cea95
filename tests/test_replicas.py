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


def _shard_rank_main(rank, world, port, out):
    import torch.distributed as dist

    from varrcwa_b200 import replicas

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = replicas.rank_queue("c3", 512, rank, world, 16)
        cost = sum(replicas.cell_cost(d) for d in mine)
        seeds = [(d["nx"], d["lam"], d["r0"]) for d in mine]
        gathered = [None] * world
        dist.all_gather_object(gathered, (cost, seeds))
        out.put((rank, gathered))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_uneven_queue_by_cost():
    """Config-3 queue (truncations 7..15 per axis: per-cell costs differ by
    ~100x) sharded over two ranks: disjoint, complete, and each rank's cost
    within the LPT bound of the mean (mean + the largest cell)."""
    import torch.multiprocessing as mp

    from varrcwa_b200 import replicas

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    gathered = res[0]
    assert gathered == res[1]
    queue = replicas.make_queue("c3", 512, 16)
    costs = [replicas.cell_cost(d) for d in queue]
    mean = sum(costs) / 2
    all_cells = [c for (_, cells) in gathered for c in cells]
    assert sorted(all_cells) == sorted((d["nx"], d["lam"], d["r0"]) for d in queue)
    assert len(set(all_cells)) == len(all_cells)
    for cost, _ in gathered:
        assert cost <= mean + max(costs)
    assert max(c for c, _ in gathered) / mean < 1.001
    # dealing by position instead would leave the ranks' costs far apart
    rr = [sum(costs[i] for i in range(r, len(costs), 2)) for r in range(2)]
    assert max(rr) / mean > max(c for c, _ in gathered) / mean
