"""The N>1 path of bench.py on CPU: two gloo ranks, each timing its own
replica, reduce to the slowest rank's time and the whole-job value; the
reference arm's non-zero ranks exit without work."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 100.0 + 50.0 * rank          # each replica's own device time
        mx = bench.max_over_ranks(ms, dist)
        value = bench.aggregate_value(1000000, 3, mx, world)
        ws, r, local = bench._dist()
        out[rank] = (mx, value, ws, r, local)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    for rank in range(world):
        mx, value, ws, r, local = out[rank]
        assert mx == 150.0                 # max over ranks, on every rank
        assert value == pytest.approx(2 * 1e6 * 3 / 0.150 / 1e6)
        assert (ws, r, local) == (world, rank, rank)


def test_reference_arm_nonzero_rank_exits_without_work(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")

    class Args:
        steps, warmup, gpus = 1, 0, 2

    called = []
    monkeypatch.setattr(bench, "_oracle_state", lambda *a, **k: called.append(1))
    assert bench.run_reference(Args(), bench.CONFIGS["c1"]) == 0
    assert not called


def _partition_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import mobydiff_b200 as M
        sizes = [m.nx * m.ny * m.nz for m in bench.ensemble_members(M, 64)]
        parts, loads = bench.partition_members(sizes, world)
        mine = parts[rank]
        # every rank computed the split on its own; gather what each took
        got = [None] * world
        dist.all_gather_object(got, mine)
        # each rank's own "result": its cell count, reduced to the whole job
        t = torch.tensor([float(sum(sizes[q] for q in mine))], dtype=torch.float64)
        dist.all_reduce(t)
        ms = bench.max_over_ranks(10.0 + rank, dist)
        out[rank] = (got, loads, float(t.item()), sum(sizes), ms, sizes)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ensemble_partition_over_gloo_ranks(world):
    """The C4 ensemble split by cell count: every rank derives the same split,
    the parts are disjoint and cover all 64 members, the cell loads differ by
    at most one member's cells, and the per-rank cell counts sum to the
    whole ensemble."""
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_partition_main, args=(world, _free_port(), out), nprocs=world, join=True)
    got0 = out[0][0]
    for rank in range(world):
        got, loads, total, cells, ms, sizes = out[rank]
        assert got == got0
        assert total == cells
        assert ms == 10.0 + world - 1
    flat = sorted(q for p in got0 for q in p)
    assert flat == list(range(64))
    assert max(loads) - min(loads) <= max(sizes)
    for rank, p in enumerate(got0):
        assert sum(sizes[q] for q in p) == loads[rank]
