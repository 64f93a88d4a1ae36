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
    monkeypatch.setattr(bench, "_oracle_sample", lambda *a, **k: called.append(1))
    assert bench.run_reference(Args(), bench.CONFIGS["c1"]) == 0
    assert not called
