"""The multi-GPU replica path of bench.py on CPU: two gloo ranks (as
torchrun would start them) reduce their per-rank timings with the same
max-over-ranks step the GPU ranks use, and the environment parsing that
picks rank and local device."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    try:
        w, r, lr = bench.dist_env()
        assert (w, r, lr) == (world, rank, rank)
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 5.0], dist, "cpu")
        dist.barrier()
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_two_rank_max_over_ranks():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:  # no fork of this multi-threaded process
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == [2.0, 10.0, 5.0]


def test_single_process_is_identity(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench.dist_env() == (1, 0, 0)
    assert bench.max_over_ranks([3.0, 4.0], None, "cpu") == [3.0, 4.0]


def test_reference_arm_runs_on_rank_zero_only(capsys):
    class Args:
        gpus, steps, warmup = 2, 1, 0
    bench.run_reference(Args(), 2, 1)  # rank 1 returns without work
    assert capsys.readouterr().out == ""
