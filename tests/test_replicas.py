"""Host logic of bench.py's multi-GPU mode (independent replicas, one process
per GPU): ranks time their own replica, the job time is the slowest rank's,
and the whole-job value counts every rank's particle-steps.  Run here as two
gloo ranks on the CPU."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as tdist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms_local = 10.0 + 5.0 * rank               # rank 1 is the slower replica
        ms_max = bench.max_over_ranks(ms_local, tdist, torch.device("cpu"))
        value = bench.replica_value(1000, world, 4, ms_max)
        seeds = [None] * world
        tdist.all_gather_object(seeds, bench.replica_seed(rank))
        out[rank] = (ms_max, value, seeds)
    finally:
        tdist.destroy_process_group()


def test_replicas_time_is_slowest_rank_and_value_counts_all_ranks():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        ms_max, value, seeds = res[rank]
        assert ms_max == 15.0
        assert value == pytest.approx(1000 * 2 * 4 / 15e-3)
        assert len(set(seeds)) == world             # independent replicas


def test_single_rank_needs_no_collective():
    assert bench.max_over_ranks(12.5, None, None) == 12.5
    assert bench.replica_value(10, 1, 2, 1000.0) == pytest.approx(20.0)
