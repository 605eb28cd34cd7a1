"""Replica runs of the bench (one process per GPU, no data exchange inside a
solve): the job's times are the maximum over the ranks. Two gloo ranks on the
CPU check the reduction bench.py applies after its timed region."""
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


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        # rank r timed (1 + r) s of device time and 10 - r s of wall time
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5], world, dist, torch, "cpu")
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_times_are_the_maximum_over_two_ranks():
    world = 2
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        results = dict(out)
    assert results[0] == results[1] == [2.0, 10.0, 0.5]


def test_single_rank_is_the_identity():
    assert bench.max_over_ranks([3.0, 4.0], 1, None, torch, "cpu") == [3.0, 4.0]
