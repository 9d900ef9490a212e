"""The bench's multi-GPU (replica) host logic on two CPU ranks with the gloo backend: every rank
gets the maximum of the per-rank step times, as the JSON line's timing requires, and a rank
that runs alone keeps its own value."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 + 7.5 * rank
        out[rank] = bench.max_over_ranks(ms, dist, device="cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        assert dict(out) == {0: 107.5, 1: 107.5}


def test_single_process_keeps_its_value():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(12.25, None) == 12.25
