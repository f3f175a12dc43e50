"""Multi-rank path of bench.py on CPU: world-size-2 gloo replicas.

bench.py --gpus N runs N independent replicas (the path does not shard); the
only collectives are the start barrier and the max-over-ranks reduction of
the timed milliseconds, which job_rate performs.  These tests run that code
with the gloo backend in two processes, no GPU.
"""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w, _ = bench.rank_info()
        dist.barrier()
        value, ms_max = bench.job_rate(10.0 + 2.0 * r, 1000, 5, w, torch.device("cpu"))
        out[rank] = (r, w, value, ms_max)
    finally:
        dist.destroy_process_group()


def test_job_rate_is_the_slowest_replica_over_two_gloo_ranks():
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert set(res) == {0, 1}
    for rank, (r, w, value, ms_max) in res.items():
        assert r == rank and w == 2
        assert ms_max == 12.0  # rank 1 is the slower replica
        assert value == pytest.approx(1000 * 2 * 5 / 0.012)


def test_job_rate_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    value, ms_max = bench.job_rate(20.0, 1000, 4, 1, torch.device("cpu"))
    assert ms_max == 20.0 and value == pytest.approx(1000 * 4 / 0.02)
