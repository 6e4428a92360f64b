"""Multi-process replica path of bench.py (one independent greedy per rank, no collective
on the data path): rank seeds and the max-over-ranks job time, with world size 2 over gloo
on CPU."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seed = bench.replica_seed(1, rank)
        local = 1.0 + rank * 0.5  # per-rank device seconds
        t = bench.job_seconds(local, world, "cpu")
        out[rank] = (seed, t)
    finally:
        dist.destroy_process_group()


def test_replicas_two_ranks_gloo():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True)
    seeds = {out[r][0] for r in range(2)}
    assert seeds == {1, 1001}
    assert out[0][1] == out[1][1] == pytest.approx(1.5)


def test_job_seconds_single_rank():
    import bench
    assert bench.job_seconds(2.5, 1, "cpu") == 2.5
