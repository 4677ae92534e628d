"""The replica path of bench.py on two CPU ranks (gloo): each rank times its own
graph, the job's time is the max over ranks, and the reference arm runs on rank 0
only."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_env() == (ws, rank, rank)
        barrier, max_over_ranks = bench.collectives(ws, "cpu")
        barrier()
        out[rank] = max_over_ranks(0.25 + rank)
        barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_ranks():
    ws, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(ws, port, out), nprocs=ws, join=True)
    assert dict(out) == {0: 1.25, 1: 1.25}


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    barrier, max_over_ranks = bench.collectives(1, "cpu")
    barrier()
    assert max_over_ranks(3.5) == 3.5


def test_reference_arm_on_non_zero_rank_prints_nothing():
    env = {**os.environ, "RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2"], capture_output=True, text=True, timeout=300, env=env,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
