"""The multi-GPU bench path on the host: replicas on two ranks (gloo on
CPU, 127.0.0.1), the whole-job aggregation (max time, summed rays) and the
reference arm, which only rank 0 runs."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [7.0, 9.5][rank]
        e2e = [8.0, 7.5][rank]
        rays = [1000, 3000][rank]
        e2e_rays = [10, 20][rank]
        out[rank] = bench.aggregate_ranks(dist, torch, ms, e2e, rays, e2e_rays, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_aggregate_over_two_gloo_ranks():
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    # every rank ends with the slowest time and the summed rays
    assert res[0] == res[1] == (9.5, 8.0, 4000, 30)


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun with N > 1, ranks other than 0 exit 0 without work and
    print nothing; the reference arm never needs a collective."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
