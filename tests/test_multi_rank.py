"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (127.0.0.1),
every rank computes its own replica's time and the job reports the maximum
over ranks, as the GPU run does over NCCL with one table per rank."""
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
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = [3.5, 7.25][rank]
        out[rank] = bench.max_over_ranks(local, dist, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        assert out[0] == out[1] == 7.25


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(4.0, None, "cpu") == 4.0


def test_reference_arm_only_rank0_prints():
    """Under torchrun the reference arm runs on rank 0 alone; other ranks exit
    0 without work."""
    import json
    import subprocess

    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip() == ""
    env = dict(os.environ, RANK="0", WORLD_SIZE="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
