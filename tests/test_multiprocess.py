"""The bench's N > 1 plumbing on CPU with world_size 2 (gloo): the whole-job rate takes the slowest
rank's time, and the reference arm under torch.distributed.run prints one line from rank 0 while
the other rank exits 0 without work.  (The path runs independent replicas per GPU: there is no
data-path collective to test beyond the max-over-ranks reduction.)"""

import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms_max, value = bench.job_rate(1.0 + rank, 1000, world, "cpu")
        out[rank] = (ms_max, value)
    finally:
        dist.destroy_process_group()


def test_job_rate_is_max_over_ranks():
    import torch.multiprocessing as mp

    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        ms_max, value = out[r]
        assert ms_max == 2.0
        assert abs(value - world * 1000 / 2e-3 / 1e6) < 1e-12


def test_reference_arm_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(port), "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference"
    if "unavailable" not in line:
        assert line["n_gpus"] == 2 and line["value"] > 0
