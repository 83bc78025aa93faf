"""The multi-GPU plumbing of bench.py on CPU (world size 2, gloo).

The scan does not shard: `bench.py --gpus N` runs N independent replicas, and
the only exchange is the max over ranks of each replica's timings. These tests
run that reduction with two gloo ranks, and check that under torchrun only
rank 0 runs the reference arm."""
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as tdist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r: step time 10 r + 1 ms, e2e time 5 - r ms
        got = bench.max_over_ranks([10.0 * rank + 1.0, 5.0 - rank], "cpu")
        if rank == 0:
            with open(out, "w") as f:
                f.write(" ".join(repr(v) for v in got))
    finally:
        tdist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    out = str(tmp_path / "max.txt")
    mp.spawn(_rank, args=(2, _free_port(), out), nprocs=2, join=True)
    got = [float(v) for v in open(out).read().split()]
    assert got == [11.0, 5.0]


def test_whole_job_rate():
    # two replicas of 5e9 tests, slowest replica 250 ms per step
    assert bench.whole_job_rate(5_000_000_000, 2, 250.0) == pytest.approx(4.0e10)


def test_reference_arm_runs_on_rank_0_only():
    env = {**os.environ, "RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
