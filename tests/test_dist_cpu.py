"""The multi-rank path of bench.py on CPU: world_size 2 over gloo (127.0.0.1). Ranks run independent
replicas, so the only cross-rank step is the max over ranks of the timed region; the reference arm runs on
rank 0 alone and the other ranks exit without work."""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out: str):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms = bench.max_over_ranks(10.0 + 5.0 * rank)
    value = bench.replica_throughput(world, 1000, 10, ms)
    dist.barrier()
    dist.destroy_process_group()
    with open(f"{out}.{rank}", "w") as f:
        f.write(f"{ms} {value}")


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp

    out = str(tmp_path / "r")
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    for r in range(2):
        ms, value = map(float, open(f"{out}.{r}").read().split())
        assert ms == 15.0  # the slower rank's time, on every rank
        assert value == pytest.approx(2 * 1000 * 10 / 0.015)


def test_reference_arm_runs_on_rank0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
