"""Host logic of the multi-GPU bench path (replicas only) on 2 CPU ranks over gloo:
barrier, max-over-ranks timing and the whole-job aggregate; and the reference arm, whose
non-zero ranks exit without work."""
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


def _worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(dist, torch)
        t = bench.reduce_max(1.5 + rank, dist, torch)  # rank 1 is the slowest
        v = bench.whole_job_value(world, 1000, 10, t)
        bench.barrier(dist, torch)
        with open(os.path.join(out, f"rank{rank}.txt"), "w") as f:
            f.write(f"{t} {v}\n")
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_aggregate(tmp_path):
    import torch.multiprocessing as mp

    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        t, v = map(float, open(tmp_path / f"rank{r}.txt").read().split())
        assert t == 2.5
        assert v == pytest.approx(2 * 1000 * 10 / 2.5)


def test_reference_arm_nonzero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
