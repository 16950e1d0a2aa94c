"""Replica aggregation of bench.py across ranks, on CPU with the gloo backend
(world size 2): whole-job points are summed, time is the maximum over ranks."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        pts, sec = bench.reduce_over_ranks(dist, points=1000 * (rank + 1), seconds=0.5 + rank, device="cpu")
        Path(out, f"r{rank}.txt").write_text(f"{pts} {sec}")
    finally:
        dist.destroy_process_group()


def test_reduce_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        pts, sec = map(float, (tmp_path / f"r{r}.txt").read_text().split())
        assert pts == 3000.0
        assert sec == 1.5


def test_reduce_over_ranks_single():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.reduce_over_ranks(None, 123, 0.25, "cpu") == (123.0, 0.25)


def test_reference_arm_other_ranks_do_nothing(capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    class A:
        steps, warmup, delta, eps, gpus = 1, 1, 1e-4, 1e-6, 2
    assert bench.run_reference(A(), rank=1, world=2) is None
    assert capsys.readouterr().out == ""
