"""Multi-rank logic of bench.py on CPU (gloo, world size 2): each rank gets an independent
system and the job time is the max over ranks."""

import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "tests"))
    import torch.distributed as dist
    from conftest import load_package
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        vp = load_package()
        fs, _ = bench.rank_workload(vp, "tangle20k", rank)
        t = bench.max_over_ranks([1.0 + rank, 5.0 - rank], "cpu", world)
        out[rank] = (float(fs[0][0, 0]), len(fs), t)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    import torch.multiprocessing as mp
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        r0, r1 = out[0], out[1]
    assert r0[1] == r1[1] == 100
    assert r0[0] != r1[0]  # independent tangles per rank
    assert r0[2] == r1[2] == [2.0, 5.0]  # max over ranks, identical on every rank
