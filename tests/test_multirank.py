"""Multi-rank logic of bench.py on CPU (gloo, world size 2): each rank gets an independent
system, the job time is the max over ranks, and the batching-form ensemble is sharded by
system (the same deterministic partition on every rank, no data exchanged)."""

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
        from vortexpasta_b200 import timestepping
        costs = [float((7 * i) % 13 + 1) for i in range(20)]
        shard = timestepping.shard_systems(costs, world)[rank]  # computed locally, nothing exchanged
        gathered = [None] * world
        dist.all_gather_object(gathered, shard)  # only to check the partition in the test
        out[rank] = (float(fs[0][0, 0]), len(fs), t, gathered)
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
    # ensemble sharding: both ranks derive the same partition, covering every system once
    assert r0[3] == r1[3]
    assert sorted(i for sh in r0[3] for i in sh) == list(range(20))


def test_shard_systems_balances_cost():
    from conftest import load_package
    load_package()
    from vortexpasta_b200 import timestepping
    costs = [100.0, 90.0, 40.0, 35.0, 30.0, 5.0, 1.0]
    shards = timestepping.shard_systems(costs, 3)
    assert sorted(i for sh in shards for i in sh) == list(range(7))
    loads = [sum(costs[i] for i in sh) for sh in shards]
    assert max(loads) - min(loads) <= max(costs)  # greedy bound
    assert shards == timestepping.shard_systems(costs, 3)  # deterministic
    assert timestepping.shard_systems(costs, 1) == [list(range(7))]
    assert timestepping.system_cost(1000, 16) == 1000 + 0.125 * 16 ** 3
    with pytest.raises(ValueError):
        timestepping.shard_systems(costs, 0)


def test_form_summary_stage_model():
    """bench.form_summary on synthetic stage times: throughput from the timed total, each stage
    against its bound, and the spread's grid-update rate Nq (2m)^3 x 3 / time."""
    import argparse
    from conftest import load_package
    vp = load_package()
    import bench
    fs, p = vp.configs.ring64()
    Np = sum(len(f) for f in fs)
    Nq = 3 * Np
    stage_ms = {k: [1.0, 1.0] for k in ("geometry", "cell_lists", "spread", "fft_forward", "fourier", "fft_inverse",
                                        "interp", "local_self", "pairs")}
    stage_ms["pairs"] = [2.0, 2.0]
    m = {"stage_ms": stage_ms, "pairs_in_range": 1000, "total_ms": 20.0, "e2e_ms": 40.0}
    args = argparse.Namespace(steps=2)
    peaks = {"hbm": 6000.0, "fp64": 30.0, "fp32": 60.0, "hbm_source": "test"}
    out = bench.form_summary(p, m, Np, Nq, 1, args, peaks)
    assert out["value"] == pytest.approx(Np * 2 / 0.020)
    assert out["e2e_value"] == pytest.approx(Np * 2 / 0.040)
    assert out["dominant"] == "pairs" and out["stages"]["pairs"]["bound"] == "fp64"
    assert out["stages"]["spread"]["grid_updates_per_s"] == pytest.approx(Nq * 8 ** 3 * 3 / 1e-3)
    # ring64's stages move far less than the L2 holds: HBM fractions are withheld, the pair stage's
    # FMA fraction is kept
    assert out["stages"]["pairs"]["frac"] > 0
    assert all(st["frac"] is None for k, st in out["stages"].items() if st["bound"] == "hbm")
    # a large workload keeps its HBM fractions
    fs1, p1 = vp.configs.tangle1m()
    out = bench.form_summary(p1, m, 1_000_000, 3_000_000, 1, args, peaks)
    assert out["stages"]["interp"]["frac"] > 0 and out["stages"]["fourier"]["frac"] > 0


def test_bench_world_size_checks(monkeypatch):
    """bench.py --gpus N fails loudly when the launcher started another number of ranks, runs in place
    for N = 1 or under a matching launcher, and relaunches itself through torchrun otherwise."""
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.check_world(4) == 2
    assert bench.check_world(2) is None
    monkeypatch.delenv("WORLD_SIZE")
    assert bench.check_world(1) is None
    assert bench.check_world(0) == 2
    cmd = bench.launch_command(4, ["--gpus", "4", "--steps", "3"], 29500)
    assert cmd[1:3] == ["-m", "torch.distributed.run"] and "--nproc-per-node=4" in cmd
    assert "--master-addr=127.0.0.1" in cmd and cmd[-4:] == ["--gpus", "4", "--steps", "3"]


def test_ensemble_workloads_are_kelvin_wave_limited():
    """The two batching-form ensembles of the bench: sizes and grids as described, and every time
    step at most the Kelvin-wave period of the system's shortest segment (the fixed 1e-3 L^2 / Gamma
    is far above it for these tangles)."""
    import math
    import sys
    from pathlib import Path
    import numpy as np
    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root))
    import bench
    from conftest import load_package
    vp = load_package()
    from vortexpasta_b200.params import kelvin_wave_period
    L = 2 * math.pi
    small = bench.small_ensemble_systems(vp, nsys=12)
    assert len(small) == 12
    for fs, p, dt in small:
        n = sum(len(f) for f in fs)
        assert 1000 <= n <= 2000 and p.splitting.Ns == (32, 32, 32) and p.precision == "mixed"
        dmin = min(float(np.linalg.norm(np.roll(f, -1, axis=0) - f, axis=1).min()) for f in fs)
        assert dt == min(1e-3 * L ** 2, kelvin_wave_period(dmin, a=1e-8, Delta=0.25, Gamma=1.0))
        assert dt < 1e-3 * L ** 2
    big = bench.ensemble_systems(vp, nsys=3)
    for fs, p, dt in big:
        assert 64 <= p.splitting.Ns[0] <= 256 and dt < 1e-3 * L ** 2
