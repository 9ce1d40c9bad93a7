"""Batching form: the on-device RK4 step against a host-driven RK4 built from public velocity
evaluations, the CUDA-graph ensemble against step-by-step RK4, and the autotuner."""

import math

import numpy as np
import pytest

from conftest import load_package

vp = load_package()
from vortexpasta_b200 import _lib, configs, curves, timestepping  # noqa: E402

L = 2 * math.pi


def host_rk4(cache, fs, dt):
    """Classic RK4 from public velocity evaluations (knots re-derived at every stage)."""
    x0 = [np.asarray(f, dtype=np.float64) for f in fs]

    def vel(xs):
        return vp.velocity_on_nodes(cache, xs)

    k1 = vel(x0)
    k2 = vel([x + 0.5 * dt * k for x, k in zip(x0, k1)])
    k3 = vel([x + 0.5 * dt * k for x, k in zip(x0, k2)])
    k4 = vel([x + dt * k for x, k in zip(x0, k3)])
    return [x + dt / 6 * (a + 2 * b + 2 * c + d) for x, a, b, c, d in zip(x0, k1, k2, k3, k4)]


@pytest.mark.gpu
def test_rk4_step_matches_host_rk4_on_translating_ring():
    import torch
    fs, p = configs.ring64()
    dt = 0.02
    c = vp.init_cache(p)
    try:
        ref = host_rk4(c, fs, dt)
        c.set_filaments(fs)
        nodes, _ = curves.concat(fs)
        t = torch.from_numpy(nodes).cuda()
        timestepping.rk4_step(c, t.data_ptr(), dt)
        torch.cuda.synchronize()
        x = t.cpu().numpy()
    finally:
        c.close()
    disp = np.linalg.norm(ref[0] - fs[0])
    # frozen knots (device) vs re-derived knots (host): the ring only translates, so the knots
    # barely change inside the step
    assert np.linalg.norm(x - ref[0]) <= 1e-6 * disp
    assert disp > 1e-3


@pytest.mark.gpu
def test_ensemble_graph_matches_stepwise_rk4():
    import torch
    # FP64 systems: separated rings (no near-collisions, so the pair sums are well conditioned and
    # run-dependent summation order stays at rounding level); mixed system: a random tangle
    ring_a = [curves.ring(64, L / 4, center=(L / 2, L / 2, L / 2))]
    ring_b = [curves.ring(48, L / 6, center=(L / 4, L / 4, L / 2)),
              curves.ring(40, L / 7, center=(3 * L / 4, 3 * L / 4, L / 2), rotation=curves.random_rotation(
                  np.random.default_rng(5)))]
    systems = [(ring_a, configs.params_for(L / 8, 3.5, 32, 4), 1e-3),
               (curves.random_tangle(20, 48, L=L, seed=101), configs.params_for(L / 8, 3.5, 48, 4, precision="mixed"),
                2e-3),
               (ring_b, configs.params_for(L / 8, 3.5, 40, 4), 3e-3)]
    ens = timestepping.Ensemble(systems)
    try:
        ens.step(3)
        got = [np.concatenate(ens.positions(k)) for k in range(len(systems))]
    finally:
        ens.close()
    for (fs, p, dt), x in zip(systems, got):
        c = vp.init_cache(p)
        try:
            c.set_filaments(fs)
            nodes, _ = curves.concat(fs)
            t = torch.from_numpy(nodes).cuda()
            for _ in range(3):
                timestepping.rk4_step(c, t.data_ptr(), dt)
            torch.cuda.synchronize()
            y = t.cpu().numpy()
        finally:
            c.close()
        moved = np.linalg.norm(y - nodes)
        assert moved > 0
        # the counting sort ranks points by atomics, so sums run in a run-dependent order: ~1e-7
        # relative in the FP32 spreading; rounding level in FP64 for well-conditioned sums
        tol = 1e-6 if p.precision == "mixed" else 1e-12
        assert np.linalg.norm(x - y) <= tol * moved


@pytest.mark.gpu
def test_autotune_keeps_results():
    fs = configs.tangle(40, 100, seed=7)
    p = configs.params_for(L / 8, 3.5, 64, 4)
    c = vp.init_cache(p)
    try:
        c.set_filaments(fs)
        c.compute(_lib.VELOCITY)
        v0 = c.get(_lib.VELOCITY)
        b = timestepping.autotune(c)
        assert b in (0, 1, 2, 3, 4)
        c.compute(_lib.VELOCITY)
        v1 = c.get(_lib.VELOCITY)
    finally:
        c.close()
    assert np.linalg.norm(v1 - v0) <= 1e-12 * np.linalg.norm(v0)


@pytest.mark.gpu
def test_spread_autotune_keeps_results():
    """The spreading autotuner picks a mode (tensor cores or CUDA cores) and the velocities stay those
    of the default mode to the run-to-run order of the FP32 spreading sums."""
    fs = configs.tangle(40, 100, seed=7)
    p = configs.params_for(L / 8, 3.5, 64, 3, precision="mixed")
    c = vp.init_cache(p)
    try:
        c.set_filaments(fs)
        c.compute(_lib.VELOCITY)
        v0 = c.get(_lib.VELOCITY)
        m = timestepping.autotune_spread(c)
        assert m in (0, 1)
        c.compute(_lib.VELOCITY)
        v1 = c.get(_lib.VELOCITY)
    finally:
        c.close()
    assert np.linalg.norm(v1 - v0) <= 1e-6 * np.linalg.norm(v0)
