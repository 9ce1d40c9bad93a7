"""RK4 time stepping of filament systems on the device: the caller side of the path
(src/Timestepping/timesteppers/explicit/RK4.jl:14-44) for the batching form.

* ``rk4_step(cache, nodes, dt)``: one RK4 step of one system, nodes in device memory
  (vpbs_rk4_step; knots frozen inside the step as the reference's RK4 does).
* ``Ensemble``: independent systems (any sizes and grids) advanced together; one RK4 step of all
  of them is captured in one CUDA graph and replayed with one launch per step
  (vpbs_ensemble_*).  ``autotune_pairs=True`` first runs the pair-kernel and spreading autotuners
  on every system.

Device memory for the node arrays comes from torch (plumbing only); every kernel is the
library's.
"""

from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib, curves
from .biotsavart import BiotSavartCache, init_cache


def system_cost(nodes: int, fft_size: int) -> float:
    """Relative cost of one velocity evaluation of a system: its nodes (pairs, spreading,
    interpolation and geometry scale with them at a fixed density) plus its FFT grid points
    (the 3-D transforms and the Fourier pass) at a lower weight."""
    return float(nodes) + 0.125 * float(fft_size) ** 3


def shard_systems(costs, world: int) -> list[list[int]]:
    """Independent systems over `world` ranks, greedy by cost (largest first onto the least
    loaded rank; ties to the lower rank): every index appears in exactly one shard, each shard
    in increasing index order.  Deterministic, so every rank computes the same partition without
    exchanging anything."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        shards[r].append(i)
        loads[r] += costs[i]
    return [sorted(sh) for sh in shards]


def rk4_step(cache: BiotSavartCache, nodes_ptr: int, dt: float) -> None:
    """One RK4 step of the filaments loaded in `cache` (vpbs_set_filaments); `nodes_ptr` is a
    device AoS [Np][3] float64 array with the same layout, advanced in place."""
    _lib.check(cache._lib.vpbs_rk4_step(cache.handle, ct.c_void_p(nodes_ptr), float(dt)), cache.handle, "rk4_step")


def autotune(cache: BiotSavartCache) -> int:
    """Pick the pair kernel's cells per CTA edge for the loaded point data (0: built-in rule)."""
    b = ct.c_int32()
    _lib.check(cache._lib.vpbs_autotune(cache.handle, ct.byref(b)), cache.handle, "autotune")
    return int(b.value)


def autotune_spread(cache: BiotSavartCache) -> int:
    """Pick the spreading mode for the loaded point data (vpbs_spread_mode: 0 tensor cores where they
    apply, 1 CUDA cores only)."""
    m = ct.c_int32()
    _lib.check(cache._lib.vpbs_autotune_spread(cache.handle, ct.byref(m)), cache.handle, "autotune_spread")
    return int(m.value)


class Ensemble:
    """Independent filament systems advanced by RK4 with one CUDA-graph launch per step.

    systems: list of (filaments, ParamsBiotSavart, dt)."""

    def __init__(self, systems, device: int = 0, autotune_pairs: bool = False):
        import torch
        self._lib = _lib.load()
        self.device = int(device)
        self.caches, self.nodes, self.layouts, self.tuned, self.spread_modes = [], [], [], [], []
        for fs, p, dt in systems:
            c = init_cache(p.with_(device=self.device))
            c.set_filaments(fs)
            if autotune_pairs:
                self.tuned.append(autotune(c))
                self.spread_modes.append(autotune_spread(c))
            nodes, offsets = curves.concat(fs)
            self.nodes.append(torch.from_numpy(nodes).to(torch.device("cuda", self.device)))
            self.layouts.append(offsets)
            self.caches.append(c)
        torch.cuda.synchronize(self.device)
        n = len(systems)
        hs = (ct.c_void_p * n)(*[c.handle.value if hasattr(c.handle, "value") else c.handle for c in self.caches])
        ps = (ct.c_void_p * n)(*[t.data_ptr() for t in self.nodes])
        dts = np.array([float(dt) for _, _, dt in systems], dtype=np.float64)
        e = ct.c_void_p()
        rc = self._lib.vpbs_ensemble_create(hs, ps, _lib.dptr(dts), n, ct.byref(e))
        if rc != 0:
            raise _lib.VpbsError(f"vpbs_ensemble_create failed ({rc}): {self._lib.vpbs_ensemble_last_error().decode()}")
        self._e = e

    def _check(self, rc, what):
        if rc != 0:
            raise _lib.VpbsError(f"{what} failed ({rc}): {self._lib.vpbs_ensemble_last_error().decode()}")

    def step(self, nsteps: int = 1):
        """Launch `nsteps` RK4 steps of every system (asynchronous)."""
        self._check(self._lib.vpbs_ensemble_step(self._e, int(nsteps)), "ensemble step")

    def synchronize(self):
        self._check(self._lib.vpbs_ensemble_synchronize(self._e), "ensemble synchronize")

    def stream(self) -> int:
        return int(self._lib.vpbs_ensemble_stream(self._e) or 0)

    def positions(self, k: int) -> list[np.ndarray]:
        """Filament nodes of system k (host copy, one array per filament)."""
        self.synchronize()
        x = self.nodes[k].cpu().numpy()
        off = self.layouts[k]
        return [x[off[i]:off[i + 1]].copy() for i in range(len(off) - 1)]

    def close(self):
        if getattr(self, "_e", None):
            self._lib.vpbs_ensemble_destroy(self._e)
            self._e = None
        for c in self.caches:
            c.close()
        self.caches = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
