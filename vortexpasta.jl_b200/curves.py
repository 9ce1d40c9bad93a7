"""Filament initial conditions used by the tests and the benchmark.

A filament is an ``(N, 3)`` float64 array of node positions of a closed curve.
Node ``i`` (1-based) sits at curve parameter ``tau_i = (2i - 1) / (2N)``, as in
``Filaments.init(S, ClosedFilament, N, method)`` (src/Filaments/closed_filament.jl:182-188).

The ring parametrisation follows ``PredefinedCurves.Ring`` (src/PredefinedCurves/ring.jl:100-108):
``S(t) = R(t) (cos 2 pi t, sin 2 pi t, 0)``, then rotated and translated.  The random
tangle follows the ``RandomRings`` benchmark shape (benchmark/benchmarks.jl:48-66) with
a seeded NumPy generator (Julia's StableRNG stream is not reproducible here), uniform
random rotations (Shoemake's quaternion method) and radial perturbations by Fourier
modes 2..8 of amplitude ``0.05 R g_k / k``.
"""

from __future__ import annotations

import math

import numpy as np


def node_parameters(n: int) -> np.ndarray:
    """tau_i = (2i - 1) / (2N), i = 1..N."""
    return (2.0 * np.arange(1, n + 1) - 1.0) / (2.0 * n)


def ring(n: int, radius: float, center=(0.0, 0.0, 0.0), rotation: np.ndarray | None = None,
         radial=None) -> np.ndarray:
    """Nodes of a (possibly perturbed) circular ring of `n` nodes."""
    t = node_parameters(n)
    r = np.full(n, float(radius))
    if radial is not None:
        r = r + radial(t)
    x = np.stack([r * np.cos(2 * np.pi * t), r * np.sin(2 * np.pi * t), np.zeros(n)], axis=1)
    if rotation is not None:
        x = x @ np.asarray(rotation).T
    return x + np.asarray(center, dtype=np.float64)


def trefoil(n: int, R: float = np.pi / 3) -> np.ndarray:
    """Trefoil knot of the reference's tests (PredefinedCurves/trefoil.jl:22-35, test/trefoil.jl:16-19):
    R (1 + (sin 2 pi t + 2 sin 4 pi t, cos 2 pi t - 2 cos 4 pi t, -sin 6 pi t)) at t = (i - 1) / n."""
    u = 2 * np.arange(n) / n
    X = np.stack([np.sin(np.pi * u) + 2 * np.sin(2 * np.pi * u), np.cos(np.pi * u) - 2 * np.cos(2 * np.pi * u),
                  -np.sin(3 * np.pi * u)], axis=1)
    return R + R * X


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    """Uniformly distributed rotation matrix (Shoemake 1992, uniform unit quaternion)."""
    u1, u2, u3 = rng.random(3)
    a = math.sqrt(1 - u1)
    b = math.sqrt(u1)
    w, x, y, z = (a * math.sin(2 * math.pi * u2), a * math.cos(2 * math.pi * u2),
                  b * math.sin(2 * math.pi * u3), b * math.cos(2 * math.pi * u3))
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def random_tangle(nrings: int, nodes_per_ring: int, L: float = 2 * np.pi, rmin: float | None = None,
                  rmax: float | None = None, modes=range(2, 9), amplitude: float = 0.05,
                  seed: int = 42, nodes_per_ring_fn=None) -> list[np.ndarray]:
    """Random tangle of perturbed rings in a periodic cube of side `L`.

    Centres are uniform in [0, L)^3, orientations uniform on SO(3), radii uniform in
    [rmin, rmax] (default [L/8, L/4]); each ring's radius is perturbed by
    sum_k amplitude*R*g_k/k*cos(2 pi k t + phi_k), g_k ~ N(0,1), phi_k ~ U[0, 2 pi).
    """
    rng = np.random.default_rng(seed)
    rmin = L / 8 if rmin is None else rmin
    rmax = L / 4 if rmax is None else rmax
    modes = list(modes)
    out = []
    for _ in range(nrings):
        R = rmin + (rmax - rmin) * rng.random()
        center = L * rng.random(3)
        rot = random_rotation(rng)
        g = rng.standard_normal(len(modes))
        phi = 2 * np.pi * rng.random(len(modes))
        amps = [amplitude * R * gk / k for gk, k in zip(g, modes)]

        def radial(t, amps=amps, phi=phi):
            return sum(a * np.cos(2 * np.pi * k * t + ph) for a, k, ph in zip(amps, modes, phi))

        n = nodes_per_ring if nodes_per_ring_fn is None else int(nodes_per_ring_fn(R))
        out.append(ring(n, R, center, rot, radial))
    return out


class InfiniteFilament(np.ndarray):
    """Nodes of an infinite, unclosed filament that repeats itself periodically: node i + N sits at
    node i + `offset` (the end-to-end offset of ``ClosedFilament``, src/Filaments/closed_filament.jl:
    118-132, 196-207).  An (N, 3) float64 array with an ``offset`` attribute."""

    def __new__(cls, nodes, offset):
        obj = np.ascontiguousarray(nodes, dtype=np.float64).view(cls)
        obj.offset = np.asarray(offset, dtype=np.float64).reshape(3).copy()
        return obj

    def __array_finalize__(self, obj):
        self.offset = getattr(obj, "offset", np.zeros(3))


def end_to_end_offset(f) -> np.ndarray:
    """end_to_end_offset(f): zero for a closed filament (closed_filament.jl:196-207)."""
    return np.asarray(getattr(f, "offset", np.zeros(3)), dtype=np.float64).reshape(3)


def periodic_line(n: int, L: float, x: float = 0.0, y: float = 0.0, r=None, sign: int = 1,
                  translate=(0.0, 0.0, 0.0)) -> InfiniteFilament:
    """``PeriodicLine`` of src/PredefinedCurves/periodic_line.jl scaled by L (``define_curve(p; scale = L,
    translate, orientation = sign)``): S(t) = translate + L (x + Re r(t), y + Im r(t), t - 1/2), nodes at
    t_j = (2j - 1) / (2N) (orientation -1 reverses t), end-to-end offset (0, 0, sign L).  `r` is a
    1-periodic complex function (None: straight line)."""
    t = node_parameters(n)
    tau = t if sign > 0 else 1.0 - t
    rr = np.zeros(n, dtype=complex) if r is None else np.asarray([r(v) for v in tau], dtype=complex)
    X = np.stack([x + rr.real, y + rr.imag, tau - 0.5], axis=1) * L + np.asarray(translate, dtype=np.float64)
    return InfiniteFilament(X, (0.0, 0.0, sign * L))


def concat(filaments) -> tuple[np.ndarray, np.ndarray]:
    """Pack a list of filaments into (AoS nodes [Np, 3], offsets [nfil + 1] int64)."""
    counts = np.array([len(f) for f in filaments], dtype=np.int64)
    offsets = np.zeros(len(filaments) + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])
    nodes = np.ascontiguousarray(np.concatenate([np.asarray(f, dtype=np.float64) for f in filaments], axis=0))
    return nodes, offsets
