"""Named workloads: the vortex configurations and Biot-Savart parameters the tests and the
benchmark run on.

* ``ring64``: single ring, L = 2 pi, R = L/4 at the box centre, N = 64 nodes, quintic
  splines, GL(3), Gamma = 1, a = 1e-8, Delta = 1/4, Gaussian splitting with beta = 3.5 and
  r_cut = L/4 (alpha = 2.228), Ns = 32 (oversampled FFT grid 48^3), NUFFT m = 4.
* ``tangle20k``: 100 random perturbed rings x 200 nodes (20,000 nodes), r_cut = L/8,
  beta = 3.5 (alpha = 4.456), Ns = 128 (FFT grid 192^3), m = 4.
* ``tangle1m``: 5000 rings x 200 nodes (1,000,000 nodes), r_cut = L/16, beta = 4
  (alpha = 10.19), Ns = 512 (FFT grid 768^3), m = 5.

The ring generator is the benchmark's RandomRings shape (benchmark/benchmarks.jl:48-66) with
radial Fourier perturbations of modes 2..8; seeds are fixed.
"""

from __future__ import annotations

import math

from . import curves
from .params import GaussianSplitting, GaussLegendre, NonuniformFFTsBackend, ParamsBiotSavart

L = 2 * math.pi


def params_for(rcut: float, beta: float, Ns: int, m: int, precision: str = "fp64", **kw) -> ParamsBiotSavart:
    alpha = beta / rcut
    return ParamsBiotSavart(Gamma=1.0, a=1e-8, Delta=0.25,
                            splitting=GaussianSplitting(Ls=L, alpha=alpha, rcut=rcut, Ns=Ns),
                            quadrature=GaussLegendre(3), backend_long=NonuniformFFTsBackend(1.5, m),
                            precision=precision, **kw)


def ring64(**kw):
    fs = [curves.ring(64, L / 4, center=(L / 2, L / 2, L / 2))]
    return fs, params_for(L / 4, 3.5, 32, 4, **kw)


def tangle(nrings: int, nodes_per_ring: int = 200, seed: int = 42):
    return curves.random_tangle(nrings, nodes_per_ring, L=L, seed=seed)


def tangle20k(seed: int = 42, **kw):
    return tangle(100, 200, seed), params_for(L / 8, 3.5, 128, 4, **kw)


def tangle1m(seed: int = 42, **kw):
    return tangle(5000, 200, seed), params_for(L / 16, 4.0, 512, 5, **kw)


WORKLOADS = {"ring64": ring64, "tangle20k": tangle20k, "tangle1m": tangle1m}


def tangle1m_cpu_sample(seed: int = 42, **kw):
    """Bounded CPU sample of ``tangle1m``: a cube of side L/4 (1/64 of the volume) holding 78 rings
    x 200 nodes (15,600 nodes: the same node density) with radii scaled by 1/4, and the same
    absolute parameters -- r_cut = L/16 (= L'/4), alpha = 4 / r_cut, the same grid spacing
    (Ns = 128, FFT 192^3), m = 5 -- so every node sees the same work as in the full workload."""
    return tangle1m_sample(4, seed, **kw)


def tangle1m_sample(k: int, seed: int = 42, **kw):
    """Volume sample of ``tangle1m``: a cube of side L/k holding round(5000/k^3) rings x 200 nodes
    (the node density of the full tangle) with radii in [L/(8k), L/(4k)], at tangle1m's absolute
    parameters (``sample_params``): r_cut = L/16, alpha = 4 / r_cut, FFT 768/k per side, m = 5.
    k = 4 gives 78 rings (15,600 nodes, FFT 192^3); k = 2 gives 625 rings (125,000 nodes, FFT 384^3)."""
    Ls = L / k
    fs = curves.random_tangle(int(round(5000 / k ** 3)), 200, L=Ls, rmin=Ls / 8, rmax=Ls / 4, seed=seed)
    return fs, sample_params(tangle1m_params(**kw), k)


def tangle1m_params(**kw) -> ParamsBiotSavart:
    return params_for(L / 16, 4.0, 512, 5, **kw)


def sample_params(p: ParamsBiotSavart, k: int) -> ParamsBiotSavart:
    """Parameters of `p` (a periodic cube of side L) carried over to a cube of side L/k with the
    same absolute cut-off, the same splitting parameter (alpha, or the Kaiser-Bessel beta and
    rtol), the same NUFFT (sigma, m) and the same grid spacing: the oversampled FFT has n/k points
    per side when n/k is an FFT size of the library (Ns then the largest count mapping to it, as
    the tuned grids are chosen), else the smallest FFT size above n/k."""
    from .params import KaiserBesselSplitting
    from . import tuning
    sp = p.splitting
    Lk = sp.Ls[0] / k
    sigma = p.backend_long.sigma
    n = tuning.fft_size(sp.Ns[0], sigma)
    target = max(n // k, 2 * p.backend_long.m)
    Ns = int(math.floor(target / sigma + 1e-9))
    while Ns > 1 and tuning.fft_size(Ns, sigma) > target:
        Ns -= 1
    if tuning.fft_size(Ns, sigma) < target:
        Ns += 1
    if isinstance(sp, KaiserBesselSplitting):
        s = KaiserBesselSplitting(Ls=Lk, beta=sp.beta, rcut=sp.rcut)
        s.Ns, s.rtol = (Ns,) * 3, sp.rtol
    else:
        s = GaussianSplitting(Ls=Lk, alpha=sp.alpha, rcut=sp.rcut, Ns=Ns)
    return p.with_(splitting=s)
