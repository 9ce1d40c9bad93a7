"""Accuracy-targeted choice of the Ewald/NUFFT parameters.

* ``default_rule``: the reference's rule for a requested tolerance -- beta from
  rtol = 10^-1.3 exp(-beta^2), alpha = beta / r_cut, k_max = 2 alpha beta and the grid from
  ``kmax_to_gridsize`` (src/BiotSavart/splitting/gaussian.jl:133-200, params.jl:156-159) with
  the NonuniformFFTsBackend defaults sigma = 1.5, m = 4 (longrange/backends/nonuniformffts.jl:
  107-126).  It is the fallback of the learned predictor.
* ``EwaldChoice`` / ``choice_from``: a parameter set (alpha, r_cut, Ns, sigma, m) built from
  the short- and long-range beta, with the grid rounded to FFT sizes that are multiples of 16
  (the register-column spreading kernel's brick) and Ns raised to the largest value that
  keeps the same FFT size (free accuracy).
* ``candidate_grid`` and ``sweep``: the parameter sweep that measures device time and
  velocity error against an FP64 reference -- the (configuration, parameters, cost, error)
  tuples the learned predictor is trained on.
"""

from __future__ import annotations

import math
from dataclasses import asdict, dataclass

import numpy as np

from . import _lib
from .params import (C_RTOL, GaussianSplitting, GaussLegendre, NonuniformFFTsBackend, ParamsBiotSavart,
                     kmax_to_gridsize)

FFT_MULTIPLE = 16
SIGMAS = (1.25, 1.5, 2.0)
HALF_SUPPORTS = (2, 3, 4, 5, 6, 7, 8)


def beta_for_rtol(rtol: float) -> float:
    """Inverse of rtol = 10^-1.3 exp(-beta^2) (gaussian.jl:175-186)."""
    return math.sqrt(-math.log(rtol / C_RTOL))


def fft_size(Ns: int, sigma: float) -> int:
    """Oversampled FFT size used by the library (smallest even 2^a 3^b 5^c >= sigma Ns)."""
    return int(_lib.load().vpbs_fft_size(int(Ns), float(sigma)))


def _smooth(n: int) -> bool:
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


def grid_for(Ns_min: int, sigma: float, m: int, multiple: int = FFT_MULTIPLE) -> int:
    """Fourier grid Ns >= Ns_min whose oversampled FFT size n is a multiple of `multiple` (and at
    least 2 multiple and 2m): the smallest such n that some Ns >= Ns_min maps to, then the
    largest Ns mapping to it."""
    n = max(int(math.ceil(sigma * Ns_min - 1e-9)), 2 * multiple, 2 * m)
    while True:
        if n % multiple == 0 and _smooth(n):
            for Ns in range(int(math.floor(n / sigma + 1e-9)), Ns_min - 1, -1):
                if fft_size(Ns, sigma) == n:
                    return Ns
        n += 1


@dataclass(frozen=True)
class EwaldChoice:
    """One parameter set of the Ewald split and its NUFFT."""
    alpha: float
    rcut: float
    Ns: int
    sigma: float
    m: int

    @property
    def beta_short(self) -> float:
        return self.alpha * self.rcut

    def beta_long(self, L: float) -> float:
        return 2 * math.pi * ((self.Ns - 1) // 2) / L / (2 * self.alpha)

    def fft_size(self) -> int:
        return fft_size(self.Ns, self.sigma)

    def params(self, L: float, precision: str = "mixed", Gamma=1.0, a=1e-8, Delta=0.25, nquad=3,
               **kw) -> ParamsBiotSavart:
        return ParamsBiotSavart(Gamma=Gamma, a=a, Delta=Delta,
                                splitting=GaussianSplitting(Ls=L, alpha=self.alpha, rcut=self.rcut, Ns=self.Ns),
                                quadrature=GaussLegendre(nquad), backend_long=NonuniformFFTsBackend(self.sigma, self.m),
                                precision=precision, **kw)

    def as_dict(self) -> dict:
        return asdict(self)


@dataclass(frozen=True)
class KBChoice:
    """One parameter set of a Kaiser-Bessel split (kaiser_bessel.jl) and its NUFFT: shape
    parameter beta (short-range weights and long-range filter alike), r_cut, the Fourier grid
    and the Chebyshev truncation rtol (C exp(-beta) unless given)."""
    beta: float
    rcut: float
    Ns: int
    sigma: float
    m: int
    rtol: float = 0.0

    @property
    def beta_short(self) -> float:
        return self.beta

    def beta_long(self, L: float) -> float:
        return 2 * math.pi * ((self.Ns - 1) // 2) / L * self.rcut

    def fft_size(self) -> int:
        return fft_size(self.Ns, self.sigma)

    def splitting(self, L: float):
        from .params import C_RTOL_KB, KaiserBesselSplitting
        sp = KaiserBesselSplitting(Ls=L, beta=self.beta, rcut=self.rcut)
        sp.Ns = (self.Ns,) * 3
        sp.rtol = self.rtol if self.rtol > 0 else C_RTOL_KB * math.exp(-self.beta)
        return sp

    def params(self, L: float, precision: str = "mixed", Gamma=1.0, a=1e-8, Delta=0.25, nquad=3,
               **kw) -> ParamsBiotSavart:
        return ParamsBiotSavart(Gamma=Gamma, a=a, Delta=Delta, splitting=self.splitting(L),
                                quadrature=GaussLegendre(nquad), backend_long=NonuniformFFTsBackend(self.sigma, self.m),
                                precision=precision, **kw)

    def as_dict(self) -> dict:
        return {**asdict(self), "splitting": "kaiser_bessel"}


def kb_choice_from(L: float, rcut: float, beta: float, sigma: float, m: int, beta_long: float | None = None) -> KBChoice:
    """Kaiser-Bessel parameters at cut-off `rcut`: the grid resolves k_max = beta_long / rcut
    (beta_long = beta by default, the reference's rule), rounded like ``choice_from``."""
    bl = beta if beta_long is None else beta_long
    Ns = grid_for(kmax_to_gridsize(bl / rcut, L), sigma, m)
    return KBChoice(beta=beta, rcut=rcut, Ns=Ns, sigma=sigma, m=m)


def choice_from(L: float, rcut: float, beta_short: float, beta_long: float, sigma: float, m: int) -> EwaldChoice:
    alpha = beta_short / rcut
    Ns = grid_for(kmax_to_gridsize(2 * alpha * beta_long, L), sigma, m)
    return EwaldChoice(alpha=alpha, rcut=rcut, Ns=Ns, sigma=sigma, m=m)


def default_rule(L: float, rtol: float, rcut: float) -> EwaldChoice:
    """The reference's parameters for tolerance `rtol` at cut-off `rcut` (sigma = 1.5, m = 4)."""
    beta = beta_for_rtol(rtol)
    alpha = beta / rcut
    Ns = kmax_to_gridsize(2 * alpha * beta, L)
    return EwaldChoice(alpha=alpha, rcut=rcut, Ns=Ns, sigma=1.5, m=4)


def rel_errors(v: np.ndarray, vref: np.ndarray) -> tuple[float, float]:
    """Relative L2 error of a node-velocity field and its largest node error relative to the
    largest reference velocity."""
    d = v - vref
    return float(np.linalg.norm(d) / np.linalg.norm(vref)), float(np.abs(d).max() / np.abs(vref).max())


def candidate_grid(L: float, rcut_fracs=(1 / 8, 1 / 12, 1 / 16, 1 / 20, 1 / 24, 1 / 32, 1 / 40),
                   betas=(2.6, 2.8, 3.0, 3.2, 3.4), sigma_m=((1.25, 3), (1.25, 4), (1.5, 3), (1.5, 4), (2.0, 3)),
                   beta_long_offsets=(0.0,)) -> list[EwaldChoice]:
    """Parameter sets of the sweep (short-range beta, long-range beta = beta + offset)."""
    out = []
    for f in rcut_fracs:
        for b in betas:
            for db in beta_long_offsets:
                for s, m in sigma_m:
                    out.append(choice_from(L, f * L, b, b + db, s, m))
    return out


def measure(fs, choice: EwaldChoice, L: float, precision: str = "mixed", reps: int = 2, fields: int = _lib.VELOCITY,
            device: int = 0):
    """Device time (ms, best of `reps`, every stage from the geometry to the interpolation, run
    one after another) of one evaluation with `choice`, and the node velocities."""
    from .biotsavart import init_cache
    cache = init_cache(choice.params(L, precision, device=device))
    try:
        cache.set_filaments(fs)
        cache.compute(fields)
        cache.stage_timing(True)
        cache.stage_times()
        best = math.inf
        for _ in range(reps):
            cache.set_filaments(fs)
            cache.compute(fields)
            best = min(best, sum(cache.stage_times().values()))
        cache.stage_timing(False)
        v = cache.get(_lib.VELOCITY)
    finally:
        cache.close()
    return best, v


def sweep(fs, L: float, vref: np.ndarray, choices, precision: str = "mixed", reps: int = 2,
          device: int = 0) -> list[dict]:
    """(parameters, cost, error) records of `choices` on the configuration `fs`."""
    recs = []
    for ch in choices:
        ms, v = measure(fs, ch, L, precision, reps, device=device)
        l2, mx = rel_errors(v, vref)
        recs.append({**ch.as_dict(), "fft": ch.fft_size(), "beta_short": ch.beta_short, "beta_long": ch.beta_long(L),
                     "ms": ms, "rel_l2": l2, "max_err": mx})
    return recs


def cheapest(recs: list[dict], rtol: float):
    """The fastest record whose relative L2 error meets `rtol` (None if none does)."""
    ok = [r for r in recs if r["rel_l2"] <= rtol]
    return min(ok, key=lambda r: r["ms"]) if ok else None
