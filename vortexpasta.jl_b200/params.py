"""Parameter types mirroring VortexPasta.BiotSavart's (src/BiotSavart/params.jl,
src/BiotSavart/splitting/gaussian.jl and kaiser_bessel.jl, the two backends and src/Quadratures).

Names, keyword arguments, defaults and the errors raised at construction follow the
reference; the backends name the CUDA implementations that replace the reference's
``CellListsBackend`` and ``NonuniformFFTsBackend``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

C_RTOL = 10 ** (-1.3)  # empirical constant of rtol(beta) ~ C exp(-beta^2) (gaussian.jl:135-140)


def kmax_to_gridsize(kmax: float, L: float) -> int:
    """params.jl:156-159."""
    m = math.ceil(kmax * L / (2 * math.pi))
    return 2 * m + 2


def maximum_wavenumber(Ns, Ls) -> float:
    """params.jl:161-166."""
    return min(2 * math.pi * ((M - 1) // 2) / L for M, L in zip(Ns, Ls))


@dataclass(frozen=True)
class GaussLegendre:
    """N-point Gauss-Legendre rule on [0, 1] (src/Quadratures/Quadratures.jl:74-76)."""
    n: int

    def rule(self):
        x, w = np.polynomial.legendre.leggauss(self.n)
        return (x + 1) / 2, w / 2

    def __len__(self):
        return self.n


class NoSplitting:
    """Open (non-periodic) domain without Ewald splitting (splitting/splitting.jl:17-37)."""
    Ls = (math.inf, math.inf, math.inf)
    rcut = math.inf
    Ns = (0, 0, 0)
    alpha = 0.0

    def __repr__(self):
        return "NoSplitting()"


@dataclass
class GaussianSplitting:
    """Gaussian Ewald splitting (splitting/gaussian.jl:109-200).

    Pass ``Ls`` and either ``beta`` or ``rtol`` plus one of ``alpha``, ``rcut``, ``Ns``;
    or all of ``alpha``, ``rcut`` and ``Ns``.
    """
    Ls: tuple
    alpha: float
    rcut: float
    Ns: tuple
    rtol: float

    def __init__(self, *, Ls, beta=None, alpha=None, rcut=None, Ns=None, rtol=None):
        Ls = tuple(float(L) for L in (Ls if np.ndim(Ls) else (Ls, Ls, Ls)))
        given = (beta is not None, alpha is not None, rcut is not None, Ns is not None, rtol is not None)
        if Ns is not None:
            Ns = tuple(int(n) for n in (Ns if np.ndim(Ns) else (Ns, Ns, Ns)))
        if given == (True, True, False, False, False):
            rcut = beta / alpha
            Ns = tuple(kmax_to_gridsize(2 * alpha * beta, L) for L in Ls)
            rtol = C_RTOL * math.exp(-beta ** 2)
        elif given == (True, False, True, False, False):
            alpha = beta / rcut
            Ns = tuple(kmax_to_gridsize(2 * alpha * beta, L) for L in Ls)
            rtol = C_RTOL * math.exp(-beta ** 2)
        elif given == (True, False, False, True, False):
            alpha = maximum_wavenumber(Ns, Ls) / (2 * beta)
            rcut = beta / alpha
            rtol = C_RTOL * math.exp(-beta ** 2)
        elif given == (False, True, True, True, False):
            rtol = C_RTOL * math.exp(-(alpha * rcut) ** 2)
        elif given[4] and sum(given[1:4]) == 1 and not given[0]:
            beta = math.sqrt(-math.log(rtol / C_RTOL))
            if alpha is not None:
                rcut = beta / alpha
                Ns = tuple(kmax_to_gridsize(2 * alpha * beta, L) for L in Ls)
            elif rcut is not None:
                alpha = beta / rcut
                Ns = tuple(kmax_to_gridsize(2 * alpha * beta, L) for L in Ls)
            else:
                alpha = maximum_wavenumber(Ns, Ls) / (2 * beta)
                rcut = beta / alpha
        else:
            raise TypeError("GaussianSplitting: pass `beta` or `rtol` and one of `alpha`, `rcut`, `Ns`;"
                            " or all of `alpha`, `rcut` and `Ns`")
        self.Ls, self.alpha, self.rcut, self.Ns, self.rtol = Ls, float(alpha), float(rcut), tuple(Ns), float(rtol)

    @property
    def beta_shortrange(self):
        return self.alpha * self.rcut

    @property
    def beta_longrange(self):
        return maximum_wavenumber(self.Ns, self.Ls) / (2 * self.alpha)


C_RTOL_KB = 10 ** (-0.2)  # empirical constant of rtol(beta) ~ C exp(-beta) (kaiser_bessel.jl:104-109)


class KaiserBesselSplitting:
    """KaiserBesselSplitting (splitting/kaiser_bessel.jl:130-223).

    Pass ``Ls`` and either ``beta`` or ``rtol`` plus one of ``rcut``, ``Ns``:
    ``beta`` and ``rcut`` give ``Ns`` from k_max = beta / rcut; ``beta`` and ``Ns`` give
    ``rcut = beta / k_max``; ``rtol`` sets ``beta = -log(rtol / C)``; ``rcut`` and ``Ns`` give
    ``beta = rcut k_max``.  When ``rtol`` is not given it is ``C exp(-beta)`` with C = 10^-0.2.
    The short-range weights 1 - F(r) and r F'(r) vanish beyond ``rcut`` (compact support); the
    long-range filter is beta / sinh(beta) sinh(q) / q with q = sqrt(beta^2 - (k rcut)^2).
    """
    beta: float
    rcut: float
    Ns: tuple
    rtol: float

    def __init__(self, *, Ls, beta=None, rcut=None, Ns=None, rtol=None):
        Ls = tuple(float(L) for L in (Ls if np.ndim(Ls) else (Ls,) * 3))
        given = (beta is not None, rcut is not None, Ns is not None, rtol is not None)
        if Ns is not None:
            Ns = tuple(int(n) for n in (Ns if np.ndim(Ns) else (Ns,) * 3))
        if given == (True, True, False, False):
            Ns = tuple(kmax_to_gridsize(beta / rcut, L) for L in Ls)
            rtol = C_RTOL_KB * math.exp(-beta)
        elif given == (False, True, True, False):
            beta = rcut * maximum_wavenumber(Ns, Ls)
            rtol = C_RTOL_KB * math.exp(-beta)
        elif given == (True, False, True, False):
            rcut = beta / maximum_wavenumber(Ns, Ls)
            rtol = C_RTOL_KB * math.exp(-beta)
        elif given == (False, True, False, True):
            beta = -math.log(rtol / C_RTOL_KB)
            Ns = tuple(kmax_to_gridsize(beta / rcut, L) for L in Ls)
        elif given == (False, False, True, True):
            beta = -math.log(rtol / C_RTOL_KB)
            rcut = beta / maximum_wavenumber(Ns, Ls)
        else:
            raise TypeError("KaiserBesselSplitting: pass `beta` or `rtol` and one of `rcut`, `Ns`; or `rcut` and `Ns`")
        self.Ls, self.beta, self.rcut, self.Ns, self.rtol = Ls, float(beta), float(rcut), Ns, float(rtol)

    def __repr__(self):
        return (f"KaiserBesselSplitting(Ls={self.Ls}, beta={self.beta}, rcut={self.rcut}, Ns={self.Ns}, "
                f"rtol={self.rtol})")

    def fourier_kernel(self, k2):
        """Long-range filter as a function of k^2 (kaiser_bessel.jl:266-278)."""
        k2 = np.asarray(k2, dtype=float)
        s = self.beta ** 2 - k2 * self.rcut ** 2
        q = np.sqrt(np.maximum(s, 0.0))
        with np.errstate(invalid="ignore", divide="ignore"):
            v = self.beta / math.sinh(self.beta) * np.where(q > 0, np.sinh(q) / np.where(q > 0, q, 1.0), 1.0)
        return np.where(s > 0, v, 0.0)


@dataclass(frozen=True)
class CellListsBackend:
    """Short-range backend: CUDA cell lists (replaces shortrange/backends/cell_lists.jl:64-87)."""
    nsubdiv: int = 2

    def max_cutoff_distance(self, L: float) -> float:
        """CellLists.jl:114-115: r_cut <= M / (2M + 1) L."""
        M = self.nsubdiv
        return M / (2 * M + 1) * L


@dataclass(frozen=True)
class NaiveShortRangeBackend:
    """Short-range backend for open domains: all pairs (shortrange/backends/naive.jl:18-30)."""

    def max_cutoff_distance(self, L: float) -> float:
        return L / 2


@dataclass(frozen=True)
class NonuniformFFTsBackend:
    """Long-range backend: CUDA NUFFT (replaces longrange/backends/nonuniformffts.jl:97-126).  Defaults
    sigma = 1.5, m = 4.  `kernel`: "es" (exponential of semicircle, the default) or "kaiser_bessel"
    (backward Kaiser-Bessel, the kind NonuniformFFTs.jl uses by default; its exact shape parameter is
    not pinned here, so results match the reference's to the NUFFT tolerance either way)."""
    sigma: float = 1.5
    m: int = 4
    kernel: str = "es"

    def __post_init__(self):
        if self.kernel not in ("es", "kaiser_bessel"):
            raise ValueError("NonuniformFFTsBackend kernel must be 'es' or 'kaiser_bessel'")


@dataclass
class ParamsBiotSavart:
    """ParamsBiotSavart (params.jl:326-376).

    ``ParamsBiotSavart(Gamma=..., a=..., splitting=GaussianSplitting(...), ...)`` or with the
    deprecated ``alpha, Ls, Ns, rcut`` keywords (``alpha=0`` selects NoSplitting).
    ``precision`` selects the arithmetic form of the CUDA library ("fp64" or "mixed").
    """
    Gamma: float
    a: float
    Delta: float
    splitting: object
    quadrature: GaussLegendre
    quadrature_near_singularity: GaussLegendre
    backend_short: object
    backend_long: object
    longrange_truncate_spherical: bool
    lia_segment_fraction: float | None
    avoid_explicit_erf: bool
    precision: str = "fp64"
    device: int = 0
    extra: dict = field(default_factory=dict)

    def __init__(self, *, Gamma, a, Delta=0.25, splitting=None, alpha=None, Ls=None, Ns=None, rcut=None,
                 quadrature=None, quadrature_near_singularity=None, backend_short=None, backend_long=None,
                 longrange_truncate_spherical=False, lia_segment_fraction=None, avoid_explicit_erf=True,
                 precision="fp64", device=0):
        if splitting is None:
            if alpha is None:
                raise TypeError("pass `splitting` or the `alpha` keyword")
            if alpha == 0:
                splitting = NoSplitting()
            else:
                splitting = GaussianSplitting(Ls=Ls, alpha=alpha, Ns=Ns, rcut=rcut)
        quadrature = quadrature or GaussLegendre(3)
        quadrature_near_singularity = quadrature_near_singularity or quadrature
        if backend_short is None:
            backend_short = NaiveShortRangeBackend() if isinstance(splitting, NoSplitting) else CellListsBackend(2)
        if backend_long is None:
            backend_long = NonuniformFFTsBackend()
        if lia_segment_fraction is not None and not (0 < lia_segment_fraction <= 1):
            raise ValueError("lia_segment_fraction must be in (0, 1]")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if not isinstance(splitting, NoSplitting):
            # params.jl:99-106
            rcut_max = min(backend_short.max_cutoff_distance(L) for L in splitting.Ls)
            if splitting.rcut > rcut_max:
                raise ValueError(f"cutoff distance `rcut = {splitting.rcut}` is larger than that allowed by the "
                                 f"{type(backend_short).__name__} backend.")
            if not 2 * splitting.rcut <= min(splitting.Ls):
                raise ValueError(f"cutoff distance `rcut = {splitting.rcut}` is too large. It must be less than half "
                                 f"the cell unit size `L` in each direction: Ls = {splitting.Ls}.")
        self.Gamma, self.a, self.Delta = float(Gamma), float(a), float(Delta)
        self.splitting = splitting
        self.quadrature = quadrature
        self.quadrature_near_singularity = quadrature_near_singularity
        self.backend_short, self.backend_long = backend_short, backend_long
        self.longrange_truncate_spherical = bool(longrange_truncate_spherical)
        self.lia_segment_fraction = None if lia_segment_fraction is None else float(lia_segment_fraction)
        self.avoid_explicit_erf = bool(avoid_explicit_erf)
        self.precision = precision
        self.device = int(device)
        self.extra = {}

    @property
    def Ls(self):
        return self.splitting.Ls

    @property
    def is_periodic(self):
        return not isinstance(self.splitting, NoSplitting)

    def with_(self, **kw):
        """Copy with some constructor keywords replaced."""
        base = dict(Gamma=self.Gamma, a=self.a, Delta=self.Delta, splitting=self.splitting,
                    quadrature=self.quadrature, quadrature_near_singularity=self.quadrature_near_singularity,
                    backend_short=self.backend_short, backend_long=self.backend_long,
                    longrange_truncate_spherical=self.longrange_truncate_spherical,
                    lia_segment_fraction=self.lia_segment_fraction, avoid_explicit_erf=self.avoid_explicit_erf,
                    precision=self.precision, device=self.device)
        base.update(kw)
        return ParamsBiotSavart(**base)


def kelvin_wave_period(lam: float, *, a: float, Delta: float, Gamma: float) -> float:
    """Period of a small-amplitude Kelvin wave of wavelength `lam` (params.jl:502-507); the
    reference's AdaptBasedOnSegmentLength sets dt = gamma * kelvin_wave_period(min segment length)."""
    return 2 * lam ** 2 / Gamma / (math.log(lam / (math.pi * a)) + 0.5 - (Delta + 0.5772156649015329))
