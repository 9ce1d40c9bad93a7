"""Diagnostics computed on the device from the long-range Fourier field: the energy and
helicity spectra of VortexPasta.Diagnostics (src/Diagnostics/spectra.jl:1-232,
spectra_helicity.jl:1-76), same names, arguments, binning and errors."""

from __future__ import annotations

import numpy as np

from . import _lib
from .biotsavart import BiotSavartCache


def init_spectrum(cache: BiotSavartCache):
    """init_spectrum (spectra.jl:63-82): wavenumbers k_n = n dk (dk = 2 pi / L_x) up to the
    largest kx of the Fourier grid, and an uninitialised spectrum of the same length."""
    sp = cache.params.splitting
    dk = 2 * np.pi / sp.Ls[0]
    M = sp.Ns[0] // 2 + 1  # kx modes with Hermitian symmetry
    ks = dk * np.arange(M)
    return ks, np.empty_like(ks)


def _spectrum(kind: int, out: np.ndarray, ks: np.ndarray, cache: BiotSavartCache):
    if len(ks) != len(out):
        raise ValueError("incompatible dimensions of vectors")
    if ks[0] != 0:
        raise ValueError("output wavenumbers should include k = 0")
    q = cache.state.quantity
    if q not in ("velocity", "vorticity") or cache.state.smoothing_scale != 0:
        raise RuntimeError(f"the current state of the long-range cache ({cache.state}) is currently not supported")
    if kind == 0 and q == "velocity":
        kind = 2  # |v_k|^2 instead of |w_k|^2 / k^2 (spectra.jl:95-98)
    dk = float(ks[1] - ks[0]) if len(ks) > 1 else 2 * np.pi / cache.params.splitting.Ls[0]
    buf = np.zeros(len(ks))
    _lib.check(cache._lib.vpbs_spectrum(cache.handle, kind, dk, _lib.dptr(buf), len(buf)), cache.handle,
               "helicity_spectrum!" if kind == 1 else "energy_spectrum!")
    out[...] = buf
    return ks, out


def energy_spectrum_(Ek: np.ndarray, ks: np.ndarray, cache: BiotSavartCache):
    """energy_spectrum! (spectra.jl:89-108) from the velocity or (unsmoothed) vorticity the
    cache holds."""
    return _spectrum(0, Ek, ks, cache)


def energy_spectrum(cache: BiotSavartCache):
    """energy_spectrum (spectra.jl:84-87) -> (ks, Ek)."""
    ks, Ek = init_spectrum(cache)
    return energy_spectrum_(Ek, ks, cache)


def helicity_spectrum_(Hk: np.ndarray, ks: np.ndarray, cache: BiotSavartCache):
    """helicity_spectrum! (spectra_helicity.jl:48-73) from the velocity or (unsmoothed)
    vorticity the cache holds (the same value from either)."""
    return _spectrum(1, Hk, ks, cache)


def helicity_spectrum(cache: BiotSavartCache):
    """helicity_spectrum (spectra_helicity.jl:43-46) -> (ks, Hk)."""
    ks, Hk = init_spectrum(cache)
    return helicity_spectrum_(Hk, ks, cache)
