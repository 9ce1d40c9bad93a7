"""CPU oracle of the long-range diagnostics (test infrastructure only).

numpy restatements, applied to the Fourier coefficients `field` (three complex arrays
(Ns0/2+1, Ns1, Ns2), x first) with wavenumbers (kx, ky, kz):

* ``spectrum``: src/Diagnostics/spectra.jl:127-232 (_compute_spectrum_impl!: bin
  n = 1 + trunc(|k|/dk + 1/2), weight 1/2 on the kx = 0 plane with Hermitian symmetry, each
  value divided by dk) with the integrands of spectra.jl:95-104 (from velocity |u|^2, from
  vorticity |w|^2 / k^2) and spectra_helicity.jl:57-67 (from velocity 2 V Re[u^* . (i k x u)],
  from vorticity 2 V Re[(i k x w)^* . w] / k^2);
* ``velocity_from_vorticity`` / ``streamfunction_from_vorticity``: fourier_biot_savart_kernel!
  and fourier_inverse_laplacian_kernel! (src/BiotSavart/longrange/longrange.jl:114-141);
* ``coarse_grained_vorticity``: coarse_grained_curl_kernel! / coarse_graining_kernel!
  (longrange.jl:160-186) as to_coarse_grained_vorticity! applies them (longrange.jl:273-293);
* ``interpolate_exact``: the ExactSumBackend type-2 sum with Hermitian doubling
  (src/BiotSavart/longrange/backends/exact_sum.jl:91-121), default callback.
"""

from __future__ import annotations

import numpy as np


def _grids(wavenumbers):
    kx, ky, kz = (np.asarray(k, dtype=np.float64) for k in wavenumbers)
    return np.meshgrid(kx, ky, kz, indexing="ij")


def _k2inv(k2):
    return np.where(k2 == 0, 0.0, 1.0 / np.where(k2 == 0, 1.0, k2))


def _cross(K, w):
    KX, KY, KZ = K
    return [KY * w[2] - KZ * w[1], KZ * w[0] - KX * w[2], KX * w[1] - KY * w[0]]


def spectrum(field, wavenumbers, ks, kind: str, V: float = 1.0, quantity: str = "vorticity"):
    K = _grids(wavenumbers)
    KX = K[0]
    k2 = sum(k ** 2 for k in K)
    beta = np.where(k2 == 0, 1.0, 1.0 / np.where(k2 == 0, 1.0, k2))
    w = [np.asarray(c, dtype=np.complex128) for c in field]
    if quantity == "velocity":
        if kind == "energy":
            v = sum(np.abs(c) ** 2 for c in w)
        else:
            om = [1j * c for c in _cross(K, w)]
            v = 2 * V * np.real(sum(np.conj(u) * o for u, o in zip(w, om)))
    elif kind == "energy":
        v = beta * sum(np.abs(c) ** 2 for c in w)
    else:
        ulap = [1j * c for c in _cross(K, w)]
        v = 2 * V * beta * np.real(sum(np.conj(u) * c for u, c in zip(ulap, w)))
    dk = ks[1] - ks[0]
    factor = np.where(KX == 0, 0.5, 1.0)
    n = (np.sqrt(k2) / dk + 0.5).astype(np.int64)
    out = np.zeros(len(ks))
    keep = n < len(ks)
    np.add.at(out, n[keep], (factor * v / dk)[keep])
    return out


def velocity_from_vorticity(field, wavenumbers):
    K = _grids(wavenumbers)
    k2inv = _k2inv(sum(k ** 2 for k in K))
    w = [np.asarray(c, dtype=np.complex128) for c in field]
    return tuple(1j * c * k2inv for c in _cross(K, w))


def streamfunction_from_vorticity(field, wavenumbers):
    K = _grids(wavenumbers)
    k2inv = _k2inv(sum(k ** 2 for k in K))
    return tuple(np.asarray(c, dtype=np.complex128) * k2inv for c in field)


def coarse_grained_vorticity(field, wavenumbers, ell: float, ell_old: float, quantity: str):
    """`field` holds the velocity (quantity "velocity": the curl i k x u is filtered) or the
    vorticity ("vorticity": filtered as is)."""
    K = _grids(wavenumbers)
    k2 = sum(k ** 2 for k in K)
    op = np.exp(-k2 * (ell ** 2 - ell_old ** 2) / 2)
    u = [np.asarray(c, dtype=np.complex128) for c in field]
    if quantity == "velocity":
        return tuple(op * 1j * c for c in _cross(K, u))
    if quantity == "vorticity":
        return tuple(op * c for c in u)
    raise ValueError(quantity)


def interpolate_exact(field, wavenumbers, points):
    kx, ky, kz = (np.asarray(k, dtype=np.float64) for k in wavenumbers)
    K = _grids(wavenumbers)
    weight = np.where((K[0] == kx[0]) | (K[0] == kx[-1]), 1.0, 2.0).ravel()
    kvec = np.stack([k.ravel() for k in K])  # (3, nmodes)
    u = np.stack([np.asarray(c, dtype=np.complex128).ravel() for c in field])  # (3, nmodes)
    pts = np.asarray(points, dtype=np.float64)
    out = np.zeros((len(pts), 3))
    for i0 in range(0, len(pts), 256):
        z = np.exp(1j * (pts[i0:i0 + 256] @ kvec))  # (n, nmodes)
        out[i0:i0 + 256] = np.real((z * weight) @ u.T)
    return out
