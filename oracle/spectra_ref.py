"""CPU oracle of the energy and helicity spectra (test infrastructure only).

numpy restatement of src/Diagnostics/spectra.jl:127-232 (_compute_spectrum_impl!: bin
n = 1 + trunc(|k|/dk + 1/2), weight 1/2 on the kx = 0 plane with Hermitian symmetry, each
value divided by dk) with the from-vorticity integrands of spectra.jl:95-104 (|w|^2 / k^2) and
spectra_helicity.jl:57-67 (2 V Re[(i k x w)^* . w] / k^2), applied to the vorticity
coefficients `field` (three complex arrays (Ns0/2+1, Ns1, Ns2), x first) with wavenumbers
(kx, ky, kz).
"""

from __future__ import annotations

import numpy as np


def spectrum(field, wavenumbers, ks, kind: str, V: float = 1.0):
    kx, ky, kz = (np.asarray(k, dtype=np.float64) for k in wavenumbers)
    KX, KY, KZ = np.meshgrid(kx, ky, kz, indexing="ij")
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    beta = np.where(k2 == 0, 1.0, 1.0 / np.where(k2 == 0, 1.0, k2))
    w = [np.asarray(c, dtype=np.complex128) for c in field]
    if kind == "energy":
        v = beta * sum(np.abs(c) ** 2 for c in w)
    else:
        c0 = KY * w[2] - KZ * w[1]
        c1 = KZ * w[0] - KX * w[2]
        c2 = KX * w[1] - KY * w[0]
        ulap = [1j * c0, 1j * c1, 1j * c2]
        v = 2 * V * beta * np.real(sum(np.conj(u) * c for u, c in zip(ulap, w)))
    dk = ks[1] - ks[0]
    factor = np.where(KX == 0, 0.5, 1.0)
    n = (np.sqrt(k2) / dk + 0.5).astype(np.int64)
    out = np.zeros(len(ks))
    keep = n < len(ks)
    np.add.at(out, n[keep], (factor * v / dk)[keep])
    return out
