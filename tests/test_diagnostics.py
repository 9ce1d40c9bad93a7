"""Energy and helicity spectra on the device against their CPU oracle (numpy restatement of
Diagnostics/spectra.jl on the same vorticity coefficients) and the oracle's own Fourier field."""

import math

import numpy as np
import pytest

from conftest import load_package
from oracle import spectra_ref

vp = load_package()
from vortexpasta_b200 import diagnostics  # noqa: E402


def test_oracle_energy_spectrum_single_mode():
    """One vorticity mode w at k = (0, 2, 0) (dk = 1): E lands in bin 2 with weight 1/2 (kx = 0
    plane) as |w|^2 / k^2 / dk."""
    Ns = 8
    kx = np.arange(Ns // 2 + 1, dtype=float)
    ky = np.fft.fftfreq(Ns, 1 / Ns)
    field = [np.zeros((Ns // 2 + 1, Ns, Ns), complex) for _ in range(3)]
    field[0][0, 2, 0] = 3.0 + 4.0j
    E = spectra_ref.spectrum(field, (kx, ky, ky), np.arange(Ns // 2 + 1, dtype=float), "energy")
    assert E[2] == pytest.approx(0.5 * 25.0 / 4.0)
    assert np.count_nonzero(E) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["energy", "helicity"])
def test_spectra_match_oracle(kind):
    fs, p = vp.configs.tangle20k()
    fs = fs[:30]
    cache = vp.init_cache(p)
    try:
        vp.velocity_on_nodes(cache, fs)
        ks, Ek = (diagnostics.energy_spectrum if kind == "energy" else diagnostics.helicity_spectrum)(cache)
        lr = vp.get_longrange_field_fourier(cache)
    finally:
        cache.close()
    V = float(np.prod(p.splitting.Ls))
    ref = spectra_ref.spectrum(lr["field"], lr["wavenumbers"], ks, kind, V)
    assert np.abs(Ek - ref).max() <= 1e-12 * np.abs(ref).max()
    assert ks[0] == 0 and len(ks) == p.splitting.Ns[0] // 2 + 1
    if kind == "energy":
        assert (Ek >= 0).all() and Ek.sum() > 0


@pytest.mark.gpu
def test_spectrum_needs_a_long_range_field():
    fs, p = vp.configs.ring64()
    cache = vp.init_cache(p)
    try:
        with pytest.raises(RuntimeError, match="not supported"):
            diagnostics.energy_spectrum(cache)
    finally:
        cache.close()
