"""Long-range diagnostics on the device against their CPU oracle (numpy restatements in
oracle/spectra_ref.py of Diagnostics/spectra.jl, spectra_helicity.jl, the coarse-graining kernels
of longrange.jl and the ExactSumBackend interpolation): energy and helicity spectra from the
velocity and from the vorticity state, coarse-grained vorticity and its values on the nodes."""

import math

import numpy as np
import pytest

from conftest import load_package
from oracle import spectra_ref

vp = load_package()
from vortexpasta_b200 import diagnostics  # noqa: E402


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def test_oracle_energy_spectrum_single_mode():
    """One vorticity mode w at k = (0, 2, 0) (dk = 1): E lands in bin 2 with weight 1/2 (kx = 0
    plane) as |w|^2 / k^2 / dk; from the velocity state the same mode holds v = i k x w / k^2
    and gives the same energy (w is orthogonal to k)."""
    Ns = 8
    kx = np.arange(Ns // 2 + 1, dtype=float)
    ky = np.fft.fftfreq(Ns, 1 / Ns)
    field = [np.zeros((Ns // 2 + 1, Ns, Ns), complex) for _ in range(3)]
    field[0][0, 2, 0] = 3.0 + 4.0j
    ks = np.arange(Ns // 2 + 1, dtype=float)
    E = spectra_ref.spectrum(field, (kx, ky, ky), ks, "energy")
    assert E[2] == pytest.approx(0.5 * 25.0 / 4.0)
    assert np.count_nonzero(E) == 1
    v = spectra_ref.velocity_from_vorticity(field, (kx, ky, ky))
    Ev = spectra_ref.spectrum(v, (kx, ky, ky), ks, "energy", quantity="velocity")
    np.testing.assert_allclose(Ev, E, rtol=1e-15)


def test_oracle_coarse_graining_and_exact_sum():
    """The curl of the Biot-Savart velocity of a solenoidal mode is the mode itself; the exact
    type-2 sum of a single mode is 2 Re[w e^{ik.x}] (Hermitian doubling)."""
    Ns = 8
    kx = np.arange(Ns // 2 + 1, dtype=float)
    ky = np.fft.fftfreq(Ns, 1 / Ns)
    ks = (kx, ky, ky)
    field = [np.zeros((Ns // 2 + 1, Ns, Ns), complex) for _ in range(3)]
    field[2][1, 1, 0] = 0.5 - 0.25j  # w along z, k = (1, 1, 0): k . w = 0
    v = spectra_ref.velocity_from_vorticity(field, ks)
    w = spectra_ref.coarse_grained_vorticity(v, ks, 0.3, 0.0, "velocity")
    op = math.exp(-2 * 0.3 ** 2 / 2)
    np.testing.assert_allclose(w[2], op * field[2], atol=1e-15)
    x = np.array([[0.3, -1.2, 2.0], [4.0, 0.1, 5.5]])
    u = spectra_ref.interpolate_exact(field, ks, x)
    np.testing.assert_allclose(u[:, 2], 2 * np.real((0.5 - 0.25j) * np.exp(1j * (x[:, 0] + x[:, 1]))), rtol=1e-14)


def evaluate(p, fs, **kw):
    cache = vp.init_cache(p)
    vs = [np.zeros_like(f) for f in fs]
    vp.compute_on_nodes_({"velocity": vs}, cache, fs, **kw)
    return cache


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["energy", "helicity"])
def test_spectra_match_oracle(kind):
    """From the velocity state (after the evaluation) and from the vorticity state (inside
    callback_vorticity), each against the oracle on the same held field."""
    fs, p = vp.configs.tangle20k()
    fs = fs[:30]
    fn = diagnostics.energy_spectrum if kind == "energy" else diagnostics.helicity_spectrum
    seen = {}

    def inside(c):
        seen["spec"] = fn(c)
        seen["lr"] = vp.get_longrange_field_fourier(c)

    cache = evaluate(p, fs, callback_vorticity=inside)
    try:
        ks, Ek = fn(cache)
        lr = vp.get_longrange_field_fourier(cache)
    finally:
        cache.close()
    V = float(np.prod(p.splitting.Ls))
    assert lr["state"].quantity == "velocity"
    ref = spectra_ref.spectrum(lr["field"], lr["wavenumbers"], ks, kind, V, quantity="velocity")
    assert np.abs(Ek - ref).max() <= 1e-12 * np.abs(ref).max()
    assert ks[0] == 0 and len(ks) == p.splitting.Ns[0] // 2 + 1
    ks_w, Ew = seen["spec"]
    ref_w = spectra_ref.spectrum(seen["lr"]["field"], lr["wavenumbers"], ks_w, kind, V, quantity="vorticity")
    assert np.abs(Ew - ref_w).max() <= 1e-12 * np.abs(ref_w).max()
    if kind == "energy":
        assert (Ek >= 0).all() and Ek.sum() > 0
        # the two states differ only by the non-solenoidal part of the discrete vorticity
        assert rel(Ek, Ew) < 1e-2
    else:
        np.testing.assert_allclose(Ek, Ew, rtol=1e-9, atol=1e-12 * np.abs(Ew).max())


@pytest.mark.gpu
def test_coarse_grained_vorticity_and_nodes():
    """to_coarse_grained_vorticity! from the velocity state (curl then filter), again from the
    resulting vorticity state (filter by exp(-k^2 (l^2 - l_old^2)/2)), then the coarse-grained
    vorticity on the nodes (type-2 NUFFT, default callback) against the exact Fourier sum."""
    fs, p = vp.configs.tangle20k()
    fs = fs[:12]
    p = p.with_(backend_long=vp.NonuniformFFTsBackend(1.5, 6))
    cache = evaluate(p, fs)
    try:
        v = vp.get_longrange_field_fourier(cache)
        lr1 = vp.to_coarse_grained_vorticity_(cache, 0.2)
        assert lr1["state"].quantity == "vorticity" and lr1["state"].smoothing_scale == 0.2
        ref1 = spectra_ref.coarse_grained_vorticity(v["field"], v["wavenumbers"], 0.2, 0.0, "velocity")
        assert rel(np.stack(lr1["field"]), np.stack(ref1)) < 1e-12
        with pytest.raises(RuntimeError, match="not supported"):
            diagnostics.energy_spectrum(cache)
        lr2 = vp.to_coarse_grained_vorticity_(cache, 0.3)
        ref2 = spectra_ref.coarse_grained_vorticity(lr1["field"], v["wavenumbers"], 0.3, 0.2, "vorticity")
        assert rel(np.stack(lr2["field"]), np.stack(ref2)) < 1e-12
        w_nodes = vp.interpolate_to_physical(cache)
    finally:
        cache.close()
    nodes = np.concatenate(fs)[:256]  # the exact sum costs O(nodes x modes) on the CPU
    ref = spectra_ref.interpolate_exact(lr2["field"], v["wavenumbers"], nodes)
    assert np.abs(w_nodes[:256] - ref).max() <= 1e-8 * np.abs(ref).max()


@pytest.mark.gpu
def test_interpolated_velocity_matches_exact_sum():
    """interpolate_to_physical of the held (unsmoothed, unfiltered) velocity field against the
    exact type-2 sum of the same coefficients."""
    fs, p = vp.configs.tangle20k()
    fs = fs[:8]
    p = p.with_(backend_long=vp.NonuniformFFTsBackend(1.5, 6))
    cache = evaluate(p, fs)
    try:
        lr = vp.get_longrange_field_fourier(cache)
        u = vp.interpolate_to_physical(cache)
    finally:
        cache.close()
    ref = spectra_ref.interpolate_exact(lr["field"], lr["wavenumbers"], np.concatenate(fs)[:256])
    assert np.abs(u[:256] - ref).max() <= 1e-8 * np.abs(ref).max()


@pytest.mark.gpu
def test_spectrum_needs_a_long_range_field():
    fs, p = vp.configs.ring64()
    cache = vp.init_cache(p)
    try:
        with pytest.raises(RuntimeError, match="not supported"):
            diagnostics.energy_spectrum(cache)
        with pytest.raises(RuntimeError, match="expected either the velocity or vorticity"):
            vp.to_coarse_grained_vorticity_(cache, 0.1)
    finally:
        cache.close()
