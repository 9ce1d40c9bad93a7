"""Unclosed (infinite) filaments with an end-to-end offset and the background-vorticity correction,
through the C ABI, against the oracle.

Reference: ClosedFilament's Xoffset (src/Filaments/closed_filament.jl:118-132, 196-207), the
periodised spline (src/Filaments/spline/spline.jl:163-194, spline/quintic.jl:9-17) and
background_vorticity_correction! (src/BiotSavart/BiotSavart.jl:255-286); test cases shaped like
test/infinite_lines.jl:19-28, 105-160 and test/background_vorticity.jl:34-81.
"""

import math

import numpy as np
import pytest

TOL = 1e-10
MIXED_TOL = 1e-5
L = 2 * math.pi


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def helical_lines(vp, Np=64, Nx=4):
    """4x4 aligned periodic lines with identical helical perturbations (test/background_vorticity.jl:34-50)."""
    xs = np.linspace(0, L, 2 * Nx + 1)[1::2]
    return [vp.curves.periodic_line(Np, L, r=lambda t: np.exp(4j * np.pi * t) / 100, translate=(x, y, L / 2))
            for x in xs for y in xs]


def opposite_lines(vp, N=32):
    """Four helical lines of alternating orientation, total offset zero (test/infinite_lines.jl:105-121)."""
    A, k, h = 0.08, 2, L / 4
    out = []
    for (x, y, sign) in ((h, h, 1), (h, 3 * h, -1), (3 * h, h, -1), (3 * h, 3 * h, 1)):
        t = np.linspace(-0.5, 0.5, N + 1)[:N]
        X = np.stack([x + A * np.cos(2 * np.pi * k * t), y + A * np.sin(2 * np.pi * k * t), (0.5 + sign * t) * L],
                     axis=1)
        out.append(vp.curves.InfiniteFilament(X, (0.0, 0.0, sign * L)))
    return out


def params(vp, splitting, Ng, **kw):
    sp = (vp.GaussianSplitting(Ls=L, rtol=1e-6, Ns=Ng) if splitting == "gaussian"
          else vp.KaiserBesselSplitting(Ls=L, rtol=1e-6, Ns=(Ng,) * 3))
    return vp.ParamsBiotSavart(Gamma=2.0, a=1e-8, splitting=sp, backend_long=vp.NonuniformFFTsBackend(1.5, 4), **kw)


def gpu_fields(vp, p, fs):
    cache = vp.init_cache(p)
    try:
        vs = [np.zeros((len(f), 3)) for f in fs]
        ps = [np.zeros((len(f), 3)) for f in fs]
        vp.compute_on_nodes_({"velocity": vs, "streamfunction": ps}, cache, fs)
    finally:
        cache.close()
    return np.concatenate(vs), np.concatenate(ps)


def test_periodic_line_geometry(vp):
    """PeriodicLine nodes and end-to-end offset (periodic_line.jl, define_curve with orientation)."""
    f = vp.curves.periodic_line(8, L, r=lambda t: 0.1 * np.exp(2j * np.pi * t), translate=(1.0, 2.0, 3.0))
    g = vp.curves.periodic_line(8, L, r=lambda t: 0.1 * np.exp(2j * np.pi * t), translate=(1.0, 2.0, 3.0), sign=-1)
    np.testing.assert_allclose(vp.curves.end_to_end_offset(f), [0, 0, L])
    np.testing.assert_allclose(vp.curves.end_to_end_offset(g), [0, 0, -L])
    np.testing.assert_allclose(g, f[::-1], atol=1e-14)  # orientation -1 reverses the parameter
    np.testing.assert_array_equal(vp.curves.end_to_end_offset(np.zeros((5, 3))), np.zeros(3))
    assert isinstance(f[1:], vp.curves.InfiniteFilament) and np.all(f[1:].offset == f.offset)


@pytest.mark.gpu
def test_point_data_of_unclosed_filaments(vp, oracle, built_lib):
    fs = helical_lines(vp)[:3] + opposite_lines(vp)[:2] + [vp.curves.ring(7, 0.5, center=(2, 2, 2))]
    p = params(vp, "gaussian", 32)
    cache = vp.init_cache(p)
    try:
        cache.set_filaments(fs)
        g = cache.pointdata()
    finally:
        cache.close()
    o = oracle.point_data(p, fs)
    for k in ("nodes", "d1", "d2", "dm", "dp", "points", "charges"):
        assert rel(g[k], o[k]) < (1e-10 if k == "d2" else 1e-12), k


@pytest.mark.gpu
@pytest.mark.parametrize("splitting", ["gaussian", "kaiser_bessel"])
def test_unclosed_filaments_match_oracle(vp, oracle, built_lib, splitting):
    """Non-zero mean vorticity (16 aligned lines): velocity and corrected streamfunction vs the oracle."""
    fs = helical_lines(vp)
    p = params(vp, splitting, 32)
    v, psi = gpu_fields(vp, p, fs)
    vo, po, _ = oracle.compute_on_nodes(p, fs, streamfunction=True)
    assert rel(v, vo) < TOL and rel(psi, po) < TOL
    vm, pm = gpu_fields(vp, p.with_(precision="mixed"), fs)
    assert rel(vm, vo) < MIXED_TOL and rel(pm, po) < MIXED_TOL


@pytest.mark.gpu
def test_opposite_lines_and_rings_match_oracle(vp, oracle, built_lib):
    """Lines of both orientations (offsets add to zero: no correction) together with closed rings."""
    fs = opposite_lines(vp) + [vp.curves.ring(40, 0.6, center=(3.0, 3.2, 1.0)),
                               vp.curves.ring(24, 0.4, center=(0.5, 5.5, 4.0))]
    p = vp.configs.params_for(L / 4, 3.5, 32, 4)
    v, psi = gpu_fields(vp, p, fs)
    vo, po, _ = oracle.compute_on_nodes(p, fs, streamfunction=True)
    assert rel(v, vo) < TOL and rel(psi, po) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("splitting", ["gaussian", "kaiser_bessel"])
def test_unclosed_filaments_independent_of_splitting(vp, built_lib, splitting):
    """test/background_vorticity.jl:57-81 on the GPU: Ns = 32 and 64 agree to 2e-6 (velocity) and 2e-7
    (streamfunction) per filament."""
    fs = helical_lines(vp)
    (v1, p1), (v2, p2) = [gpu_fields(vp, params(vp, splitting, Ng), fs) for Ng in (32, 64)]
    Np = 64
    for i in range(len(fs)):
        s = slice(i * Np, (i + 1) * Np)
        assert np.linalg.norm(v1[s] - v2[s]) <= 2e-6 * np.linalg.norm(v2[s])
        assert np.linalg.norm(p1[s] - p2[s]) <= 2e-7 * np.linalg.norm(p2[s])


@pytest.mark.gpu
def test_straight_line_has_no_velocity(vp, built_lib):
    f = vp.curves.periodic_line(32, L, translate=(L / 3, L / 5, L / 2))
    v, psi = gpu_fields(vp, vp.configs.params_for(L / 4, 3.5, 32, 5), [f])
    assert np.abs(v).max() < 1e-7 * np.abs(psi).max()
    assert np.ptp(psi[:, 2]) < 1e-8 * np.abs(psi[:, 2]).max()


@pytest.mark.gpu
def test_offsets_must_match_filament_count(vp, built_lib):
    from vortexpasta_b200 import _lib
    p = vp.configs.params_for(L / 4, 3.5, 32, 4)
    cache = vp.init_cache(p)
    try:
        cache.set_end_to_end_offsets(np.array([[0, 0, L], [0, 0, L]]))
        nodes, offsets = vp.curves.concat([vp.curves.periodic_line(16, L)])
        with pytest.raises(vp.VpbsError, match="offsets were set for 2 filaments"):
            _lib.check(cache._lib.vpbs_set_filaments(cache.handle, 1, offsets.ctypes.data_as(_lib.c_int64_p),
                                                     nodes.ctypes.data_as(_lib.ct.c_void_p), 0), cache.handle, "set")
    finally:
        cache.close()
