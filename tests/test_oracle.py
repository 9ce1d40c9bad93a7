"""Pin the CPU oracle against the reference's own known-answer tests.

The reference (Julia) cannot run here, so the oracle is checked against what its tests
assert: analytic vortex-ring velocity/streamfunction (test/ring.jl), NUFFT vs exact Fourier
sums (test/trefoil.jl:135-245), cell lists vs naive pair enumeration (test/cell_lists.jl,
test/trefoil.jl:247-282) and independence from the Ewald parameter (test/trefoil.jl:299-329).
"""

import math

import numpy as np
import pytest


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def ring_velocity(Gamma, R, a, Delta):
    """test/ring.jl:41: U = Gamma/(4 pi R) (ln(8R/a) - Delta)."""
    return Gamma / (4 * math.pi * R) * (math.log(8 * R / a) - Delta)


def ring_streamfunction(Gamma, R, a, Delta):
    """test/ring.jl:43: psi . t = Gamma/(2 pi) (ln(8R/a) - (1 + Delta))."""
    return Gamma / (2 * math.pi) * (math.log(8 * R / a) - (1 + Delta))


def test_gauss_legendre(oracle):
    for n in (1, 2, 3, 4, 8):
        z, w = oracle.gl_rule(n)
        x, ww = np.polynomial.legendre.leggauss(n)
        np.testing.assert_allclose(z, (x + 1) / 2, rtol=0, atol=1e-15)
        np.testing.assert_allclose(w, ww / 2, rtol=0, atol=1e-15)


def test_fft_size_rule(oracle, vp):
    from vortexpasta_b200 import _lib
    assert [oracle.fft_size(n, 1.5) for n in (32, 128, 512)] == [48, 192, 768]
    for n in (7, 30, 90, 100, 120, 250):
        for s in (1.25, 1.5, 2.0):
            m = oracle.fft_size(n, s)
            assert m >= s * n - 1e-9 and m % 2 == 0
            assert _lib.load().vpbs_fft_size(n, s) == m


@pytest.mark.parametrize("quad,lia_fraction,rtol_v,rtol_psi", [(4, 0.4, 1e-4, 1e-4), (3, None, 1e-4, 1e-3)])
def test_ring_open_domain_analytic(vp, oracle, quad, lia_fraction, rtol_v, rtol_psi):
    """test/ring.jl:43-157: non-periodic ring, N = 32, Gamma = 2.4, a = 1e-6, quintic, GL(4)."""
    R, N, Gamma, a, Delta = math.pi / 3, 32, 2.4, 1e-6, 0.25
    f = vp.curves.ring(N, R, center=(math.pi,) * 3)
    p = vp.ParamsBiotSavart(Gamma=Gamma, a=a, Delta=Delta, alpha=0, quadrature=vp.GaussLegendre(quad),
                            lia_segment_fraction=lia_fraction)
    v, psi, _ = oracle.compute_on_nodes(p, [f], velocity=True, streamfunction=True)
    U = np.linalg.norm(v.mean(axis=0))
    assert abs(U - ring_velocity(Gamma, R, a, Delta)) / U < rtol_v
    assert v[:, 2].std() < 1e-12 * U  # uniform translation along the normal
    t = vp.curves.node_parameters(N)
    tang = np.stack([-np.sin(2 * np.pi * t), np.cos(2 * np.pi * t), np.zeros(N)], axis=1)
    psi_para = (psi * tang).sum(axis=1)
    psi_perp = np.linalg.norm(psi - psi_para[:, None] * tang, axis=1)
    assert np.max(psi_perp / np.abs(psi_para)) < 1e-10  # psi parallel to the tangent
    assert abs(psi_para.mean() - ring_streamfunction(Gamma, R, a, Delta)) / abs(psi_para.mean()) < rtol_psi


def test_lia_only_plus_nonlia_is_total(vp, oracle):
    """test/ring.jl:139-143: v_total = v_LIA + v_nonLIA."""
    f = vp.curves.ring(32, math.pi / 3, center=(math.pi,) * 3)
    p = vp.ParamsBiotSavart(Gamma=2.4, a=1e-6, alpha=0, quadrature=vp.GaussLegendre(4), lia_segment_fraction=0.4)
    vt, _, _ = oracle.compute_on_nodes(p, [f])
    vl, _, _ = oracle.compute_on_nodes(p, [f], LIA="only")
    vn, _, _ = oracle.compute_on_nodes(p, [f], LIA=False)
    np.testing.assert_allclose(vt, vl + vn, rtol=1e-12, atol=1e-12 * np.abs(vt).max())


def test_lia_segment_fraction_ring(vp, oracle):
    """test/ring.jl:236-270: N = 64 quintic ring, fraction 0.2, GL(8) near singularity: error < 2e-6."""
    R, N = math.pi / 3, 64
    f = vp.curves.ring(N, R, center=(math.pi,) * 3)
    p = vp.ParamsBiotSavart(Gamma=1.0, a=1e-8, alpha=0, lia_segment_fraction=0.2,
                            quadrature_near_singularity=vp.GaussLegendre(8))
    v, _, _ = oracle.compute_on_nodes(p, [f])
    vz = v[:, 2]
    assert vz.std() / vz.mean() < 1e-12
    assert abs(vz.mean() - ring_velocity(1.0, R, 1e-8, 0.25)) / vz.mean() < 2e-6


@pytest.mark.parametrize("m,tol", [(4, 3e-6), (5, 1e-7), (6, 1e-9)])
def test_nufft_vs_exact_sum(vp, oracle, m, tol):
    """test/trefoil.jl:135-245: long-range velocity/streamfunction by NUFFT vs ExactSumBackend."""
    fs, p = vp.configs.ring64()
    p = p.with_(backend_long=vp.NonuniformFFTsBackend(1.5, m))
    vn, pn, _ = oracle.compute_on_nodes(p, fs, streamfunction=True, shortrange=False)
    ve, pe, _ = oracle.compute_on_nodes(p, fs, streamfunction=True, shortrange=False, exact=True)
    assert rel(vn, ve) < tol
    assert rel(pn, pe) < tol


def test_vorticity_fourier_vs_exact(vp, oracle):
    fs, p = vp.configs.ring64()
    pd = oracle.point_data(p, fs)
    un = oracle.vorticity_fourier(p, pd["points"], pd["charges"])
    ue = oracle.vorticity_fourier(p, pd["points"], pd["charges"], exact=True)
    assert np.abs(un - ue).max() < 1e-5 * np.abs(ue).max()
    # Hermitian-symmetry zeroing (longrange.jl:556-583)
    assert np.all(ue[:, :, :, -1] == 0) and np.all(ue[:, :, 16, :] == 0) and np.all(ue[:, 16, :, :] == 0)


def test_alpha_independence(vp, oracle):
    """test/trefoil.jl:299-329: results independent of the splitting parameter."""
    fs = vp.configs.tangle(3, 40, seed=3)
    L = vp.configs.L
    outs = []
    for rcut in (0.8, 1.0, 1.3):
        beta = 5.0
        alpha = beta / rcut
        Ns = vp.kmax_to_gridsize(2 * alpha * beta, L)
        p = vp.ParamsBiotSavart(Gamma=1.0, a=1e-8, splitting=vp.GaussianSplitting(Ls=L, alpha=alpha, rcut=rcut, Ns=Ns),
                                backend_long=vp.NonuniformFFTsBackend(1.5, 6))
        outs.append(oracle.compute_on_nodes(p, fs, streamfunction=True)[:2])
    for v, psi in outs[1:]:
        assert rel(v, outs[0][0]) < 1e-6
        assert rel(psi, outs[0][1]) < 1e-6


def test_cell_lists_vs_naive_pairs(vp, oracle):
    """test/cell_lists.jl:184-282 and test/trefoil.jl:247-282: identical pairs and sums."""
    fs, p = vp.configs.tangle20k()
    fs = fs[:20]
    vc, pc, sc = oracle.compute_on_nodes(p, fs, streamfunction=True, longrange=False)
    pn = p.with_(backend_short=vp.NaiveShortRangeBackend())
    vn, pnn, sn = oracle.compute_on_nodes(pn, fs, streamfunction=True, longrange=False)
    assert sc["pairs_in_range"] == sn["pairs_in_range"]
    assert sc["pairs_candidates"] < sn["pairs_candidates"]
    assert rel(vc, vn) < 1e-12 and rel(pc, pnn) < 1e-12


def test_avoid_explicit_erf_equivalence(vp, oracle):
    """avoid_explicit_erf = true/false give the same result (test/trefoil.jl:299-329 loop)."""
    fs, p = vp.configs.ring64()
    v1, p1, _ = oracle.compute_on_nodes(p, fs, streamfunction=True)
    v2, p2, _ = oracle.compute_on_nodes(p.with_(avoid_explicit_erf=False), fs, streamfunction=True)
    assert rel(v1, v2) < 1e-10 and rel(p1, p2) < 1e-10


def test_golden_ring64(vp, oracle):
    """Regression against the committed fixture (tests/golden/make_golden.py)."""
    from pathlib import Path
    g = np.load(Path(__file__).parent / "golden" / "ring64.npz")
    fs, p = vp.configs.ring64()
    np.testing.assert_array_equal(np.concatenate(fs), g["nodes"])
    v, psi, st = oracle.compute_on_nodes(p, fs, streamfunction=True)
    assert rel(v, g["velocity"]) < 1e-13 and rel(psi, g["streamfunction"]) < 1e-13
    assert st["pairs_in_range"] == int(g["pairs_in_range"])


def _helical_lines(vp, Np=64, Nx=4):
    """The 4x4 array of aligned periodic lines with identical helical perturbations of the
    reference's test/background_vorticity.jl:34-50 (L = 2 pi, PeriodicLine(r = t -> cispi(4t) / 100))."""
    L = 2 * math.pi
    xs = np.linspace(0, L, 2 * Nx + 1)[1::2]
    return [vp.curves.periodic_line(Np, L, r=lambda t: np.exp(4j * np.pi * t) / 100, translate=(x, y, L / 2))
            for x in xs for y in xs]


@pytest.mark.parametrize("splitting", ["gaussian", "kaiser_bessel"])
def test_infinite_lines_independent_of_splitting(vp, oracle, splitting):
    """test/background_vorticity.jl:57-81: infinite lines with a non-zero mean vorticity give the same
    velocity (rtol 2e-6) and streamfunction (rtol 2e-7, thanks to the background-vorticity correction
    of BiotSavart.jl:255-286) with Ns = 32 and 64 (alpha changes by a factor 2)."""
    L = 2 * math.pi
    fs = _helical_lines(vp)
    assert all(np.allclose(vp.curves.end_to_end_offset(f), [0, 0, L]) for f in fs)
    res = []
    for Ng in (32, 64):
        sp = (vp.GaussianSplitting(Ls=L, rtol=1e-6, Ns=Ng) if splitting == "gaussian"
              else vp.KaiserBesselSplitting(Ls=L, rtol=1e-6, Ns=(Ng,) * 3))
        p = vp.ParamsBiotSavart(Gamma=2.0, a=1e-8, splitting=sp, backend_long=vp.NonuniformFFTsBackend(1.5, 4))
        v, psi, _ = oracle.compute_on_nodes(p, fs, streamfunction=True)
        # the correction the oracle applied: -(sum of offsets) Gamma / V * C
        back = -(16 * L) * 2.0 / L ** 3 * oracle.background_factor(p)
        res.append((v, psi, back))
    Np = 64
    for i in range(len(fs)):
        s = slice(i * Np, (i + 1) * Np)
        (v1, p1, b1), (v2, p2, b2) = res
        assert np.linalg.norm(v1[s] - v2[s]) <= 2e-6 * np.linalg.norm(v2[s])
        assert np.linalg.norm(p1[s] - p2[s]) <= 2e-7 * np.linalg.norm(p2[s])
        # without the correction the streamfunction would depend on the splitting
        q1, q2 = p1[s].copy(), p2[s].copy()
        q1[:, 2] -= b1
        q2[:, 2] -= b2
        assert np.linalg.norm(q1 - q2) > 100 * 2e-7 * np.linalg.norm(q2)


def test_straight_infinite_line(vp, oracle):
    """A straight periodic line along z: zero velocity (no curvature, images cancel), streamfunction
    along z and uniform along the line; closing spline segment and offset handled (s' = L / T along z)."""
    L = 2 * math.pi
    f = vp.curves.periodic_line(32, L, translate=(L / 3, L / 5, L / 2))
    p = vp.configs.params_for(L / 4, 3.5, 32, 5)
    v, psi, _ = oracle.compute_on_nodes(p, [f], streamfunction=True)
    assert np.abs(v).max() < 1e-7 * np.abs(psi).max()
    assert np.abs(psi[:, :2]).max() < 1e-10 * np.abs(psi[:, 2]).max()
    assert np.ptp(psi[:, 2]) < 1e-8 * np.abs(psi[:, 2]).max()
    pd = oracle.point_data(p, [f])
    np.testing.assert_allclose(pd["d1"][:, 2], 1.0, rtol=1e-12)  # chordal knots: |s'| = 1
    np.testing.assert_allclose(pd["dp"], L / 32, rtol=1e-12)


@pytest.mark.parametrize("kernel,bounds", [("es", {2: 3e-3, 3: 5e-5, 4: 1e-6, 5: 2e-8, 6: 3e-10}),
                                           ("kaiser_bessel", {2: 6e-3, 3: 1.2e-4, 4: 2e-6, 5: 5e-8, 6: 1e-9})])
def test_nufft_kernels_against_exact_sums(vp, oracle, kernel, bounds):
    """Long-range velocity of the trefoil with the NUFFT against the exact Fourier sums
    (ExactSumBackend, exact_sum.jl:15-121; test/trefoil.jl:135-245 holds the NonuniformFFTs.jl
    backend to 1e-5 against them), sigma = 1.5, for both spreading kernels and m = 2..6.  The
    reference's own kernel (NonuniformFFTs.jl's default) is not in its tree; both kernels here meet
    the accuracy the reference documents per m (nonuniformffts.jl:69-88: 6 digits at m = 4, 8 at
    m = 5, 10 at m = 6)."""
    fs = [vp.curves.trefoil(64)]
    for m, bound in bounds.items():
        p = vp.configs.params_for(math.pi / 2, 3.5, 32, m).with_(backend_long=vp.NonuniformFFTsBackend(1.5, m, kernel))
        v, _, _ = oracle.compute_on_nodes(p, fs, shortrange=False)
        ve, _, _ = oracle.compute_on_nodes(p, fs, shortrange=False, exact=True)
        assert np.linalg.norm(v - ve) / np.linalg.norm(ve) < bound, (m, kernel)
