"""Parity of the CUDA library (through its C ABI) with the CPU oracle.

Bar: the plain FP64 GPU form matches the FP64 oracle to <= 1e-10 relative L2
per node-velocity (and streamfunction) field.  Pair counts are integers and must match
exactly.
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10  # relative L2, FP64 form vs FP64 oracle


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def gpu_fields(vp, p, fs, **kw):
    cache = vp.init_cache(p)
    vs = [np.zeros_like(f) for f in fs]
    ps = [np.zeros_like(f) for f in fs]
    vp.compute_on_nodes_({"velocity": vs, "streamfunction": ps}, cache, fs, **kw)
    return np.concatenate(vs), np.concatenate(ps), cache


def test_point_data_matches_oracle(vp, oracle, built_lib):
    fs, p = vp.configs.tangle20k()
    fs = fs[:10] + [vp.curves.ring(5, 0.3, center=(1, 1, 1)), vp.curves.ring(7, 0.5, center=(6.2, 0.1, 3))]
    cache = vp.init_cache(p)
    cache.set_filaments(fs)
    g = cache.pointdata()
    o = oracle.point_data(p, fs)
    # s'' is a second divided difference of the spline coefficients (factors 1/dt^2), so its
    # rounding differences are amplified ~1e3-1e4 times; everything else agrees to ~1e-15.
    tol = {"d2": 1e-10}
    for k in ("nodes", "d1", "d2", "dm", "dp", "points", "charges"):
        assert rel(g[k], o[k]) < tol.get(k, 1e-12), k
    np.testing.assert_array_equal(g["idx_prev"], o["idx_prev"])


@pytest.mark.parametrize("workload", ["ring64", "tangle20k"])
def test_full_velocity_streamfunction(vp, oracle, built_lib, workload):
    fs, p = vp.configs.WORKLOADS[workload]()
    v, psi, cache = gpu_fields(vp, p, fs)
    vo, po, st = oracle.compute_on_nodes(p, fs, streamfunction=True)
    assert rel(v, vo) < TOL
    assert rel(psi, po) < TOL
    assert cache.pair_counts()[0] == st["pairs_in_range"]


def test_golden_ring64(vp, built_lib):
    from pathlib import Path
    g = np.load(Path(__file__).parent / "golden" / "ring64.npz")
    fs, p = vp.configs.ring64()
    v, psi, _ = gpu_fields(vp, p, fs)
    assert rel(v, g["velocity"]) < TOL and rel(psi, g["streamfunction"]) < TOL


@pytest.mark.parametrize("LIA", [True, False, "only"])
@pytest.mark.parametrize("short,long", [(True, True), (True, False), (False, True)])
def test_flags(vp, oracle, built_lib, LIA, short, long):
    fs, p = vp.configs.ring64()
    if not short and LIA == "only":
        pytest.skip("no contribution")
    v, psi, _ = gpu_fields(vp, p, fs, LIA=LIA, shortrange=short, longrange=long)
    vo, po, _ = oracle.compute_on_nodes(p, fs, streamfunction=True, LIA=LIA, shortrange=short, longrange=long)
    assert rel(v, vo) < TOL and rel(psi, po) < TOL


@pytest.mark.parametrize("variant", ["explicit_erf", "lia_fraction", "truncate", "m5", "m6", "m8", "sigma125_m3",
                                     "gl2", "nsubdiv1", "kb_kernel_m4", "kb_kernel_m6"])
def test_parameter_variants(vp, oracle, built_lib, variant):
    fs, p = vp.configs.tangle20k()
    fs = fs[:30]
    kw = {
        "explicit_erf": dict(avoid_explicit_erf=False),
        "lia_fraction": dict(lia_segment_fraction=0.3, quadrature_near_singularity=vp.GaussLegendre(6)),
        "truncate": dict(longrange_truncate_spherical=True),
        "m5": dict(backend_long=vp.NonuniformFFTsBackend(1.5, 5)),
        "m6": dict(backend_long=vp.NonuniformFFTsBackend(1.5, 6)),
        "m8": dict(backend_long=vp.NonuniformFFTsBackend(2.0, 8)),
        "sigma125_m3": dict(backend_long=vp.NonuniformFFTsBackend(1.25, 3)),
        "gl2": dict(quadrature=vp.GaussLegendre(2)),
        "nsubdiv1": dict(backend_short=vp.CellListsBackend(1)),
        "kb_kernel_m4": dict(backend_long=vp.NonuniformFFTsBackend(1.5, 4, "kaiser_bessel")),
        "kb_kernel_m6": dict(backend_long=vp.NonuniformFFTsBackend(1.5, 6, "kaiser_bessel")),
    }[variant]
    p = p.with_(**kw)
    v, psi, _ = gpu_fields(vp, p, fs)
    vo, po, _ = oracle.compute_on_nodes(p, fs, streamfunction=True)
    assert rel(v, vo) < TOL and rel(psi, po) < TOL


def test_vorticity_fourier_coefficients(vp, oracle, built_lib):
    """The vorticity coefficients (what callback_vorticity sees, BiotSavart.jl:436-438) and the
    velocity coefficients the cache holds after the evaluation (compute_velocity_fourier!,
    longrange.jl:128-156) against the oracle's vorticity and its Biot-Savart transform."""
    from oracle import spectra_ref
    fs, p = vp.configs.tangle20k()
    fs = fs[:20]
    seen = {}

    def grab(c):
        seen["lr"] = vp.get_longrange_field_fourier(c)

    cache = vp.init_cache(p)
    vs = [np.zeros_like(f) for f in fs]
    vp.compute_on_nodes_({"velocity": vs}, cache, fs, callback_vorticity=grab)
    lr = seen["lr"]
    assert lr["state"].quantity == "vorticity" and lr["state"].smoothing_scale == 0
    o = oracle.point_data(p, fs)
    uo = oracle.vorticity_fourier(p, o["points"], o["charges"])  # [3, Ns2, Ns1, nkx]
    ug = np.stack([c.transpose(2, 1, 0) for c in lr["field"]])
    assert np.linalg.norm(ug - uo) / np.linalg.norm(uo) < TOL
    kx, ky, kz = lr["wavenumbers"]
    assert kx[-1] > 0 and len(ky) == p.splitting.Ns[1]
    after = vp.get_longrange_field_fourier(cache)
    assert after["state"].quantity == "velocity"
    vo = spectra_ref.velocity_from_vorticity(tuple(uo[c].transpose(2, 1, 0) for c in range(3)), lr["wavenumbers"])
    vg = np.stack(after["field"])
    assert np.linalg.norm(vg - np.stack(vo)) / np.linalg.norm(np.stack(vo)) < TOL
    vp.compute_on_nodes_({"streamfunction": [np.zeros_like(f) for f in fs]}, cache, fs)
    psi = vp.get_longrange_field_fourier(cache)
    assert psi["state"].quantity == "streamfunction"
    po = spectra_ref.streamfunction_from_vorticity(tuple(uo[c].transpose(2, 1, 0) for c in range(3)),
                                                    lr["wavenumbers"])
    assert np.linalg.norm(np.stack(psi["field"]) - np.stack(po)) / np.linalg.norm(np.stack(po)) < TOL
    cache.close()


def test_open_domain_ring_analytic(vp, oracle, built_lib):
    """NoSplitting on the GPU (naive pair kernel): test/ring.jl analytic answers."""
    R, N, Gamma, a, Delta = math.pi / 3, 32, 2.4, 1e-6, 0.25
    f = vp.curves.ring(N, R, center=(math.pi,) * 3)
    p = vp.ParamsBiotSavart(Gamma=Gamma, a=a, Delta=Delta, alpha=0, quadrature=vp.GaussLegendre(4),
                            lia_segment_fraction=0.4)
    v, psi, _ = gpu_fields(vp, p, [f])
    vo, po, _ = oracle.compute_on_nodes(p, [f], streamfunction=True)
    assert rel(v, vo) < TOL and rel(psi, po) < TOL
    U = np.linalg.norm(v.mean(axis=0))
    Uex = Gamma / (4 * math.pi * R) * (math.log(8 * R / a) - Delta)
    assert abs(U - Uex) / Uex < 1e-4


def test_set_points_plugin_contract(vp, oracle, built_lib):
    """Point data computed by the caller (host add_point_charges!), as in the reference plugin API."""
    fs, p = vp.configs.tangle20k()
    fs = fs[:15]
    pd = oracle.point_data(p, fs)
    cache = vp.init_cache(p)
    cache.set_points(pd)
    cache.compute(3)
    v = cache.get(1)
    psi = cache.get(2)
    vo, po, _ = oracle.compute_on_nodes(p, fs, streamfunction=True)
    assert rel(v, vo) < TOL and rel(psi, po) < TOL


def test_integration_cutoff(vp, oracle, built_lib):
    fs, p = vp.configs.ring64()
    v1, _, _ = gpu_fields(vp, p, fs, LIA="only")
    v2, _, _ = gpu_fields(vp, p, fs, LIA="only", integration_cutoff=1e-3)
    # ln(delta / r) scaling: v ~ ln(delta / r_cut)
    assert np.all(np.abs(v2[:, 2]) < np.abs(v1[:, 2]))


def test_ragged_sizes_and_reuse(vp, oracle, built_lib):
    fs, p = vp.configs.tangle20k()
    cache = vp.init_cache(p)
    for sub in (fs[:3] + [vp.curves.ring(5, 0.4, center=(3, 3, 3))], fs[:40], fs[:2]):
        vs = [np.zeros_like(f) for f in sub]
        vp.velocity_on_nodes_(vs, cache, sub)
        vo, _, _ = oracle.compute_on_nodes(p, sub)
        assert rel(np.concatenate(vs), vo) < TOL


def test_repeatable(vp, built_lib):
    fs, p = vp.configs.tangle20k()
    fs = fs[:20]
    cache = vp.init_cache(p)
    a = np.concatenate(vp.velocity_on_nodes(cache, fs))
    b = np.concatenate(vp.velocity_on_nodes(cache, fs))
    assert rel(a, b) < 1e-14


MIXED_TOL = 1e-5  # relative L2 of the mixed (FP32 bulk) form vs the FP64 oracle


@pytest.mark.parametrize("workload", ["ring64", "tangle20k"])
def test_mixed_precision_form(vp, oracle, built_lib, workload):
    """Precision form: FP32 pair sum, spreading, FFT and interpolation; FP64 positions,
    separations, local/self terms and final accumulation.  Target: <= 1e-5 relative L2."""
    fs, p = vp.configs.WORKLOADS[workload](precision="mixed")
    v, psi, _ = gpu_fields(vp, p, fs)
    vo, po, _ = oracle.compute_on_nodes(p, fs, streamfunction=True)
    ev, ep = rel(v, vo), rel(psi, po)
    print(f"{workload} mixed: velocity rel L2 {ev:.2e} (max {np.abs(v - vo).max() / np.abs(vo).max():.2e}), "
          f"streamfunction rel L2 {ep:.2e}")
    assert ev < MIXED_TOL and ep < MIXED_TOL


@pytest.mark.parametrize("LIA", [True, False, "only"])
def test_mixed_precision_flags(vp, oracle, built_lib, LIA):
    fs, p = vp.configs.tangle20k(precision="mixed")
    fs = fs[:25]
    v, psi, _ = gpu_fields(vp, p, fs, LIA=LIA)
    vo, po, _ = oracle.compute_on_nodes(p, fs, streamfunction=True, LIA=LIA)
    assert rel(v, vo) < MIXED_TOL and rel(psi, po) < MIXED_TOL


@pytest.mark.parametrize("sigma,m", [(1.5, 6), (1.25, 3), (2.0, 8), (2.0, 2), (1.5, 1)])
def test_mixed_precision_kernel_widths(vp, oracle, built_lib, sigma, m):
    """Mixed form with other NUFFT widths: plane-owner spreading with 8- and 4-wide patches
    (m = 3, 2, 1), register columns (m = 6, 8), interpolation tables of up to 3 x 16 entries."""
    fs, p = vp.configs.tangle20k(precision="mixed")
    fs = fs[:25]
    p = p.with_(backend_long=vp.NonuniformFFTsBackend(sigma, m))
    v, psi, _ = gpu_fields(vp, p, fs)
    vo, po, _ = oracle.compute_on_nodes(p, fs, streamfunction=True)
    assert rel(v, vo) < MIXED_TOL and rel(psi, po) < MIXED_TOL


def test_errors_surface(vp, built_lib):
    fs, p = vp.configs.ring64()
    cache = vp.init_cache(p)
    with pytest.raises(vp.VpbsError, match="no point data"):
        cache.compute(1)
    with pytest.raises(vp.VpbsError, match="at least 5 nodes"):
        cache.set_filaments([vp.curves.ring(4, 0.5, center=(3, 3, 3))])
    with pytest.raises(ValueError, match="not recognised"):
        vp.compute_on_nodes_({"vorticity": [np.zeros_like(fs[0])]}, cache, fs)


@pytest.mark.gpu
def test_spline_solve_at_exactly_48k_shared_memory(vp):
    """Filaments of 128 nodes make the spline solve ask for exactly 48 KB of shared memory;
    this must work in a fresh process-wide state (no earlier larger launch)."""
    fs = vp.configs.tangle(5, 128, seed=11)
    p = vp.configs.params_for(2 * np.pi / 8, 3.5, 32, 4)
    c = vp.init_cache(p)
    try:
        c.set_filaments(fs)
        c.compute(1)
        v = c.get(1)
    finally:
        c.close()
    assert np.isfinite(v).all() and np.abs(v).max() > 0


@pytest.mark.gpu
def test_host_entry_points_agree(vp):
    """Staged list input (velocity_on_nodes), the flat host-buffer call and the per-filament
    pointer-list C entry points give the same velocities."""
    import ctypes as ct
    from vortexpasta_b200 import _lib
    fs, p = vp.configs.tangle20k()
    fs = fs[:40]
    c = vp.init_cache(p)
    try:
        v_list = np.concatenate(vp.velocity_on_nodes(c, fs))
        nodes, offsets = vp.curves.concat(fs)
        c.set_filaments_flat(nodes, offsets)
        c.compute(_lib.VELOCITY)
        v_flat = c.get(_lib.VELOCITY)
        lib = _lib.load()
        fsc = [np.ascontiguousarray(f, dtype=np.float64) for f in fs]
        ptrs = (ct.c_void_p * len(fsc))(*[f.ctypes.data for f in fsc])
        counts = np.array([len(f) for f in fsc], dtype=np.int64)
        _lib.check(lib.vpbs_set_filament_list(c.handle, len(fsc), ptrs, counts.ctypes.data_as(_lib.c_int64_p)),
                   c.handle, "set_filament_list")
        c.compute(_lib.VELOCITY)
        outs = [np.zeros_like(f) for f in fsc]
        optr = (ct.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
        _lib.check(lib.vpbs_get_filament_list(c.handle, _lib.VELOCITY, optr, len(outs)), c.handle,
                   "get_filament_list")
        v_ptr = np.concatenate(outs)
    finally:
        c.close()
    assert np.abs(v_flat - v_list).max() <= 1e-13 * np.abs(v_list).max()
    assert np.abs(v_ptr - v_list).max() <= 1e-13 * np.abs(v_list).max()


@pytest.mark.parametrize("sigma,m,kernel", [(1.5, 3, "es"), (1.5, 4, "es"), (2.0, 2, "es"), (1.25, 3, "es"),
                                            (1.5, 4, "kaiser_bessel"), (2.0, 1, "es")])
def test_tensor_core_spreading(vp, oracle, built_lib, sigma, m, kernel):
    """Mixed form: the tensor-core brick product (tcgen05, 3xTF32) against the CUDA-core plane
    kernel and the oracle -- vorticity coefficients (the spread grid after the forward FFT) and
    velocities."""
    from vortexpasta_b200 import _lib
    fs, p = vp.configs.tangle20k(precision="mixed")
    fs = fs[:40]
    p = p.with_(backend_long=vp.NonuniformFFTsBackend(sigma, m, kernel))
    assert _lib.load().vpbs_fft_size(p.splitting.Ns[0], sigma) % 16 == 0  # brick spreading applies
    out = {}
    for mode in (0, 1):
        c = vp.init_cache(p)
        try:
            _lib.check(c._lib.vpbs_spread_mode(c.handle, mode), c.handle, "spread_mode")
            vs = [np.zeros_like(f) for f in fs]
            vp.compute_on_nodes_({"velocity": vs}, c, fs)
            out[mode] = (np.concatenate(vs), np.stack(vp.get_longrange_field_fourier(c)["field"]))
        finally:
            c.close()
    (v_tc, u_tc), (v_cc, u_cc) = out[0], out[1]
    assert rel(v_tc, v_cc) < 1e-6
    vo, _, _ = oracle.compute_on_nodes(p, fs)
    assert rel(v_tc, vo) < MIXED_TOL
    assert np.linalg.norm(u_tc - u_cc) / np.linalg.norm(u_cc) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_split_devices_match_single_handle(vp, built_lib, precision):
    """The reference's device split (short range and long range on two handles, the short-range field
    added into the long-range one) gives the single-handle result.  Here both handles share GPU 0 (a
    test box has one GPU); across GPUs the same call adds a peer copy."""
    import torch
    fs, p = vp.configs.tangle20k(precision=precision)
    fs = fs[:30]
    v1, p1, _ = gpu_fields(vp, p, fs)
    long_dev = 0
    short_dev = 1 if torch.cuda.device_count() > 1 else 0
    c = vp.SplitDevicesCache(p, long_device=long_dev, short_device=short_dev)
    try:
        vs = [np.zeros_like(f) for f in fs]
        ps = [np.zeros_like(f) for f in fs]
        c.compute_on_nodes_({"velocity": vs, "streamfunction": ps}, fs)
        vl = [np.zeros_like(f) for f in fs]
        c.compute_on_nodes_({"velocity": vl}, fs, LIA="only")
    finally:
        c.close()
    tol = 1e-14 if precision == "fp64" else 1e-6
    assert rel(np.concatenate(vs), v1) < tol and rel(np.concatenate(ps), p1) < tol
    vo, _, _ = gpu_fields(vp, p, fs, LIA="only")
    assert rel(np.concatenate(vl), vo) < 1e-14


def test_handles_release_device_memory(vp, built_lib):
    """Create / evaluate / read back / destroy cycles leave the device's free memory where it was
    (no buffer of the handle outlives it)."""
    import torch
    from vortexpasta_b200 import _lib
    fs, p = vp.configs.tangle20k(precision="mixed")

    def cycle():
        c = vp.init_cache(p)
        try:
            c.set_filaments(fs)
            c.compute(_lib.VELOCITY | _lib.STREAMFUNCTION)
            c.get(_lib.VELOCITY)
            c.get(_lib.STREAMFUNCTION)
        finally:
            c.close()

    cycle()  # first use: module loading, library workspaces
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(10):
        cycle()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 < 16 << 20, f"{(free0 - free1) / 2**20:.1f} MiB not released after 10 cycles"
