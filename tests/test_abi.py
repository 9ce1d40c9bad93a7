"""CPU-side checks of the C ABI: the library loads, exports exactly what include/vpbs.h
declares, rejects bad parameters before touching a GPU, and reports errors through
vpbs_last_error (host-side fault injection, no GPU needed)."""

import ctypes as ct
import math
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    src = (ROOT / "include" / "vpbs.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vpbs_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(vp, built_lib):
    from vortexpasta_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES), "ctypes prototypes out of sync with include/vpbs.h"


def test_params_struct_layout(vp):
    from vortexpasta_b200 import _lib
    # offsets of the C struct computed by the C compiler rules for the declared members
    P = _lib.VpbsParams
    assert P.L.offset == 24 and P.Ns.offset == 64 and P.sigma.offset == 80
    # the Kaiser-Bessel fields appended after `device`: int32 then two doubles (8-byte aligned)
    assert P.splitting.offset == P.device.offset + 4
    assert P.kb_beta.offset % 8 == 0 and P.kb_rtol.offset == P.kb_beta.offset + 8
    assert P.nufft_kernel.offset == P.kb_rtol.offset + 8
    assert ct.sizeof(P) == P.nufft_kernel.offset + 8  # int32 plus tail padding to 8-byte alignment


def _params(vp, **kw):
    from vortexpasta_b200.biotsavart import _c_params
    fs, p = vp.configs.ring64()
    return _c_params(p), p


def test_create_rejects_bad_parameters_without_gpu(vp):
    from vortexpasta_b200 import _lib
    lib = _lib.load()
    c, _ = _params(vp)
    bad = []
    c1 = _lib.VpbsParams.from_buffer_copy(c)
    c1.rcut = 3.0  # > 2/5 L with nsubdiv = 2 (CellLists.jl:114-115)
    bad.append(c1)
    c2 = _lib.VpbsParams.from_buffer_copy(c)
    c2.nquad = 0
    bad.append(c2)
    c3 = _lib.VpbsParams.from_buffer_copy(c)
    c3.a = -1.0
    bad.append(c3)
    c4 = _lib.VpbsParams.from_buffer_copy(c)
    c4.m = 20
    bad.append(c4)
    c5 = _lib.VpbsParams.from_buffer_copy(c)
    c5.sigma = 1.0
    bad.append(c5)
    for cp in bad:
        h = ct.c_void_p()
        rc = lib.vpbs_create(ct.byref(cp), ct.byref(h))
        assert rc == -2, rc
        assert not h.value
        assert lib.vpbs_last_error(None)
    assert lib.vpbs_create(ct.byref(bad[0]), ct.byref(ct.c_void_p())) == -2
    assert b"larger than that allowed" in lib.vpbs_last_error(None)


def test_null_arguments(vp):
    from vortexpasta_b200 import _lib
    lib = _lib.load()
    assert lib.vpbs_create(None, None) == -1
    assert lib.vpbs_destroy(None) == 0
    assert lib.vpbs_compute(None, 1, 1, 1, 1, 0.0) == -1
    assert lib.vpbs_launch_count(None) == 0
    # long-range diagnostics entry points check their arguments before any device work
    buf = np.zeros(6)
    assert lib.vpbs_spectrum(None, 0, 1.0, _lib.dptr(buf), 6) == -1
    assert lib.vpbs_coarse_grain(None, 0.1, 1) == -1
    assert lib.vpbs_get_field_fourier(None, 1, _lib.dptr(buf), 6) == -1
    assert lib.vpbs_interpolate_field(None, 1, _lib.dptr(buf)) == -1
    assert lib.vpbs_kb_weights(14.0, 0.5, 1e-6, None, 1, None, None, None, None) == -1
    assert lib.vpbs_kb_weights(-1.0, 0.5, 1e-6, _lib.dptr(buf), 1, None, None, None, None) == -1


def test_python_params_mirror_reference_errors(vp):
    L = vp.configs.L
    with pytest.raises(ValueError, match="larger than that allowed"):
        vp.ParamsBiotSavart(Gamma=1.0, a=1e-8, splitting=vp.GaussianSplitting(Ls=L, alpha=1.0, rcut=2.6, Ns=32))
    with pytest.raises(ValueError, match="NaiveShortRangeBackend"):
        vp.ParamsBiotSavart(Gamma=1.0, a=1e-8, splitting=vp.GaussianSplitting(Ls=L, alpha=1.0, rcut=3.2, Ns=32),
                            backend_short=vp.NaiveShortRangeBackend())
    # the naive backend allows up to L/2 (naive.jl:8-16)
    vp.ParamsBiotSavart(Gamma=1.0, a=1e-8, splitting=vp.GaussianSplitting(Ls=L, alpha=1.0, rcut=3.1, Ns=32),
                        backend_short=vp.NaiveShortRangeBackend())
    with pytest.raises(TypeError):
        vp.GaussianSplitting(Ls=L, alpha=1.0)


def test_gaussian_splitting_derivations(vp):
    """splitting/gaussian.jl:133-200 and its docstring example (Ns = 128, beta = 3.5 => alpha = 9)."""
    L = vp.configs.L
    g = vp.GaussianSplitting(Ls=L, beta=3.5, Ns=128)
    assert abs(g.alpha - 9.0) < 1e-12 and abs(g.rcut - 3.5 / 9) < 1e-12
    assert abs(g.rtol - 2.398239748342885e-7) < 1e-18
    g2 = vp.GaussianSplitting(Ls=L, beta=3.5, rcut=L / 4)
    assert abs(g2.alpha - 3.5 / (L / 4)) < 1e-12
    assert g2.Ns == (vp.kmax_to_gridsize(2 * g2.alpha * 3.5, L),) * 3
    g3 = vp.GaussianSplitting(Ls=L, rtol=g.rtol, alpha=9.0)
    assert abs(g3.rcut - g.rcut) < 1e-12
    assert vp.maximum_wavenumber((128,) * 3, (L,) * 3) == pytest.approx(63.0)


def test_ewald_weight_tables_accuracy(vp):
    """The pair kernel's Taylor tables of erfc(x) and erfc(x) + 2/sqrt(pi) x exp(-x^2)
    (replacing the reference's erfc/exp calls, splitting/gaussian.jl:273-279) against scipy."""
    import numpy as np
    from scipy.special import erfc
    from vortexpasta_b200 import _lib
    lib = _lib.load()
    for xmax in (3.5, 4.0, 6.5):
        x = np.concatenate([np.linspace(0, xmax, 20001), np.random.default_rng(1).uniform(0, xmax, 20000)])
        a = np.empty_like(x)
        g = np.empty_like(x)
        assert lib.vpbs_ewald_table_eval(xmax, _lib.dptr(x), len(x), _lib.dptr(a), _lib.dptr(g)) == 0
        ea = erfc(x)
        eg = ea + 2 / np.sqrt(np.pi) * x * np.exp(-x * x)
        # absolute error (the weights multiply 1/r^3 and 1/r; they are <= 1 and smooth)
        assert np.max(np.abs(a - ea)) < 1e-15  # a few ulp of 1
        assert np.max(np.abs(g - eg)) < 1e-15
        small = x <= 4.0  # relative accuracy where erfc is not yet negligible (erfc(4) ~ 1.5e-8)
        assert np.max(np.abs(a - ea)[small] / ea[small]) < 1e-13


def test_periodic_helpers_on_host(vp, built_lib):
    """The device's folding and cell-index helpers (the same inline code, run on the CPU): the
    reference's subtraction loops within a few periods (min_distance.jl:5-20), O(1) beyond, NaN
    for a non-finite coordinate, and the sentinel cell nc for it (so that a blown-up point is
    left out of every neighbourhood instead of stalling the pair search)."""
    from vortexpasta_b200 import _lib
    lib = _lib.load()
    L, nc = 2 * math.pi, 16
    x = np.array([0.0, 1.0, -1e-17, L, -L, 3.5 * L + 0.25, -3.9 * L, 1e6, -1e300, 1e300,
                  np.inf, -np.inf, np.nan, L - 1e-16, 5 * L])
    folded = np.zeros_like(x)
    cell = np.zeros(len(x), dtype=np.int64)
    assert lib.vpbs_periodic_eval(L, nc, _lib.dptr(x), len(x), _lib.dptr(folded), cell.ctypes.data_as(_lib.c_int64_p)) == 0
    fin = np.isfinite(x)
    assert np.all(np.isnan(folded[~fin]))
    assert np.all(cell[~fin] == nc)
    f = folded[fin]
    assert np.all((f >= 0) & (f < L))
    # folded values are congruent to x modulo L (to the rounding of one subtraction per period)
    mod = fin & (np.abs(x) < 1e7)
    k = np.round((x[mod] - folded[mod]) / L)
    assert np.allclose(x[mod] - k * L, folded[mod], rtol=0, atol=1e-8)
    assert np.all((cell[fin] >= 0) & (cell[fin] < nc))
    np.testing.assert_array_equal(cell[fin], np.minimum((f / L * nc).astype(np.int64), nc - 1))
    # within four periods: the reference's loops exactly
    for xi, fi in zip(x[:7], folded[:7]):
        y = xi
        while y < 0:
            y += L
        while y >= L:
            y -= L
        assert fi == y


@pytest.mark.parametrize("case", ["gaussian_beta4", "gaussian_beta5.5", "kaiser_bessel_12.44", "kaiser_bessel_30"])
def test_f32_pair_weights(vp, built_lib, case):
    """The mixed form's FP32 pair-kernel weights (cubic tables on 1/32-wide intervals in x = alpha r)
    against FP64: erfc / erfc + 2x/sqrt(pi) e^-x^2 (gaussian.jl:273-279) and the oracle's Kaiser-Bessel
    series (kaiser_bessel.jl:139-147), to 2e-7 absolute over [0, r_cut]."""
    from scipy.special import erfc
    from vortexpasta_b200 import _lib
    from oracle import oracle as O
    lib = _lib.load()
    rcut = 0.3
    r = np.linspace(0.0, rcut, 20001)
    a = np.zeros(len(r), dtype=np.float32)
    g = np.zeros(len(r), dtype=np.float32)
    fp = lambda x: x.ctypes.data_as(_lib.c_float_p)
    if case.startswith("gaussian"):
        beta = float(case.split("beta")[1])
        alpha = beta / rcut
        assert lib.vpbs_f32_weights_eval(0, alpha, rcut, 0.0, 0.0, _lib.dptr(r), len(r), fp(a), fp(g)) == 0
        x = alpha * r
        ea, eg = erfc(x), erfc(x) + 2 / math.sqrt(math.pi) * x * np.exp(-x * x)
    else:
        beta = float(case.split("_")[-1])
        rtol = 10 ** (-0.2) * math.exp(-beta)
        assert lib.vpbs_f32_weights_eval(1, 0.0, rcut, beta, rtol, _lib.dptr(r), len(r), fp(a), fp(g)) == 0
        ea, eg, _ = O.kb_weights(beta, rcut, rtol, r)
    assert np.abs(a - ea).max() < 2e-7
    assert np.abs(g - eg).max() < 2e-7


def _host_copies(lib, dsts, srcs):
    from vortexpasta_b200 import _lib  # noqa: F401
    n = len(dsts)
    dp = (ct.c_void_p * max(n, 1))(*[d.ctypes.data for d in dsts])
    sp = (ct.c_void_p * max(n, 1))(*[s.ctypes.data for s in srcs])
    nb = (ct.c_size_t * max(n, 1))(*[s.nbytes for s in srcs])
    return lib.vpbs_host_copies(n, dp, sp, nb)


def test_host_copy_threads(built_lib):
    """The staging copies of the host-buffer entry points: every byte of every block arrives, for one
    large block (split into pieces), many small blocks (grouped), mixed sizes and empty blocks, over
    repeated jobs on the same thread pool."""
    from vortexpasta_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(5)
    cases = [[24 << 20], [4800] * 3000, [0, 17, 3 << 20, 1 << 20, 5, 0, (1 << 20) + 3, 999_999],
             [1 << 10], [(2 << 20) + 8]]
    for rep in range(3):
        for sizes in cases:
            srcs = [rng.integers(0, 256, size=b, dtype=np.uint8) for b in sizes]
            dsts = [np.zeros(b, dtype=np.uint8) for b in sizes]
            assert _host_copies(lib, dsts, srcs) == 0
            for s, d in zip(srcs, dsts):
                assert np.array_equal(s, d)
    assert lib.vpbs_host_copies(-1, None, None, None) != 0


def _copy_in_child(q):
    from vortexpasta_b200 import _lib
    lib = _lib.load()
    src = [np.arange(3 << 20, dtype=np.uint8)]
    dst = [np.zeros(3 << 20, dtype=np.uint8)]
    rc = _host_copies(lib, dst, src)
    q.put(rc == 0 and np.array_equal(src[0], dst[0]))


@pytest.mark.filterwarnings("ignore:This process .* is multi-threaded:DeprecationWarning")
def test_host_copy_threads_after_fork(built_lib):
    """A child forked after the parent's copy threads started has none of them: its first large copy
    starts its own pool instead of waiting for threads that do not exist."""
    import multiprocessing as mp
    from vortexpasta_b200 import _lib
    lib = _lib.load()
    src = [np.ones(4 << 20, dtype=np.uint8)]
    dst = [np.zeros(4 << 20, dtype=np.uint8)]
    assert _host_copies(lib, dst, src) == 0  # the parent's pool exists now
    ctx = mp.get_context("fork")
    q = ctx.Queue()
    p = ctx.Process(target=_copy_in_child, args=(q,))
    p.start()
    p.join(60)
    alive = p.is_alive()
    if alive:
        p.kill()
    assert not alive and p.exitcode == 0
    assert q.get(timeout=5)


def test_destroy_frees_every_device_buffer():
    """Every device buffer of the handle (a DevBuf member in vpbs_internal.cuh) is in vpbs_destroy's
    list of buffers to free: a buffer left out leaks device memory on every create / destroy cycle."""
    csrc = Path(__file__).resolve().parents[1] / "vortexpasta.jl_b200" / "csrc"
    header = (csrc / "vpbs_internal.cuh").read_text()
    names = []
    for m in re.finditer(r"vpbs::DevBuf ([^;]+);", header):
        names += [x.strip() for x in m.group(1).split(",")]
    assert len(names) > 40
    api = (csrc / "api.cu").read_text()
    i = api.index("DevBuf* bufs[] = {")
    listed = api[i:api.index("};", i)]
    missing = [n for n in names if f"&h->{n}" not in listed]
    assert not missing, f"not freed by vpbs_destroy: {missing}"
