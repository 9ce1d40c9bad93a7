"""ctypes front end of the CPU oracle (oracle/vp_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg as the checker; never by the product package.  Parity status: pinned to the
reference's known-answer tests (see vp_oracle.c), not to reference outputs.
"""

from __future__ import annotations

import ctypes as ct
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "build" / "libvporacle.so"


class OParams(ct.Structure):
    _fields_ = [
        ("Gamma", ct.c_double), ("a", ct.c_double), ("Delta", ct.c_double), ("L", ct.c_double * 3),
        ("alpha", ct.c_double), ("rcut", ct.c_double), ("Ns", ct.c_int * 3), ("sigma", ct.c_double),
        ("m", ct.c_int), ("nquad", ct.c_int), ("nquad_near", ct.c_int), ("lia_segment_fraction", ct.c_double),
        ("avoid_explicit_erf", ct.c_int), ("truncate_spherical", ct.c_int), ("nsubdiv", ct.c_int),
        ("longrange_exact", ct.c_int), ("nthreads", ct.c_int), ("splitting", ct.c_int), ("kb_beta", ct.c_double),
        ("kb_rtol", ct.c_double), ("fil_offsets", ct.c_void_p), ("nufft_kernel", ct.c_int),
    ]


class OStats(ct.Structure):
    _fields_ = [("pairs_in_range", ct.c_int64), ("pairs_candidates", ct.c_int64), ("fft_n", ct.c_int * 3),
                ("es_beta", ct.c_double)]


_lib = None


def build():
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = ct.CDLL(str(LIB))
        dp = ct.POINTER(ct.c_double)
        i64p = ct.POINTER(ct.c_int64)
        lib.vpo_compute_on_nodes.restype = ct.c_int
        lib.vpo_compute_on_nodes.argtypes = [ct.POINTER(OParams), ct.c_int, i64p, dp, ct.c_int, ct.c_int, ct.c_int,
                                             dp, dp, ct.POINTER(OStats)]
        lib.vpo_point_data.restype = ct.c_int
        lib.vpo_point_data.argtypes = [ct.POINTER(OParams), ct.c_int, i64p, dp, dp, ct.POINTER(ct.c_int32), dp, dp,
                                       dp, dp, dp, dp]
        lib.vpo_vorticity_fourier.restype = ct.c_int
        lib.vpo_vorticity_fourier.argtypes = [ct.POINTER(OParams), ct.c_int64, dp, dp, dp, ct.POINTER(OStats)]
        lib.vpo_gl_rule.argtypes = [ct.c_int, dp, dp]
        lib.vpo_kb_weights.restype = ct.c_int
        lib.vpo_kb_weights.argtypes = [ct.c_double, ct.c_double, ct.c_double, dp, ct.c_long, dp, dp]
        lib.vpo_fft_size.restype = ct.c_int
        lib.vpo_fft_size.argtypes = [ct.c_int, ct.c_double]
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def make_params(p, *, exact=False, nthreads=0) -> OParams:
    """Oracle parameters from a ParamsBiotSavart-like object (duck typed)."""
    o = OParams()
    o.Gamma, o.a, o.Delta = p.Gamma, p.a, p.Delta
    sp = p.splitting
    if hasattr(sp, "beta") and not hasattr(sp, "alpha"):  # KaiserBesselSplitting
        o.splitting, o.kb_beta, o.kb_rtol = 1, sp.beta, sp.rtol
        o.alpha, o.rcut = 0.0, sp.rcut
        for d in range(3):
            o.L[d] = sp.Ls[d]
            o.Ns[d] = sp.Ns[d]
    elif getattr(sp, "alpha", 0.0) == 0.0:
        o.alpha = 0.0
        o.rcut = math.inf
        for d in range(3):
            o.L[d] = 0.0
            o.Ns[d] = 0
    else:
        o.alpha, o.rcut = sp.alpha, sp.rcut
        for d in range(3):
            o.L[d] = sp.Ls[d]
            o.Ns[d] = sp.Ns[d]
    o.sigma = p.backend_long.sigma
    o.m = p.backend_long.m
    o.nufft_kernel = {"es": 0, "kaiser_bessel": 1}[getattr(p.backend_long, "kernel", "es")]
    o.nquad = len(p.quadrature)
    o.nquad_near = len(p.quadrature_near_singularity)
    o.lia_segment_fraction = p.lia_segment_fraction if p.lia_segment_fraction is not None else 0.0
    o.avoid_explicit_erf = int(p.avoid_explicit_erf)
    o.truncate_spherical = int(p.longrange_truncate_spherical)
    o.nsubdiv = getattr(p.backend_short, "nsubdiv", 0)
    o.longrange_exact = int(exact)
    o.nthreads = nthreads
    return o


def _pack(fs):
    counts = np.array([len(f) for f in fs], dtype=np.int64)
    offsets = np.zeros(len(fs) + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])
    nodes = np.ascontiguousarray(np.concatenate([np.asarray(f, dtype=np.float64) for f in fs]))
    return nodes, offsets


def end_to_end_offsets(fs):
    """[nfil, 3] end-to-end offsets (a filament's `offset` attribute, zero when absent), or None
    when every filament is closed."""
    offs = np.array([np.asarray(getattr(f, "offset", np.zeros(3)), dtype=np.float64) for f in fs]).reshape(len(fs), 3)
    return np.ascontiguousarray(offs) if np.any(offs != 0) else None


def compute_on_nodes(p, fs, *, velocity=True, streamfunction=False, LIA=True, shortrange=True, longrange=True,
                     exact=False, nthreads=0):
    """Oracle compute_on_nodes!: returns (vel [Np,3] or None, psi [Np,3] or None, stats dict)."""
    lib = load()
    o = make_params(p, exact=exact, nthreads=nthreads)
    nodes, offsets = _pack(fs)
    foff = end_to_end_offsets(fs)
    o.fil_offsets = foff.ctypes.data if foff is not None else None
    Np = int(offsets[-1])
    vel = np.zeros((Np, 3)) if velocity else None
    psi = np.zeros((Np, 3)) if streamfunction else None
    st = OStats()
    lia = {True: 1, False: 0, "only": 2}[LIA]
    rc = lib.vpo_compute_on_nodes(ct.byref(o), len(fs), offsets.ctypes.data_as(ct.POINTER(ct.c_int64)), _dp(nodes),
                                  lia, int(shortrange), int(longrange), _dp(vel) if vel is not None else None,
                                  _dp(psi) if psi is not None else None, ct.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle compute_on_nodes failed ({rc})")
    return vel, psi, {"pairs_in_range": st.pairs_in_range, "pairs_candidates": st.pairs_candidates,
                      "fft_n": tuple(st.fft_n), "es_beta": st.es_beta}


def point_data(p, fs):
    """Oracle add_point_charges!: dict of arrays (AoS [.,3] for vectors; idx_prev 0-based)."""
    lib = load()
    o = make_params(p)
    nodes, offsets = _pack(fs)
    foff = end_to_end_offsets(fs)
    o.fil_offsets = foff.ctypes.data if foff is not None else None
    Np = int(offsets[-1])
    nq = o.nquad
    out = {k: np.zeros((Np, 3)) for k in ("nodes", "d1", "d2")}
    out["idx_prev"] = np.zeros(Np, dtype=np.int32)
    out["dm"] = np.zeros(Np)
    out["dp"] = np.zeros(Np)
    out["points"] = np.zeros((Np * nq, 3))
    out["charges"] = np.zeros((Np * nq, 3))
    rc = lib.vpo_point_data(ct.byref(o), len(fs), offsets.ctypes.data_as(ct.POINTER(ct.c_int64)), _dp(nodes),
                            _dp(out["nodes"]), out["idx_prev"].ctypes.data_as(ct.POINTER(ct.c_int32)),
                            _dp(out["d1"]), _dp(out["d2"]), _dp(out["dm"]), _dp(out["dp"]), _dp(out["points"]),
                            _dp(out["charges"]))
    if rc != 0:
        raise RuntimeError(f"oracle point_data failed ({rc})")
    return out


def vorticity_fourier(p, points, charges, *, exact=False):
    """Oracle vorticity coefficients: complex array [3, Ns2, Ns1, Ns0//2+1]."""
    lib = load()
    o = make_params(p, exact=exact)
    Ns = p.splitting.Ns
    nkx = Ns[0] // 2 + 1
    buf = np.zeros(2 * 3 * nkx * Ns[1] * Ns[2])
    pts = np.ascontiguousarray(points, dtype=np.float64)
    chg = np.ascontiguousarray(charges, dtype=np.float64)
    rc = lib.vpo_vorticity_fourier(ct.byref(o), len(pts), _dp(pts), _dp(chg), _dp(buf), None)
    if rc != 0:
        raise RuntimeError("oracle vorticity_fourier failed")
    return buf.view(np.complex128).reshape(3, Ns[2], Ns[1], nkx)


def kb_weights(beta, rcut, rtol, r):
    """Kaiser-Bessel short-range weights (1 - F(r), 1 - F(r) + r f(r)) from the oracle's series,
    and the number of even Chebyshev coefficients kept in f."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    a = np.zeros_like(r)
    g = np.zeros_like(r)
    ne = load().vpo_kb_weights(beta, rcut, rtol, _dp(r), len(r), _dp(a), _dp(g))
    if ne < 0:
        raise RuntimeError("oracle Kaiser-Bessel series did not converge")
    return a, g, ne


def gl_rule(n):
    lib = load()
    z = np.zeros(n)
    w = np.zeros(n)
    lib.vpo_gl_rule(n, _dp(z), _dp(w))
    return z, w


def background_factor(p):
    """Streamfunction factor of a uniform background vorticity (1/(4 alpha^2), or the Kaiser-Bessel
    integral), as the oracle applies it."""
    lib = load()
    lib.vpo_background_factor.restype = ct.c_double
    lib.vpo_background_factor.argtypes = [ct.POINTER(OParams)]
    return lib.vpo_background_factor(ct.byref(make_params(p)))


def fft_size(Ns, sigma):
    return load().vpo_fft_size(Ns, sigma)


def default_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
