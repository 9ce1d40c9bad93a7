"""Host-side mirror of VortexPasta.BiotSavart's public API on top of libvpbs.so.

``init_cache``, ``velocity_on_nodes(_)``, ``compute_on_nodes_`` and
``get_longrange_field_fourier`` keep the reference's names, argument meaning and error
behaviour (src/BiotSavart/BiotSavart.jl:85-161, 288-612; cache.jl:40-83). A trailing
underscore stands for Julia's ``!`` (the outputs are overwritten in place).

Filaments are closed curves given as ``(N, 3)`` float64 node arrays (N >= 5, quintic
splines with chordal knots as in the reference's defaults); fields are lists of
``(N, 3)`` arrays, one per filament.
"""

from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib, curves
from .curves import concat
from .params import KaiserBesselSplitting, NoSplitting, ParamsBiotSavart


def _c_params(p: ParamsBiotSavart) -> _lib.VpbsParams:
    c = _lib.VpbsParams()
    c.Gamma, c.a, c.Delta = p.Gamma, p.a, p.Delta
    sp = p.splitting
    if isinstance(sp, NoSplitting):
        c.alpha = 0.0
        c.rcut = 0.0
        for d in range(3):
            c.L[d] = 0.0
            c.Ns[d] = 0
    elif isinstance(sp, KaiserBesselSplitting):
        c.splitting = _lib.SPLITTING_KAISER_BESSEL
        c.alpha, c.rcut, c.kb_beta, c.kb_rtol = 0.0, sp.rcut, sp.beta, sp.rtol
        for d in range(3):
            c.L[d] = sp.Ls[d]
            c.Ns[d] = sp.Ns[d]
    else:
        c.alpha, c.rcut = sp.alpha, sp.rcut
        for d in range(3):
            c.L[d] = sp.Ls[d]
            c.Ns[d] = sp.Ns[d]
    c.sigma = p.backend_long.sigma
    c.m = p.backend_long.m
    c.nufft_kernel = {"es": 0, "kaiser_bessel": 1}[getattr(p.backend_long, "kernel", "es")]
    z, w = p.quadrature.rule()
    c.nquad = len(z)
    for q in range(len(z)):
        c.quad_zeta[q], c.quad_w[q] = z[q], w[q]
    zn, wn = p.quadrature_near_singularity.rule()
    c.nquad_near = len(zn)
    for q in range(len(zn)):
        c.quad_near_zeta[q], c.quad_near_w[q] = zn[q], wn[q]
    c.lia_segment_fraction = p.lia_segment_fraction if p.lia_segment_fraction is not None else 0.0
    c.avoid_explicit_erf = int(p.avoid_explicit_erf)
    c.truncate_spherical = int(p.longrange_truncate_spherical)
    c.nsubdiv = getattr(p.backend_short, "nsubdiv", 0)  # 0: NaiveShortRangeBackend
    c.precision = _lib.PRECISION[p.precision]
    c.device = p.device
    return c


class LongRangeCacheState:
    """longrange/cache_common.jl:17-31."""

    def __init__(self, quantity="undef", smoothing_scale=0.0):
        self.quantity = quantity
        self.smoothing_scale = smoothing_scale

    def __repr__(self):
        return f"LongRangeCacheState(quantity = {self.quantity}, smoothing_scale = {self.smoothing_scale})"


class BiotSavartCache:
    """Owns one libvpbs handle (device memory, cuFFT plans, stream, pinned staging)."""

    def __init__(self, params: ParamsBiotSavart):
        self.params = params
        self._lib = _lib.load()
        self._cparams = _c_params(params)
        h = ct.c_void_p()
        rc = self._lib.vpbs_create(ct.byref(self._cparams), ct.byref(h))
        _lib.check(rc, None, "init_cache")
        self._h = h
        self.state = LongRangeCacheState()
        self.Np = 0
        self._out = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.vpbs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr: int | None):
        _lib.check(self._lib.vpbs_set_stream(self._h, ct.c_void_p(stream_ptr or 0)), self._h, "set_stream")

    def set_end_to_end_offsets(self, offs):
        """End-to-end offsets of the next filaments ([nfil, 3], or None for closed filaments), the
        ``Xoffset`` of unclosed filaments (closed_filament.jl:118-132); re-sent only when changed."""
        offs = None if offs is None else np.ascontiguousarray(offs, dtype=np.float64).reshape(-1, 3)
        if offs is not None and not np.any(offs):
            offs = None
        prev = getattr(self, "_fil_off", None)
        if (offs is None and prev is None) or (offs is not None and prev is not None and prev.shape == offs.shape
                                               and np.array_equal(prev, offs)):
            return
        if offs is None:
            rc = self._lib.vpbs_set_filament_offsets(self._h, 0, None)
        else:
            rc = self._lib.vpbs_set_filament_offsets(self._h, len(offs), _lib.dptr(offs))
        _lib.check(rc, self._h, "set_filament_offsets")
        self._fil_off = None if offs is None else offs.copy()

    def set_filaments(self, fs, on_device_ptr: int | None = None, offsets=None, end_to_end=None):
        """add_point_charges! on the device. `fs`: list of (N, 3) arrays (assembled straight into
        the handle's pinned staging buffer; an array with an ``offset`` attribute is an unclosed
        filament, ``curves.InfiniteFilament``), or None with a device pointer to AoS nodes plus host
        `offsets` (and the filaments' end-to-end offsets `end_to_end`, [nfil, 3], if any)."""
        if on_device_ptr is None:
            self.set_end_to_end_offsets(np.array([curves.end_to_end_offset(f) for f in fs]))
        else:
            self.set_end_to_end_offsets(end_to_end)
        if on_device_ptr is None:
            n = len(fs)
            counts = np.fromiter(map(len, fs), dtype=np.int64, count=n)
            Np = int(counts.sum())
            po, pn = _lib.c_int64_p(), _lib.c_double_p()
            _lib.check(self._lib.vpbs_stage_filaments(self._h, n, Np, ct.byref(po), ct.byref(pn)), self._h,
                       "add_point_charges!")
            off = np.ctypeslib.as_array(po, shape=(n + 1,))
            off[0] = 0
            np.cumsum(counts, out=off[1:])
            np.concatenate(fs, axis=0, out=np.ctypeslib.as_array(pn, shape=(Np, 3)))
            offsets = off.copy()
            rc = self._lib.vpbs_set_staged_filaments(self._h, n)
        else:
            offsets = np.ascontiguousarray(offsets, dtype=np.int64)
            rc = self._lib.vpbs_set_filaments(self._h, len(offsets) - 1, offsets.ctypes.data_as(_lib.c_int64_p),
                                              ct.c_void_p(on_device_ptr), 1)
        _lib.check(rc, self._h, "add_point_charges!")
        self.Np = int(offsets[-1])
        self._offsets = np.asarray(offsets)

    def set_filaments_flat(self, nodes: np.ndarray, offsets: np.ndarray, end_to_end=None):
        """add_point_charges! from one host AoS array [Np][3] and filament offsets (the flat C-ABI
        call vpbs_set_filaments with host nodes); `end_to_end`: [nfil, 3] offsets of unclosed filaments."""
        self.set_end_to_end_offsets(end_to_end)
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        rc = self._lib.vpbs_set_filaments(self._h, len(offsets) - 1, offsets.ctypes.data_as(_lib.c_int64_p),
                                          nodes.ctypes.data_as(ct.c_void_p), 0)
        _lib.check(rc, self._h, "add_point_charges!")
        self.Np = int(offsets[-1])
        self._offsets = offsets

    def get_list(self, field_mask: int, outs) -> None:
        """Copy a computed field into per-filament host arrays laid out like the last filaments."""
        p = _lib.c_double_p()
        _lib.check(self._lib.vpbs_get_staged(self._h, field_mask, ct.byref(p)), self._h,
                   "copy_output_values_on_nodes!")
        flat = np.ctypeslib.as_array(p, shape=(self.Np, 3))
        off = self._offsets.tolist()
        for k, u in enumerate(outs):
            u[...] = flat[off[k]:off[k + 1]]

    def compute(self, fields_mask: int, lia_mode: int = _lib.LIA_TRUE, shortrange=True, longrange=True,
                integration_cutoff=None):
        rc = self._lib.vpbs_compute(self._h, fields_mask, lia_mode, int(bool(shortrange)), int(bool(longrange)),
                                    0.0 if integration_cutoff is None else float(integration_cutoff))
        _lib.check(rc, self._h, "compute_on_nodes!")
        if longrange and lia_mode != _lib.LIA_ONLY and self.params.is_periodic:
            # the field the reference's cache holds afterwards (BiotSavart.jl:540-580): the velocity
            # when it was requested, else the streamfunction; the device keeps the vorticity
            # coefficients and converts on request
            q = "velocity" if fields_mask & _lib.VELOCITY else "streamfunction"
            self.state = LongRangeCacheState(q, 0.0)

    def get(self, field_mask: int, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.Np, 3))
        rc = self._lib.vpbs_get(self._h, field_mask, _lib.dptr(out), 0)
        _lib.check(rc, self._h, "copy_output_values_on_nodes!")
        return out

    def device_field(self, field_mask: int):
        x, y, z = ct.c_void_p(), ct.c_void_p(), ct.c_void_p()
        _lib.check(self._lib.vpbs_device_field(self._h, field_mask, ct.byref(x), ct.byref(y), ct.byref(z)),
                   self._h, "device_field")
        return x.value, y.value, z.value

    def features(self) -> np.ndarray:
        """Configuration features of the loaded filaments (vpbs_features): the inputs of the
        learned parameter predictor."""
        out = np.zeros(_lib.NUM_FEATURES, dtype=np.float32)
        _lib.check(self._lib.vpbs_features(self._h, _lib.fptr(out), _lib.NUM_FEATURES), self._h, "features")
        return out

    def pair_counts(self):
        a, b = ct.c_int64(), ct.c_int64()
        _lib.check(self._lib.vpbs_pair_counts(self._h, ct.byref(a), ct.byref(b)), self._h, "pair_counts")
        return a.value, b.value

    def launch_count(self) -> int:
        return int(self._lib.vpbs_launch_count(self._h))

    def stage_timing(self, enable: bool = True):
        _lib.check(self._lib.vpbs_stage_timing(self._h, int(enable)), self._h, "stage_timing")

    def stage_times(self) -> dict:
        """Milliseconds per stage since the previous query (CUDA events on the handle's stream)."""
        buf = np.zeros(_lib.NUM_STAGES)
        _lib.check(self._lib.vpbs_stage_times(self._h, _lib.dptr(buf), _lib.NUM_STAGES), self._h, "stage_times")
        return {self._lib.vpbs_stage_name(i).decode(): float(buf[i]) for i in range(_lib.NUM_STAGES)}

    def pointdata(self) -> dict:
        """Device point data (cache.pointdata of the reference) as AoS numpy arrays."""
        Np = self.Np
        Nq = Np * len(self.params.quadrature)
        out = {}
        for which, name, n in ((0, "nodes", Np), (1, "d1", Np), (2, "d2", Np), (5, "points", Nq), (6, "charges", Nq)):
            buf = np.empty(3 * n)
            _lib.check(self._lib.vpbs_get_pointdata(self._h, which, buf.ctypes.data_as(ct.c_void_p), 3 * n),
                       self._h, "get_pointdata")
            out[name] = buf.reshape(3, n).T.copy()
        for which, name in ((3, "dm"), (4, "dp")):
            buf = np.empty(Np)
            _lib.check(self._lib.vpbs_get_pointdata(self._h, which, buf.ctypes.data_as(ct.c_void_p), Np),
                       self._h, "get_pointdata")
            out[name] = buf
        idx = np.empty(Np, dtype=np.int32)
        _lib.check(self._lib.vpbs_get_pointdata(self._h, 7, idx.ctypes.data_as(ct.c_void_p), Np), self._h,
                   "get_pointdata")
        out["idx_prev"] = idx
        return out

    def set_points(self, pd: dict):
        """Plugin-contract input: PointData arrays (AoS [.,3]; idx_prev 0-based here, passed
        1-based to the C ABI as in the reference)."""
        def soa(a):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)
            return a, _lib.CVec3(_lib.dptr(a[0]), _lib.dptr(a[1]), _lib.dptr(a[2]))
        keep = {k: soa(pd[k]) for k in ("nodes", "d1", "d2", "points", "charges")}
        idx1 = np.ascontiguousarray(pd["idx_prev"], dtype=np.int32) + 1
        dm = np.ascontiguousarray(pd["dm"], dtype=np.float64)
        dp = np.ascontiguousarray(pd["dp"], dtype=np.float64)
        Np = len(dm)
        rc = self._lib.vpbs_set_points(self._h, Np, keep["nodes"][1], idx1.ctypes.data_as(_lib.c_int32_p),
                                       keep["d1"][1], keep["d2"][1], _lib.dptr(dm), _lib.dptr(dp),
                                       keep["points"][1], keep["charges"][1])
        _lib.check(rc, self._h, "set_points")
        self.Np = Np
        self._offsets = np.array([0, Np])


def init_cache(params: ParamsBiotSavart, fs=None) -> BiotSavartCache:
    """BiotSavart.init_cache (src/BiotSavart/cache.jl:40-49)."""
    return BiotSavartCache(params)


def _lia_mode(LIA) -> int:
    if LIA is True:
        return _lib.LIA_TRUE
    if LIA is False:
        return _lib.LIA_FALSE
    if LIA == "only":
        return _lib.LIA_ONLY
    raise ValueError("LIA must be True, False or 'only'")


def compute_on_nodes_(fields: dict, cache: BiotSavartCache, fs, *, LIA=True, shortrange=True, longrange=True,
                      integration_cutoff=None, callback_vorticity=None):
    """compute_on_nodes! (src/BiotSavart/BiotSavart.jl:395-612): overwrite `fields`
    (keys "velocity" and/or "streamfunction", each a list of (N_f, 3) arrays)."""
    names = set(fields)
    if not names or not names <= {"velocity", "streamfunction"}:
        raise ValueError(f"some of these fields were not recognised: {tuple(fields)}")
    for us in fields.values():
        if len(us) != len(fs):
            raise ValueError("wrong dimensions of vector")
        for u, f in zip(us, fs):
            if np.shape(u) != np.shape(f):
                raise ValueError("wrong dimensions of vector")
    mask = (_lib.VELOCITY if "velocity" in names else 0) | (_lib.STREAMFUNCTION if "streamfunction" in names else 0)
    cache.set_filaments(fs)
    cache.compute(mask, _lia_mode(LIA), shortrange, longrange, integration_cutoff)
    if callback_vorticity is not None and longrange and LIA != "only" and cache.params.is_periodic:
        # the reference fires the callback while the cache holds the unsmoothed vorticity
        # (BiotSavart.jl:436-438); here the evaluation is already complete, so the state is set to
        # the vorticity for the callback and put back afterwards unless the callback changed it
        after = cache.state
        cache.state = LongRangeCacheState("vorticity", 0.0)
        callback_vorticity(cache)
        if cache.state.quantity == "vorticity" and cache.state.smoothing_scale == 0.0:
            cache.state = after
    for name, bit in (("velocity", _lib.VELOCITY), ("streamfunction", _lib.STREAMFUNCTION)):
        if name in names:
            cache.get_list(bit, fields[name])
    return fields


def velocity_on_nodes_(vs, cache: BiotSavartCache, fs, **kws):
    """velocity_on_nodes! (src/BiotSavart/BiotSavart.jl:152-161)."""
    compute_on_nodes_({"velocity": vs}, cache, fs, **kws)
    return vs


def velocity_on_nodes(cache: BiotSavartCache, fs, **kws):
    """velocity_on_nodes (src/BiotSavart/BiotSavart.jl:94-102)."""
    vs = [np.empty_like(np.asarray(f, dtype=np.float64)) for f in fs]
    return velocity_on_nodes_(vs, cache, fs, **kws)


class SplitDevicesCache:
    """The reference's default placement of the two halves of compute_on_nodes! on two GPUs
    (src/BiotSavart/BiotSavart.jl:535-605): the long range on `long_device` (its cache holds the
    Fourier field, for the diagnostics) and the short range (local term, pairs) on `short_device`,
    evaluated concurrently; the short-range fields then cross once, by a peer copy, and are added on
    the long-range device (vpbs_add_field).  The two devices may be the same."""

    def __init__(self, params: ParamsBiotSavart, long_device: int = 0, short_device: int = 1):
        if not params.is_periodic:
            raise ValueError("the device split needs a periodic domain (Ewald splitting)")
        self.params = params
        self.long = BiotSavartCache(params.with_(device=long_device))
        self.short = BiotSavartCache(params.with_(device=short_device))
        self._lib = self.long._lib

    def close(self):
        self.long.close()
        self.short.close()

    def compute_on_nodes_(self, fields: dict, fs, *, LIA=True, shortrange=True, longrange=True,
                          integration_cutoff=None):
        names = set(fields)
        if not names or not names <= {"velocity", "streamfunction"}:
            raise ValueError(f"some of these fields were not recognised: {tuple(fields)}")
        mask = ((_lib.VELOCITY if "velocity" in names else 0) |
                (_lib.STREAMFUNCTION if "streamfunction" in names else 0))
        lia = _lia_mode(LIA)
        self.short.set_filaments(fs)
        self.long.set_filaments(fs)
        # both halves are queued before either is waited for: they run concurrently
        self.short.compute(mask, lia, shortrange, False, integration_cutoff)
        self.long.compute(mask, lia, False, longrange, integration_cutoff)
        _lib.check(self._lib.vpbs_add_field(self.long.handle, self.short.handle, mask), self.long.handle,
                   "add_field")
        for name, bit in (("velocity", _lib.VELOCITY), ("streamfunction", _lib.STREAMFUNCTION)):
            if name in names:
                self.long.get_list(bit, fields[name])
        return fields


def _wavenumbers(sp):
    Ns = sp.Ns
    return (np.fft.rfftfreq(Ns[0], 1 / Ns[0]) * 2 * np.pi / sp.Ls[0],
            np.fft.fftfreq(Ns[1], 1 / Ns[1]) * 2 * np.pi / sp.Ls[1],
            np.fft.fftfreq(Ns[2], 1 / Ns[2]) * 2 * np.pi / sp.Ls[2])


def get_longrange_field_fourier(cache: BiotSavartCache):
    """get_longrange_field_fourier (src/BiotSavart/cache.jl:72-83): returns
    ``{"field": (ux, uy, uz), "wavenumbers": (kx, ky, kz), "state": LongRangeCacheState}``
    with each component a complex array of shape (Ns0/2+1, Ns1, Ns2) (x first, as in Julia).
    The field is the cache state's quantity: the velocity after a velocity evaluation, the
    streamfunction after a streamfunction-only one, the vorticity inside ``callback_vorticity``
    and after ``to_coarse_grained_vorticity_``."""
    q = cache.state.quantity
    if q not in _lib.QUANTITY:
        raise RuntimeError(f"no long-range field in the cache ({cache.state})")
    sp = cache.params.splitting
    Ns = sp.Ns
    nkx = Ns[0] // 2 + 1
    buf = np.empty(2 * 3 * nkx * Ns[1] * Ns[2])
    _lib.check(cache._lib.vpbs_get_field_fourier(cache.handle, _lib.QUANTITY[q], _lib.dptr(buf), buf.size),
               cache.handle, "get_longrange_field_fourier")
    u = buf.view(np.complex128).reshape(3, Ns[2], Ns[1], nkx)
    field = tuple(np.ascontiguousarray(u[c].transpose(2, 1, 0)) for c in range(3))
    return {"field": field, "wavenumbers": _wavenumbers(sp),
            "state": LongRangeCacheState(q, cache.state.smoothing_scale)}


def to_coarse_grained_vorticity_(cache: BiotSavartCache, ell: float):
    """to_coarse_grained_vorticity! (src/BiotSavart/longrange/longrange.jl:273-293): Gaussian
    filter exp(-k^2 (ell^2 - ell_old^2) / 2) of the vorticity -- the curl of the held velocity,
    or the held vorticity -- on the device; the state becomes (vorticity, ell).  Returns
    ``get_longrange_field_fourier(cache)``."""
    q = cache.state.quantity
    if q not in ("velocity", "vorticity"):
        raise RuntimeError(f"expected either the velocity or vorticity to be in the cache (got state.quantity = {q})")
    ell_old = cache.state.smoothing_scale
    factor = (float(ell) ** 2 - ell_old ** 2) / 2
    _lib.check(cache._lib.vpbs_coarse_grain(cache.handle, factor, int(q == "velocity")), cache.handle,
               "to_coarse_grained_vorticity!")
    cache.state = LongRangeCacheState("vorticity", float(ell))
    return get_longrange_field_fourier(cache)


def interpolate_to_physical(cache: BiotSavartCache) -> np.ndarray:
    """interpolate_to_physical! with the default callback + copy_long_range_output!
    (longrange.jl:360-378): the held field of the cache state (no Ewald filter) at the nodes of
    the last evaluation, as an (N_p, 3) array in filament order."""
    q = cache.state.quantity
    if q not in _lib.QUANTITY:
        raise RuntimeError(f"no long-range field in the cache ({cache.state})")
    out = np.empty((cache.Np, 3))
    _lib.check(cache._lib.vpbs_interpolate_field(cache.handle, _lib.QUANTITY[q], _lib.dptr(out)), cache.handle,
               "interpolate_to_physical!")
    return out
