"""ctypes binding of libvpbs.so (the C ABI declared in include/vpbs.h).

There is no fallback: if the shared library is missing or no CUDA device is usable, every
call raises.
"""

from __future__ import annotations

import ctypes as ct
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libvpbs.so"

VELOCITY = 1
STREAMFUNCTION = 2
LIA_FALSE, LIA_TRUE, LIA_ONLY = 0, 1, 2
PRECISION = {"fp64": 0, "mixed": 1}
QUANTITY = {"vorticity": 1, "streamfunction": 2, "velocity": 3}  # held long-range field
SPLITTING_GAUSSIAN = 0
SPLITTING_KAISER_BESSEL = 1

c_double_p = ct.POINTER(ct.c_double)
c_int32_p = ct.POINTER(ct.c_int32)
c_int64_p = ct.POINTER(ct.c_int64)
c_float_p = ct.POINTER(ct.c_float)


class VpbsParams(ct.Structure):
    _fields_ = [
        ("Gamma", ct.c_double), ("a", ct.c_double), ("Delta", ct.c_double),
        ("L", ct.c_double * 3), ("alpha", ct.c_double), ("rcut", ct.c_double),
        ("Ns", ct.c_int32 * 3), ("sigma", ct.c_double), ("m", ct.c_int32),
        ("nquad", ct.c_int32), ("quad_zeta", ct.c_double * 16), ("quad_w", ct.c_double * 16),
        ("nquad_near", ct.c_int32), ("quad_near_zeta", ct.c_double * 16), ("quad_near_w", ct.c_double * 16),
        ("lia_segment_fraction", ct.c_double), ("avoid_explicit_erf", ct.c_int32),
        ("truncate_spherical", ct.c_int32), ("nsubdiv", ct.c_int32), ("precision", ct.c_int32),
        ("device", ct.c_int32), ("splitting", ct.c_int32), ("kb_beta", ct.c_double), ("kb_rtol", ct.c_double),
        ("nufft_kernel", ct.c_int32),
    ]


class CVec3(ct.Structure):
    _fields_ = [("x", c_double_p), ("y", c_double_p), ("z", c_double_p)]


# name -> (restype, argtypes); every function of include/vpbs.h
SIGNATURES = {
    "vpbs_create": (ct.c_int, [ct.POINTER(VpbsParams), ct.POINTER(ct.c_void_p)]),
    "vpbs_destroy": (ct.c_int, [ct.c_void_p]),
    "vpbs_last_error": (ct.c_char_p, [ct.c_void_p]),
    "vpbs_set_stream": (ct.c_int, [ct.c_void_p, ct.c_void_p]),
    "vpbs_set_filaments": (ct.c_int, [ct.c_void_p, ct.c_int64, c_int64_p, ct.c_void_p, ct.c_int32]),
    "vpbs_set_filament_offsets": (ct.c_int, [ct.c_void_p, ct.c_int64, c_double_p]),
    "vpbs_set_points": (ct.c_int, [ct.c_void_p, ct.c_int64, CVec3, c_int32_p, CVec3, CVec3, c_double_p, c_double_p,
                                   CVec3, CVec3]),
    "vpbs_compute": (ct.c_int, [ct.c_void_p, ct.c_int32, ct.c_int32, ct.c_int32, ct.c_int32, ct.c_double]),
    "vpbs_add_field": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_int32]),
    "vpbs_get": (ct.c_int, [ct.c_void_p, ct.c_int32, c_double_p, ct.c_int32]),
    "vpbs_get_soa": (ct.c_int, [ct.c_void_p, ct.c_int32, CVec3, ct.c_int32]),
    "vpbs_device_field": (ct.c_int, [ct.c_void_p, ct.c_int32, ct.POINTER(ct.c_void_p), ct.POINTER(ct.c_void_p),
                                     ct.POINTER(ct.c_void_p)]),
    "vpbs_get_uhat": (ct.c_int, [ct.c_void_p, c_double_p, ct.c_int64]),
    "vpbs_pair_counts": (ct.c_int, [ct.c_void_p, c_int64_p, c_int64_p]),
    "vpbs_get_pointdata": (ct.c_int, [ct.c_void_p, ct.c_int32, ct.c_void_p, ct.c_int64]),
    "vpbs_fft_size": (ct.c_int32, [ct.c_int32, ct.c_double]),
    "vpbs_launch_count": (ct.c_int64, [ct.c_void_p]),
    "vpbs_stage_timing": (ct.c_int, [ct.c_void_p, ct.c_int32]),
    "vpbs_stage_times": (ct.c_int, [ct.c_void_p, c_double_p, ct.c_int32]),
    "vpbs_stage_name": (ct.c_char_p, [ct.c_int32]),
    "vpbs_fma_throughput": (ct.c_int, [ct.c_int32, ct.c_int32, c_double_p]),
    "vpbs_ewald_table_eval": (ct.c_int, [ct.c_double, c_double_p, ct.c_int64, c_double_p, c_double_p]),
    "vpbs_kb_weights": (ct.c_int, [ct.c_double, ct.c_double, ct.c_double, c_double_p, ct.c_int64, c_double_p,
                                   c_double_p, c_double_p, c_double_p]),
    "vpbs_f32_weights_eval": (ct.c_int, [ct.c_int32, ct.c_double, ct.c_double, ct.c_double, ct.c_double, c_double_p,
                                         ct.c_int64, c_float_p, c_float_p]),
    "vpbs_periodic_eval": (ct.c_int, [ct.c_double, ct.c_int32, c_double_p, ct.c_int64, c_double_p, c_int64_p]),
    "vpbs_host_copies": (ct.c_int, [ct.c_int64, ct.POINTER(ct.c_void_p), ct.POINTER(ct.c_void_p),
                                    ct.POINTER(ct.c_size_t)]),
    "vpbs_point_data_noalloc": (ct.c_int, [ct.POINTER(VpbsParams), ct.c_int64, c_int64_p, ct.c_void_p, ct.c_void_p,
                                           ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                           ct.c_void_p, ct.c_void_p, ct.c_void_p]),
    "vpbs_features": (ct.c_int, [ct.c_void_p, c_float_p, ct.c_int32]),
    "vpbs_spectrum": (ct.c_int, [ct.c_void_p, ct.c_int32, ct.c_double, c_double_p, ct.c_int64]),
    "vpbs_coarse_grain": (ct.c_int, [ct.c_void_p, ct.c_double, ct.c_int32]),
    "vpbs_get_field_fourier": (ct.c_int, [ct.c_void_p, ct.c_int32, c_double_p, ct.c_int64]),
    "vpbs_interpolate_field": (ct.c_int, [ct.c_void_p, ct.c_int32, c_double_p]),
    "vpbs_set_filament_list": (ct.c_int, [ct.c_void_p, ct.c_int64, ct.c_void_p, c_int64_p]),
    "vpbs_stage_filaments": (ct.c_int, [ct.c_void_p, ct.c_int64, ct.c_int64, ct.POINTER(c_int64_p),
                                        ct.POINTER(c_double_p)]),
    "vpbs_set_staged_filaments": (ct.c_int, [ct.c_void_p, ct.c_int64]),
    "vpbs_get_staged": (ct.c_int, [ct.c_void_p, ct.c_int32, ct.POINTER(c_double_p)]),
    "vpbs_get_filament_list": (ct.c_int, [ct.c_void_p, ct.c_int32, ct.c_void_p, ct.c_int64]),
    "vpbs_rk4_step": (ct.c_int, [ct.c_void_p, ct.c_void_p, ct.c_double]),
    "vpbs_ensemble_create": (ct.c_int, [ct.POINTER(ct.c_void_p), ct.POINTER(ct.c_void_p), c_double_p, ct.c_int32,
                                        ct.POINTER(ct.c_void_p)]),
    "vpbs_ensemble_step": (ct.c_int, [ct.c_void_p, ct.c_int32]),
    "vpbs_ensemble_synchronize": (ct.c_int, [ct.c_void_p]),
    "vpbs_ensemble_stream": (ct.c_void_p, [ct.c_void_p]),
    "vpbs_ensemble_destroy": (ct.c_int, [ct.c_void_p]),
    "vpbs_ensemble_last_error": (ct.c_char_p, []),
    "vpbs_autotune": (ct.c_int, [ct.c_void_p, c_int32_p]),
    "vpbs_autotune_spread": (ct.c_int, [ct.c_void_p, c_int32_p]),
    "vpbs_pair_block": (ct.c_int, [ct.c_void_p, ct.c_int32]),
    "vpbs_spread_mode": (ct.c_int, [ct.c_void_p, ct.c_int32]),
    "vpbs_mlp_create": (ct.c_int, [ct.c_int32, ct.c_int32, ct.POINTER(ct.c_void_p)]),
    "vpbs_mlp_destroy": (ct.c_int, [ct.c_void_p]),
    "vpbs_mlp_last_error": (ct.c_char_p, [ct.c_void_p]),
    "vpbs_mlp_set_params": (ct.c_int, [ct.c_void_p, c_float_p, ct.c_int64]),
    "vpbs_mlp_get_params": (ct.c_int, [ct.c_void_p, c_float_p, ct.c_int64]),
    "vpbs_mlp_set_loss_weights": (ct.c_int, [ct.c_void_p, c_float_p]),
    "vpbs_mlp_set_weight_decay": (ct.c_int, [ct.c_void_p, ct.c_float]),
    "vpbs_mlp_forward": (ct.c_int, [ct.c_void_p, c_float_p, ct.c_int32, c_float_p]),
    "vpbs_mlp_gradient": (ct.c_int, [ct.c_void_p, c_float_p, c_float_p, ct.c_int32, c_float_p, c_float_p]),
    "vpbs_mlp_train_step": (ct.c_int, [ct.c_void_p, c_float_p, c_float_p, ct.c_int32, ct.c_float, c_float_p]),
}

NUM_FEATURES = 16
MLP_IN, MLP_HIDDEN, MLP_OUT = 16, 64, 5
MLP_NPARAMS = MLP_HIDDEN * MLP_IN + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_OUT * MLP_HIDDEN + MLP_OUT

NUM_STAGES = 9

_lib = None


def load(path: Path | str | None = None):
    """Load libvpbs.so and declare its prototypes (raises if the library is missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"libvpbs.so not found at {p}; build it with vortexpasta.jl_b200/build.py")
    lib = ct.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class VpbsError(RuntimeError):
    pass


def check(rc: int, handle=None, what: str = ""):
    if rc != 0:
        lib = load()
        msg = lib.vpbs_last_error(handle)
        raise VpbsError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")


def dptr(a):
    """ctypes double* of a contiguous float64 numpy array."""
    return a.ctypes.data_as(c_double_p)


def fptr(a):
    """ctypes float* of a contiguous float32 numpy array."""
    return a.ctypes.data_as(c_float_p)
