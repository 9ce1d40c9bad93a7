"""CUDA (sm_100a) drop-in for VortexPasta.BiotSavart's Ewald-split velocity and
streamfunction evaluation on vortex-filament nodes.

The compute path is libvpbs.so (C ABI in include/vpbs.h); this package mirrors the
reference's BiotSavart API on top of it.
"""

from . import configs, curves, diagnostics, learned, timestepping, tuning
from ._lib import LIB_PATH, VpbsError
from .biotsavart import (BiotSavartCache, LongRangeCacheState, SplitDevicesCache, compute_on_nodes_, get_longrange_field_fourier,
                         init_cache, interpolate_to_physical, to_coarse_grained_vorticity_, velocity_on_nodes,
                         velocity_on_nodes_)
from .params import (CellListsBackend, GaussianSplitting, GaussLegendre, KaiserBesselSplitting, NaiveShortRangeBackend,
                     NonuniformFFTsBackend, NoSplitting, ParamsBiotSavart, kmax_to_gridsize, maximum_wavenumber)

__all__ = [
    "configs", "curves", "diagnostics", "learned", "timestepping", "tuning", "LIB_PATH", "VpbsError", "BiotSavartCache", "LongRangeCacheState", "compute_on_nodes_",
    "get_longrange_field_fourier", "init_cache", "SplitDevicesCache", "interpolate_to_physical", "to_coarse_grained_vorticity_",
    "velocity_on_nodes", "velocity_on_nodes_", "CellListsBackend",
    "GaussianSplitting", "GaussLegendre", "KaiserBesselSplitting", "NaiveShortRangeBackend", "NonuniformFFTsBackend", "NoSplitting",
    "ParamsBiotSavart", "kmax_to_gridsize", "maximum_wavenumber",
]
