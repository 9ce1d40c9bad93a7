"""The allocation-free point-data entry point (vpbs_point_data_noalloc).

It exists for callers that cannot allocate device memory (an external pool owns the GPU's
memory, cudaMalloc is not allowed where they run, or their binding can only pass buffers it
already holds).  The caller owns every input and output buffer; the library keeps its
intermediates in a fixed file-scope device array.  This file is collected last on purpose.
"""

import ctypes as ct

import numpy as np
import pytest


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _call_noalloc(vp, p, fs, torch):
    from vortexpasta_b200 import _lib
    from vortexpasta_b200.biotsavart import _c_params
    lib = _lib.load()
    nodes, offsets = vp.curves.concat(fs)
    Np = int(offsets[-1])
    Nq = Np * len(p.quadrature)
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(nodes).to(dev)
    out = {
        "nodes": torch.empty(3 * Np, dtype=torch.float64, device=dev),
        "idx_prev": torch.empty(Np, dtype=torch.int32, device=dev),
        "d1": torch.empty(3 * Np, dtype=torch.float64, device=dev),
        "d2": torch.empty(3 * Np, dtype=torch.float64, device=dev),
        "dm": torch.empty(Np, dtype=torch.float64, device=dev),
        "dp": torch.empty(Np, dtype=torch.float64, device=dev),
        "points": torch.empty(3 * Nq, dtype=torch.float64, device=dev),
        "charges": torch.empty(3 * Nq, dtype=torch.float64, device=dev),
    }
    cp = _c_params(p)
    stream = torch.cuda.current_stream(dev)
    rc = lib.vpbs_point_data_noalloc(
        ct.byref(cp), len(fs), offsets.ctypes.data_as(_lib.c_int64_p), ct.c_void_p(x.data_ptr()),
        ct.c_void_p(stream.cuda_stream),
        *[ct.c_void_p(out[k].data_ptr()) for k in ("nodes", "idx_prev", "d1", "d2", "dm", "dp", "points", "charges")])
    assert rc == 0, lib.vpbs_last_error(None)
    torch.cuda.synchronize()
    res = {}
    for k, t in out.items():
        a = t.cpu().numpy()
        res[k] = a.reshape(3, -1).T if k in ("nodes", "d1", "d2", "points", "charges") else a
    return res


def _check_against_set_filaments(vp, p, fs, got):
    tol = {"d2": 1e-10}  # same tolerances as test_gpu_parity.test_point_data_matches_oracle
    cache = vp.init_cache(p)
    cache.set_filaments(fs)
    ref = cache.pointdata()
    cache.close()
    for k in ("nodes", "d1", "d2", "dm", "dp", "points", "charges"):
        assert rel(got[k], ref[k]) < tol.get(k, 1e-12), k
    np.testing.assert_array_equal(got["idx_prev"], ref["idx_prev"])


@pytest.mark.gpu
def test_noalloc_matches_set_filaments_two_calls(vp, built_lib):
    import torch
    _, p = vp.configs.tangle20k()
    for seed, nrings in ((7, 40), (8, 25)):  # two calls in a row, different sizes
        fs = vp.configs.tangle(nrings, 200, seed=seed) + [vp.curves.ring(5, 0.3, center=(1, 1, 1))]
        got = _call_noalloc(vp, p, fs, torch)
        _check_against_set_filaments(vp, p, fs, got)


@pytest.mark.gpu
def test_noalloc_with_lia_segment_fraction(vp, built_lib):
    """With lia_segment_fraction the library's own path writes the quadrature points in a separate
    kernel; the allocation-free call must give the same point data."""
    import torch
    _, p = vp.configs.tangle20k()
    p = p.with_(lia_segment_fraction=0.3, quadrature_near_singularity=vp.GaussLegendre(6))
    fs = vp.configs.tangle(30, 200, seed=9) + [vp.curves.ring(6, 0.4, center=(2, 5, 1))]
    for _ in range(2):
        _check_against_set_filaments(vp, p, fs, _call_noalloc(vp, p, fs, torch))


@pytest.mark.gpu
def test_noalloc_allocates_no_device_memory(vp, built_lib):
    """After one warm-up call (which may load the module and its array), further calls leave the
    device's free memory and torch's allocation unchanged."""
    import torch
    _, p = vp.configs.tangle20k()
    fs = vp.configs.tangle(20, 200, seed=5)
    _call_noalloc(vp, p, fs, torch)
    torch.cuda.synchronize()
    # the output tensors of _call_noalloc are freed by now; the caching allocator keeps their blocks
    free0, _ = torch.cuda.mem_get_info(0)
    alloc0 = torch.cuda.memory_allocated(0)
    reserved0 = torch.cuda.memory_reserved(0)
    _call_noalloc(vp, p, fs, torch)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    assert torch.cuda.memory_allocated(0) == alloc0
    assert torch.cuda.memory_reserved(0) == reserved0


@pytest.mark.gpu
def test_noalloc_rejects_host_pointers(vp, built_lib):
    """Node and output arrays must be device memory of params->device; a host array is refused
    before any kernel runs."""
    import torch
    from vortexpasta_b200 import _lib
    from vortexpasta_b200.biotsavart import _c_params
    lib = _lib.load()
    _, p = vp.configs.tangle20k()
    fs = vp.configs.tangle(2, 200, seed=3)
    nodes, offsets = vp.curves.concat(fs)
    host = np.zeros(3 * 3 * len(nodes))
    dev = torch.zeros(3 * 3 * len(nodes), dtype=torch.float64, device="cuda:0")
    outs = [ct.c_void_p(dev.data_ptr())] * 8
    rc = lib.vpbs_point_data_noalloc(ct.byref(_c_params(p)), len(fs), offsets.ctypes.data_as(_lib.c_int64_p),
                                     ct.c_void_p(nodes.ctypes.data), None, *outs)
    assert rc == -1 and b"device memory" in lib.vpbs_last_error(None)
    outs[3] = ct.c_void_p(host.ctypes.data)
    x = torch.from_numpy(nodes).to("cuda:0")
    rc = lib.vpbs_point_data_noalloc(ct.byref(_c_params(p)), len(fs), offsets.ctypes.data_as(_lib.c_int64_p),
                                     ct.c_void_p(x.data_ptr()), None, *outs)
    assert rc == -1 and b"device memory" in lib.vpbs_last_error(None)


def test_noalloc_rejects_oversized_input(vp, built_lib):
    """Sizes beyond the fixed array are rejected before any device work (no GPU needed)."""
    from vortexpasta_b200 import _lib
    from vortexpasta_b200.biotsavart import _c_params
    lib = _lib.load()
    _, p = vp.configs.tangle20k()
    n = 40000  # > VPBS_NOALLOC_MAX_NODES
    offsets = np.array([0, n], dtype=np.int64)
    dummy = ct.c_void_p(1)
    rc = lib.vpbs_point_data_noalloc(ct.byref(_c_params(p)), 1, offsets.ctypes.data_as(_lib.c_int64_p), dummy, None,
                                     *([dummy] * 8))
    assert rc == -1
    assert b"at most 32768 nodes" in lib.vpbs_last_error(None)


def _reject(vp, offsets):
    from vortexpasta_b200 import _lib
    from vortexpasta_b200.biotsavart import _c_params
    lib = _lib.load()
    _, p = vp.configs.tangle20k()
    offsets = np.asarray(offsets, dtype=np.int64)
    dummy = ct.c_void_p(1)
    rc = lib.vpbs_point_data_noalloc(ct.byref(_c_params(p)), len(offsets) - 1, offsets.ctypes.data_as(_lib.c_int64_p),
                                     dummy, None, *([dummy] * 8))
    return rc, lib.vpbs_last_error(None)


def test_noalloc_rejects_too_many_filaments(vp, built_lib):
    """4097 filaments of 5 nodes (20,485 nodes, under the node limit) exceed the filament limit."""
    rc, msg = _reject(vp, np.arange(0, 5 * 4098, 5))
    assert rc == -1 and b"4096 filaments" in msg


def test_noalloc_rejects_short_filament(vp, built_lib):
    rc, msg = _reject(vp, [0, 10, 14])
    assert rc == -1 and b"at least 5 nodes" in msg


def test_noalloc_rejects_offsets_not_starting_at_zero(vp, built_lib):
    rc, msg = _reject(vp, [1, 11])
    assert rc == -1 and b"bad offsets" in msg
