"""The allocation-free entry point (smcrt_run_device_static) for callers that cannot
allocate device memory -- e.g. code running under CUDA stream capture or inside an
application-owned memory pool.  Through the C ABI it must give the same tallies
and event counters as the context-based smcrt_run_device on the same packets, on
two calls in a row (the static scratch keeps the previous call's contents, so
the second call checks that what must start at zero is cleared)."""
import ctypes as C

import numpy as np
import pytest

from signedmcrt_b200 import abi, presets as P
from signedmcrt_b200.scene import FlatScene

pytestmark = pytest.mark.gpu

KEYS = ("packets", "nscatt", "sdf_evals", "voxel_segments", "trace_steps", "scatters", "fresnel_events",
        "reflections", "rng_draws", "kills_error", "kills_step_cap")


def test_static_entry_point_matches_context_path(gpu):
    import torch
    from signedmcrt_b200 import _lib
    lib = _lib.lib()
    st = P.benchmark_settings("layered_vessels")
    flat = FlatScene(P.setup_simulation(st))
    n, first, seed = 40000, 1000, 77
    with gpu.Transport(flat, st, precision="fp32", stream=0) as tr:
        jm_ref = torch.zeros(tr.ncell, dtype=torch.float64, device="cuda")
        bins_ref = torch.zeros(tr.nbins, dtype=torch.float64, device="cuda")
        ref = tr.run_device(first, n, seed, jm_ref.data_ptr(), bins_ref.data_ptr(), stats=True)
        ncell, nbins, opts = tr.ncell, tr.nbins, tr.options
        grid, src, dets, ndet = tr.grid, tr.source, tr._dets, tr.ndet

    assert lib.smcrt_static_scratch_bytes() >= 512
    want_j = jm_ref.cpu().numpy()
    want_b = bins_ref.cpu().numpy()
    jm = torch.empty(ncell, dtype=torch.float64, device="cuda")
    bins = torch.empty(nbins, dtype=torch.float64, device="cuda")
    for call in range(2):
        jm.zero_()
        bins.zero_()
        torch.cuda.synchronize()
        stats = abi.Stats()
        rc = lib.smcrt_run_device_static(flat.ptr(), C.byref(grid), C.byref(src), dets, ndet, C.byref(opts), first,
                                         n, seed, C.c_void_p(jm.data_ptr()), C.c_void_p(bins.data_ptr()),
                                         C.byref(stats))
        assert rc == abi.OK, lib.smcrt_last_error().decode()
        got = stats.to_dict()
        for k in KEYS:
            assert got[k] == ref[k], (call, k, got[k], ref[k])
        assert got["device_status"] == 0
        j = jm.cpu().numpy()
        # same kernel, same packets: only the order of the FP64 atomic additions differs
        assert np.allclose(j, want_j, rtol=1e-12, atol=1e-12 * want_j.max()), call
        assert np.array_equal(bins.cpu().numpy(), want_b), call


def test_static_entry_point_rejects_bad_arguments(gpu):
    from signedmcrt_b200 import _lib
    lib = _lib.lib()
    st = P.benchmark_settings("box_slab")
    flat = FlatScene(P.setup_simulation(st))
    grid, src = st.grid_c(), st.source_c()
    dets = (abi.Detector * 1)()
    opts = abi.Options()
    rc = lib.smcrt_run_device_static(flat.ptr(), C.byref(grid), C.byref(src), dets, 0, C.byref(opts), 0, 10, 1,
                                     None, None, None)
    assert rc == abi.ERR_ARG and b"fluence buffer" in lib.smcrt_last_error()


def test_static_entry_point_leaves_device_memory_untouched(gpu):
    """Callers whose device memory is owned by their own pool (or budgeted up front)
    need the call to take no memory of its own: the device's free memory is the
    same before and after an allocation-free run (after a first call, which only
    looks up the static array's device address)."""
    import torch
    from signedmcrt_b200 import _lib
    lib = _lib.lib()
    st = P.benchmark_settings("box_slab")
    flat = FlatScene(P.setup_simulation(st))
    grid, src = st.grid_c(), st.source_c()
    dets = (abi.Detector * 1)()
    opts = abi.Options()
    ncell = st.grid.nxg * st.grid.nyg * st.grid.nzg
    jm = torch.zeros(ncell, dtype=torch.float64, device="cuda")

    def call():
        stats = abi.Stats()
        rc = lib.smcrt_run_device_static(flat.ptr(), C.byref(grid), C.byref(src), dets, 0, C.byref(opts), 0, 20000,
                                         5, C.c_void_p(jm.data_ptr()), None, C.byref(stats))
        assert rc == abi.OK, lib.smcrt_last_error().decode()
        return stats.to_dict()

    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    st1 = call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert st1["packets"] == 20000
    assert free1 == free0, (free0, free1)
