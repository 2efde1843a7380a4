"""mlbm_phase_stats_noalloc: phase statistics for callers that cannot
allocate device memory when they need them (an application whose own pool
holds the GPU's memory, or a host that forbids library allocations because
cudaMalloc may synchronise the device).

It takes device fields the caller owns and keeps its scratch in a fixed
static device array, so it must give the same statistics as the allocating
mlbm_phase_stats -- on two calls in a row, since the second call reuses the
array the first one left behind.  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import sphere_case

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    from multiphase_lbm_b200 import capi
    fn = capi.lib().mlbm_phase_stats_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                   C.POINTER(capi.Params), C.c_void_p, C.POINTER(capi.Stats)]
    return fn


def test_noalloc_stats_match_allocating_entry_point_twice():
    import torch
    from multiphase_lbm_b200 import capi
    shape = (48, 40, 36)
    fluid, rho = sphere_case(shape, seed=31, rho0=0.7, amp=0.01)
    params = capi.default_params(G=-6.0, tau=1.0, rhos=0.182322)
    lat = capi.Lattice(shape)
    lat.set_params(params)
    lat.upload(fluid, rho)
    lat.initialize()
    lat.iterate(0, 300)
    ref = lat.stats()  # the existing (allocating) entry point

    rho_dev = torch.empty(shape, dtype=torch.float32, device="cuda")
    fl_dev = torch.empty(shape, dtype=torch.uint8, device="cuda")
    capi.check(capi.lib().mlbm_download_field_device(
        lat.h, capi.FIELD_RHO, capi.DTYPE_F32, C.c_void_p(rho_dev.data_ptr())))
    capi.check(capi.lib().mlbm_download_field_device(
        lat.h, capi.FIELD_FLUID, capi.DTYPE_U8, C.c_void_p(fl_dev.data_ptr())))
    torch.cuda.synchronize()

    fn = _noalloc_fn()
    results = []
    for _ in range(2):
        out = capi.Stats()
        capi.check(fn(C.c_void_p(rho_dev.data_ptr()),
                      C.c_void_p(fl_dev.data_ptr()), *shape, C.byref(params),
                      None, C.byref(out)))
        results.append(out.as_dict())

    for got in results:
        for k in ("n_fluid", "n_liquid", "n_vapour", "n_liquid_solid_boundary",
                  "n_liquid_vapour_boundary"):
            assert got[k] == ref[k], k
        for k in ("min_rho", "max_rho", "min_p", "max_p"):
            assert got[k] == ref[k], k
        for k in ("mass", "sum_p_liquid", "sum_p_vapour", "sum_rho_liquid",
                  "sum_rho_vapour", "saturation", "avg_p_liquid",
                  "avg_p_vapour", "suction", "avg_rho_liquid",
                  "avg_rho_vapour"):
            assert got[k] == pytest.approx(ref[k], rel=1e-9, abs=1e-12), k
    assert results[0] == results[1]
    assert 0 < ref["n_liquid"] < ref["n_fluid"]
    lat.close()


def test_noalloc_on_a_user_stream_and_at_the_largest_lx():
    """On a stream of the caller's (not the legacy default), and at lx equal
    to MLBM_NOALLOC_MAX_LX, the largest the scratch array holds: the same
    statistics as the allocating entry point."""
    import torch
    from multiphase_lbm_b200 import capi
    shape = (4096, 3, 4)
    fluid, rho = sphere_case(shape, seed=5, rmin=1.0, rmax=1.5, porosity=0.7,
                             rho0=0.7, amp=0.5)
    params = capi.default_params(G=-6.0, tau=1.0, rhos=0.182322)
    lat = capi.Lattice(shape)
    lat.set_params(params)
    lat.upload(fluid, rho)
    lat.initialize()
    lat.iterate(0, 3)
    ref = lat.stats()
    rho_dev = torch.empty(shape, dtype=torch.float32, device="cuda")
    fl_dev = torch.empty(shape, dtype=torch.uint8, device="cuda")
    capi.check(capi.lib().mlbm_download_field_device(
        lat.h, capi.FIELD_RHO, capi.DTYPE_F32, C.c_void_p(rho_dev.data_ptr())))
    capi.check(capi.lib().mlbm_download_field_device(
        lat.h, capi.FIELD_FLUID, capi.DTYPE_U8, C.c_void_p(fl_dev.data_ptr())))
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    out = capi.Stats()
    capi.check(_noalloc_fn()(C.c_void_p(rho_dev.data_ptr()),
                             C.c_void_p(fl_dev.data_ptr()), *shape,
                             C.byref(params), C.c_void_p(stream.cuda_stream),
                             C.byref(out)))
    got = out.as_dict()
    for k in ("n_fluid", "n_liquid", "n_vapour", "min_rho", "max_rho"):
        assert got[k] == ref[k], k
    assert got["mass"] == pytest.approx(ref["mass"], rel=1e-9)
    lat.close()


def test_noalloc_rejects_lattices_beyond_its_scratch():
    from multiphase_lbm_b200 import capi
    fn = _noalloc_fn()
    params = capi.default_params()
    out = capi.Stats()
    big_lx = 4097  # MLBM_NOALLOC_MAX_LX + 1
    st = fn(C.c_void_p(16), C.c_void_p(16), big_lx, 4, 4, C.byref(params),
            None, C.byref(out))
    assert st == 1  # MLBM_ERR_ARG, nothing launched
    assert b"MLBM_NOALLOC_MAX_LX" in capi.lib().mlbm_last_error()
