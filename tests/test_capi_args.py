"""Argument checks of the newer C ABI entry points, on the CPU: each call
below is refused with MLBM_ERR_ARG and a message before it touches the
device, as the reference's own entry points would fail loudly on bad input
(they exit instead, include/iteration_host.h:6-15)."""
import ctypes as C

import numpy as np
import pytest

from multiphase_lbm_b200 import capi, driver

ERR_ARG = 1


def _refused(status, words):
    assert status == ERR_ARG
    msg = capi.lib().mlbm_last_error().decode()
    assert words in msg, msg


def test_slab_entry_points_refuse_bad_arguments():
    L = capi.lib()
    _refused(L.mlbm_set_slab(None, 1), "null lattice")
    _refused(L.mlbm_step_pass(None, 0, 0, 1, 0, 0), "null lattice")
    _refused(L.mlbm_step_pass(None, 0, 2, 1, 0, 0), "pass must be 0")
    ptrs = (C.c_void_p * capi.HALO_MAX_SEGMENTS)()
    nb = np.zeros(capi.HALO_MAX_SEGMENTS, np.int64)
    n = C.c_int32()
    _refused(L.mlbm_halo_segments(None, 0, 0, None, None, None), "null output")
    _refused(L.mlbm_halo_segments(None, 0, 2, ptrs, nb.ctypes.data, C.byref(n)),
             "side must be")
    _refused(L.mlbm_halo_segments(None, 9, 0, ptrs, nb.ctypes.data, C.byref(n)),
             "unknown kind")
    _refused(L.mlbm_halo_segments(None, 0, 0, ptrs, nb.ctypes.data, C.byref(n)),
             "null lattice")


def test_slab_ring_refuses_bad_arguments():
    L = capi.lib()
    out = C.c_void_p()
    _refused(L.mlbm_slab_ring_create(None, 0, C.byref(out)), "bad arguments")
    arr = (C.c_void_p * 1)(None)
    _refused(L.mlbm_slab_ring_create(arr, 1, C.byref(out)), "null lattice")
    assert not out.value
    _refused(L.mlbm_slab_ring_exchange(None, 0), "null ring")
    assert L.mlbm_slab_ring_destroy(None) == 0


def test_statistics_entry_points_refuse_bad_arguments():
    L = capi.lib()
    raw = np.zeros(capi.STATS_RAW_LEN, np.float64)
    _refused(L.mlbm_phase_stats_async(None, raw.ctypes.data), "null lattice")
    _refused(L.mlbm_bulk_stats_async(None, raw.ctypes.data), "null lattice")
    s = capi.Stats()
    _refused(L.mlbm_stats_from_raw(None, raw.ctypes.data, C.byref(s)),
             "null lattice")


def test_gpu_cluster_statistics_refuse_bad_arguments():
    row = driver.StatsRow()
    L = driver.dlib()
    rho = np.zeros(8, np.float32)
    fl = np.ones(8, np.uint8)
    _refused(L.mlbm_cluster_stats_gpu(None, fl.ctypes.data, None, 2, 2, 2,
                                      0.27, 0.05, 0, 0, None, None,
                                      C.byref(row)), "bad arguments")
    _refused(L.mlbm_cluster_stats_gpu(rho.ctypes.data, fl.ctypes.data, None, 0,
                                      2, 2, 0.27, 0.05, 0, 0, None, None,
                                      C.byref(row)), "bad arguments")


def test_async_stats_buffer_checked_in_python():
    with pytest.raises(ValueError):
        capi.Lattice.stats_async(object.__new__(capi.Lattice),
                                 np.zeros(3, np.float64))


def test_checkpoint_entry_points_refuse_bad_arguments():
    L = capi.lib()
    n = C.c_uint64()
    _refused(L.mlbm_checkpoint_bytes(None, C.byref(n)), "null argument")
    _refused(L.mlbm_checkpoint_save(None, 0, None, 0), "null argument")
    _refused(L.mlbm_checkpoint_load(None, None, 0, None), "null argument")
    _refused(L.mlbm_checkpoint_write(None, 0, b"x"), "null argument")
    _refused(L.mlbm_checkpoint_read(None, b"x", None), "null argument")
    _refused(L.mlbm_checkpoint_info(None, 0, None, None, None), "null argument")
    img = np.zeros(4096, np.uint8)
    _refused(L.mlbm_checkpoint_info(img.ctypes.data, 16, None, None, None),
             "truncated")
    _refused(L.mlbm_checkpoint_info(img.ctypes.data, img.nbytes, None, None,
                                    None), "not a checkpoint")
    img[:8] = np.frombuffer(b"MLBMCKPT", np.uint8)
    img[8:12] = np.frombuffer(np.uint32(99).tobytes(), np.uint8)
    _refused(L.mlbm_checkpoint_info(img.ctypes.data, img.nbytes, None, None,
                                    None), "unsupported format version")

