"""ctypes binding of the host driver (``include/mlbm_driver.h``): command
files, the GPU run loop, Stats.txt / VTK output, cluster statistics."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .capi import Params, check, lib

_VP = C.c_void_p


class StatsRow(C.Structure):
    """``mlbm_stats_row`` -- one Stats.txt row."""
    _fields_ = [("step", C.c_int64), ("min_rho", C.c_double),
                ("max_rho", C.c_double), ("min_p", C.c_double),
                ("max_p", C.c_double), ("avg_liq_press", C.c_double),
                ("avg_vap_press", C.c_double), ("suction", C.c_double),
                ("saturation", C.c_double), ("avg_liq_rho", C.c_double),
                ("avg_vap_rho", C.c_double), ("liq_cluster_count", C.c_int64),
                ("cluster_order", C.c_double), ("wet_coord_num", C.c_double),
                ("gas_cluster_count", C.c_int64),
                ("liquid_solid_boundary", C.c_double),
                ("liquid_vapor_boundary", C.c_double),
                ("cluster_radius", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


DRIVER_SIGNATURES = [
    ("mlbm_driver_create", C.c_int, [C.POINTER(_VP)]),
    ("mlbm_driver_destroy", C.c_int, [_VP]),
    ("mlbm_driver_read", C.c_int, [_VP, C.c_char_p]),
    ("mlbm_driver_init", C.c_int, [_VP]),
    ("mlbm_driver_run", C.c_int, [_VP, C.c_int32]),
    ("mlbm_driver_write_vtk", C.c_int, [_VP, C.c_int64]),
    ("mlbm_driver_dims", C.c_int, [_VP, _VP]),
    ("mlbm_driver_arrays", C.c_int, [_VP, C.POINTER(_VP), C.POINTER(_VP),
                                     C.POINTER(_VP)]),
    ("mlbm_driver_params", C.c_int, [_VP, C.POINTER(Params)]),
    ("mlbm_driver_last_stats", C.c_int, [_VP, C.POINTER(StatsRow)]),
    ("mlbm_driver_info", C.c_int, [_VP] + [_VP] * 7),
    ("mlbm_driver_lattice", _VP, [_VP]),
    ("mlbm_cluster_stats", C.c_int, [_VP, _VP, _VP, C.c_int32, C.c_int32,
                                     C.c_int32, C.c_float, C.c_float,
                                     C.c_int64, _VP, _VP, C.POINTER(StatsRow)]),
    ("mlbm_cluster_stats_gpu", C.c_int, [_VP, _VP, _VP, C.c_int32, C.c_int32,
                                         C.c_int32, C.c_float, C.c_float,
                                         C.c_int64, C.c_int32, _VP, _VP,
                                         C.POINTER(StatsRow)]),
]

_bound = False


def dlib() -> C.CDLL:
    global _bound
    L = lib()
    if not _bound:
        for name, res, args in DRIVER_SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _bound = True
    return L


class Driver:
    """The reference's MultiphaseLBM run surface: read / init / run."""

    def __init__(self):
        h = C.c_void_p()
        check(dlib().mlbm_driver_create(C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            dlib().mlbm_driver_destroy(self.h)
            self.h = None

    __del__ = close

    def read(self, path: str):
        check(dlib().mlbm_driver_read(self.h, path.encode()))

    def init(self):
        check(dlib().mlbm_driver_init(self.h))

    def run(self, quiet: bool = True):
        check(dlib().mlbm_driver_run(self.h, 1 if quiet else 0))

    def dims(self):
        d = np.zeros(3, np.int32)
        check(dlib().mlbm_driver_dims(self.h, d.ctypes.data))
        return tuple(d.tolist())

    def arrays(self):
        """(rho, is_fluid, solid_number) host arrays (copies)."""
        r, f, s = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(dlib().mlbm_driver_arrays(self.h, C.byref(r), C.byref(f),
                                        C.byref(s)))
        shape = self.dims()
        n = int(np.prod(shape))
        rho = np.ctypeslib.as_array((C.c_float * n).from_address(r.value)).reshape(shape).copy()
        fl = np.ctypeslib.as_array((C.c_uint8 * n).from_address(f.value)).reshape(shape).copy()
        sn = np.ctypeslib.as_array((C.c_int64 * n).from_address(s.value)).reshape(shape).copy()
        return rho, fl, sn

    def params(self) -> Params:
        p = Params()
        check(dlib().mlbm_driver_params(self.h, C.byref(p)))
        return p

    def last_stats(self) -> dict:
        r = StatsRow()
        check(dlib().mlbm_driver_last_stats(self.h, C.byref(r)))
        return r.as_dict()

    def info(self) -> dict:
        vals = [C.c_int64() for _ in range(5)]
        pd, st = C.c_double(), C.c_int32()
        check(dlib().mlbm_driver_info(self.h, *[C.byref(v) for v in vals],
                                      C.byref(pd), C.byref(st)))
        keys = ["step", "step_max", "statPeriod", "vtkPeriod", "solid_count"]
        d = {k: v.value for k, v in zip(keys, vals)}
        d["packing_density"] = pd.value
        d["storage"] = st.value
        return d


def cluster_stats(rho, fluid, solid_number, rhol, rhog, solid_count,
                  device=None):
    """Cluster columns of a Stats.txt row plus liquid / gas labels; on the
    host, or on GPU `device` (an int) when given."""
    shape = rho.shape
    r = np.ascontiguousarray(rho, np.float32)
    f = np.ascontiguousarray(fluid, np.uint8)
    sn = np.ascontiguousarray(solid_number, np.int64)
    liq = np.zeros(shape, np.int64)
    gas = np.zeros(shape, np.int64)
    row = StatsRow()
    if device is None:
        check(dlib().mlbm_cluster_stats(
            r.ctypes.data, f.ctypes.data, sn.ctypes.data, *shape, rhol, rhog,
            solid_count, liq.ctypes.data, gas.ctypes.data, C.byref(row)))
    else:
        check(dlib().mlbm_cluster_stats_gpu(
            r.ctypes.data, f.ctypes.data, sn.ctypes.data, *shape, rhol, rhog,
            solid_count, int(device), liq.ctypes.data, gas.ctypes.data,
            C.byref(row)))
    return row.as_dict(), liq, gas
