"""ctypes binding of the host-side driver surface (``include/mlbm_host.h``):
geometry, initial density and positions files.  Arrays use the reference
layout ``[x][y][z]`` (z fastest)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .capi import check, lib

_VP = C.c_void_p
HOST_SIGNATURES = [
    ("mlbm_place_sphere", C.c_int, [_VP, _VP, C.c_int32, C.c_int32, C.c_int32,
                                    C.c_float, C.c_float, C.c_float, C.c_float,
                                    C.c_int64]),
    ("mlbm_read_positions", C.c_int, [C.c_char_p, C.c_float, _VP, _VP,
                                      C.c_int32, C.c_int32, C.c_int32, _VP]),
    ("mlbm_init_density", C.c_int, [_VP, C.c_int32, C.c_int32, C.c_int32,
                                    C.c_float, C.c_float]),
    ("mlbm_generate_packing", C.c_int, [C.c_int32, C.c_int32, C.c_int32,
                                        C.c_float, C.c_float, C.c_double,
                                        C.c_uint64, C.c_int64, _VP, _VP, _VP,
                                        _VP]),
    ("mlbm_generate_packing_gpu", C.c_int, [C.c_int32, C.c_int32, C.c_int32,
                                            C.c_float, C.c_float, C.c_double,
                                            C.c_uint64, C.c_int64, C.c_int32,
                                            _VP, _VP, _VP, _VP]),
    ("mlbm_generate_solids", C.c_int, [_VP, _VP, C.c_int32, C.c_int32,
                                       C.c_int32, C.c_int32] + [C.c_float] * 8
     + [_VP]),
    ("mlbm_write_positions", C.c_int, [C.c_char_p, _VP, C.c_int64]),
    ("mlbm_packing_density", C.c_double, [_VP, C.c_int32, C.c_int32,
                                          C.c_int32]),
    ("mlbm_read_density_vtk", C.c_int, [C.c_char_p, _VP, C.c_int32, C.c_int32,
                                        C.c_int32]),
]

_bound = False


def hlib() -> C.CDLL:
    global _bound
    L = lib()
    if not _bound:
        for name, res, args in HOST_SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _bound = True
    return L


def place_sphere(fluid: np.ndarray, x, y, z, r, solid_number=None, sid=0):
    assert fluid.dtype == np.uint8 and fluid.flags.c_contiguous
    sn = solid_number.ctypes.data if solid_number is not None else None
    check(hlib().mlbm_place_sphere(fluid.ctypes.data, sn, *fluid.shape,
                                   x, y, z, r, sid))


def read_positions(path: str, shape, resolution: float = 1.0, fluid=None,
                   solid_number=None, count: int = 0):
    """Place every grain of a positions file; returns (fluid, solid_number,
    grain count)."""
    if fluid is None:
        fluid = np.ones(shape, np.uint8)
    if solid_number is None:
        solid_number = np.zeros(shape, np.int64)
    n = C.c_int64(count)
    check(hlib().mlbm_read_positions(path.encode(), resolution,
                                     fluid.ctypes.data, solid_number.ctypes.data,
                                     *shape, C.byref(n)))
    return fluid, solid_number, n.value


def init_density(shape, rho0: float, rate: float) -> np.ndarray:
    rho = np.empty(shape, np.float32)
    check(hlib().mlbm_init_density(rho.ctypes.data, *shape, rho0, rate))
    return rho


def generate_packing(shape, rmin: float, rmax: float, porosity: float,
                     seed: int, max_spheres: int = 10_000_000, device=None):
    """Seeded sphere packing to a porosity target: (fluid, spheres[n, 4]).
    With `device` (a GPU index) the voxelisation runs on that GPU; the
    result is the same, bit for bit."""
    fluid = np.ones(shape, np.uint8)
    cap = int(min(max_spheres, 2 + np.prod(shape) // 4))
    xyzr = np.zeros((cap, 4), np.float32)
    n = C.c_int64()
    por = C.c_double()
    if device is None:
        check(hlib().mlbm_generate_packing(*shape, rmin, rmax, porosity,
                                           seed & (2**64 - 1), cap,
                                           fluid.ctypes.data, xyzr.ctypes.data,
                                           C.byref(n), C.byref(por)))
    else:
        check(hlib().mlbm_generate_packing_gpu(*shape, rmin, rmax, porosity,
                                               seed & (2**64 - 1), cap,
                                               int(device), fluid.ctypes.data,
                                               xyzr.ctypes.data, C.byref(n),
                                               C.byref(por)))
    return fluid, xyzr[: n.value].copy()


def write_positions(path: str, xyzr: np.ndarray) -> None:
    a = np.ascontiguousarray(xyzr, np.float32)
    check(hlib().mlbm_write_positions(path.encode(), a.ctypes.data, len(a)))


def packing_density(fluid: np.ndarray) -> float:
    f = np.ascontiguousarray(fluid, np.uint8)
    return hlib().mlbm_packing_density(f.ctypes.data, *f.shape)


def read_density_vtk(path: str, shape) -> np.ndarray:
    rho = np.empty(shape, np.float32)
    check(hlib().mlbm_read_density_vtk(path.encode(), rho.ctypes.data, *shape))
    return rho
