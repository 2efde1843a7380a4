"""ctypes binding of ``include/mlbm_batch.h``: many independent domains of
uneven size advanced together by persistent batched launches."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .capi import Lattice, Params, STORE_F32, check, lib

_VP = C.c_void_p
BATCH_SIGNATURES = [
    ("mlbm_batch_create", C.c_int, [C.c_int32, C.c_int32, C.POINTER(_VP)]),
    ("mlbm_batch_destroy", C.c_int, [_VP]),
    ("mlbm_batch_add", C.c_int, [_VP, C.c_int32, C.c_int32, C.c_int32,
                                 C.POINTER(Params), _VP, _VP, C.c_int64,
                                 C.POINTER(C.c_int32)]),
    ("mlbm_batch_add_checkpoint", C.c_int, [_VP, _VP, C.c_uint64,
                                            C.POINTER(C.c_int32)]),
    ("mlbm_batch_remove", C.c_int, [_VP, C.c_int32]),
    ("mlbm_batch_count", C.c_int32, [_VP]),
    ("mlbm_batch_bytes", C.c_uint64, [_VP]),
    ("mlbm_batch_iterate", C.c_int, [_VP, C.c_int32, C.c_int32, C.c_uint32]),
    ("mlbm_batch_lattice", _VP, [_VP, C.c_int32]),
    ("mlbm_batch_domain_step", C.c_int64, [_VP, C.c_int32]),
    ("mlbm_batch_synchronize", C.c_int, [_VP]),
    ("mlbm_batch_set_tuning", C.c_int, [_VP] + [C.c_int32] * 5),
    ("mlbm_batch_autotune", C.c_int, [_VP, C.c_int32, _VP]),
]
_bound = False


def blib() -> C.CDLL:
    global _bound
    L = lib()
    if not _bound:
        for name, res, args in BATCH_SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _bound = True
    return L


class _View(Lattice):
    """A domain's lattice owned by the batch (not destroyed by Python)."""

    def __init__(self, handle, shape, storage):  # noqa: D401
        self.h = C.c_void_p(handle)
        self.shape = tuple(shape)
        self.storage = storage

    def close(self):
        self.h = None

    __del__ = close


class Batch:
    def __init__(self, storage: int = STORE_F32, device: int = 0):
        h = C.c_void_p()
        check(blib().mlbm_batch_create(storage, device, C.byref(h)))
        self.h = h
        self.storage = storage
        self.shapes = {}

    def close(self):
        if getattr(self, "h", None):
            blib().mlbm_batch_destroy(self.h)
            self.h = None

    __del__ = close

    def add(self, fluid, rho, params: Params, step0: int = 0) -> int:
        fl = np.ascontiguousarray(fluid, np.uint8)
        r = np.ascontiguousarray(rho, np.float32)
        did = C.c_int32()
        check(blib().mlbm_batch_add(self.h, *fl.shape, C.byref(params),
                                    fl.ctypes.data, r.ctypes.data, step0,
                                    C.byref(did)))
        self.shapes[did.value] = fl.shape
        return did.value

    def add_checkpoint(self, image: np.ndarray) -> int:
        """Admit a domain from a checkpoint image (Lattice.checkpoint); it
        resumes at the image's step, bit for bit."""
        a = np.ascontiguousarray(image, np.uint8)
        did = C.c_int32()
        check(blib().mlbm_batch_add_checkpoint(self.h, a.ctypes.data, a.nbytes,
                                               C.byref(did)))
        dims = (C.c_int32 * 3)()
        check(lib().mlbm_checkpoint_info(a.ctypes.data, a.nbytes, dims, None,
                                         None))
        self.shapes[did.value] = tuple(dims)
        return did.value

    def remove(self, did: int):
        check(blib().mlbm_batch_remove(self.h, did))
        self.shapes.pop(did, None)

    def count(self) -> int:
        return blib().mlbm_batch_count(self.h)

    def nbytes(self) -> int:
        return int(blib().mlbm_batch_bytes(self.h))

    def iterate(self, nsteps: int, reverse: int = 1, inject_type: int = 0):
        check(blib().mlbm_batch_iterate(self.h, nsteps, reverse, inject_type))

    def synchronize(self):
        check(blib().mlbm_batch_synchronize(self.h))

    def lattice(self, did: int) -> Lattice:
        h = blib().mlbm_batch_lattice(self.h, did)
        if not h:
            raise KeyError(did)
        return _View(h, self.shapes[did], self.storage)

    def domain_step(self, did: int) -> int:
        return int(blib().mlbm_batch_domain_step(self.h, did))

    def set_tuning(self, rows_density=4, rows_update=4, planes=8,
                   blocks_per_sm=0, graphs=True):
        check(blib().mlbm_batch_set_tuning(self.h, rows_density, rows_update,
                                           planes, blocks_per_sm, int(graphs)))

    def autotune(self, trial_steps: int = 4):
        out = np.zeros(4, np.int32)
        check(blib().mlbm_batch_autotune(self.h, trial_steps, out.ctypes.data))
        return dict(zip(["rows_density", "rows_update", "planes",
                         "blocks_per_sm"], out.tolist()))
