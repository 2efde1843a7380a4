"""ctypes binding of the C ABI in ``include/mlbm.h`` (``libmlbm.so``).

This is the Python face of the library: every call goes through the same
``extern "C"`` entry points a C, C++ or Fortran host would bind.  There is no
CPU fallback -- if ``libmlbm.so`` is missing or no GPU is usable, the calls
raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmlbm.so")

STORE_F32, STORE_F16, STORE_F64 = 0, 1, 2
FIELD_RHO, FIELD_PRESSURE, FIELD_PSI, FIELD_VELOCITY, FIELD_POPULATIONS, \
    FIELD_FLUID = range(6)
DTYPE_F32, DTYPE_F64, DTYPE_U8 = 0, 1, 2
ITER_WRITE_VELOCITY = 1
HALO_PSI_EDGE, HALO_PSI_GHOST, HALO_POP_EDGE, HALO_POP_GHOST = 0, 1, 2, 3
HALO_MAX_SEGMENTS = 5
STATS_RAW_LEN = 15
KERNEL_AUTO, KERNEL_TWO_PASS, KERNEL_COMPACT, KERNEL_BAND = 0, 2, 3, 6
Q = 19

STATUS = {0: "MLBM_OK", 1: "MLBM_ERR_ARG", 2: "MLBM_ERR_CUDA",
          3: "MLBM_ERR_NOMEM", 4: "MLBM_ERR_STATE", 5: "MLBM_ERR_TIMEOUT",
          6: "MLBM_ERR_IO", 7: "MLBM_ERR_PARSE"}


class MlbmError(RuntimeError):
    """A non-zero mlbm_status; ``.status`` holds the code."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Params(C.Structure):
    """``mlbm_params`` (include/mlbm.h)."""
    _fields_ = [("tau", C.c_float), ("G", C.c_float), ("T_Tc", C.c_float),
                ("rhol_spinodal", C.c_float), ("rhog_spinodal", C.c_float),
                ("rho_increment", C.c_float), ("rhos", C.c_float),
                ("inject_position", C.c_float), ("carn_star", C.c_int32),
                ("inject_density", C.c_int32),
                ("rho_inject_period", C.c_uint64),
                ("stat_period", C.c_uint64), ("inlet_width", C.c_int32),
                ("outlet_width", C.c_int32), ("rho_inlet", C.c_float),
                ("rho_outlet", C.c_float), ("rho_shift", C.c_float),
                ("reserved", C.c_int32)]


class Stats(C.Structure):
    """``mlbm_stats`` (include/mlbm.h)."""
    _fields_ = [("n_fluid", C.c_int64), ("n_liquid", C.c_int64),
                ("n_vapour", C.c_int64), ("n_liquid_solid_boundary", C.c_int64),
                ("n_liquid_vapour_boundary", C.c_int64), ("mass", C.c_double),
                ("sum_p_liquid", C.c_double), ("sum_p_vapour", C.c_double),
                ("sum_rho_liquid", C.c_double), ("sum_rho_vapour", C.c_double),
                ("saturation", C.c_double), ("avg_p_liquid", C.c_double),
                ("avg_p_vapour", C.c_double), ("suction", C.c_double),
                ("avg_rho_liquid", C.c_double), ("avg_rho_vapour", C.c_double),
                ("ratio_liquid_solid_boundary", C.c_double),
                ("ratio_liquid_vapour_boundary", C.c_double),
                ("min_rho", C.c_double), ("max_rho", C.c_double),
                ("min_p", C.c_double), ("max_p", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def default_params(**kw) -> Params:
    """Reference defaults (src/multiphase_lbm.cu:35-80) overridden by ``kw``."""
    d = dict(tau=1.0, G=-1.0, T_Tc=0.7, rhol_spinodal=0.2726,
             rhog_spinodal=0.0484, rho_increment=0.0, rhos=0.0,
             inject_position=1.0, carn_star=0, inject_density=0,
             rho_inject_period=100, stat_period=10, inlet_width=0,
             outlet_width=0, rho_inlet=0.0, rho_outlet=0.0, rho_shift=1.0,
             reserved=0)
    d.update(kw)
    return Params(**d)


_lib = None

# (name, restype, argtypes) of every exported entry point of include/mlbm.h
_VP = C.c_void_p
SIGNATURES = [
    ("mlbm_abi_version", C.c_int32, []),
    ("mlbm_status_string", C.c_char_p, [C.c_int32]),
    ("mlbm_last_error", C.c_char_p, []),
    ("mlbm_d3q19", None, [_VP, _VP]),
    ("mlbm_lattice_create", C.c_int, [C.c_int32, C.c_int32, C.c_int32,
                                      C.c_int32, C.c_int32, C.POINTER(_VP)]),
    ("mlbm_lattice_destroy", C.c_int, [_VP]),
    ("mlbm_lattice_bytes", C.c_uint64, [C.c_int32] * 4),
    ("mlbm_set_stream", C.c_int, [_VP, _VP]),
    ("mlbm_set_params", C.c_int, [_VP, C.POINTER(Params)]),
    ("mlbm_upload_fluid_mask", C.c_int, [_VP, _VP]),
    ("mlbm_upload_rho", C.c_int, [_VP, _VP]),
    ("mlbm_upload_fluid_mask_device", C.c_int, [_VP, _VP]),
    ("mlbm_upload_rho_device", C.c_int, [_VP, _VP]),
    ("mlbm_initialize", C.c_int, [_VP]),
    ("mlbm_iterate", C.c_int, [_VP, C.c_int64, C.c_int32, C.c_int32,
                               C.c_uint32, C.c_uint32]),
    ("mlbm_download_field", C.c_int, [_VP, C.c_int32, C.c_int32, _VP]),
    ("mlbm_download_field_device", C.c_int, [_VP, C.c_int32, C.c_int32, _VP]),
    ("mlbm_phase_stats", C.c_int, [_VP, C.POINTER(Stats)]),
    ("mlbm_plane_profile", C.c_int, [_VP, _VP, _VP]),
    ("mlbm_lattice_info", C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    ("mlbm_set_step_kernel", C.c_int, [_VP, C.c_int32]),
    ("mlbm_synchronize", C.c_int, [_VP]),
    ("mlbm_set_update_shape", C.c_int, [_VP, C.c_int32, C.c_int32]),
    ("mlbm_set_band_shape", C.c_int, [_VP, C.c_int32, C.c_int32]),
    ("mlbm_set_wait_limit", C.c_int, [_VP, C.c_uint64]),
    ("mlbm_test_stall_wait", C.c_int, [_VP]),
    ("mlbm_get_step_kernel", C.c_int32, [_VP]),
    ("mlbm_autotune", C.c_int, [_VP, C.c_int64, C.c_int32, _VP, _VP]),
    ("mlbm_set_slab", C.c_int, [_VP, C.c_int32]),
    ("mlbm_step_pass", C.c_int, [_VP, C.c_int64, C.c_int32, C.c_int32,
                                 C.c_uint32, C.c_uint32]),
    ("mlbm_halo_segments", C.c_int, [_VP, C.c_int32, C.c_int32, _VP, _VP,
                                     _VP]),
    ("mlbm_phase_stats_async", C.c_int, [_VP, _VP]),
    ("mlbm_bulk_stats_async", C.c_int, [_VP, _VP]),
    ("mlbm_stats_from_raw", C.c_int, [_VP, _VP, C.POINTER(Stats)]),
    ("mlbm_slab_ring_create", C.c_int, [_VP, C.c_int32, C.POINTER(_VP)]),
    ("mlbm_slab_ring_exchange", C.c_int, [_VP, C.c_int32]),
    ("mlbm_slab_ring_destroy", C.c_int, [_VP]),
    ("mlbm_checkpoint_bytes", C.c_int, [_VP, C.POINTER(C.c_uint64)]),
    ("mlbm_checkpoint_info", C.c_int, [_VP, C.c_uint64, _VP, _VP, _VP]),
    ("mlbm_checkpoint_save", C.c_int, [_VP, C.c_int64, _VP, C.c_uint64]),
    ("mlbm_checkpoint_load", C.c_int, [_VP, _VP, C.c_uint64,
                                       C.POINTER(C.c_int64)]),
    ("mlbm_checkpoint_write", C.c_int, [_VP, C.c_int64, C.c_char_p]),
    ("mlbm_checkpoint_read", C.c_int, [_VP, C.c_char_p, C.POINTER(C.c_int64)]),
    ("mlbm_phase_stats_noalloc", C.c_int, [_VP, _VP, C.c_int32, C.c_int32,
                                           C.c_int32, C.POINTER(Params), _VP,
                                           C.POINTER(Stats)]),
]


def lib() -> C.CDLL:
    """Load ``libmlbm.so`` (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} not built: run `python -m multiphase_lbm_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != 0:
        raise MlbmError(status, lib().mlbm_last_error().decode())


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Lattice:
    """One porous domain resident on one GPU (an ``mlbm_lattice`` handle).

    Mirrors the reference boundary: :meth:`set_params` =
    ``transfer_parameter``, :meth:`upload` + :meth:`initialize` =
    ``multiphaselbm_initialization``, :meth:`iterate` =
    ``multiphaselbm_iteration`` (include/iteration_host.h:30-60).
    Arrays are in the reference layout ``[x][y][z]`` (z fastest).
    """

    def __init__(self, shape, storage: int = STORE_F32, device: int = 0):
        self.shape = tuple(int(v) for v in shape)
        self.storage = storage
        h = C.c_void_p()
        check(lib().mlbm_lattice_create(*self.shape, storage, device,
                                        C.byref(h)))
        self.h = h

    def close(self) -> None:
        h = getattr(self, "h", None)
        if h:
            self.h = None
            lib().mlbm_lattice_destroy(h)

    def __del__(self):
        # at interpreter exit the module may already be torn down; the
        # process exit releases the device memory then
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream_ptr: int) -> None:
        check(lib().mlbm_set_stream(self.h, C.c_void_p(stream_ptr)))

    def set_step_kernel(self, kind: int) -> None:
        check(lib().mlbm_set_step_kernel(self.h, kind))

    def set_update_shape(self, rows: int = 4, planes: int = 16) -> None:
        check(lib().mlbm_set_update_shape(self.h, rows, planes))

    @property
    def step_kernel(self) -> int:
        """The kernel the next iterate runs (KERNEL_COMPACT, ... ; AUTO
        resolved)."""
        return int(lib().mlbm_get_step_kernel(self.h))

    def checkpoint(self, step: int, out: "np.ndarray | None" = None) -> np.ndarray:
        """Exact image of the lattice's state (uint8 array; `out`, if given,
        must be a large enough uint8 array, e.g. pinned memory)."""
        n = C.c_uint64()
        check(lib().mlbm_checkpoint_bytes(self.h, C.byref(n)))
        if out is None:
            out = np.empty(n.value, np.uint8)
        if out.dtype != np.uint8 or out.nbytes < n.value:
            raise ValueError(f"checkpoint needs a uint8 buffer of {n.value} bytes")
        check(lib().mlbm_checkpoint_save(self.h, int(step), out.ctypes.data,
                                         out.nbytes))
        return out

    def restore(self, image: np.ndarray) -> int:
        """Load an image made by checkpoint(); returns its step counter."""
        a = np.ascontiguousarray(image, np.uint8)
        step = C.c_int64()
        check(lib().mlbm_checkpoint_load(self.h, a.ctypes.data, a.nbytes,
                                         C.byref(step)))
        return int(step.value)

    def write_checkpoint(self, path: str, step: int) -> None:
        check(lib().mlbm_checkpoint_write(self.h, int(step), path.encode()))

    def read_checkpoint(self, path: str) -> int:
        step = C.c_int64()
        check(lib().mlbm_checkpoint_read(self.h, path.encode(), C.byref(step)))
        return int(step.value)

    def set_wait_limit(self, ns: int) -> None:
        """Limit of the step kernels' bounded device waits (0 = 1 s)."""
        check(lib().mlbm_set_wait_limit(self.h, int(ns)))

    def test_stall_wait(self) -> None:
        """Make one wait of the next BAND launch run out (testing)."""
        check(lib().mlbm_test_stall_wait(self.h))

    def set_band_shape(self, rows: int = 4, planes: int = 24) -> None:
        """Tiling of KERNEL_BAND: rows per band (y) and planes per chunk (z)."""
        check(lib().mlbm_set_band_shape(self.h, rows, planes))

    def autotune(self, step0: int, trial_steps: int = 4):
        """Pick the shape of the lattice's step kernel by timing; returns
        (rows, planes, steps the lattice advanced)."""
        out = np.zeros(2, np.int32)
        done = C.c_int32()
        check(lib().mlbm_autotune(self.h, step0, trial_steps, out.ctypes.data,
                                  C.byref(done)))
        return int(out[0]), int(out[1]), done.value

    def synchronize(self) -> None:
        check(lib().mlbm_synchronize(self.h))

    def set_params(self, params: Params) -> None:
        check(lib().mlbm_set_params(self.h, C.byref(params)))

    def upload(self, fluid_xyz, rho_xyz) -> None:
        fl = np.ascontiguousarray(fluid_xyz, dtype=np.uint8)
        rho = np.ascontiguousarray(rho_xyz, dtype=np.float32)
        if fl.shape != self.shape or rho.shape != self.shape:
            raise ValueError(f"arrays must have shape {self.shape}")
        check(lib().mlbm_upload_fluid_mask(self.h, _ptr(fl)))
        check(lib().mlbm_upload_rho(self.h, _ptr(rho)))

    def upload_device(self, fluid_dev_ptr: int, rho_dev_ptr: int) -> None:
        check(lib().mlbm_upload_fluid_mask_device(self.h, C.c_void_p(fluid_dev_ptr)))
        check(lib().mlbm_upload_rho_device(self.h, C.c_void_p(rho_dev_ptr)))

    def initialize(self) -> None:
        check(lib().mlbm_initialize(self.h))

    def iterate(self, step0: int, nsteps: int = 1, reverse: int = 1,
                inject_type: int = 0, write_velocity: bool = False) -> None:
        check(lib().mlbm_iterate(self.h, step0, nsteps, reverse, inject_type,
                                 ITER_WRITE_VELOCITY if write_velocity else 0))

    # ---- slab decomposition (include/mlbm.h; driven by slab.py) ----
    def set_slab(self, enable: bool = True) -> None:
        """Planes 0 and nz - 1 become halo planes that the step reads but
        does not advance."""
        check(lib().mlbm_set_slab(self.h, 1 if enable else 0))

    def step_pass(self, step: int, pass_: int, reverse: int = 1,
                  inject_type: int = 0, write_velocity: bool = False) -> None:
        """One pass (0 density, 1 update) of time step `step`."""
        check(lib().mlbm_step_pass(self.h, step, pass_, reverse, inject_type,
                                   ITER_WRITE_VELOCITY if write_velocity else 0))

    def halo_segments(self, kind: int, side: int):
        """[(device pointer, bytes)] of one halo kind on one side."""
        ptrs = (C.c_void_p * HALO_MAX_SEGMENTS)()
        nbytes = np.zeros(HALO_MAX_SEGMENTS, np.int64)
        n = C.c_int32()
        check(lib().mlbm_halo_segments(self.h, kind, side, ptrs, _ptr(nbytes),
                                       C.byref(n)))
        return [(int(ptrs[i] or 0), int(nbytes[i])) for i in range(n.value)]

    def field(self, which: str, f64: bool = False) -> np.ndarray:
        code, extra = {"rho": (FIELD_RHO, ()), "pressure": (FIELD_PRESSURE, ()),
                       "psi": (FIELD_PSI, ()), "velocity": (FIELD_VELOCITY, (3,)),
                       "f": (FIELD_POPULATIONS, (Q,)),
                       "fluid": (FIELD_FLUID, ())}[which]
        if which == "fluid":
            out = np.empty(self.shape, np.uint8)
            check(lib().mlbm_download_field(self.h, code, DTYPE_U8, _ptr(out)))
            return out
        out = np.empty(self.shape + extra, np.float64 if f64 else np.float32)
        check(lib().mlbm_download_field(self.h, code,
                                        DTYPE_F64 if f64 else DTYPE_F32,
                                        _ptr(out)))
        return out

    def stats(self) -> dict:
        s = Stats()
        check(lib().mlbm_phase_stats(self.h, C.byref(s)))
        return s.as_dict()

    def stats_async(self, raw: np.ndarray) -> None:
        """Enqueue the phase statistics into `raw` (float64[STATS_RAW_LEN],
        page-locked host memory) without waiting; read them with
        :meth:`stats_from_raw` once the lattice's stream has passed this
        call."""
        if raw.dtype != np.float64 or raw.size < STATS_RAW_LEN:
            raise ValueError(f"raw must be float64[{STATS_RAW_LEN}]")
        check(lib().mlbm_phase_stats_async(self.h, _ptr(raw)))

    def bulk_stats_async(self, raw: np.ndarray) -> None:
        """As :meth:`stats_async` for the bulk columns only (counts, mass,
        liquid/vapour density sums, saturation, min/max rho, bit-identical
        to the full statistics; the boundary counts and the pressures read
        0)."""
        if raw.dtype != np.float64 or raw.size < STATS_RAW_LEN:
            raise ValueError(f"raw must be float64[{STATS_RAW_LEN}]")
        check(lib().mlbm_bulk_stats_async(self.h, _ptr(raw)))

    def stats_from_raw(self, raw: np.ndarray) -> dict:
        s = Stats()
        check(lib().mlbm_stats_from_raw(self.h, _ptr(raw), C.byref(s)))
        return s.as_dict()

    def plane_profile(self):
        nf = np.zeros(self.shape[0], np.int64)
        nl = np.zeros(self.shape[0], np.int64)
        check(lib().mlbm_plane_profile(self.h, _ptr(nf), _ptr(nl)))
        return nf, nl

    def info(self) -> dict:
        dims = np.zeros(3, np.int32)
        st, ph, ini = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().mlbm_lattice_info(self.h, _ptr(dims), C.byref(st),
                                      C.byref(ph), C.byref(ini)))
        return dict(dims=tuple(dims.tolist()), storage=st.value,
                    phase=ph.value, initialized=bool(ini.value))


def lattice_bytes(shape, storage: int = STORE_F32) -> int:
    return int(lib().mlbm_lattice_bytes(*shape, storage))
