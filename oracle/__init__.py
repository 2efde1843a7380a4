"""The oracle: CPU restatements of the D3Q19 Shan-Chen time step that the
tests compare the library against.

TEST INFRASTRUCTURE ONLY.  Imported by ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` -- to
verify results or as the timed CPU baseline, never by the product library.

Two implementations, both on the reference layout (scalars ``[x][y][z]`` with
z fastest, populations ``[x][y][z][19]``):

* :class:`Port` -- ``oracle/mlbm_oracle.c``, a C restatement of the
  reference's update with runtime sizes (FP32 = the reference arithmetic,
  FP64 = the same update in double precision).
* :class:`Reference` -- ``oracle/_ref/libref_<size>.so``, the reference's own
  kernels and host driver compiled for the CPU (``oracle/build_ref.py``); it
  exists only for the lattice sizes it was compiled for.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
Q = 19

# include/lbm_model.cuh:35-54
EX = np.array([0, -1, 0, 0, -1, -1, -1, -1, 0, 0, 1, 0, 0, 1, 1, 1, 1, 0, 0])
EY = np.array([0, 0, -1, 0, -1, 1, 0, 0, -1, -1, 0, 1, 0, 1, -1, 0, 0, 1, 1])
EZ = np.array([0, 0, 0, -1, 0, 0, -1, 1, -1, 1, 0, 0, 1, 0, 0, 1, -1, 1, -1])
T = np.array([1 / 3] + [1 / 18] * 3 + [1 / 36] * 6 + [1 / 18] * 3
             + [1 / 36] * 6, dtype=np.float32)


class Params(C.Structure):
    """Physics parameters (the reference's transfer_parameter arguments,
    include/iteration_host.h:30-41, plus the drainage boundary)."""
    _fields_ = [("tau", C.c_float), ("G", C.c_float), ("T_Tc", C.c_float),
                ("rhol_spinodal", C.c_float), ("rhog_spinodal", C.c_float),
                ("rho_increment", C.c_float), ("rhos", C.c_float),
                ("inject_position", C.c_float), ("carn_star", C.c_int32),
                ("inject_density", C.c_int32),
                ("rho_inject_period", C.c_uint64),
                ("stat_period", C.c_uint64), ("inlet_width", C.c_int32),
                ("outlet_width", C.c_int32), ("rho_inlet", C.c_float),
                ("rho_outlet", C.c_float)]


def make_params(**kw) -> Params:
    """Reference defaults (src/multiphase_lbm.cu:35-80) overridden by ``kw``."""
    d = dict(tau=1.0, G=-1.0, T_Tc=0.7, rhol_spinodal=0.2726,
             rhog_spinodal=0.0484, rho_increment=0.0, rhos=0.0,
             inject_position=1.0, carn_star=0, inject_density=0,
             rho_inject_period=100, stat_period=10, inlet_width=0,
             outlet_width=0, rho_inlet=0.0, rho_outlet=0.0)
    d.update(kw)
    return Params(**d)


def build() -> None:
    """Compile the C restatement (and, where the reference is present, the
    reference's own code into ``oracle/_ref``)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    from . import build_ref  # noqa: WPS433
    build_ref.build()
    build_ref.build_dropin(["40x40x40", "200x200x200"])
    build_ref.build_cuda()  # the reference's CUDA program, timing only


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `python -c 'import oracle; oracle.build()'`")
    return C.CDLL(path)


class Port:
    """C restatement of the update (``oracle/mlbm_oracle.c``)."""

    _libs: dict = {}

    def __init__(self, rho_xyz, fluid_xyz, params: Params, f64: bool = False):
        key = "f64" if f64 else "f32"
        if key not in Port._libs:
            lib = _load(os.path.join(HERE, f"liboracle_{key}.so"))
            pre = "mlbmo64_" if f64 else "mlbmo32_"
            for name in ("create", "destroy", "step", "get", "phase_stats"):
                setattr(lib, name, getattr(lib, pre + name))
            lib.create.restype = C.c_void_p
            lib.create.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(Params),
                                   C.c_void_p, C.c_void_p]
            lib.destroy.argtypes = [C.c_void_p]
            lib.step.argtypes = [C.c_void_p, C.c_int64, C.c_int32, C.c_int32,
                                 C.c_uint32]
            lib.get.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
            lib.phase_stats.argtypes = [C.c_void_p, C.c_void_p]
            Port._libs[key] = lib
        self.lib = Port._libs[key]
        self.dtype = np.float64 if f64 else np.float32
        rho = np.ascontiguousarray(rho_xyz, dtype=np.float32)
        fl = np.ascontiguousarray(fluid_xyz, dtype=np.uint8)
        self.shape = rho.shape
        self.params = params
        self.h = self.lib.create(*self.shape, C.byref(params),
                                 rho.ctypes.data, fl.ctypes.data)
        if not self.h:
            raise MemoryError("oracle allocation failed")

    def step(self, step0: int, nsteps: int = 1, reverse: int = 1,
             inject_type: int = 0) -> None:
        self.lib.step(self.h, step0, nsteps, reverse, inject_type)

    def get(self, which: str) -> np.ndarray:
        code, extra = {"rho": (0, ()), "pressure": (1, ()), "psi": (2, ()),
                       "force": (3, (3,)), "f": (4, (Q,)),
                       "velocity": (5, (3,))}[which]
        out = np.empty(self.shape + extra, dtype=self.dtype)
        self.lib.get(self.h, code, out.ctypes.data)
        return out

    def phase_stats(self) -> np.ndarray:
        out = np.zeros(12, dtype=np.float64)
        self.lib.phase_stats(self.h, out.ctypes.data)
        return out

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.destroy(self.h)
            self.h = None


def reference_sizes() -> list[tuple[int, int, int]]:
    """Lattice sizes for which ``oracle/_ref`` holds a compiled reference."""
    out = []
    if os.path.isdir(REF_DIR):
        for f in sorted(os.listdir(REF_DIR)):
            if f.startswith("libref_") and f.endswith(".so"):
                out.append(tuple(int(v) for v in f[7:-3].split("x")))
    return out


class Reference:
    """The reference's own kernels and host driver compiled for the CPU at a
    fixed lattice size (``oracle/_ref/libref_<lx>x<ly>x<lz>.so``)."""

    _libs: dict = {}

    def __init__(self, shape):
        shape = tuple(int(v) for v in shape)
        if shape not in Reference._libs:
            lib = _load(os.path.join(
                REF_DIR, "libref_{}x{}x{}.so".format(*shape)))
            lib.ref_setup.argtypes = [C.POINTER(Params), C.c_void_p, C.c_void_p]
            lib.ref_step.argtypes = [C.c_int64, C.c_int32, C.c_int32, C.c_uint32]
            lib.ref_get_field.argtypes = [C.c_int32, C.c_void_p]
            lib.ref_driver_read.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p]
            lib.ref_driver_stats.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_float, C.c_float, C.c_void_p]
            lib.ref_driver_clusters.argtypes = [
                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
            Reference._libs[shape] = lib
        self.lib = Reference._libs[shape]
        self.shape = shape

    def setup(self, rho_xyz, fluid_xyz, params: Params) -> None:
        rho = np.ascontiguousarray(rho_xyz, dtype=np.float32)
        fl = np.ascontiguousarray(fluid_xyz, dtype=np.uint8)
        assert rho.shape == self.shape
        if self.lib.ref_setup(C.byref(params), rho.ctypes.data, fl.ctypes.data):
            raise MemoryError("reference harness allocation failed")

    def step(self, step0: int, nsteps: int = 1, reverse: int = 1,
             inject_type: int = 0) -> None:
        self.lib.ref_step(step0, nsteps, reverse, inject_type)

    def get(self, which: str) -> np.ndarray:
        code, extra = {"rho": (0, ()), "pressure": (1, ()), "psi": (2, ()),
                       "force": (3, (3,)), "f": (4, (Q,))}[which]
        out = np.empty(self.shape + extra, dtype=np.float32)
        self.lib.ref_get_field(code, out.ctypes.data)
        return out

    def driver_read(self, cmdfile: str):
        """Run the reference command-file parser / geometry builder."""
        n = int(np.prod(self.shape))
        rho = np.empty(self.shape, np.float32)
        fl = np.empty(self.shape, np.uint8)
        sn = np.empty(self.shape, np.int64)
        info = np.zeros(12, np.float64)
        self.lib.ref_driver_read(cmdfile.encode(), rho.ctypes.data,
                                 fl.ctypes.data, sn.ctypes.data,
                                 info.ctypes.data)
        assert rho.size == n
        keys = ["packing_density", "solid_count", "step", "step_max",
                "statPeriod", "tau", "G", "rhos", "rho0", "IniPerturbRate",
                "rhol_spinodal", "rhog_spinodal"]
        return rho, fl, sn, dict(zip(keys, info.tolist()))

    def driver_stats(self, rho, pressure, fluid, rhol, rhog) -> dict:
        """Run the reference calc_cluster statistics on given fields."""
        out = np.zeros(13, np.float64)
        r = np.ascontiguousarray(rho, np.float32)
        p = np.ascontiguousarray(pressure, np.float32)
        f = np.ascontiguousarray(fluid, np.uint8)
        self.lib.ref_driver_stats(r.ctypes.data, p.ctypes.data, f.ctypes.data,
                                  rhol, rhog, out.ctypes.data)
        keys = ["saturation", "avg_liq_p", "avg_vap_p", "avg_liq_rho",
                "avg_vap_rho", "ratio_liquid_solid", "ratio_liquid_vapor",
                "liq_clusters", "gas_clusters", "min_rho", "max_rho", "min_p",
                "max_p"]
        return dict(zip(keys, out.tolist()))

    def driver_clusters(self, rho, pressure, fluid, solid_number, solid_count,
                        rhol, rhog):
        """Run the reference calc_cluster (with solid numbers): returns
        (dict of cluster columns, liquid labels, gas labels)."""
        out = np.zeros(8, np.float64)
        liq = np.zeros(self.shape, np.int64)
        gas = np.zeros(self.shape, np.int64)
        r = np.ascontiguousarray(rho, np.float32)
        p = np.ascontiguousarray(pressure, np.float32)
        f = np.ascontiguousarray(fluid, np.uint8)
        sn = np.ascontiguousarray(solid_number, np.int64)
        self.lib.ref_driver_clusters(r.ctypes.data, p.ctypes.data, f.ctypes.data,
                                     sn.ctypes.data, solid_count, rhol, rhog,
                                     out.ctypes.data, liq.ctypes.data,
                                     gas.ctypes.data)
        keys = ["liq_cluster_count", "gas_cluster_count", "cluster_order",
                "wet_coord_num", "cluster_radius", "liquid_solid_boundary",
                "liquid_vapor_boundary", "saturation"]
        return dict(zip(keys, out.tolist())), liq, gas
