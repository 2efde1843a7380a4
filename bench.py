"""Benchmark of the D3Q19 Shan-Chen time step on B200.

Workload (one GPU): the 200^3 drainage case -- seeded sphere packing
(radius U[5,15], centres uniform, overlap allowed, added until porosity
<= 0.50), pores start at rho = 2.0, inlet slab x < 8 held at rho = 0.10,
outlet plane x = 199 held at rho = 1.95, periodic in y and z, G = -6.0,
tau = 1.0, G_ads = -1.0 (rhos = -ln(1 - G_ads/G) = 0.182322).  Synthetic
input: the packing comes from libmlbm's seeded generator.

One bench step = one lattice time step over the whole domain.  ``value`` is
MLUPS (lattice nodes x steps / s, the reference's convention, all nodes)
timed on the device with CUDA events around K steps whose inputs are
resident in HBM (the lattice, 0.6 GB, is far larger than L2, so no flush is
needed).  ``e2e`` is the same metric through the C ABI with host buffers:
geometry and initial density copied in from pinned host memory, then every
step an ``mlbm_iterate`` call and a device->host read of its phase
statistics, and the final density field copied out.

``--impl reference`` times the reference's own kernels compiled for the CPU
(``oracle/_ref``, OpenMP over all host cores) on a bounded sample of the same
workload.  ``--gpus N`` (under torchrun) runs N independent replicas, one per
GPU (the single-domain step has no exchange to shard); value = all ranks'
node updates / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (200, 200, 200)
RHO_S = 0.182322  # -ln(1 - G_ads/G) for G_ads = -1, G = -6


def phys(n=200):
    """Drainage parameters of the n^3 case (slab scaled as round(8 n / 200))."""
    return dict(G=-6.0, tau=1.0, rhos=RHO_S, inlet_width=max(1, round(8 * n / 200)),
                outlet_width=1, rho_inlet=0.10, rho_outlet=1.95,
                rhol_spinodal=0.2726, rhog_spinodal=0.0484)


PHYS = phys(200)
BYTES_PER_FLUID = {"f32": 152, "f16": 76, "f64": 304}


def workload(shape=SHAPE, seed=2024):
    from multiphase_lbm_b200 import host
    fluid, spheres = host.generate_packing(shape, 5.0, 15.0, 0.50, seed)
    rho = np.full(shape, 2.0, np.float32)
    return fluid, rho, len(spheres)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(kernel, storage):
    """DRAM bytes per time step of `kernel` at 200^3 from the committed ncu
    summary (profiles/traffic.json), if present."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        d = json.load(open(p)).get(kernel, {})
        v = d.get(storage)
        if v is not None:
            return float(v)
    return None


# roofline label and launches per step of each step kernel
KERNEL_INFO = {5: ("wave", "k_cwave (wavefront step, compact layout)", 1),
               4: ("single-pass", "k_compact_step (single pass, compact layout)", 1),
               3: ("compact", "time step (k_cdensity + k_cupdate, compact layout)", 2),
               2: ("two-pass", "time step (k_density + k_update_zm)", 2),
               1: ("fused", "k_step_fused (persistent)", 1)}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[2:6]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_sample(fluid, rho, budget_s=15.0, max_steps=200):
    """Reference kernels on the host cores (oracle/_ref) at the bench size."""
    import oracle
    if tuple(fluid.shape) not in oracle.reference_sizes():
        return None
    ref = oracle.Reference(fluid.shape)
    p = oracle.make_params(**PHYS)
    ref.setup(rho, fluid, p)
    t0 = time.perf_counter()
    ref.step(0, 1)
    t1 = time.perf_counter() - t0
    n = int(max(1, min(max_steps, budget_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    ref.step(1, n)
    dt = time.perf_counter() - t0
    cores = len(os.sched_getaffinity(0))
    mlups = fluid.size * n / dt / 1e6
    return {"value": round(mlups, 3), "unit": "MLUPS", "cores": cores,
            "kind": "reference",
            "sample": f"{n} steps of the 200^3 drainage case (reference "
                      f"kernels compiled for the CPU, OpenMP {cores} threads, "
                      f"race-free two-sweep collision)"}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    fluid, rho, _ = workload()
    import oracle
    if tuple(fluid.shape) not in oracle.reference_sizes():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref has no 200^3 build"}))
        return 0
    ref = oracle.Reference(fluid.shape)
    ref.setup(rho, fluid, oracle.make_params(**PHYS))
    cores = len(os.sched_getaffinity(0))
    steps_per = 1  # each bench step = a bounded sample of 1 lattice step
    for w in range(args.warmup):
        ref.step(w * steps_per, steps_per)
    t0 = time.perf_counter()
    for k in range(args.steps):
        ref.step((args.warmup + k) * steps_per, steps_per)
    dt = time.perf_counter() - t0
    mlups = fluid.size * steps_per * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": "MLUPS", "value": round(mlups, 3),
        "unit": "MLUPS", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "drainage 200^3, sphere packing porosity 0.50, "
                               "inlet x<8 rho 0.10, outlet x=199 rho 1.95",
                   "sample_steps_per_bench_step": steps_per},
        "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS",
                         "cores": cores, "kind": "reference",
                         "sample": f"{steps_per} lattice steps per bench step"},
        "e2e": {"value": round(mlups, 3), "unit": "MLUPS",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "f64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--size", type=int, default=200,
                    help="lattice edge (profiling runs use a smaller case)")
    ap.add_argument("--kernel", default="auto",
                    choices=["auto", "wave", "compact", "single-pass", "fused",
                             "two-pass"])
    ap.add_argument("--wave-shape", default=None,
                    help="tile_nodes,lookahead of the wavefront step")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from multiphase_lbm_b200 import capi
    storage = {"f32": capi.STORE_F32, "f16": capi.STORE_F16,
               "f64": capi.STORE_F64}[args.storage]
    fluid, rho, nspheres = workload((args.size,) * 3)
    n_nodes = fluid.size
    n_fluid = int(fluid.sum())
    params = capi.default_params(**phys(args.size), rho_shift=1.0)

    lat = capi.Lattice(fluid.shape, storage=storage, device=local)
    lat.set_params(params)
    lat.upload(fluid, rho)
    lat.initialize()
    kernel_id = {"auto": capi.KERNEL_AUTO, "wave": capi.KERNEL_WAVE,
                 "compact": capi.KERNEL_COMPACT,
                 "single-pass": capi.KERNEL_SINGLE_PASS,
                 "fused": capi.KERNEL_FUSED,
                 "two-pass": capi.KERNEL_TWO_PASS}[args.kernel]
    lat.set_step_kernel(kernel_id)
    if args.wave_shape:
        lat.set_wave_shape(*[int(v) for v in args.wave_shape.split(",")])
    kname, klabel, klaunches = KERNEL_INFO[lat.step_kernel]
    step = 0
    lat.iterate(step, args.warmup)
    step += args.warmup
    torch.cuda.synchronize()

    # ---- device-timed region (inputs resident) --------------------------
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ev0.record()
        lat.iterate(step, args.steps)
        ev1.record()
        torch.cuda.synchronize()
    step += args.steps
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    from multiphase_lbm_b200.shard import max_over_ranks
    t_max = max_over_ranks(ms)
    s_per_step = t_max / 1e3 / args.steps
    mlups = n_nodes * world * args.steps / (t_max / 1e3) / 1e6

    # ---- roofline of the time step ----------------------------------------
    peak, peak_kind = load_peaks()
    alg_bytes = n_fluid * BYTES_PER_FLUID[args.storage] + n_nodes / 8
    achieved = alg_bytes / s_per_step / 1e9
    traffic = load_traffic(kname, args.storage) if args.size == 200 else None

    # ---- end to end through the C ABI with host buffers --------------------
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(capi, torch, fluid, rho, params, storage, local,
                      args.steps, dist, kernel_id)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.size == 200:
        cpu = cpu_reference_sample(fluid, rho)

    line = {
        "metric": "MLUPS", "value": round(mlups, 2), "unit": "MLUPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(s_per_step * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.storage,
        "data": "synthetic (seeded sphere packing)",
        "config": {"workload": "drainage 200^3: spheres r~U[5,15] to porosity "
                               "0.50, pores rho 2.0, inlet x<8 rho 0.10, outlet "
                               "x=199 rho 1.95, G -6, tau 1, rhos 0.182322",
                   "lattice": list(fluid.shape), "fluid_nodes": n_fluid,
                   "porosity": round(n_fluid / n_nodes, 5),
                   "spheres": nspheres, "storage": args.storage,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (lattice "
                         f"{capi.lattice_bytes(fluid.shape, storage) / 1e9:.2f} GB)"},
        "mflups": round(n_fluid * world * args.steps / (t_max / 1e3) / 1e6, 2),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1),
                     "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": klabel,
                     "alg_bytes_per_step": int(alg_bytes)},
        "clocks": clocks.summary(),
        "gpu_launches": klaunches * args.steps,
    }
    if e2e:
        line["e2e"] = e2e
    if cpu:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line))
    lat.close()
    if dist:
        dist.destroy_process_group()
    return 0


def run_e2e(capi, torch, fluid, rho, params, storage, device, steps, dist,
            kernel_id=0):
    """MLUPS through the public C ABI with host buffers (pinned).  Every
    step's phase statistics are read back: enqueued without waiting
    (mlbm_phase_stats_async) and read on the host one step later, while the
    next step runs, so the GPU does not idle on the host's read."""
    fl_h = torch.from_numpy(fluid).pin_memory().numpy()
    rho_h = torch.from_numpy(rho).pin_memory().numpy()
    out_h = torch.empty(fluid.shape, dtype=torch.float32).pin_memory().numpy()
    raw = [torch.zeros(capi.STATS_RAW_LEN, dtype=torch.float64).pin_memory().numpy()
           for _ in range(2)]
    done = [torch.cuda.Event() for _ in range(2)]
    lat = capi.Lattice(fluid.shape, storage=storage, device=device)
    lat.set_step_kernel(kernel_id)
    lat.set_params(params)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lat.upload(fl_h, rho_h)
    lat.initialize()
    sat = []
    for k in range(steps):
        lat.iterate(k, 1)
        lat.stats_async(raw[k % 2])  # device->host read of the step's stats
        done[k % 2].record()
        if k > 0:
            done[(k - 1) % 2].synchronize()
            sat.append(lat.stats_from_raw(raw[(k - 1) % 2])["saturation"])
    done[(steps - 1) % 2].synchronize()
    sat.append(lat.stats_from_raw(raw[(steps - 1) % 2])["saturation"])
    from multiphase_lbm_b200.capi import DTYPE_F32, FIELD_RHO, check, lib
    check(lib().mlbm_download_field(lat.h, FIELD_RHO, DTYPE_F32,
                                    out_h.ctypes.data))
    dt = time.perf_counter() - t0
    from multiphase_lbm_b200.shard import max_over_ranks
    dt = max_over_ranks(dt)
    lat.close()
    world = dist.get_world_size() if dist else 1
    n = fluid.size
    stats_bytes = 8 * capi.STATS_RAW_LEN
    assert len(sat) == steps
    return {"value": round(n * world * steps / dt / 1e6, 2), "unit": "MLUPS",
            "h2d_bytes_per_step": int((n + 4 * n) / steps),
            "d2h_bytes_per_step": int(stats_bytes + 4 * n / steps)}


if __name__ == "__main__":
    sys.exit(main())
