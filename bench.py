"""Benchmark of the D3Q19 Shan-Chen time step on B200.

Workload (one GPU): the 200^3 drainage case -- the sphere packing of
``multiphase_lbm_b200/workloads/drainage_200_seed2024.positions`` (radius
U[5,15], centres uniform, overlap allowed, added until porosity <= 0.50,
written by that folder's ``make_positions.py``), pores start at rho = 2.0,
inlet slab x < 8 held at rho = 0.10, outlet plane x = 199 held at rho = 1.95,
periodic in y and z, G = -6.0, tau = 1.0, G_ads = -1.0
(rhos = -ln(1 - G_ads/G) = 0.182322).  Both arms read the same positions
file: this library through mlbm_read_positions, the reference arm through
the reference's own read_positions.

One bench step = one lattice time step over the whole domain.  ``value`` is
MLUPS (lattice nodes x steps / s, the reference's convention, all nodes)
timed on the device with CUDA events around blocks of K steps whose inputs
are resident in HBM (the lattice, >= 0.3 GB, is larger than L2, so no flush
is needed); blocks are repeated until at least a second has been timed and
the median block is reported.  FP32 storage is the headline; the FP16-store
form is timed in the same run (``fp16``).  ``e2e`` is the same metric
through the C ABI with host buffers: geometry and initial density copied in
from pinned host memory, then every step an ``mlbm_iterate`` call and a
device->host read of its saturation and mass (the bulk statistics), and the
final density field copied out, over a job of max(K, 500) steps
(``e2e.steps``); ``e2e.with_full_stats_every_step`` reads every column of
the phase statistics each step instead (the 18-neighbour boundary counts
and the pressures included).

``--impl reference`` runs the reference's own code: its time step compiled
for the CPU (``oracle/_ref``, OpenMP over all host cores) on a bounded
sample of the same workload (the line's ``value``), and its CUDA build
(``oracle/_ref/ref_cuda_timer_200x200x200``: the reference's unmodified
kernels between CUDA events, periodic boundaries as the reference has no
drainage boundary) on the same GPU (``reference_cuda``), and that build at
64^3 on the periodic case (``reference_cuda_64``; this library's step on it
is the ``periodic_64`` object of the other arm).  It loads nothing
of this library.  ``--gpus N`` (under torchrun) runs N independent replicas,
one per GPU (the single-domain step has no exchange to shard); value = all
ranks' node updates / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (200, 200, 200)
RHO_S = 0.182322  # -ln(1 - G_ads/G) for G_ads = -1, G = -6
POSITIONS = os.path.join(ROOT, "multiphase_lbm_b200", "workloads",
                         "drainage_200_seed2024.positions")
MIN_TIMED_S = 1.0  # timed blocks repeat until this much device time
# The 64^3 periodic case (phase separation from rho 0.70 +- 0.01, the
# reference's srand(1)/rand() stream): a second speed comparison against the
# reference's CUDA build on identical geometry and boundaries.
SHAPE_64 = (64, 64, 64)
POSITIONS_64 = os.path.join(ROOT, "multiphase_lbm_b200", "workloads",
                            "periodic_64_seed64.positions")
RATE_64 = 0.02 / 0.70  # IniPerturbRate: rho0 (1 + rate (U - 0.5)), rho0 0.70


def phys(n=200):
    """Drainage parameters of the n^3 case (slab scaled as round(8 n / 200))."""
    return dict(G=-6.0, tau=1.0, rhos=RHO_S, inlet_width=max(1, round(8 * n / 200)),
                outlet_width=1, rho_inlet=0.10, rho_outlet=1.95,
                rhol_spinodal=0.2726, rhog_spinodal=0.0484)


PHYS = phys(200)
# The end-to-end leg runs a job of at least this many steps (its one-time
# upload and layout change are part of it), whatever --steps is.
E2E_MIN_STEPS = 500
BYTES_PER_FLUID = {"f32": 152, "f16": 76, "f64": 304}


def workload(shape=SHAPE, seed=2024):
    """(fluid mask, initial density, sphere count) of the n^3 case through
    this library: the committed positions file at 200^3, the seeded
    generator at other (profiling) sizes."""
    from multiphase_lbm_b200 import host
    if tuple(shape) == SHAPE:
        fluid, _, n = host.read_positions(POSITIONS, shape)
    else:
        fluid, spheres = host.generate_packing(shape, 5.0, 15.0, 0.50, seed)
        n = len(spheres)
    rho = np.full(shape, 2.0, np.float32)
    return fluid, rho, n


def command_file(folder: str) -> str:
    """The 200^3 case as a command file in the reference's format (read by
    its read_data, src/multiphase_lbm.cu:619-745): density 2.0 everywhere,
    the committed positions file, statistics never due, one OpenMP thread
    per host core this process may use."""
    text = f"""! 200^3 drainage benchmark packing
result_folder {folder}/RES
num_threads {len(os.sched_getaffinity(0))}
statPeriod 1000000000
lx 200
ly 200
lz 200
rho0 2.0
IniPerturbRate 0.0
G -6.0
rhos {RHO_S}
tau 1.0
rhol_spinodal 0.2726
rhog_spinodal 0.0484
resize
resolution 1
read_positions {POSITIONS}
step_max 1000000000
"""
    path = os.path.join(folder, "bench_200.txt")
    with open(path, "w") as fh:
        fh.write(text)
    return path


def command_file_64(folder: str) -> str:
    """The 64^3 periodic case as a reference command file."""
    text = f"""! 64^3 periodic phase-separation case
result_folder {folder}/RES64
num_threads {len(os.sched_getaffinity(0))}
statPeriod 1000000000
lx 64
ly 64
lz 64
rho0 0.70
IniPerturbRate {RATE_64:.9g}
G -6.0
rhos {RHO_S}
tau 1.0
rhol_spinodal 0.2726
rhog_spinodal 0.0484
resize
resolution 1
read_positions {POSITIONS_64}
step_max 1000000000
"""
    path = os.path.join(folder, "bench_64.txt")
    with open(path, "w") as fh:
        fh.write(text)
    return path


def bench_config(fluid_nodes: int, spheres: int, n: int = 200) -> dict:
    """The workload description both arms print (identical dicts)."""
    return {"workload": f"drainage {n}^3: spheres r~U[5,15] to porosity 0.50 "
                        f"(positions file, seed 2024), pores rho 2.0, inlet "
                        f"x<{phys(n)['inlet_width']} rho 0.10, outlet "
                        f"x={n - 1} rho 1.95, G -6, tau 1, rhos 0.182322",
            "lattice": [n, n, n], "fluid_nodes": int(fluid_nodes),
            "porosity": round(fluid_nodes / n ** 3, 5), "spheres": int(spheres),
            "l2": "inputs larger than L2 (FP32 populations 0.61 GB, FP16 "
                  "0.30 GB per step), no flush"}


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
KERNEL_INFO = {6: ("band", "k_band (one-pass step, compact layout, two buffers)", 1),
               3: ("compact", "time step (k_cdensity + k_cupdate, compact layout)", 2),
               2: ("two-pass", "time step (k_density + k_update_zm)", 2)}


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
                 "-lms", "100"], stdout=subprocess.PIPE,
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


# ---- the reference's own code -------------------------------------------------

def reference_read(folder: str):
    """Geometry and initial density through the reference's own command-file
    parser and read_positions (oracle/_ref), and its harness at 200^3."""
    import oracle
    if SHAPE not in oracle.reference_sizes():
        return None
    ref = oracle.Reference(SHAPE)
    rho, fluid, _, info = ref.driver_read(command_file(folder))
    ref.setup(rho, fluid, oracle.make_params(**PHYS))
    return ref, fluid, int(info["solid_count"])


def reference_cpu_steps(ref, step0: int, steps: int, budget_s: float):
    """Time up to `steps` reference steps on the host cores, stopping once
    `budget_s` is spent: (steps run, seconds)."""
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        ref.step(step0 + done, 1)
        done += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    return done, time.perf_counter() - t0


def cpu_reference_sample(budget_s=15.0, max_steps=200):
    """cpu_baseline of this library's line: the reference's time step on the
    host cores, a bounded sample of the 200^3 case."""
    with tempfile.TemporaryDirectory() as folder:
        got = reference_read(folder)
    if got is None:
        return None
    ref, fluid, _ = got
    ref.step(0, 1)
    n, dt = reference_cpu_steps(ref, 1, max_steps, budget_s)
    cores = len(os.sched_getaffinity(0))
    return {"value": round(fluid.size * n / dt / 1e6, 3), "unit": "MLUPS",
            "cores": cores, "kind": "reference",
            "sample": f"{n} steps of the 200^3 drainage case (the reference's "
                      f"kernels compiled for the CPU, OpenMP {cores} threads, "
                      f"race-free two-sweep collision)"}


def reference_cuda(folder: str, steps: int, warmup: int, device: int,
                   n: int = 200):
    """The reference's CUDA build on this GPU: its unmodified
    multiphaselbm_iteration timed between CUDA events by
    oracle/_ref/ref_cuda_timer_<n>x<n>x<n> (n = 200: the drainage packing;
    n = 64: the periodic case), blocks of `steps` steps repeated for about a
    second; median block."""
    name = f"ref_cuda_timer_{n}x{n}x{n}"
    exe = os.path.join(ROOT, "oracle", "_ref", name)
    if not os.path.exists(exe):
        return {"unavailable": f"oracle/_ref/{name} not built"}
    cmd = command_file(folder) if n == 200 else command_file_64(folder)
    # ~3 ms per step at 200^3: enough blocks for about a second of steps
    est = 0.003 * (n / 200) ** 3 + 2e-5
    repeats = max(3, int(MIN_TIMED_S / (est * steps)) + 1)
    with ClockSampler(device) as clocks:
        r = subprocess.run(
            ["bash", "-c", f"ulimit -s unlimited; exec {exe} {cmd} "
                           f"{warmup} {steps} {repeats}"],
            cwd=folder, capture_output=True, text=True, timeout=600)
    blocks = [float(ln.split()[-1]) for ln in r.stdout.splitlines()
              if ln.startswith("block ")]
    if r.returncode != 0 or not blocks:
        return {"unavailable": f"reference CUDA timer exited {r.returncode}: "
                               f"{(r.stderr or r.stdout)[-200:]}"}
    ms = statistics.median(blocks)
    return {"ms_per_step": round(ms, 4),
            "value": round(n ** 3 / (ms / 1e3) / 1e6, 2),
            "unit": "MLUPS", "steps": steps, "blocks": len(blocks),
            "boundaries": "periodic (the reference has no drainage boundary)"
                          if n == 200 else "periodic (as configured)",
            "clocks": clocks.summary()}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    with tempfile.TemporaryDirectory() as folder:
        got = reference_read(folder)
        if got is None:
            print(json.dumps({"impl": "reference",
                              "unavailable": "oracle/_ref has no 200^3 build"}))
            return 0
        ref, fluid, spheres = got
        cores = len(os.sched_getaffinity(0))
        for w in range(args.warmup):
            ref.step(w, 1)
        # each bench step is one lattice step; the sample stops after ~60 s
        n, dt = reference_cpu_steps(ref, args.warmup, args.steps, 60.0)
        mlups = fluid.size * n / dt / 1e6
        cuda = cuda64 = None
        if not args.no_reference_cuda:
            dev = int(os.environ.get("LOCAL_RANK", "0"))
            cuda = reference_cuda(folder, max(args.steps, 20), args.warmup, dev)
            cuda64 = reference_cuda(folder, max(args.steps, 20), args.warmup,
                                    dev, n=64)
    sample = (f"{n} of {args.steps} timed lattice steps (each bench step one "
              f"lattice step; stops after 60 s) of the 200^3 drainage case")
    line = {
        "impl": "reference", "metric": "MLUPS", "value": round(mlups, 3),
        "unit": "MLUPS", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dt / n * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded sphere packing)",
        "config": bench_config(int(fluid.sum()), spheres),
        "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS",
                         "cores": cores, "kind": "reference",
                         "sample": sample + f", OpenMP {cores} threads"},
        "e2e": {"value": round(mlups, 3), "unit": "MLUPS",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if cuda is not None:
        line["reference_cuda"] = cuda
    if cuda64 is not None:
        line["reference_cuda_64"] = cuda64
    print(json.dumps(line))
    return 0


# ---- this library ------------------------------------------------------------

def timed_blocks(lat, torch, step, steps, dist, min_s=MIN_TIMED_S):
    """Blocks of `steps` steps between CUDA events on the lattice's stream
    (the current stream), repeated until min_s seconds of device time (and
    at least three blocks); returns (median ms per block, blocks, next
    step)."""
    from multiphase_lbm_b200.shard import max_over_ranks
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    times = []
    total = 0.0
    while total < min_s * 1e3 or len(times) < 3:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record()
        lat.iterate(step, steps)
        ev1.record()
        torch.cuda.synchronize()
        step += steps
        ms = max_over_ranks(ev0.elapsed_time(ev1))
        times.append(ms)
        total += ms
    return statistics.median(times), len(times), step


def measure(capi, torch, fluid, rho, storage_name, args, local, dist,
            kernel_id):
    """Median device time per step (seconds) of one storage format."""
    storage = {"f32": capi.STORE_F32, "f16": capi.STORE_F16,
               "f64": capi.STORE_F64}[storage_name]
    params = capi.default_params(**phys(args.size), rho_shift=1.0)
    lat = capi.Lattice(fluid.shape, storage=storage, device=local)
    lat.set_params(params)
    lat.upload(fluid, rho)
    lat.initialize()
    if kernel_id is not None:
        lat.set_step_kernel(kernel_id)
    if args.band_shape:
        lat.set_band_shape(*[int(v) for v in args.band_shape.split(",")])
    kernel = lat.step_kernel
    lat.iterate(0, args.warmup)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ms, blocks, _ = timed_blocks(lat, torch, args.warmup, args.steps, dist,
                                     args.min_time)
    lat.close()
    return ms / 1e3 / args.steps, blocks, clocks.summary(), kernel


def measure_64(capi, torch, args, local):
    """The default FP32 step on the 64^3 periodic case (the committed 64^3
    positions file, rho 0.70 with the reference's srand(1)/rand()
    perturbation, no inlet or outlet): median device time per step, in blocks
    as long as the reference's CUDA timing uses."""
    from multiphase_lbm_b200 import host
    fluid, _, nsph = host.read_positions(POSITIONS_64, SHAPE_64)
    rho = host.init_density(SHAPE_64, 0.70, RATE_64)
    params = capi.default_params(G=-6.0, tau=1.0, rhos=RHO_S,
                                 rhol_spinodal=0.2726, rhog_spinodal=0.0484,
                                 rho_shift=1.0)
    lat = capi.Lattice(SHAPE_64, storage=capi.STORE_F32, device=local)
    lat.set_params(params)
    lat.upload(fluid, rho)
    lat.initialize()
    steps = max(args.steps, 20)
    lat.iterate(0, args.warmup)
    torch.cuda.synchronize()
    ms, blocks, _ = timed_blocks(lat, torch, args.warmup, steps, None,
                                 min(args.min_time, 0.5))
    kernel = KERNEL_INFO.get(lat.step_kernel, ("", str(lat.step_kernel)))[1]
    lat.close()
    per = ms / steps
    return {"ms_per_step": round(per, 5),
            "value": round(64 ** 3 / (per / 1e3) / 1e6, 2), "unit": "MLUPS",
            "fluid_nodes": int(fluid.sum()), "spheres": int(nsph),
            "steps": steps, "blocks": blocks, "kernel": kernel,
            "boundaries": "periodic"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "f64"])
    ap.add_argument("--min-time", type=float, default=MIN_TIMED_S,
                    help="seconds of timed blocks (profiling runs use less)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp16", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true")
    ap.add_argument("--no-64", action="store_true",
                    help="skip the 64^3 periodic comparison case")
    ap.add_argument("--size", type=int, default=200,
                    help="lattice edge (profiling runs use a smaller case)")
    ap.add_argument("--kernel", default="auto",
                    choices=["auto", "band", "compact", "two-pass"])
    ap.add_argument("--band-shape", default=None,
                    help="rows,planes of the one-pass step's bands")
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
    fluid, rho, nspheres = workload((args.size,) * 3)
    n_nodes = fluid.size
    n_fluid = int(fluid.sum())
    kernel_id = {"auto": None, "band": capi.KERNEL_BAND,
                 "compact": capi.KERNEL_COMPACT,
                 "two-pass": capi.KERNEL_TWO_PASS}[args.kernel]

    # ---- device-timed region (inputs resident) --------------------------
    s_per_step, blocks, clocks, kernel = measure(
        capi, torch, fluid, rho, args.storage, args, local, dist, kernel_id)
    kname, klabel, klaunches = KERNEL_INFO[kernel]
    mlups = n_nodes * world / s_per_step / 1e6

    # ---- roofline of the time step ----------------------------------------
    peak, peak_kind = load_peaks()
    alg_bytes = n_fluid * BYTES_PER_FLUID[args.storage] + n_nodes / 8
    achieved = alg_bytes / s_per_step / 1e9
    traffic = load_traffic(kname, args.storage) if args.size == 200 else None

    fp16 = None
    if args.storage == "f32" and not args.no_fp16:
        s16, b16, c16, _ = measure(capi, torch, fluid, rho, "f16", args, local,
                                   dist, kernel_id)
        alg16 = n_fluid * BYTES_PER_FLUID["f16"] + n_nodes / 8
        fp16 = {"ms_per_step": round(s16 * 1e3, 4),
                "value": round(n_nodes * world / s16 / 1e6, 2), "unit": "MLUPS",
                "speedup_vs_fp32": round(s_per_step / s16, 3),
                "roofline": {"achieved": round(alg16 / s16 / 1e9, 1),
                             "peak": peak, "unit": "GB/s",
                             "frac": round(alg16 / s16 / 1e9 / peak, 4),
                             "alg_bytes_per_step": int(alg16),
                             "traffic": load_traffic(kname, "f16")
                             if args.size == 200 else None},
                "timed_blocks": b16, "clocks": c16}

    # ---- end to end through the C ABI with host buffers --------------------
    e2e = None
    if not args.no_e2e:
        e2e_args = (capi, torch, fluid, rho, capi.default_params(
            **phys(args.size), rho_shift=1.0),
            {"f32": capi.STORE_F32, "f16": capi.STORE_F16,
             "f64": capi.STORE_F64}[args.storage],
            local, max(args.steps, E2E_MIN_STEPS), dist, kernel_id)
        e2e = run_e2e(*e2e_args)
        full = run_e2e(*e2e_args, full_stats=True)
        e2e["with_full_stats_every_step"] = {
            k: full[k] for k in ("value", "unit", "breakdown_ms")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.size == 200:
        cpu = cpu_reference_sample()
    case64 = None
    if world == 1 and not args.no_64 and args.size == 200:
        case64 = measure_64(capi, torch, args, local)

    line = {
        "metric": "MLUPS", "value": round(mlups, 2), "unit": "MLUPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(s_per_step * 1e3, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.storage,
        "data": "synthetic (seeded sphere packing)",
        "config": bench_config(n_fluid, nspheres, args.size),
        "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
        "timed_blocks": blocks,
        "mflups": round(n_fluid * world / s_per_step / 1e6, 2),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1),
                     "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": traffic,
                     "traffic_source": "committed ncu summary "
                                       "(profiles/traffic.json), not this run",
                     "peak_kind": peak_kind, "kernel": klabel,
                     "alg_bytes_per_step": int(alg_bytes)},
        "clocks": clocks,
        "gpu_launches": klaunches * args.steps * blocks,
    }
    if fp16:
        line["fp16"] = fp16
    if e2e:
        line["e2e"] = e2e
    if cpu:
        line["cpu_baseline"] = cpu
    if case64:
        line["periodic_64"] = case64
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


def run_e2e(capi, torch, fluid, rho, params, storage, device, steps, dist,
            kernel_id=None, full_stats=False):
    """MLUPS through the public C ABI with host buffers (pinned).  Every
    step's result is read back: its saturation and mass (the bulk
    statistics, mlbm_bulk_stats_async; with full_stats every column of the
    phase statistics, mlbm_phase_stats_async), enqueued without waiting and
    read on the host one step later, while the next step runs, so the GPU
    does not idle on the host's read."""
    fl_h = torch.from_numpy(fluid).pin_memory().numpy()
    rho_h = torch.from_numpy(rho).pin_memory().numpy()
    out_h = torch.empty(fluid.shape, dtype=torch.float32).pin_memory().numpy()
    raw = [torch.zeros(capi.STATS_RAW_LEN, dtype=torch.float64).pin_memory().numpy()
           for _ in range(2)]
    done = [torch.cuda.Event() for _ in range(2)]
    lat = capi.Lattice(fluid.shape, storage=storage, device=device)
    if kernel_id is not None:
        lat.set_step_kernel(kernel_id)
    lat.set_params(params)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    marks = []

    def mark():
        torch.cuda.synchronize()
        marks.append(time.perf_counter())

    t0 = time.perf_counter()
    lat.upload(fl_h, rho_h)
    mark()
    lat.initialize()
    mark()
    sat = []
    for k in range(steps):
        lat.iterate(k, 1)
        # device->host read of the step's statistics
        (lat.stats_async if full_stats else lat.bulk_stats_async)(raw[k % 2])
        done[k % 2].record()
        if k == 0:
            mark()  # the first step builds the fluid-only tables
        if k > 0:
            done[(k - 1) % 2].synchronize()
            sat.append(lat.stats_from_raw(raw[(k - 1) % 2])["saturation"])
    done[(steps - 1) % 2].synchronize()
    sat.append(lat.stats_from_raw(raw[(steps - 1) % 2])["saturation"])
    mark()
    from multiphase_lbm_b200.capi import DTYPE_F32, FIELD_RHO, check, lib
    check(lib().mlbm_download_field(lat.h, FIELD_RHO, DTYPE_F32,
                                    out_h.ctypes.data))
    dt = time.perf_counter() - t0
    edges = [t0] + marks + [t0 + dt]
    parts = ["upload", "initialize", "first_step", "steps_after_first",
             "download"]
    breakdown = {k: round((b - a) * 1e3, 3)
                 for k, a, b in zip(parts, edges[:-1], edges[1:])}
    from multiphase_lbm_b200.shard import max_over_ranks
    dt = max_over_ranks(dt)
    lat.close()
    world = dist.get_world_size() if dist else 1
    n = fluid.size
    stats_bytes = 8 * capi.STATS_RAW_LEN
    assert len(sat) == steps
    return {"value": round(n * world * steps / dt / 1e6, 2), "unit": "MLUPS",
            "steps": steps,
            "per_step_read": "all phase statistics" if full_stats
                             else "bulk statistics (saturation, mass, ...)",
            "breakdown_ms": breakdown,
            "h2d_bytes_per_step": int((n + 4 * n) / steps),
            "d2h_bytes_per_step": int(stats_bytes + 4 * n / steps)}


if __name__ == "__main__":
    sys.exit(main())
