"""Batching form: many independent porous domains of uneven size.

Workload (defaults): 512 domains; every box edge drawn independently from
{32, 48, ..., 128}; each domain its own seeded sphere packing (radius
U[2.5, 7.5], porosity target U[0.35, 0.65]) and wall adhesion G_ads in
U[-2, 0] (rhos = -ln(1 - G_ads/G), G = -6); the drainage boundaries of the
200^3 case scaled to the box (inlet slab round(8 lx / 200) >= 1 at rho 0.10,
outlet plane x = lx - 1 at rho 1.95, pores start at rho 2.0); FP16 storage.

Two executions of the same steps, bit-identical results:
  * batched -- mlbm_batch_iterate: one persistent density launch and one
    persistent update launch per step for all domains, CUDA graphs, work-item
    shape from the autotuner;
  * plain   -- each domain advanced by its own mlbm_iterate calls, one domain
    after the other (sequential per-domain launches), with the same two-pass
    kernels as the batch.
Two more executions advance the domains one after the other with the
fluid-only kernels: plain_compact (the compact two-pass step, two launches
per step and domain) and plain_band (the one-pass step, one launch per step
and domain); both bit-identical to the batch.
All are timed with CUDA events over `--steps` steps (default 5,000, the
configured run); solves/s = domains / (time for 5,000 steps).

Run: python -m multiphase_lbm_b200.batchbench [--domains 512 --steps 5000]
(N GPUs: torchrun --nproc-per-node N -m multiphase_lbm_b200.batchbench; every
rank advances its share of the domains, shard.partition.)
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

from . import batch, capi, host

EDGES = list(range(32, 129, 16))


def make_domains_meta(n, seed=3):
    """(shape, porosity, G_ads, packing seed) of every domain: cheap, so every
    rank draws the whole list and builds only its own share."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        shape = tuple(int(v) for v in rng.choice(EDGES, 3))
        por = float(rng.uniform(0.35, 0.65))
        gads = float(rng.uniform(-2.0, 0.0))
        out.append((shape, por, gads, seed * 100003 + i))
    return out


def build_domain(shape, por, gads, pseed):
    fluid, _ = host.generate_packing(shape, 2.5, 7.5, por, pseed)
    rhos = -math.log(1.0 - gads / -6.0)
    params = capi.default_params(
        G=-6.0, tau=1.0, rhos=rhos, inlet_width=max(1, round(8 * shape[0] / 200)),
        outlet_width=1, rho_inlet=0.10, rho_outlet=1.95, rho_shift=1.0)
    return shape, fluid, np.full(shape, 2.0, np.float32), params


def make_domains(n, seed=3):
    return [build_domain(*m) for m in make_domains_meta(n, seed)]


def run(ndomains=512, steps=100, storage=capi.STORE_F16, solve_steps=5000,
        seed=3, log=print, compact=True, rank=0, world=1) -> dict:
    """On `world` GPUs (one process each, under torchrun) every rank builds
    and advances its own share of the domains (shard.partition by lattice
    size); times are the slowest rank's, throughputs are whole-job."""
    import torch
    from .shard import max_over_ranks, partition
    t0 = time.time()
    all_doms = make_domains_meta(ndomains, seed)
    mine = partition([int(np.prod(m[0])) for m in all_doms], world)[rank]
    doms = [build_domain(*all_doms[i]) for i in mine]
    nodes_all = sum(int(np.prod(m[0])) for m in all_doms)
    nodes = sum(int(np.prod(s)) for s, _, _, _ in doms)
    log(f"{ndomains} domains, {nodes / 1e6:.1f} M nodes, geometry in "
        f"{time.time() - t0:.1f} s")

    # ---- batched --------------------------------------------------------
    b = batch.Batch(storage)
    for shape, fl, rho, p in doms:
        b.add(fl, rho, p)
    tuning = b.autotune(2)
    b.iterate(3)
    b.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    e0.record()
    b.iterate(steps)
    b.synchronize()
    e1.record()
    torch.cuda.synchronize()
    wall_b = time.perf_counter() - t_wall
    ms_b = max_over_ranks(e0.elapsed_time(e1) / steps)
    mem = b.nbytes()
    b.close()

    # ---- plain sequential per-domain launches ---------------------------
    def plain(kernel):
        lats = []
        for shape, fl, rho, p in doms:
            lat = capi.Lattice(shape, storage=storage)
            lat.set_step_kernel(kernel)
            lat.set_params(p)
            lat.upload(fl, rho)
            lat.initialize()
            lat.iterate(0, 3)
            lats.append(lat)
        torch.cuda.synchronize()
        t_wall = time.perf_counter()
        e0.record()
        for k in range(steps):
            for lat in lats:
                lat.iterate(3 + k, 1)
        e1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t_wall
        ms = max_over_ranks(e0.elapsed_time(e1) / steps)
        for lat in lats:
            lat.close()
        return ms, wall

    ms_p, wall_p = plain(capi.KERNEL_TWO_PASS)
    ms_c, wall_c = plain(capi.KERNEL_COMPACT) if compact else (None, None)
    ms_band, wall_band = plain(capi.KERNEL_BAND) if compact else (None, None)

    nodes = nodes_all  # whole-job throughputs below
    res = {
        "domains": ndomains, "nodes": nodes, "storage": storage,
        "n_gpus": world, "domains_per_rank": len(mine),
        "sample_steps": steps, "solve_steps": solve_steps,
        "batched_ms_per_step": round(ms_b, 4),
        "plain_ms_per_step": round(ms_p, 4),
        "batched_mlups": round(nodes / ms_b / 1e3, 1),
        "plain_mlups": round(nodes / ms_p / 1e3, 1),
        "batched_solves_per_s": round(ndomains / (ms_b * solve_steps / 1e3), 4),
        "plain_solves_per_s": round(ndomains / (ms_p * solve_steps / 1e3), 4),
        "speedup": round(ms_p / ms_b, 3),
        "form": "batching",
        "wall_s": {"batched": round(wall_b, 2), "plain": round(wall_p, 2),
                   "plain_compact": None if wall_c is None else round(wall_c, 2),
                   "plain_band": None if wall_band is None else round(wall_band, 2)},
        "plain_compact_ms_per_step": None if ms_c is None else round(ms_c, 4),
        "speedup_vs_plain_compact": None if ms_c is None else round(ms_c / ms_b, 3),
        "plain_band_ms_per_step": None if ms_band is None else round(ms_band, 4),
        "speedup_vs_plain_band": None if ms_band is None else round(ms_band / ms_b, 3),
        "tuning": tuning, "device_bytes": mem,
    }
    return res


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--domains", type=int, default=512)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--storage", default="f16", choices=["f16", "f32"])
    ap.add_argument("--seed", type=int, default=3)
    a = ap.parse_args(argv)
    st = capi.STORE_F16 if a.storage == "f16" else capi.STORE_F32
    import os
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:  # one process per GPU under torchrun
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res = run(a.domains, a.steps, st, seed=a.seed, rank=rank, world=world,
              log=lambda s: print(s, file=sys.stderr, flush=True))
    if rank == 0:
        print(json.dumps(res))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
