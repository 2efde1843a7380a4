"""One lattice over several GPUs: time the slab decomposition (slab.py).

Workload: the 200^3 drainage packing of bench.py (radii U[5, 15] to porosity
0.50, seed 2024; pores at rho 2.0; inlet slab x < 8 at rho 0.10, outlet plane
x = lx - 1 at rho 1.95), any cubic size, FP32 or FP16 storage.

* under torchrun (one process per GPU): rank r steps slab r of the z-split,
  exchanging halos with its neighbours through RankExchange (NCCL
  point-to-point batches); strong scaling, the lattice is fixed;
* in one process: ``--parts P`` slabs on the current GPU through the ring
  exchange (one kernel per exchange), to measure the decomposition's
  overhead against the undecomposed lattice on one GPU.

Timing: CUDA events around `--steps` steps after `--warmup` steps, on each
rank; the slowest rank's time (shard.max_over_ranks).  Prints one JSON line
on rank 0: MLUPS over all lattice nodes.

Run: python -m torch.distributed.run --nproc-per-node N --master-addr
127.0.0.1 -m multiphase_lbm_b200.slabbench --size 400 --steps 200
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

from . import capi, host, slab


def workload(n: int):
    fluid, _ = host.generate_packing((n, n, n), 5.0, 15.0, 0.50, 2024)
    rho = np.full((n, n, n), 2.0, np.float32)
    params = capi.default_params(G=-6.0, tau=1.0, rhos=0.182322,
                                 inlet_width=max(1, round(8 * n / 200)),
                                 outlet_width=1, rho_inlet=0.10,
                                 rho_outlet=1.95, rho_shift=1.0)
    return fluid, rho, params


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--size", type=int, default=200)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--parts", type=int, default=0,
                    help="slabs in this process (single-process mode)")
    ap.add_argument("--storage", default="f32", choices=["f32", "f16"])
    a = ap.parse_args(argv)
    import torch

    from .shard import max_over_ranks
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    st = capi.STORE_F16 if a.storage == "f16" else capi.STORE_F32
    fluid, rho, params = workload(a.size)
    dev = torch.cuda.current_device()
    if world > 1:
        z0, m = slab.slab_bounds(fluid, world)[rank]
        mine = slab.Slab(fluid, rho, params, z0, m, st, dev)
        run = slab.SlabRun([mine], slab.RankExchange(mine))
        parts = world
    else:
        parts = max(1, a.parts)
        run = slab.decompose(fluid, rho, params, parts, st, [dev] * parts)
    run.run(0, a.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run.run(a.warmup, a.steps)
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / a.steps)
    if rank == 0:
        n = fluid.size
        print(json.dumps({
            "metric": "MLUPS", "value": round(n / (ms * 1e-3) / 1e6, 2),
            "unit": "MLUPS", "ms_per_step": round(ms, 4), "n_gpus": world,
            "slabs": parts, "lattice": [a.size] * 3, "storage": a.storage,
            "steps": a.steps, "warmup": a.warmup,
            "scaling": "strong", "transport": "nccl" if world > 1 else "ring"}))
    run.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
