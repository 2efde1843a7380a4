"""Serving form: a request loop with continuous batching.

Each request is one porous domain: box edges drawn from {48, 64, ..., 192},
a seeded sphere packing (radius U[2.5, 7.5], porosity U[0.35, 0.65]), inlet
density U[0.05, 0.3], wall adhesion G_ads U[-2, 0] (G = -5, see SERVE_G), a step budget
U[2000, 50000] (times --budget-scale), and a tolerance that picks FP32 or
FP16 storage.  A request is done when its budget is spent or its saturation
changed by less than 1e-5 over the last 1000 steps.

Batched server: requests arrive as a Poisson stream; the loop admits
arrived requests, the one with the least work left first, while they fit
under the HBM cap into the FP32 or FP16 batch (mlbm_batch_add; the geometry
is built on the host while the GPU runs the previous chunk), preempts a
long request for a much shorter one (exact checkpoint to host memory,
mlbm_batch_add_checkpoint to resume), advances both batches by `chunk`
steps (their launches overlap on the device), and retires finished requests
(mlbm_batch_remove), freeing memory for the queue.  FIFO baseline: the same
requests, in arrival order, each run alone on the whole GPU with
mlbm_iterate.

Reported, one JSON line per arrival rate: solves/s, p50/p95/p99
time-to-result (arrival to result on the host), the fraction of the run with
nothing to compute (idle_fraction) and the throughput while busy, for both.  Each result (final saturation and density field) is the
same in the batch as alone: the batched kernels are bit-identical to the
single-domain ones (tests/test_gpu_batch.py, tests/test_gpu_serve.py).

Run: python -m multiphase_lbm_b200.serve --requests 48 --rates 5,20,50,200
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time
from dataclasses import dataclass, field

import numpy as np

from . import batch, capi, host

EDGES = list(range(48, 193, 16))
# Coupling of the served drainage runs.  The configured G = -6 with pores at
# rho 2.0 turns to NaN within a few hundred steps in the reference's own
# scheme (the liquid cavitates at the walls), so no run could converge;
# G = -5 is the nearest coupling that stays finite and lets the convergence
# test end requests.  The step cost does not depend on G.
SERVE_G = -5.0
CONVERGENCE_DS = 1e-5
CONVERGENCE_STEPS = 1000
# Active lattice nodes beyond which arrivals wait (about twice what fills
# every SM of a B200 with the compact kernels).
DEFAULT_NODE_CAP = 16_000_000


# Preemption: a waiting request displaces the running request with the most
# work left when its own work is below this fraction of that.
PREEMPT_RATIO = 0.25


@dataclass
class Request:
    rid: int
    arrival: float
    shape: tuple
    seed: int
    porosity: float
    rho_in: float
    g_ads: float
    budget: int
    fp16_ok: bool
    # filled by the server
    done_at: float = -1.0
    steps: int = 0
    saturation: float = float("nan")
    converged: bool = False
    history: list = field(default_factory=list)
    image: object = None        # checkpoint of a preempted request
    preemptions: int = 0

    def nodes(self) -> int:
        return int(np.prod(self.shape))

    def work_left(self) -> int:
        return self.nodes() * max(0, self.budget - self.steps)


def make_requests(n, rate, seed=7, budget_scale=1.0, edges=EDGES):
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        shape = tuple(int(v) for v in rng.choice(edges, 3))
        budget = max(CONVERGENCE_STEPS,
                     int(round(rng.uniform(2000, 50000) * budget_scale)))
        out.append(Request(i, t, shape, int(rng.integers(1 << 30)),
                           float(rng.uniform(0.35, 0.65)),
                           float(rng.uniform(0.05, 0.3)),
                           float(rng.uniform(-2.0, 0.0)), budget,
                           bool(rng.random() < 0.5)))
    return out


def geometry(req: Request):
    fluid, _ = host.generate_packing(req.shape, 2.5, 7.5, req.porosity, req.seed)
    rho = np.full(req.shape, 2.0, np.float32)
    rhos = -math.log(1.0 - req.g_ads / SERVE_G)
    params = capi.default_params(
        G=SERVE_G, tau=1.0, rhos=rhos,
        inlet_width=max(1, round(8 * req.shape[0] / 200)), outlet_width=1,
        rho_inlet=req.rho_in, rho_outlet=1.95, rho_shift=1.0)
    return fluid, rho, params


def _finished(req: Request) -> bool:
    if req.steps >= req.budget:
        return True
    h = req.history
    if len(h) >= 2 and h[-1][0] - h[-2][0] >= CONVERGENCE_STEPS:
        if abs(h[-1][1] - h[-2][1]) < CONVERGENCE_DS:
            req.converged = True
            return True
    return False


def serve_batched(reqs, hbm_cap=150e9, chunk=CONVERGENCE_STEPS, log=None,
                  node_cap=DEFAULT_NODE_CAP, preempt=True):
    """Continuous batching; returns (makespan_s, requests).

    Arrived requests wait in order of the work they have left (shortest
    first) and are admitted while their lattices fit under the HBM cap and
    the active lattices hold fewer than `node_cap` nodes in total: enough
    resident work to keep every SM busy, but no more, since requests that
    share the GPU beyond saturation only wait longer for their results
    without raising throughput.  With `preempt`, a waiting request whose work
    is below PREEMPT_RATIO of the running request with the most work left
    displaces it: that request is saved (an exact checkpoint in host memory),
    removed from its batch and queued again with its work left; it resumes
    from the image, bit for bit, when there is room.  Requests change batch
    only at chunk boundaries, where their convergence test runs, so every
    result is the one the request gives alone."""
    batches = {True: batch.Batch(capi.STORE_F16), False: batch.Batch(capi.STORE_F32)}
    pending = sorted(reqs, key=lambda r: r.arrival)
    waiting = []     # arrived, not running (new or preempted)
    ready = {}       # rid -> geometry built ahead of admission
    active = {}      # rid -> (req, batch, domain id, bytes)
    used = 0
    nodes = 0        # lattice nodes of the active requests
    t0 = time.perf_counter()
    qi = 0
    idle = 0.0       # seconds with nothing to run

    def fits(r, need):
        return not active or (used + need <= hbm_cap and nodes + r.nodes() <= node_cap)

    def suspend(rid):
        nonlocal used, nodes
        r, b, did, need = active.pop(rid)
        r.image = b.lattice(did).checkpoint(r.steps)
        b.remove(did)
        used -= need
        nodes -= r.nodes()
        r.preemptions += 1
        waiting.append(r)

    while qi < len(pending) or active or waiting:
        now = time.perf_counter() - t0
        while qi < len(pending) and pending[qi].arrival <= now:
            waiting.append(pending[qi])
            qi += 1
        waiting.sort(key=lambda q: (q.work_left(), q.arrival))
        # admit (shortest work first), preempting where that pays
        for r in list(waiting):
            storage = capi.STORE_F16 if r.fp16_ok else capi.STORE_F32
            need = capi.lattice_bytes(r.shape, storage)
            if not fits(r, need) and preempt and active:
                victim = max(active, key=lambda rid: active[rid][0].work_left())
                if r.work_left() < PREEMPT_RATIO * active[victim][0].work_left():
                    suspend(victim)
            if not fits(r, need):
                break
            waiting.remove(r)
            b = batches[r.fp16_ok]
            if r.image is not None:
                did = b.add_checkpoint(r.image)
                r.image = None
            else:
                fl, rho, p = ready.pop(r.rid, None) or geometry(r)
                did = b.add(fl, rho, p)
            active[r.rid] = (r, b, did, need)
            used += need
            nodes += r.nodes()
        if not active:
            if qi < len(pending):
                wait = max(0.0, pending[qi].arrival - now)
                time.sleep(wait)
                idle += wait
            continue
        # advance every batch by one chunk (asynchronous, overlapping)
        for b in batches.values():
            if b.count():
                b.iterate(chunk)
        # build geometry of the next arrivals while the GPU works
        for r in pending[qi:qi + 4]:
            if r.rid not in ready:
                ready[r.rid] = geometry(r)
        for b in batches.values():
            b.synchronize()
        done = []
        for rid, (r, b, did, need) in active.items():
            r.steps += chunk
            sat = b.lattice(did).stats()["saturation"]
            r.history.append((r.steps, sat))
            if _finished(r):
                r.saturation = sat
                r.done_at = time.perf_counter() - t0
                done.append(rid)
        for rid in done:
            r, b, did, need = active.pop(rid)
            b.remove(did)
            used -= need
            nodes -= r.nodes()
        if log and done:
            log(f"t={time.perf_counter() - t0:.2f}s active={len(active)} "
                f"done+={len(done)} waiting={len(waiting)} "
                f"queue={len(pending) - qi}")
    makespan = time.perf_counter() - t0
    for b in batches.values():
        b.close()
    return makespan, reqs, idle


def serve_fifo(reqs, chunk=CONVERGENCE_STEPS, log=None,
               kernel=capi.KERNEL_AUTO):
    """Requests one at a time in arrival order, each alone on the GPU, with
    the fastest plain kernels (AUTO: the compact two-pass step, bit-identical
    to the batch's kernels, so every result equals the batched one bit for
    bit)."""
    t0 = time.perf_counter()
    idle = 0.0
    for r in sorted(reqs, key=lambda q: q.arrival):
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
            idle += r.arrival - now
        fl, rho, p = geometry(r)
        lat = capi.Lattice(r.shape, storage=capi.STORE_F16 if r.fp16_ok
                           else capi.STORE_F32)
        lat.set_step_kernel(kernel)
        lat.set_params(p)
        lat.upload(fl, rho)
        lat.initialize()
        while True:
            lat.iterate(r.steps, chunk)
            r.steps += chunk
            s = lat.stats()["saturation"]
            r.history.append((r.steps, s))
            if _finished(r):
                r.saturation = s
                break
        r.done_at = time.perf_counter() - t0
        lat.close()
    return time.perf_counter() - t0, reqs, idle


def summarise(makespan, reqs, idle=0.0):
    ttr = np.array([r.done_at - r.arrival for r in reqs])
    node_steps = int(sum(np.prod(r.shape) * r.steps for r in reqs))
    busy = max(1e-9, makespan - idle)
    return {"requests": len(reqs), "makespan_s": round(makespan, 3),
            "idle_fraction": round(idle / makespan, 4),
            "mlups_while_busy": round(node_steps / busy / 1e6, 1),
            "solves_per_s": round(len(reqs) / makespan, 4),
            "p50_s": round(float(np.percentile(ttr, 50)), 3),
            "p95_s": round(float(np.percentile(ttr, 95)), 3),
            "p99_s": round(float(np.percentile(ttr, 99)), 3),
            "converged": int(sum(r.converged for r in reqs)),
            "preemptions": int(sum(r.preemptions for r in reqs)),
            "node_steps": node_steps}


def run_rate(a, rate, log):
    """Batched and FIFO serving of the same request stream at one rate: one
    JSON-able dict."""
    reqs = make_requests(a.requests, rate, a.seed, a.budget_scale)
    mk, done, idle = serve_batched(reqs, a.hbm_cap_gb * 1e9, log=log,
                                   node_cap=a.node_cap,
                                   preempt=not a.no_preempt)
    out = {"form": "serving", "config": {
               "requests": a.requests, "rate_per_s": rate,
               "budget_scale": a.budget_scale, "hbm_cap_gb": a.hbm_cap_gb,
               "node_cap": a.node_cap, "seed": a.seed,
               "preempt": not a.no_preempt, "G": SERVE_G},
           "batched": summarise(mk, done, idle)}
    if not a.no_fifo:
        reqs2 = make_requests(a.requests, rate, a.seed, a.budget_scale)
        kern = {"auto": capi.KERNEL_AUTO, "two-pass": capi.KERNEL_TWO_PASS,
                "compact": capi.KERNEL_COMPACT,
                "band": capi.KERNEL_BAND}[a.fifo_kernel]
        mk2, done2, idle2 = serve_fifo(reqs2, log=log, kernel=kern)
        out["fifo_kernel"] = a.fifo_kernel
        out["fifo"] = summarise(mk2, done2, idle2)
        same = [abs(x.saturation - y.saturation) <= 0.0 and x.steps == y.steps
                for x, y in zip(sorted(done, key=lambda r: r.rid),
                                sorted(done2, key=lambda r: r.rid))]
        out["results_identical"] = int(sum(same))
        out["solves_ratio"] = round(out["batched"]["solves_per_s"] /
                                    out["fifo"]["solves_per_s"], 3)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--rate", type=float, default=None,
                    help="one arrival rate (req/s); default: the sweep")
    ap.add_argument("--rates", default="5,20,50,200",
                    help="arrival rates swept, one JSON line each")
    ap.add_argument("--budget-scale", type=float, default=1.0)
    ap.add_argument("--hbm-cap-gb", type=float, default=150.0)
    ap.add_argument("--node-cap", type=float, default=DEFAULT_NODE_CAP,
                    help="active lattice nodes beyond which arrivals wait")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--no-fifo", action="store_true")
    ap.add_argument("--no-preempt", action="store_true")
    ap.add_argument("--fifo-kernel", default="auto",
                    choices=["auto", "two-pass", "compact", "band"])
    a = ap.parse_args(argv)
    log = lambda s: print(s, file=sys.stderr, flush=True)  # noqa: E731
    rates = [a.rate] if a.rate else [float(v) for v in a.rates.split(",")]
    for rate in rates:
        print(json.dumps(run_rate(a, rate, log)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
