"""Work across several GPUs (one process per GPU, launched by torchrun).

A single lattice has no exchange-free split (every step needs a halo of
populations and psi), so the single-domain step runs as independent
replicas, one per GPU.  Batches and served requests shard by domain: the
domains are independent lattices, so each rank advances its own share with
no collective on the data path; only the timing (the slowest rank) and the
results are gathered.

* `partition(weights, world)` -- domains to ranks, heaviest first onto the
  least loaded rank (deterministic: ties go to the lower rank, equal weights
  keep their input order), so every rank computes the same assignment
  without communicating;
* `max_over_ranks(value, group)` -- the slowest rank's time, through the
  process group of any backend (NCCL on GPUs, gloo on the CPU);
* `gather_results(obj, group)` -- per-rank result objects on every rank.
"""
from __future__ import annotations

import heapq
from typing import Any, List, Sequence


def partition(weights: Sequence[float], world: int) -> List[List[int]]:
    """Indices of `weights` for each of `world` ranks, balancing the sums
    (longest-processing-time-first)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    for part in out:
        part.sort()
    return out


def _device_for(group) -> str:
    import torch.distributed as dist
    return "cuda" if dist.get_backend(group) == "nccl" else "cpu"


def max_over_ranks(value: float, group=None) -> float:
    """max(value) over the ranks of the process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=_device_for(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_results(obj: Any, group=None) -> List[Any]:
    """Every rank's `obj`, in rank order, on every rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out: List[Any] = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, obj, group=group)
    return out
