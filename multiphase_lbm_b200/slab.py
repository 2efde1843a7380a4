"""One lattice split along z into slabs, one per GPU (or several on one GPU).

The reference runs one lattice on one GPU and has no multi-GPU path; this is
the decomposition for lattices that should span GPUs.  Each slab is an
``mlbm_lattice`` holding its own planes [z0, z0 + m) of the whole lattice
plus one halo plane on each side (periodic in z), marked with
``mlbm_set_slab``: the step advances only the own planes.  A time step is

1. (AA phase 0 only) halo planes <- neighbours' edge planes: the five
   populations each face streams through (``HALO_POP_*``);
2. density pass on every slab (``mlbm_step_pass(..., 0, ...)``);
3. psi halo planes <- neighbours' psi edge planes (``HALO_PSI_*``);
4. update pass on every slab;
5. (AA phase 0 only) neighbours' edge planes <- halo planes: what this
   slab's nodes pushed across the face.  Merged slot by slot: slot s of an
   edge node y came across the face only if y - e_s (the pusher, in the
   other slab) is fluid; where it is solid, y itself wrote that slot (its
   halfway bounce-back) and the received value is stale.

The result is the undecomposed lattice's state bit for bit.  Why z: z is the
outermost dimension of the library's layout, so every halo segment is one
contiguous range (a padded psi plane; one population slot of one plane of
the fluid-only layout) and moves with one copy or one send, no packing.

Transports:
* :class:`RingExchange` -- all slabs in this process, one kernel per
  exchange (``mlbm_slab_ring``, peer loads and stores between GPUs);
* :class:`LocalExchange` -- all slabs in this process: device-to-device
  copies on the current torch stream (the slabs' lattices run on it too);
* :class:`RankExchange` -- one slab per rank (torchrun): the same moves as
  ``torch.distributed`` point-to-point sends and receives in one batch per
  exchange (NCCL over NVLink between GPUs; gloo on CPU tensors in tests).

Both perform the moves of :data:`MOVES_IN` / :data:`MOVES_OUT`, written once:
a move ``(src kind, src side, dir, dst kind, dst side)`` copies segments of
slab i into slab i + dir.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import capi

EDGE_POP, GHOST_POP = capi.HALO_POP_EDGE, capi.HALO_POP_GHOST
EDGE_PSI, GHOST_PSI = capi.HALO_PSI_EDGE, capi.HALO_PSI_GHOST

# D3Q19 velocities in the library's order (csrc/lattice.cuh)
_EX = [0, -1, 0, 0, -1, -1, -1, -1, 0, 0, 1, 0, 0, 1, 1, 1, 1, 0, 0]
_EY = [0, 0, -1, 0, -1, 1, 0, 0, -1, -1, 0, 1, 0, 1, -1, 0, 0, 1, 1]
_EZ = [0, 0, 0, -1, 0, 0, -1, 1, -1, 1, 0, 0, 1, 0, 0, 1, -1, 1, -1]

# halo <- neighbour's edge (before a phase-0 step, and psi between passes)
MOVES_IN = ((1, +1, 0), (0, -1, 1))      # (src side, dir, dst side)
# neighbour's edge <- halo (after a phase-0 step)
MOVES_OUT = ((1, +1, 0), (0, -1, 1))


def slab_bounds(fluid: np.ndarray, parts: int) -> List[Tuple[int, int]]:
    """Contiguous z-ranges (z0, m) of a [x][y][z] fluid mask for `parts`
    slabs, each >= 1 plane, balancing the fluid nodes (what the step
    costs)."""
    nz = fluid.shape[2]
    if not 1 <= parts <= nz:
        raise ValueError(f"cannot split {nz} planes into {parts} slabs")
    per = np.asarray(fluid, bool).sum(axis=(0, 1)).astype(np.float64)
    cum = np.concatenate([[0.0], np.cumsum(per)])
    cuts = [0]
    for i in range(1, parts):
        z = int(np.searchsorted(cum, cum[-1] * i / parts))
        z = min(max(z, cuts[-1] + 1), nz - (parts - i))
        cuts.append(z)
    cuts.append(nz)
    return [(cuts[i], cuts[i + 1] - cuts[i]) for i in range(parts)]


def slab_view(arr: np.ndarray, z0: int, m: int) -> np.ndarray:
    """Planes z0 - 1 .. z0 + m of a [x][y][z] array (periodic in z)."""
    nz = arr.shape[2]
    idx = [(z0 - 1) % nz] + list(range(z0, z0 + m)) + [(z0 + m) % nz]
    return np.ascontiguousarray(np.take(arr, idx, axis=2))


class _DeviceBytes:
    """A device range as an object torch can view (CUDA array interface)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {
            "shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
            "version": 3, "strides": None}


def device_bytes(ptr: int, nbytes: int, device: int):
    """A torch uint8 tensor over `nbytes` of device memory at `ptr`."""
    import torch
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device=f"cuda:{device}")


def push_masks(fluid_slab: np.ndarray, side: int) -> List[np.ndarray]:
    """For the edge plane of `side` of a slab ([x][y][z] mask with its halo
    planes), one boolean array per population segment of HALO_POP_EDGE
    (directions with e_z = +1 for side 0, -1 for side 1, ascending): True
    where the node's slot is written from across the face, i.e. where
    y - e_s is fluid.  Entries follow the fluid-only layout of the plane
    (rows y ascending, x ascending within a row, one hole slot -- False --
    when the plane's fluid count is odd)."""
    f = np.asarray(fluid_slab, bool)
    lx, ly, lz = f.shape
    z = 1 if side == 0 else lz - 2
    dz = 1 if side == 0 else -1
    ys, xs = np.nonzero(f[:, :, z].T)  # (y, x) in layout order
    out = []
    if len(xs) == 0:
        return out
    for d in range(1, 19):
        if _EZ[d] != dz:
            continue
        px, py = (xs - _EX[d]) % lx, (ys - _EY[d]) % ly
        m = f[px, py, z - dz]
        if len(m) % 2:
            m = np.concatenate([m, [False]])
        out.append(m)
    return out


class Slab:
    """One slab: its own planes [z0, z0 + m) and the two halo planes, as a
    lattice on `device` stepping on the current torch stream of that
    device."""

    def __init__(self, fluid: np.ndarray, rho: np.ndarray, params, z0: int,
                 m: int, storage: int = capi.STORE_F32, device: int = 0):
        import torch
        self.z0, self.m, self.device = int(z0), int(m), int(device)
        sub_f = slab_view(fluid, z0, m)
        self.lat = capi.Lattice(sub_f.shape, storage, device)
        self.lat.set_params(params)
        self.lat.upload(sub_f, slab_view(rho, z0, m))
        self.lat.set_stream(torch.cuda.current_stream(device).cuda_stream)
        self.lat.initialize()
        self.lat.set_slab(True)
        pop_t = torch.int16 if storage == capi.STORE_F16 else torch.int32
        self._types = {EDGE_POP: pop_t, GHOST_POP: pop_t,
                       EDGE_PSI: torch.int32, GHOST_PSI: torch.int32}
        self._masks = {}
        for side in (0, 1):
            ms = push_masks(sub_f, side)
            segs = self.segments(EDGE_POP, side)
            if [len(m) for m in ms] != [t.numel() for t in segs]:
                raise RuntimeError("halo segments do not follow the plane layout")
            self._masks[side] = [torch.as_tensor(m, device=f"cuda:{device}")
                                 for m in ms]

    def segments(self, kind: int, side: int):
        """Element views (int32 / int16: bits, not values) of the halo
        segments of one kind on one side; cached, since the layout stays put
        while the lattice steps."""
        if not hasattr(self, "_segs"):
            self._segs = {}
        key = (kind, side)
        if key not in self._segs:
            self._segs[key] = [
                device_bytes(p, n, self.device).view(self._types[kind])
                for p, n in self.lat.halo_segments(kind, side) if n > 0]
        return self._segs[key]

    def push_mask(self, side: int):
        """Per EDGE_POP segment of `side`: where received values apply."""
        return self._masks[side]

    def field(self, which: str) -> np.ndarray:
        """A field of the own planes, [x][y][z]."""
        return self.lat.field(which)[:, :, 1:-1]

    def close(self) -> None:
        self._segs = {}
        self.lat.close()


def _merge(dst, src, mask) -> None:
    """dst[mask] = src[mask], without a host synchronisation."""
    import torch
    torch.where(mask, src, dst, out=dst)


class LocalExchange:
    """Halo moves between slabs held by this process, in ring order (the
    list order along z, periodic)."""

    def __init__(self, slabs: Sequence[Slab]):
        self.slabs = list(slabs)

    def _move(self, src_kind: int, dst_kind: int, moves) -> None:
        n = len(self.slabs)
        for i, s in enumerate(self.slabs):
            for src_side, d, dst_side in moves:
                dst = self.slabs[(i + d) % n]
                masks = (dst.push_mask(dst_side) if dst_kind == EDGE_POP
                         else None)
                for j, (a, b) in enumerate(zip(s.segments(src_kind, src_side),
                                               dst.segments(dst_kind, dst_side))):
                    if masks is None:
                        b.copy_(a)
                    else:
                        _merge(b, a, masks[j])

    def pops_in(self) -> None:
        self._move(EDGE_POP, GHOST_POP, MOVES_IN)

    def psi(self) -> None:
        self._move(EDGE_PSI, GHOST_PSI, MOVES_IN)

    def pops_out(self) -> None:
        self._move(GHOST_POP, EDGE_POP, MOVES_OUT)


class RingExchange:
    """All slabs of this process, one kernel per exchange
    (``mlbm_slab_ring``): the same moves and merge as
    :class:`LocalExchange`, issued from C as one launch, with the slabs on
    one GPU or on GPUs with peer access (loads and stores over NVLink)."""

    def __init__(self, slabs: Sequence[Slab]):
        import ctypes as C
        self.slabs = list(slabs)
        arr = (C.c_void_p * len(self.slabs))(*[s.lat.h.value for s in self.slabs])
        h = C.c_void_p()
        capi.check(capi.lib().mlbm_slab_ring_create(arr, len(self.slabs),
                                                    C.byref(h)))
        self.h = h

    def _run(self, what: int) -> None:
        capi.check(capi.lib().mlbm_slab_ring_exchange(self.h, what))

    def pops_in(self) -> None:
        self._run(0)

    def psi(self) -> None:
        self._run(1)

    def pops_out(self) -> None:
        self._run(2)

    def close(self) -> None:
        h = getattr(self, "h", None)
        if h:
            self.h = None
            capi.lib().mlbm_slab_ring_destroy(h)

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


class RankExchange:
    """Halo moves between ranks of a process group, one slab per rank, rank
    order = z order (periodic).  Each exchange is one batch of sends and
    receives; every rank issues the same batch shape, so the batches match
    (NCCL pairs them in order, gloo by tag)."""

    def __init__(self, slab, group=None):
        import torch.distributed as dist
        self.slab = slab
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def _peer(self, r: int) -> int:
        import torch.distributed as dist
        r %= self.world
        return r if self.group is None else dist.get_global_rank(self.group, r)

    def _move(self, src_kind: int, dst_kind: int, moves) -> None:
        import torch.distributed as dist
        if self.world == 1:
            LocalExchange([self.slab])._move(src_kind, dst_kind, moves)
            return
        ops, merges = [], []
        for j, (src_side, d, dst_side) in enumerate(moves):
            out = self.slab.segments(src_kind, src_side)
            inn = self.slab.segments(dst_kind, dst_side)
            masks = (self.slab.push_mask(dst_side) if dst_kind == EDGE_POP
                     else None)
            for k, t in enumerate(out):
                ops.append(dist.P2POp(dist.isend, t, self._peer(self.rank + d),
                                      self.group, tag=8 * j + k))
            for k, t in enumerate(inn):
                if masks is not None:  # receive aside, then merge
                    buf = self._staging(j, k, t)
                    merges.append((t, buf, masks[k]))
                    t = buf
                ops.append(dist.P2POp(dist.irecv, t, self._peer(self.rank - d),
                                      self.group, tag=8 * j + k))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for dst, buf, mask in merges:
            _merge(dst, buf, mask)

    def _staging(self, j: int, k: int, like):
        if not hasattr(self, "_bufs"):
            self._bufs = {}
        key = (j, k)
        if key not in self._bufs or self._bufs[key].numel() != like.numel():
            self._bufs[key] = like.clone()
        return self._bufs[key]

    def pops_in(self) -> None:
        self._move(EDGE_POP, GHOST_POP, MOVES_IN)

    def psi(self) -> None:
        self._move(EDGE_PSI, GHOST_PSI, MOVES_IN)

    def pops_out(self) -> None:
        self._move(GHOST_POP, EDGE_POP, MOVES_OUT)


class SlabRun:
    """Time steps of a decomposed lattice: `slabs` are the slabs this
    process steps (all of them with :class:`LocalExchange`, its own one
    with :class:`RankExchange`)."""

    def __init__(self, slabs: Sequence[Slab], exchange):
        self.slabs = list(slabs)
        self.exchange = exchange
        self.phase = self.slabs[0].lat.info()["phase"]

    def step(self, step: int, reverse: int = 1, inject_type: int = 0,
             write_velocity: bool = False) -> None:
        if self.phase == 0:
            self.exchange.pops_in()
        for s in self.slabs:
            s.lat.step_pass(step, 0, reverse, inject_type)
        self.exchange.psi()
        for s in self.slabs:
            s.lat.step_pass(step, 1, reverse, inject_type, write_velocity)
        if self.phase == 0:
            self.exchange.pops_out()
        self.phase ^= 1

    def run(self, step0: int, nsteps: int, **kw) -> None:
        for s in range(nsteps):
            self.step(step0 + s, **kw)

    def close(self) -> None:
        """Release the transport, then the slabs (a ring holds their device
        addresses, so it goes first)."""
        close = getattr(self.exchange, "close", None)
        if close:
            close()
        for s in self.slabs:
            s.close()


def decompose(fluid: np.ndarray, rho: np.ndarray, params, parts: int,
              storage: int = capi.STORE_F32,
              devices: Optional[Sequence[int]] = None,
              transport: str = "ring") -> SlabRun:
    """All slabs of a lattice in this process (`devices[i]` for slab i,
    default GPU 0), exchanging through :class:`RingExchange` ("ring", one
    kernel per exchange) or :class:`LocalExchange` ("local", torch ops)."""
    bounds = slab_bounds(fluid, parts)
    devs = list(devices) if devices is not None else [0] * parts
    slabs = [Slab(fluid, rho, params, z0, m, storage, devs[i])
             for i, (z0, m) in enumerate(bounds)]
    if transport == "ring":
        return SlabRun(slabs, RingExchange(slabs))
    if transport == "local":
        return SlabRun(slabs, LocalExchange(slabs))
    raise ValueError(f"unknown transport {transport!r}")


def gather(slabs: Sequence[Slab], which: str) -> np.ndarray:
    """A field of the whole lattice from its slabs (in z order)."""
    return np.concatenate([s.field(which) for s in slabs], axis=2)
