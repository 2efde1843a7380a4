"""The slab decomposition's host logic on the CPU (slab.py): z-ranges that
balance the fluid nodes, halo planes with periodic wrap, and the halo moves
of both transports.  Fake slabs hold CPU tensors in place of the device
segments; ranks run over gloo (world sizes 2 and 3) and must leave every
halo equal to the neighbour's edge -- and after the outbound move every edge
equal to the neighbour's halo -- exactly as the in-process transport does."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from multiphase_lbm_b200 import slab

KINDS = (slab.EDGE_POP, slab.GHOST_POP, slab.EDGE_PSI, slab.GHOST_PSI)


class FakeSlab:
    """Segments of a slab as CPU tensors: POP kinds have 5 segments of a
    plane-dependent size, PSI kinds one; edges carry rank-stamped values,
    halos start at -1."""

    def __init__(self, r, world):
        self.segs = {}
        for kind in KINDS:
            for side in (0, 1):
                # the global plane this segment belongs to fixes its size, so
                # a halo and the edge it pairs with have equal sizes
                edge = kind in (slab.EDGE_POP, slab.EDGE_PSI)
                plane = (2 * r + side) if edge else \
                    (2 * r - 1 if side == 0 else 2 * r + 2)
                plane %= 2 * world
                n = 1 if kind in (slab.EDGE_PSI, slab.GHOST_PSI) else 5
                seg = []
                for j in range(n):
                    size = 3 + (plane * 7 + j) % 5
                    val = 1000 * r + 100 * kind + 10 * side + j if edge else -1
                    seg.append(torch.full((size,), float(val)))
                self.segs[(kind, side)] = seg

        # where a received push applies (the pusher is fluid); seeded by
        # rank so every process builds the same fake
        g = torch.Generator().manual_seed(97 * r + 5)
        self.masks = {side: [torch.rand(t.numel(), generator=g) < 0.7
                             for t in self.segs[(slab.EDGE_POP, side)]]
                      for side in (0, 1)}

    def segments(self, kind, side):
        return self.segs[(kind, side)]

    def push_mask(self, side):
        return self.masks[side]


def _fake_world(world):
    """FakeSlabs of a ring of 2 * world planes, slab r owning planes 2r and
    2r + 1, so a halo and the neighbour's edge it pairs with have the same
    plane and the same segment sizes."""
    return [FakeSlab(r, world) for r in range(world)]


def _expected(world):
    """Expected halo contents after MOVES_IN and edge contents after
    MOVES_OUT, from the in-process transport."""
    s = _fake_world(world)
    ex = slab.LocalExchange(s)
    ex.pops_in()
    ex.psi()
    after_in = {r: {k: [t.clone() for t in v] for k, v in s[r].segs.items()}
                for r in range(world)}
    for r in range(world):  # mark the halos, then send them back
        for kind in (slab.GHOST_POP,):
            for side in (0, 1):
                for j, t in enumerate(s[r].segs[(kind, side)]):
                    t.fill_(-(1000 * r + 10 * side + j + 1))
    ex.pops_out()
    after_out = {r: {k: [t.clone() for t in v] for k, v in s[r].segs.items()}
                 for r in range(world)}
    return after_in, after_out


def test_local_moves_fill_halos_from_neighbours():
    world = 3
    s = _fake_world(world)
    edges = {r: {k: [t.clone() for t in v] for k, v in s[r].segs.items()}
             for r in range(world)}
    ex = slab.LocalExchange(s)
    ex.pops_in()
    ex.psi()
    for r in range(world):
        up, down = (r + 1) % world, (r - 1) % world
        for kind, ekind in ((slab.GHOST_POP, slab.EDGE_POP),
                            (slab.GHOST_PSI, slab.EDGE_PSI)):
            for a, b in zip(s[r].segs[(kind, 1)], edges[up][(ekind, 0)]):
                assert torch.equal(a, b)
            for a, b in zip(s[r].segs[(kind, 0)], edges[down][(ekind, 1)]):
                assert torch.equal(a, b)


def test_local_moves_return_pushes_to_neighbours():
    world = 3
    _, after_out = _expected(world)
    fakes = _fake_world(world)
    for r in range(world):
        up, down = (r + 1) % world, (r - 1) % world
        # r's lower edge holds what the slab below pushed (its upper halo)
        # where the push applies, and its own value elsewhere
        for side, src, sside in ((0, down, 1), (1, up, 0)):
            for j, t in enumerate(after_out[r][(slab.EDGE_POP, side)]):
                own = fakes[r].segs[(slab.EDGE_POP, side)][j]
                mask = fakes[r].masks[side][j]
                pushed = torch.full_like(own, -(1000 * src + 10 * sside + j + 1))
                assert torch.equal(t, torch.where(mask, pushed, own))
    allm = torch.cat([m for f in fakes for side in (0, 1) for m in f.masks[side]])
    assert allm.any() and (~allm).any()  # both branches of the merge ran


def test_bounds_balance_fluid_and_cover_planes():
    rng = np.random.default_rng(3)
    fl = (rng.random((8, 6, 40)) < np.linspace(0.1, 0.9, 40)).astype(np.uint8)
    for parts in (1, 2, 3, 7, 40):
        b = slab.slab_bounds(fl, parts)
        assert b[0][0] == 0 and sum(m for _, m in b) == 40
        assert all(m >= 1 for _, m in b)
        assert all(b[i][0] + b[i][1] == b[i + 1][0] for i in range(parts - 1))
    per = fl.sum(axis=(0, 1))
    b = slab.slab_bounds(fl, 4)
    loads = [per[z0:z0 + m].sum() for z0, m in b]
    assert max(loads) - min(loads) <= 2 * per.max()
    with pytest.raises(ValueError):
        slab.slab_bounds(fl, 41)


def test_slab_view_wraps_halo_planes():
    a = np.arange(2 * 3 * 5).reshape(2, 3, 5)
    v = slab.slab_view(a, 0, 2)
    assert np.array_equal(v, a[:, :, [4, 0, 1, 2]])
    v = slab.slab_view(a, 3, 2)
    assert np.array_equal(v, a[:, :, [2, 3, 4, 0]])
    v = slab.slab_view(a, 0, 5)
    assert np.array_equal(v, a[:, :, [4, 0, 1, 2, 3, 4, 0]])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from multiphase_lbm_b200 import slab as sl
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        me = FakeSlab(rank, world)
        ex = sl.RankExchange(me)
        ex.pops_in()
        ex.psi()
        # plain lists: tensors sent through a queue would share memory with
        # a process that has exited by the time they are read
        after_in = {k: [t.tolist() for t in v] for k, v in me.segs.items()}
        for side in (0, 1):
            for j, t in enumerate(me.segs[(sl.GHOST_POP, side)]):
                t.fill_(-(1000 * rank + 10 * side + j + 1))
        ex.pops_out()
        after_out = {k: [t.tolist() for t in v] for k, v in me.segs.items()}
        dist.barrier()
        q.put((rank, after_in, after_out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_rank_moves_over_gloo_match_local_moves(world):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, a, b = q.get(timeout=120)
        res[r] = (a, b)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want_in, want_out = _expected(world)
    for r in range(world):
        for key, segs in want_in[r].items():
            assert res[r][0][key] == [t.tolist() for t in segs], (r, key)
        for key, segs in want_out[r].items():
            assert res[r][1][key] == [t.tolist() for t in segs], (r, key)


def test_push_masks_match_brute_force():
    """slab.push_masks against a direct walk of the plane: for each fluid node
    of the edge plane in layout order (rows y, then x) and each direction s
    crossing the face, whether the node y - e_s that would push into it is
    fluid; a hole entry (False) pads an odd count."""
    rng = np.random.default_rng(8)
    f = (rng.random((7, 5, 6)) < 0.6).astype(np.uint8)
    lx, ly, lz = f.shape
    for side, dz in ((0, 1), (1, -1)):
        z = 1 if side == 0 else lz - 2
        got = slab.push_masks(f, side)
        dirs = [d for d in range(1, 19) if slab._EZ[d] == dz]
        nodes = [(x, y) for y in range(ly) for x in range(lx) if f[x, y, z]]
        assert len(got) == len(dirs)
        for m, d in zip(got, dirs):
            want = [bool(f[(x - slab._EX[d]) % lx, (y - slab._EY[d]) % ly, z - dz])
                    for x, y in nodes]
            if len(want) % 2:
                want.append(False)
            assert m.tolist() == want
