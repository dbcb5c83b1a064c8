"""z-slab decomposition on the CPU: how split() cuts a problem, and the halo
exchange of SlabRank over two and three gloo ranks, as a chain and as a ring (planes
stand in for lattices: each interior plane carries its global z, ghosts start
as -1)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fluidmaxxer_b200 import problems, slabs


def test_split_cuts_the_problem_into_slabs_with_ghosts():
    p = problems.channel_small(nx=20, ny=12, nz=37)          # periodic y and z: a ring of slabs
    parts = slabs.split(p, 3)
    assert [(s.z0, s.z1, s.lo, s.hi) for s in parts] == [(0, 12, 1, 1), (12, 25, 1, 1), (25, 37, 1, 1)]
    full = p.solid.reshape(p.nz, p.ny, p.nx)
    for s in parts:
        q = s.problem
        assert (q.nx, q.ny, q.nz) == (p.nx, p.ny, s.nz_local) and q.periodic[2] is False
        zs = [z % p.nz for z in range(s.z0 - s.lo, s.z1 + s.hi)]
        assert np.array_equal(q.solid.reshape(q.nz, q.ny, q.nx), full[zs])
        assert q.ns_inlet == p.ns_inlet and q.ns_outlet == p.ns_outlet and q.sample_every == p.sample_every
        m = slabs.interior_outlet(s).reshape(q.nz, q.ny, q.nx)
        assert m.sum() == (s.z1 - s.z0) * p.ny and m[:, :, -1].all(axis=1)[s.first:s.last + 1].all()
    closed = problems.channel_small(nx=20, ny=12, nz=16)
    closed.periodic = (False, True, False)
    assert [(s.lo, s.hi) for s in slabs.split(closed, 2)] == [(0, 1), (1, 0)]


def test_split_rejects_what_it_cannot_cut():
    with pytest.raises(ValueError):
        slabs.split(problems.channel_small(nz=5), 3)
    q = problems.channel_small(nz=16)
    q.outlet = np.zeros(q.n_cells, np.uint8)
    with pytest.raises(ValueError):
        slabs.split(q, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class FakeIO:
    """Planes stand in for a slab lattice: each interior plane holds its global
    z, ghosts start as None; pack puts (z value, dir) in the buffer and unpack
    records it, so the test sees which plane and which populations arrived."""

    def __init__(self, slab, split):
        self.split = split
        self.planes = [None] * slab.nz_local
        for z in range(slab.first, slab.last + 1):
            self.planes[z] = float(slab.z0 + z - slab.first)
        self.log = []

    def pack(self, z, direction, t):
        self.log.append(("pack", z, direction))
        t[0] = self.planes[z]
        t[1] = float(direction)

    def unpack(self, z, direction, t):
        self.log.append(("unpack", z, direction))
        assert float(t[1]) == float(direction), "halo of the wrong direction"
        self.planes[z] = float(t[0])

    def step_planes(self, z0, z1):
        self.log.append(("planes", z0, z1))

    def finish(self):
        self.log.append(("finish",))

    def step_all(self):
        self.log.append(("all",))

    def make_buffer(self):
        import torch

        return torch.zeros(8, dtype=torch.float64)


def _rank(rank, world, port, ring, split, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    p = problems.channel_small(nx=6, ny=4, nz=20)
    p.periodic = (False, True, ring)
    s = slabs.split(p, world)[rank]
    io = FakeIO(s, split)
    sr = slabs.SlabRank(s, rank, world, ring, io)
    sr.step()
    # the reductions: a series and sums known per rank
    rows = s.z1 - s.z0
    bt = sr.breakthrough(np.array([rank + 1.0, 2.0 * (rank + 1.0)]))
    sums = sr.reduce(np.array([1.0, rank, rows]))
    out.put((rank, s.z0, s.z1, s.lo, s.hi, s.first, s.last, io.planes, io.log, bt.tolist(), sums.tolist()))
    dist.destroy_process_group()


@pytest.mark.parametrize("split", [True, False])
@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("ring", [False, True])
def test_slab_step_exchanges_the_crossing_halos(ring, world, split):
    """Every ghost ends up holding its neighbour's boundary plane, with the
    populations that cross towards it (c_z = +1 into a low ghost, c_z = -1
    into a high ghost).  With two ranks on a ring the slab below and the slab
    above are one peer: the exchange must still put each plane into the right
    ghost.  A split step updates the boundary planes, packs, updates the
    interior while the halos travel, unpacks, then finishes; otherwise the
    slab steps whole first.  The cross-rank reductions of the breakthrough
    (weighted by interior rows) and of the sums are checked too."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, world, port, ring, split, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    nz = 20
    rows = [z1 - z0 for _, z0, z1, *_ in res]
    want_bt = np.array([sum(r * (i + 1.0) for i, r in enumerate(rows)),
                        sum(r * 2.0 * (i + 1.0) for i, r in enumerate(rows))]) / nz
    for rank, z0, z1, lo, hi, first, last, planes, log, bt, sums in res:
        expect = [float(z % nz) for z in range(z0 - lo, z1 + hi)]   # ghosts hold the neighbours' planes
        assert planes == expect, (rank, planes)
        kinds = [e[0] for e in log]
        if split:
            assert log[0] == ("planes", first, first + 1) and log[1] == ("planes", last, last + 1)
            assert kinds.index("unpack") > kinds.index("planes", 2) > max(i for i, k in enumerate(kinds) if k == "pack")
            assert log[-1] == ("finish",) and ("planes", first + 1, last) in log
        else:
            assert kinds[0] == "all" and "finish" not in kinds
        for e in log:
            if e[0] == "unpack":
                assert e[2] == (+1 if e[1] == 0 else -1)
        assert np.allclose(bt, want_bt)
        assert np.allclose(sums, [world, sum(range(world)), nz])
