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


def _rank(rank, world, port, ring, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    p = problems.channel_small(nx=6, ny=4, nz=20)
    p.periodic = (False, True, ring)
    s = slabs.split(p, world)[rank]
    planes = np.full(s.nz_local, -1.0)
    planes[s.first:s.last + 1] = np.arange(s.z0, s.z1)

    def pack(z, t):
        t.fill_(float(planes[z]))

    def unpack(z, t):
        planes[z] = float(t[0])

    sr = slabs.SlabRank(s, rank, world, ring, pack, unpack, lambda: torch.zeros(8, dtype=torch.float64))
    sr.exchange()
    out.put((rank, s.z0, s.z1, s.lo, s.hi, planes.tolist()))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("ring", [False, True])
def test_slab_exchange_fills_every_ghost_with_its_neighbours_plane(ring, world):
    """With two ranks on a ring the slab below and the slab above are one peer:
    the exchange must still put each plane into the right ghost."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, world, port, ring, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, z0, z1, lo, hi, planes in res:
        expect = [z % 20 for z in range(z0 - lo, z1 + hi)]   # ghosts hold the neighbours' planes (wrapped)
        assert planes == [float(v) for v in expect], (rank, planes)
