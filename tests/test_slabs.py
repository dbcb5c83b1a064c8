"""x-slab decomposition on the CPU: how split() cuts a problem, and the halo
exchange of SlabRank over three gloo ranks (planes stand in for lattices: each
interior plane carries its global x, ghosts start as -1)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fluidmaxxer_b200 import problems, slabs


def test_split_cuts_the_problem_into_slabs_with_ghosts():
    p = problems.channel_small(nx=37, ny=12, nz=10)
    parts = slabs.split(p, 3)
    assert [(s.x0, s.x1, s.lo, s.hi) for s in parts] == [(0, 12, 0, 1), (12, 25, 1, 1), (25, 37, 1, 0)]
    full = p.solid.reshape(p.nz, p.ny, p.nx)
    for s in parts:
        q = s.problem
        assert q.nx == s.nx_local and q.ny == p.ny and q.nz == p.nz
        local = q.solid.reshape(q.nz, q.ny, q.nx)
        assert np.array_equal(local, full[:, :, s.x0 - s.lo:s.x1 + s.hi])
    assert [s.problem.ns_inlet for s in parts] == ["neq", "none", "none"]
    assert [s.problem.ns_outlet for s in parts] == ["none", "none", "pressure"]
    assert [s.problem.ad_outlet for s in parts] == ["none", "none", "neumann"]
    assert [s.problem.sample_every for s in parts] == [0, 0, p.sample_every]


def test_split_rejects_what_it_cannot_cut():
    with pytest.raises(ValueError):
        slabs.split(problems.channel_small(nx=5), 3)
    q = problems.channel_small(nx=16)
    q.periodic = (True, True, True)
    with pytest.raises(ValueError):
        slabs.split(q, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    p = problems.channel_small(nx=20, ny=4, nz=3)
    s = slabs.split(p, world)[rank]
    planes = np.full(s.nx_local, -1.0)
    planes[s.lo:s.lo + s.x1 - s.x0] = np.arange(s.x0, s.x1)

    def pack(x, t):
        t.fill_(float(planes[x]))

    def unpack(x, t):
        planes[x] = float(t[0])

    sr = slabs.SlabRank(s, rank, world, pack, unpack, lambda: torch.zeros(8, dtype=torch.float64))
    sr.exchange()
    out.put((rank, s.x0, s.x1, s.lo, s.hi, planes.tolist()))
    dist.destroy_process_group()


def test_slab_exchange_fills_every_ghost_with_its_neighbours_plane():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 3, port, q)) for r in range(3)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, x0, x1, lo, hi, planes in res:
        expect = list(range(x0 - lo, x1 + hi))    # every plane, ghosts included, now holds its global x
        assert planes == [float(v) for v in expect], (rank, planes)
