"""z-slab decomposition of one coupled lattice.

The slowest axis z is cut into slabs.  Each slab is an ordinary lattice holding
its cells (every x and y) plus one ghost plane per inner face; with periodic z
the first and last slabs are neighbours too (a ring).  Every slab keeps its
share of the x = 0 inlet and x = nx-1 outlet planes, so the fused boundary
planes work in each slab unchanged.  A step is the fused step on every slab,
then the halo exchange: each slab sends the stored populations (19 + 7
directions) of the plane next to an inner face into the neighbour's ghost plane
(``fm_pack_zplane`` / ``fm_unpack_zplane``; a z-plane is one contiguous run of
nx*ny cells per population, so packing is a coalesced copy).  Every interior
cell then pulls exactly what it pulls in the unsplit lattice, so the slabs
reproduce the unsplit run bit for bit; the ghost cells' own updates are
overwritten by the exchange.  The outlet mean C_out is the cell-weighted mean of
the slabs' outlet means over their interior rows.

:class:`SlabRun` runs all slabs of a problem in one process on one GPU (the
slabs step one after another on one stream; the exchange is host-ordered, no
kernel waits for another).  :class:`SlabRank` is one slab per process with the
exchange over ``torch.distributed`` point-to-point (NCCL on GPUs); packing and
transport are separate, so the exchange pattern also runs on CPU ranks.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import lattice as _lattice
from ._abi import check
from .problems import Problem

ELEMENT_BYTES = {"f32": 4, "f64": 8, "f16": 2, "bf16": 2, "f16q": 2}


@dataclasses.dataclass
class Slab:
    index: int
    z0: int            # first interior z of this slab (global)
    z1: int            # one past the last interior z (global)
    lo: int            # ghost planes below z0
    hi: int            # ghost planes above z1 - 1
    problem: Problem   # the slab's own lattice problem (ghosts included, z not periodic)

    @property
    def nz_local(self) -> int:
        return self.z1 - self.z0 + self.lo + self.hi

    @property
    def first(self) -> int:   # local z of the first interior plane
        return self.lo

    @property
    def last(self) -> int:    # local z of the last interior plane
        return self.lo + self.z1 - self.z0 - 1


def _crop(a, p: Problem, zs):
    return np.ascontiguousarray(np.asarray(a).reshape(p.nz, p.ny, p.nx)[zs]).reshape(-1)


def split(problem: Problem, nslabs: int) -> list:
    """Cut `problem` into `nslabs` z-slabs of near-equal thickness (at least 2 planes each)."""
    p = problem
    if nslabs < 1 or p.nz < 2 * nslabs:
        raise ValueError("split: each slab needs at least 2 planes")
    if p.inlet is not None or p.outlet is not None:
        raise ValueError("split: custom inlet / outlet masks are not split; use the x = 0 / x = nx-1 planes")
    ring = bool(p.periodic[2])
    edges = [round(i * p.nz / nslabs) for i in range(nslabs + 1)]
    region = p.solid if p.region is None else p.region
    parts = []
    for i in range(nslabs):
        z0, z1 = edges[i], edges[i + 1]
        lo = int(ring or i > 0)
        hi = int(ring or i < nslabs - 1)
        zs = [z % p.nz for z in range(z0 - lo, z1 + hi)]
        q = dataclasses.replace(p)
        q.nz = len(zs)
        q.periodic = (p.periodic[0], p.periodic[1], False)
        q.solid = _crop(p.solid, p, zs).astype(np.uint8)
        q.region = _crop(region, p, zs).astype(np.uint8)
        if not np.isscalar(p.tau_ad):
            q.tau_ad = _crop(p.tau_ad, p, zs)
        if p.porosity is not None:
            q.porosity = _crop(p.porosity, p, zs)
        q.name = f"{p.name}_zslab{i}"
        q.notes = {}
        parts.append(Slab(i, z0, z1, lo, hi, q))
    return parts


def interior_outlet(slab: Slab) -> np.ndarray:
    """The slab's x = nx-1 plane restricted to its interior z planes (the probe)."""
    q = slab.problem
    m = np.zeros((q.nz, q.ny, q.nx), np.uint8)
    m[slab.first:slab.last + 1, :, q.nx - 1] = 1
    return m.reshape(-1)


def _neighbours(n: int, index: int, ring: bool):
    """(slab below, slab above), None where the chain ends."""
    below = index - 1 if index > 0 else (n - 1 if ring else None)
    above = index + 1 if index < n - 1 else (0 if ring else None)
    return below, above


class SlabRun:
    """All slabs of `problem` on the current GPU, stepped in turn on one stream."""

    def __init__(self, problem: Problem, nslabs: int, precision="f32"):
        import torch

        self.problem = problem
        self.ring = bool(problem.periodic[2])
        self.slabs = split(problem, nslabs)
        self.stream = torch.cuda.Stream()
        self.lats = []
        for s in self.slabs:
            L = _lattice.from_problem(s.problem, precision, stream=self.stream.cuda_stream, probe=False)
            if problem.sample_every > 0:
                L.set_outlet_probe(interior_outlet(s), problem.sample_every)
            self.lats.append(L)
        nbytes = 26 * problem.nx * problem.ny * ELEMENT_BYTES[precision]
        self.buf = torch.empty(nbytes, dtype=torch.uint8, device="cuda")

    def _move(self, src, zs, dst, zd):
        check(src._lib.fm_pack_zplane(src.h, zs, self.buf.data_ptr()))
        check(dst._lib.fm_unpack_zplane(dst.h, zd, self.buf.data_ptr()))

    def exchange(self):
        n = len(self.slabs)
        for i, (s, L) in enumerate(zip(self.slabs, self.lats)):
            below, above = _neighbours(n, i, self.ring)
            if above is not None:                      # my last interior plane -> the low ghost above
                self._move(L, s.last, self.lats[above], 0)
            if below is not None:                      # my first interior plane -> the high ghost below
                b = self.slabs[below]
                self._move(L, s.first, self.lats[below], b.nz_local - 1)

    def step(self, nsteps=1):
        for _ in range(nsteps):
            for L in self.lats:
                L.step(1)
            self.exchange()

    def fields(self):
        """The unsplit lattice's fields, assembled from the slabs' interior planes."""
        p = self.problem
        out = {}
        for k in ("rho", "ux", "uy", "uz", "phi", "q"):
            parts = []
            for s, L in zip(self.slabs, self.lats):
                parts.append(L.field(k).reshape(s.nz_local, p.ny, p.nx)[s.first:s.last + 1])
            out[k] = np.ascontiguousarray(np.concatenate(parts, axis=0)).reshape(-1)
        return out

    def breakthrough(self):
        """C_out(t): the slabs' outlet means weighted by their interior outlet cells."""
        series = [L.breakthrough() for L in self.lats]
        counts = np.array([(s.z1 - s.z0) * self.problem.ny for s in self.slabs], dtype=np.float64)
        return sum(c * b for c, b in zip(counts, series)) / counts.sum()

    def close(self):
        for L in self.lats:
            L.close()
        self.lats = []


class SlabRank:
    """One slab per process.  `pack(z, tensor)` / `unpack(z, tensor)` move one
    plane between the slab and a flat buffer; the exchange pairs them with
    point-to-point sends to the neighbouring ranks (a ring when z is periodic)."""

    def __init__(self, slab: Slab, rank: int, world: int, ring: bool, pack, unpack, make_buffer):
        self.slab, self.rank, self.world = slab, rank, world
        self.below, self.above = _neighbours(world, rank, ring)
        self.pack, self.unpack = pack, unpack
        self.send_lo, self.recv_lo = make_buffer(), make_buffer()
        self.send_hi, self.recv_hi = make_buffer(), make_buffer()

    def exchange(self):
        s = self.slab
        if self.world == 1:                            # a ring of one: the slab is its own neighbour
            if self.above is not None:
                self.pack(s.last, self.send_hi)
                self.unpack(0, self.send_hi)
                self.pack(s.first, self.send_lo)
                self.unpack(s.nz_local - 1, self.send_lo)
            return
        import torch.distributed as dist

        # Point-to-point operations between one pair of ranks match in the
        # order they are queued.  With two ranks on a ring the slab below and
        # the slab above are the same peer, so the order is fixed on both
        # sides: every rank sends its last plane (to the slab above) before
        # its first plane (to the slab below), and receives its low ghost
        # (from the slab below) before its high ghost (from the slab above).
        # The k-th send of one rank then meets the k-th receive of its peer.
        if self.below is not None:
            self.pack(s.first, self.send_lo)
        if self.above is not None:
            self.pack(s.last, self.send_hi)
        ops = []
        if self.above is not None:
            ops.append(dist.P2POp(dist.isend, self.send_hi, self.above))
        if self.below is not None:
            ops.append(dist.P2POp(dist.isend, self.send_lo, self.below))
        if self.below is not None:
            ops.append(dist.P2POp(dist.irecv, self.recv_lo, self.below))
        if self.above is not None:
            ops.append(dist.P2POp(dist.irecv, self.recv_hi, self.above))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if self.below is not None:
            self.unpack(0, self.recv_lo)
        if self.above is not None:
            self.unpack(s.nz_local - 1, self.recv_hi)


def lattice_rank(problem: Problem, rank: int, world: int, precision="f32", *, stream):
    """This rank's slab lattice and its :class:`SlabRank` (device buffers).

    `stream` (a raw ``cudaStream_t`` value) must be torch's current stream:
    ``torch.distributed`` orders its sends and receives against that stream
    only, and the lattice queues its steps, ``fm_pack_zplane`` and
    ``fm_unpack_zplane`` on the stream it is given.  On any other stream a send
    could read the buffer before the pack has finished, or an unpack could run
    before the receive has landed."""
    import torch

    if stream is None or int(stream) != int(torch.cuda.current_stream().cuda_stream):
        raise ValueError("lattice_rank: stream must be torch.cuda.current_stream().cuda_stream")
    slab = split(problem, world)[rank]
    L = _lattice.from_problem(slab.problem, precision, stream=stream, probe=False)
    if problem.sample_every > 0:
        L.set_outlet_probe(interior_outlet(slab), problem.sample_every)
    nbytes = 26 * problem.nx * problem.ny * ELEMENT_BYTES[precision]

    def pack(z, t):
        check(L._lib.fm_pack_zplane(L.h, z, t.data_ptr()))

    def unpack(z, t):
        check(L._lib.fm_unpack_zplane(L.h, z, t.data_ptr()))

    return L, SlabRank(slab, rank, world, bool(problem.periodic[2]), pack, unpack,
                       lambda: torch.empty(nbytes, dtype=torch.uint8, device="cuda"))
