"""z-slab decomposition of one coupled lattice.

The slowest axis z is cut into slabs.  Each slab is an ordinary lattice holding
its cells (every x and y) plus one ghost plane per inner face; with periodic z
the first and last slabs are neighbours too (a ring).  Every slab keeps its
share of the x = 0 inlet and x = nx-1 outlet planes, so the fused boundary
planes work in each slab unchanged.

A step of a slab is split so that its halo travels while its interior updates
(``fm_step_planes`` / ``fm_step_finish``):

1. the fused step on the slab's first and last interior planes;
2. the halo of those planes is packed -- only the populations that cross a
   z-face, 5 D3Q19 + 1 D3Q7 of the 26 (``fm_pack_zhalo``): the c_z = +1 ones of
   the last plane for the slab above, the c_z = -1 ones of the first plane for
   the slab below -- and sent;
3. the fused step on the remaining interior planes, while the halo is in flight;
4. the received halos are unpacked into the ghost planes (``fm_unpack_zhalo``)
   and the step is finished.

Ghost planes are never stepped: interior cells pull from a ghost plane exactly
the populations the halo brings, so the slabs reproduce the unsplit run bit
for bit.  A slab whose step is not one fused launch (list-path boundaries, or
nx * ny not a multiple of 64) steps whole, ghost planes included, and then
receives whole planes -- all 26 populations (``fm_pack_zplane``): a boundary
kernel that runs before the next collision, such as the NEQ velocity inlet on
its list path, rewrites a ghost cell from its neighbours in the ghost plane,
so every population of that plane must be the neighbour slab's.  The outlet mean C_out is the cell-weighted mean of the slabs' outlet
means over their interior rows; the domain sums add the slabs' interior sums
(``fm_reduce_zrange``).

:class:`SlabRun` runs all slabs of a problem in one process on one GPU (the
slabs' parts run one after another on one stream, and the halos move between
them in host order; no kernel waits for another).  :class:`SlabRank` is one
slab per process with the halos over ``torch.distributed`` point-to-point
(NCCL on GPUs); it drives its slab through a small adapter (``pack``,
``unpack``, ``step_planes``, ``finish``, ``make_buffer``), so the same
exchange also runs on CPU ranks in the tests.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import lattice as _lattice
from ._abi import check
from .problems import Problem

ELEMENT_BYTES = {"f32": 4, "f64": 8, "f16": 2, "bf16": 2, "f16q": 2}
HALO_POPULATIONS = 6    # per plane cell: the 5 D3Q19 and 1 D3Q7 populations crossing a z-face
PLANE_POPULATIONS = 26  # per plane cell: every population (the whole-step fallback)


def halo_bytes(L, precision) -> int:
    """Bytes of one halo message of slab lattice `L`: the crossing populations
    of a plane with split steps, the whole plane otherwise."""
    nx, ny, _ = L.shape
    pops = HALO_POPULATIONS if split_capable(L) else PLANE_POPULATIONS
    return pops * nx * ny * ELEMENT_BYTES[precision]


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


def split_capable(L) -> bool:
    """A slab lattice can step its planes in parts (fm_step_planes) when its
    step is one launch and nx * ny is a multiple of 64; otherwise it steps
    whole (ghost planes included, their updates unread) and the halo moves
    after the step."""
    nx, ny, _ = L.shape
    return L.launches_per_step() == 1 and (nx * ny) % 64 == 0


def _neighbours(n: int, index: int, ring: bool):
    """(slab below, slab above), None where the chain ends."""
    below = index - 1 if index > 0 else (n - 1 if ring else None)
    above = index + 1 if index < n - 1 else (0 if ring else None)
    return below, above


class SlabRun:
    """All slabs of `problem` on the current GPU, their parts run in turn on one stream."""

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
        self.split = all(split_capable(L) for L in self.lats)
        nbytes = max(halo_bytes(L, precision) for L in self.lats)
        self.buf = torch.empty(nbytes, dtype=torch.uint8, device="cuda")

    def _move(self, src, zs, dst, zd, direction):
        if self.split:
            check(src._lib.fm_pack_zhalo(src.h, zs, direction, self.buf.data_ptr()))
            check(dst._lib.fm_unpack_zhalo(dst.h, zd, direction, self.buf.data_ptr()))
        else:
            check(src._lib.fm_pack_zplane(src.h, zs, self.buf.data_ptr()))
            check(dst._lib.fm_unpack_zplane(dst.h, zd, self.buf.data_ptr()))

    @property
    def split_steps(self):
        """Whether the slabs step their interior planes only (see split_capable)."""
        return self.split

    def step(self, nsteps=1):
        n = len(self.slabs)
        split = self.split
        for _ in range(nsteps):
            for s, L in zip(self.slabs, self.lats):
                if split:
                    check(L._lib.fm_step_planes(L.h, s.first, s.last + 1))
                else:
                    L.step(1)
            for i, (s, L) in enumerate(zip(self.slabs, self.lats)):
                below, above = _neighbours(n, i, self.ring)
                if above is not None:      # my last plane's c_z = +1 populations -> the low ghost above
                    self._move(L, s.last, self.lats[above], 0, +1)
                if below is not None:      # my first plane's c_z = -1 populations -> the high ghost below
                    self._move(L, s.first, self.lats[below], self.slabs[below].nz_local - 1, -1)
            if split:
                for L in self.lats:
                    check(L._lib.fm_step_finish(L.h))

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

    def reduce(self):
        """Sums of rho, C and q over the unsplit lattice (the slabs' interiors)."""
        tot = np.zeros(3)
        for s, L in zip(self.slabs, self.lats):
            out = np.empty(3)
            check(L._lib.fm_reduce_zrange(L.h, s.first, s.last + 1, out.ctypes.data))
            tot += out
        return tot

    def close(self):
        for L in self.lats:
            L.close()
        self.lats = []


class SlabRank:
    """One slab per process.  `io` drives the slab: ``pack(z, dir, buf)`` /
    ``unpack(z, dir, buf)`` move the crossing populations of plane z (dir +1:
    c_z = +1, dir -1: c_z = -1) between the slab and a flat buffer; with
    ``io.split`` true, ``step_planes(z0, z1)`` runs the fused step on planes
    [z0, z1) and ``finish()`` completes the step, else ``step_all()`` steps
    the whole slab; ``make_buffer()`` gives a buffer.  The
    halos go to the neighbouring ranks (a ring when z is periodic) by
    point-to-point operations."""

    def __init__(self, slab: Slab, rank: int, world: int, ring: bool, io):
        self.slab, self.rank, self.world, self.io = slab, rank, world, io
        self.below, self.above = _neighbours(world, rank, ring)
        self.send_lo, self.recv_lo = io.make_buffer(), io.make_buffer()
        self.send_hi, self.recv_hi = io.make_buffer(), io.make_buffer()

    def step(self):
        """One time step of the slab.  With split steps (``io.split``) the halo
        exchange overlaps the interior update; otherwise the slab steps whole
        and the halo moves after it."""
        s, io = self.slab, self.io
        if io.split:
            io.step_planes(s.first, s.first + 1)
            if s.last > s.first:
                io.step_planes(s.last, s.last + 1)
        else:
            io.step_all()
        if self.below is not None:
            io.pack(s.first, -1, self.send_lo)
        if self.above is not None:
            io.pack(s.last, +1, self.send_hi)
        reqs = self._start()
        if io.split and s.last - s.first > 1:
            io.step_planes(s.first + 1, s.last)      # the interior, while the halos travel
        for req in reqs:
            req.wait()
        if self.world == 1:
            if self.above is not None:             # a ring of one: the slab is its own neighbour
                io.unpack(0, +1, self.send_hi)
                io.unpack(s.nz_local - 1, -1, self.send_lo)
        else:
            if self.below is not None:
                io.unpack(0, +1, self.recv_lo)
            if self.above is not None:
                io.unpack(s.nz_local - 1, -1, self.recv_hi)
        if io.split:
            io.finish()

    def _start(self):
        if self.world == 1:
            return []
        import torch.distributed as dist

        # Point-to-point operations between one pair of ranks match in the
        # order they are queued.  With two ranks on a ring the slab below and
        # the slab above are the same peer, so the order is fixed on both
        # sides: every rank sends its last plane's halo (to the slab above)
        # before its first plane's (to the slab below), and receives its low
        # ghost (from the slab below) before its high ghost (from the slab
        # above).  The k-th send of one rank then meets the k-th receive of
        # its peer.
        ops = []
        if self.above is not None:
            ops.append(dist.P2POp(dist.isend, self.send_hi, self.above))
        if self.below is not None:
            ops.append(dist.P2POp(dist.isend, self.send_lo, self.below))
        if self.below is not None:
            ops.append(dist.P2POp(dist.irecv, self.recv_lo, self.below))
        if self.above is not None:
            ops.append(dist.P2POp(dist.irecv, self.recv_hi, self.above))
        return dist.batch_isend_irecv(ops) if ops else []

    def breakthrough(self, series, device=None):
        """The whole lattice's C_out(t) from this rank's outlet series: the
        interior-row-weighted mean over all ranks (one all-reduce, FP64)."""
        import torch
        import torch.distributed as dist

        rows = float((self.slab.z1 - self.slab.z0))
        t = torch.tensor(np.concatenate([[rows], rows * np.asarray(series, dtype=np.float64)]), dtype=torch.float64,
                         device=device)
        if self.world > 1:
            dist.all_reduce(t)
        t = t.cpu().numpy()
        return t[1:] / t[0]

    def reduce(self, sums, device=None):
        """The whole lattice's sums of rho, C and q from this rank's interior sums."""
        import torch
        import torch.distributed as dist

        t = torch.tensor(np.asarray(sums, dtype=np.float64), device=device)
        if self.world > 1:
            dist.all_reduce(t)
        return t.cpu().numpy()


class LatticeIO:
    """The adapter of :class:`SlabRank` for a slab lattice on this rank's GPU:
    halos of the crossing populations with split steps, whole planes when the
    slab steps whole (see :func:`halo_bytes`)."""

    def __init__(self, L, precision):
        self.L = L
        self.split = split_capable(L)
        self.nbytes = halo_bytes(L, precision)

    def step_all(self):
        self.L.step(1)

    def pack(self, z, direction, t):
        if self.split:
            check(self.L._lib.fm_pack_zhalo(self.L.h, z, direction, t.data_ptr()))
        else:
            check(self.L._lib.fm_pack_zplane(self.L.h, z, t.data_ptr()))

    def unpack(self, z, direction, t):
        if self.split:
            check(self.L._lib.fm_unpack_zhalo(self.L.h, z, direction, t.data_ptr()))
        else:
            check(self.L._lib.fm_unpack_zplane(self.L.h, z, t.data_ptr()))

    def step_planes(self, z0, z1):
        check(self.L._lib.fm_step_planes(self.L.h, z0, z1))

    def finish(self):
        check(self.L._lib.fm_step_finish(self.L.h))

    def make_buffer(self):
        import torch

        return torch.empty(self.nbytes, dtype=torch.uint8, device="cuda")


def lattice_rank(problem: Problem, rank: int, world: int, precision="f32", *, stream):
    """This rank's slab lattice and its :class:`SlabRank` (device buffers).

    `stream` (a raw ``cudaStream_t`` value) must be torch's current stream:
    ``torch.distributed`` orders its sends and receives against that stream
    only, and the lattice queues its steps, ``fm_pack_zhalo`` and
    ``fm_unpack_zhalo`` on the stream it is given.  On any other stream a send
    could read the buffer before the pack has finished, or an unpack could run
    before the receive has landed."""
    import torch

    if stream is None or int(stream) != int(torch.cuda.current_stream().cuda_stream):
        raise ValueError("lattice_rank: stream must be torch.cuda.current_stream().cuda_stream")
    slab = split(problem, world)[rank]
    L = _lattice.from_problem(slab.problem, precision, stream=stream, probe=False)
    if problem.sample_every > 0:
        L.set_outlet_probe(interior_outlet(slab), problem.sample_every)
    return L, SlabRank(slab, rank, world, bool(problem.periodic[2]), LatticeIO(L, precision))
