"""x-slab decomposition of one coupled lattice.

The flow axis x is cut into slabs.  Each slab is an ordinary lattice holding
its cells plus one ghost plane per inner face; the first slab keeps the inlet
boundaries, the last keeps the outlet boundaries and the outlet probe.  A step
is the fused step on every slab, then the halo exchange: each slab sends the
stored populations (19 + 7 directions) of the plane next to an inner face into
the neighbour's ghost plane (``fm_pack_xplane`` / ``fm_unpack_xplane``).  Every
interior cell then pulls exactly what it pulls in the unsplit lattice, so the
slabs reproduce the unsplit run bit for bit; the ghost cells' own updates are
discarded by the exchange.

:class:`SlabRun` runs all slabs of a problem in one process on one GPU (the
slabs step one after another on one stream; the exchange is host-ordered, no
kernel waits for another).  :class:`SlabRank` is one slab per process with the
exchange over ``torch.distributed`` (NCCL on GPUs); its packing and transport
are separable so the exchange pattern runs on CPU ranks too.
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
    x0: int            # first interior x of this slab (global)
    x1: int            # one past the last interior x (global)
    lo: int            # ghost planes below x0 (0 for the first slab)
    hi: int            # ghost planes above x1 - 1 (0 for the last slab)
    problem: Problem   # the slab's own lattice problem (ghosts included)

    @property
    def nx_local(self) -> int:
        return self.x1 - self.x0 + self.lo + self.hi


def _crop(a, p: Problem, xa: int, xb: int):
    return np.ascontiguousarray(np.asarray(a).reshape(p.nz, p.ny, p.nx)[:, :, xa:xb]).reshape(-1)


def split(problem: Problem, nslabs: int) -> list:
    """Cut `problem` into `nslabs` x-slabs of near-equal width (at least 2 planes each)."""
    p = problem
    if p.periodic[0]:
        raise ValueError("split: periodic x has no slab ends")
    if nslabs < 1 or p.nx < 2 * nslabs:
        raise ValueError("split: each slab needs at least 2 planes")
    if p.inlet is not None or p.outlet is not None:
        raise ValueError("split: custom inlet / outlet masks are not split; use the x = 0 / x = nx-1 planes")
    edges = [round(i * p.nx / nslabs) for i in range(nslabs + 1)]
    region = p.solid if p.region is None else p.region
    slabs = []
    for i in range(nslabs):
        x0, x1 = edges[i], edges[i + 1]
        lo, hi = int(i > 0), int(i < nslabs - 1)
        xa, xb = x0 - lo, x1 + hi
        q = dataclasses.replace(p)
        q.nx = xb - xa
        q.solid = _crop(p.solid, p, xa, xb).astype(np.uint8)
        q.region = _crop(region, p, xa, xb).astype(np.uint8)
        if not np.isscalar(p.tau_ad):
            q.tau_ad = _crop(p.tau_ad, p, xa, xb)
        if p.porosity is not None:
            q.porosity = _crop(p.porosity, p, xa, xb)
        if i > 0:
            q.ns_inlet, q.ad_inlet = "none", "none"
        if i < nslabs - 1:
            q.ns_outlet, q.ad_outlet = "none", "none"
            q.sample_every = 0
        q.name = f"{p.name}_slab{i}"
        q.notes = {}
        slabs.append(Slab(i, x0, x1, lo, hi, q))
    return slabs


class SlabRun:
    """All slabs of `problem` on the current GPU, stepped in turn on one stream."""

    def __init__(self, problem: Problem, nslabs: int, precision="f32"):
        import torch

        self.problem = problem
        self.slabs = split(problem, nslabs)
        self.stream = torch.cuda.Stream()
        self.lats = [_lattice.from_problem(s.problem, precision, stream=self.stream.cuda_stream) for s in self.slabs]
        rows = problem.ny * problem.nz
        nbytes = 26 * rows * ELEMENT_BYTES[precision]
        self.buf = torch.empty(nbytes, dtype=torch.uint8, device="cuda")

    def _move(self, src, xs, dst, xd):
        check(src._lib.fm_pack_xplane(src.h, xs, self.buf.data_ptr()))
        check(dst._lib.fm_unpack_xplane(dst.h, xd, self.buf.data_ptr()))

    def exchange(self):
        for r in range(len(self.slabs) - 1):
            a, b = self.slabs[r], self.slabs[r + 1]
            La, Lb = self.lats[r], self.lats[r + 1]
            self._move(La, a.nx_local - 2, Lb, 0)          # a's last interior plane -> b's low ghost
            self._move(Lb, 1, La, a.nx_local - 1)          # b's first interior plane -> a's high ghost

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
                a = L.field(k).reshape(p.nz, p.ny, s.nx_local)
                parts.append(a[:, :, s.lo:s.lo + (s.x1 - s.x0)])
            out[k] = np.ascontiguousarray(np.concatenate(parts, axis=2)).reshape(-1)
        return out

    def breakthrough(self):
        return self.lats[-1].breakthrough()

    def close(self):
        for L in self.lats:
            L.close()
        self.lats = []


class SlabRank:
    """One slab per process.  `pack(x, tensor)` / `unpack(x, tensor)` move one
    plane between the slab and a flat buffer; the exchange pairs them with
    point-to-point sends to the neighbouring ranks."""

    def __init__(self, slab: Slab, rank: int, world: int, pack, unpack, make_buffer):
        self.slab, self.rank, self.world = slab, rank, world
        self.pack, self.unpack = pack, unpack
        self.send_lo, self.recv_lo = make_buffer(), make_buffer()
        self.send_hi, self.recv_hi = make_buffer(), make_buffer()

    def exchange(self):
        import torch.distributed as dist

        s, ops = self.slab, []
        if self.rank > 0:
            self.pack(s.lo, self.send_lo)                   # first interior plane
            ops += [dist.P2POp(dist.isend, self.send_lo, self.rank - 1),
                    dist.P2POp(dist.irecv, self.recv_lo, self.rank - 1)]
        if self.rank < self.world - 1:
            self.pack(s.nx_local - 2, self.send_hi)         # last interior plane
            ops += [dist.P2POp(dist.isend, self.send_hi, self.rank + 1),
                    dist.P2POp(dist.irecv, self.recv_hi, self.rank + 1)]
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if self.rank > 0:
            self.unpack(0, self.recv_lo)
        if self.rank < self.world - 1:
            self.unpack(s.nx_local - 1, self.recv_hi)


def lattice_rank(problem: Problem, rank: int, world: int, precision="f32", stream=None):
    """This rank's slab lattice and its :class:`SlabRank` (device buffers, NCCL)."""
    import torch

    slab = split(problem, world)[rank]
    L = _lattice.from_problem(slab.problem, precision, stream=stream)
    nbytes = 26 * problem.ny * problem.nz * ELEMENT_BYTES[precision]

    def pack(x, t):
        check(L._lib.fm_pack_xplane(L.h, x, t.data_ptr()))

    def unpack(x, t):
        check(L._lib.fm_unpack_xplane(L.h, x, t.data_ptr()))

    return L, SlabRank(slab, rank, world, pack, unpack,
                       lambda: torch.empty(nbytes, dtype=torch.uint8, device="cuda"))
