"""Python host binding of the coupled lattice (thin wrapper over ``include/fm.h``).

:class:`CoupledLattice` owns one ``fm_lattice``: the reference's
``Lattice<D3Q19>`` + ``ADLattice<D3Q7>`` + ``AdsorbedField`` with their
operators and boundary conditions.  Method names follow the reference classes
(``set_obstacle_mask`` <-> ``Lattice::setObstacleMask`` ...); every error is an
:class:`~fluidmaxxer_b200._abi.FmError` at the point the reference throws.

:func:`from_problem` performs the set-up of ``src/main.cpp:101-303`` for a
:class:`~fluidmaxxer_b200.problems.Problem`.
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _abi
from ._abi import check

PRECISIONS = {"f32": _abi.FM_F32, "f16": _abi.FM_F16_SHIFTED, "bf16": _abi.FM_BF16_SHIFTED, "f64": _abi.FM_F64,
              "f16q": _abi.FM_F16_FIXED_AD}


def _u8(a, n):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    if a.size != n:
        raise ValueError("mask size mismatch")
    return a


def _f64(a, n):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.size != n:
        raise ValueError("field size mismatch")
    return a


class CoupledLattice:
    def __init__(self, nx, ny, nz, rho0=1.0, tau=0.8, tau_ad=0.7, phi0=0.0, min_concentration=1e-8,
                 periodic=(False, True, True), precision="f32", stream=None):
        self._lib = _abi.lib()
        p = _abi.FmParams(nx, ny, nz, rho0, tau, tau_ad, phi0, min_concentration,
                          int(periodic[0]), int(periodic[1]), int(periodic[2]))
        h = C.c_void_p()
        check(self._lib.fm_lattice_create(C.byref(p), PRECISIONS[precision], stream, C.byref(h)))
        self.h = h
        self.shape = (nx, ny, nz)
        self.n = nx * ny * nz
        self.precision = precision

    # -- lifetime ------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            # a batch holding this lattice goes first (the C ABI destroys
            # batches before their lattices; the garbage collector may finalise
            # a lattice before the batch that refers to it)
            for B in list(getattr(self, "_batches", ())):
                B.close()
            self._lib.fm_lattice_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- geometry / fields ---------------------------------------------------
    def set_obstacle_mask(self, mask):
        m = _u8(mask, self.n)
        check(self._lib.fm_set_obstacle_mask(self.h, m.ctypes.data, m.size))

    def set_obstacle_bits(self, bits):
        b = np.ascontiguousarray(bits, dtype=np.uint32)
        check(self._lib.fm_set_obstacle_bits(self.h, b.ctypes.data, b.size))

    def set_porosity_from_mask(self, mask, phi_masked, phi_else):
        m = _u8(mask, self.n)
        check(self._lib.fm_set_porosity_from_mask(self.h, m.ctypes.data, m.size, phi_masked, phi_else))

    def set_porosity(self, porosity):
        a = _f64(porosity, self.n)
        check(self._lib.fm_set_porosity(self.h, a.ctypes.data, a.size))

    def set_tau_field(self, tau):
        a = _f64(tau, self.n)
        check(self._lib.fm_set_tau_field(self.h, a.ctypes.data, a.size))

    # -- operators -------------------------------------------------------------
    def set_collision(self, kind):
        check(self._lib.fm_set_collision(self.h, {"bgk": _abi.FM_COLL_BGK, "porous": _abi.FM_COLL_POROUS}[kind]))

    def set_coupling(self, enabled=True):
        check(self._lib.fm_set_coupling(self.h, int(bool(enabled))))

    def set_isotherm_linear(self, region, k_henry, k_ldf):
        m = _u8(region, self.n)
        check(self._lib.fm_set_isotherm_linear(self.h, m.ctypes.data, m.size, k_henry, k_ldf))

    def set_isotherm_langmuir(self, region, q_max, b, k_ldf):
        m = _u8(region, self.n)
        check(self._lib.fm_set_isotherm_langmuir(self.h, m.ctypes.data, m.size, q_max, b, k_ldf))

    def clear_isotherm(self):
        check(self._lib.fm_clear_isotherm(self.h))

    # -- boundaries ------------------------------------------------------------
    def add_ns_velocity_eq(self, mask, ux, uy=0.0, uz=0.0):
        m = _u8(mask, self.n)
        check(self._lib.fm_add_ns_velocity_eq(self.h, m.ctypes.data, m.size, ux, uy, uz))

    def add_ns_velocity_neq(self, mask, ux, uy=0.0, uz=0.0):
        m = _u8(mask, self.n)
        check(self._lib.fm_add_ns_velocity_neq(self.h, m.ctypes.data, m.size, ux, uy, uz))

    def add_ns_pressure(self, mask, rho_out):
        m = _u8(mask, self.n)
        check(self._lib.fm_add_ns_pressure(self.h, m.ctypes.data, m.size, rho_out))

    def add_ns_bounceback(self, mask):
        m = _u8(mask, self.n)
        check(self._lib.fm_add_ns_bounceback(self.h, m.ctypes.data, m.size))

    def add_ad_dirichlet(self, mask, phi):
        m = _u8(mask, self.n)
        check(self._lib.fm_add_ad_dirichlet(self.h, m.ctypes.data, m.size, phi))

    def add_ad_tanh_pulse(self, mask, phi_base, phi_amp, t_on, t_off, k):
        m = _u8(mask, self.n)
        check(self._lib.fm_add_ad_tanh_pulse(self.h, m.ctypes.data, m.size, phi_base, phi_amp, int(t_on), int(t_off), k))

    def add_ad_neumann(self, mask):
        m = _u8(mask, self.n)
        check(self._lib.fm_add_ad_neumann(self.h, m.ctypes.data, m.size))

    # -- stepping --------------------------------------------------------------
    def init_equilibrium(self):
        check(self._lib.fm_init_equilibrium(self.h))

    def step(self, nsteps=1):
        check(self._lib.fm_step(self.h, int(nsteps)))

    def synchronize(self):
        check(self._lib.fm_synchronize(self.h))

    @property
    def step_count(self):
        return int(self._lib.fm_step_count(self.h))

    # -- outputs ---------------------------------------------------------------
    def field(self, name, out=None, dtype=np.float64):
        """One field as `dtype` (float64, or float32 through ``fm_get_field_f32``) [n];
        `out` (optional, contiguous [n] of that dtype, e.g. page-locked) receives it
        without a new allocation."""
        code = {"rho": _abi.FM_FIELD_RHO, "ux": _abi.FM_FIELD_UX, "uy": _abi.FM_FIELD_UY,
                "uz": _abi.FM_FIELD_UZ, "C": _abi.FM_FIELD_C, "phi": _abi.FM_FIELD_C, "q": _abi.FM_FIELD_Q}[name]
        dtype = np.dtype(dtype)
        if dtype not in (np.float64, np.float32):
            raise ValueError("field: dtype float64 or float32")
        if out is None:
            out = np.empty(self.n, dtype=dtype)
        elif out.dtype != dtype or out.size != self.n or not out.flags.c_contiguous:
            raise ValueError(f"field: out must be a contiguous {dtype} array of n values")
        fn = self._lib.fm_get_field if dtype == np.float64 else self._lib.fm_get_field_f32
        check(fn(self.h, code, out.ctypes.data, out.size))
        return out

    def fields(self, out=None, dtype=np.float64):
        """rho, ux, uy, uz, phi, q in one call (``fm_get_fields`` / ``fm_get_fields_f32``);
        `out` (optional) maps names to contiguous arrays of `dtype` [n] to fill."""
        names = ("rho", "ux", "uy", "uz", "phi", "q")
        dtype = np.dtype(dtype)
        if dtype not in (np.float64, np.float32):
            raise ValueError("fields: dtype float64 or float32")
        res = {}
        for k in names:
            a = np.empty(self.n, dtype=dtype) if out is None else out[k]
            if a.dtype != dtype or a.size != self.n or not a.flags.c_contiguous:
                raise ValueError(f"fields: out[{k!r}] must be a contiguous {dtype} array of n values")
            res[k] = a
        ptrs = (C.c_void_p * 6)(*[res[k].ctypes.data for k in names])
        fn = self._lib.fm_get_fields if dtype == np.float64 else self._lib.fm_get_fields_f32
        check(fn(self.h, ptrs, self.n))
        return res

    def set_outlet_probe(self, mask, every):
        m = _u8(mask, self.n)
        check(self._lib.fm_set_outlet_probe(self.h, m.ctypes.data, m.size, int(every)))

    def breakthrough(self):
        cnt = C.c_int(0)
        check(self._lib.fm_get_breakthrough(self.h, None, 0, C.byref(cnt)))
        out = np.empty(max(cnt.value, 1))
        check(self._lib.fm_get_breakthrough(self.h, out.ctypes.data, out.size, C.byref(cnt)))
        return out[: cnt.value]

    def outlet_stats(self):
        """(mean, min, max) of C over the outlet probe cells, reduced on the device."""
        out = np.empty(3)
        check(self._lib.fm_outlet_stats(self.h, out.ctypes.data))
        return tuple(out)

    def reduce(self):
        out = np.empty(4)
        check(self._lib.fm_reduce(self.h, out.ctypes.data))
        return out

    def get_state(self):
        f = np.empty(19 * self.n); g = np.empty(7 * self.n); phi = np.empty(self.n); q = np.empty(self.n)
        check(self._lib.fm_get_state(self.h, f.ctypes.data, g.ctypes.data, phi.ctypes.data, q.ctypes.data))
        return dict(f=f.reshape(19, self.n), g=g.reshape(7, self.n), phi=phi, q=q)

    def set_state(self, f=None, g=None, phi=None, q=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (f, g, phi, q)]
        check(self._lib.fm_set_state(self.h, *[None if a is None else a.ctypes.data for a in arrs]))

    def profile_enable(self, enabled=True):
        check(self._lib.fm_profile_enable(self.h, int(bool(enabled))))

    def profile_read(self):
        ms = C.c_double(0.0)
        cnt = C.c_longlong(0)
        check(self._lib.fm_profile_read(self.h, C.byref(ms), C.byref(cnt)))
        return ms.value, cnt.value

    def bench_pull_copy(self, reps=20):
        """(ms per launch, bytes per launch) of the pure pull-copy of the step's
        access pattern (fm_bench_pull_copy); overwrites the write buffers only."""
        ms, nb = C.c_double(0.0), C.c_double(0.0)
        check(self._lib.fm_bench_pull_copy(self.h, int(reps), C.byref(ms), C.byref(nb)))
        return ms.value, nb.value

    def set_monitor(self, every):
        """Monitor every `every`-th step inside the fused kernel (``fm_set_monitor``; 0 = off)."""
        check(self._lib.fm_set_monitor(self.h, int(every)))

    def monitor(self):
        """The monitor's rows as a dict of arrays: step, mass, C, q, outlet_flux, bad_cells."""
        cnt = C.c_int(0)
        check(self._lib.fm_get_monitor(self.h, None, 0, C.byref(cnt)))
        out = np.empty((max(cnt.value, 1), 6))
        check(self._lib.fm_get_monitor(self.h, out.ctypes.data, out.shape[0], C.byref(cnt)))
        out = out[: cnt.value]
        return {k: out[:, i] for i, k in enumerate(("step", "mass", "C", "q", "outlet_flux", "bad_cells"))}

    def set_pair_layout(self, enabled=True):
        """Allow or forbid (the default) the pair layout of the 16-bit forms (``fm_set_pair_layout``)."""
        check(self._lib.fm_set_pair_layout(self.h, int(bool(enabled))))

    def storage_layout(self):
        """'pair' or 'natural': the population layout the next step runs on."""
        rc = int(self._lib.fm_storage_layout(self.h))
        if rc < 0:
            check(rc)
        return "pair" if rc == 1 else "natural"

    def set_pair_kernel(self, staged=True):
        """Pair layout: the staged kernel where it applies (default) or k_coupled_pair (``fm_set_pair_kernel``)."""
        check(self._lib.fm_set_pair_kernel(self.h, int(bool(staged))))

    def step_kernel(self):
        """The kernel the next step runs: 'one-cell', 'pair', 'pair-staged', or
        'one-cell-wide' (the one-cell kernel with unsigned pull offsets, for a
        16-bit lattice too large for signed ones) (``fm_step_kernel``)."""
        rc = int(self._lib.fm_step_kernel(self.h))
        if rc < 0:
            check(rc)
        return ("one-cell", "pair", "pair-staged", "one-cell-wide")[rc]

    def step_status(self):
        """The step kernels' status word since the last call (0: no wait gave up); clears it."""
        st = C.c_int(0)
        check(self._lib.fm_step_status(self.h, C.byref(st)))
        return st.value

    def set_prefetch_distance(self, blocks):
        check(self._lib.fm_set_prefetch_distance(self.h, int(blocks)))

    def launches_per_step(self):
        return int(self._lib.fm_launches_per_step(self.h))

    def adjoint_breakthrough(self, nsteps, target, checkpoint_every=0, max_stored_states=0, porosity_grad=True):
        """Loss sum_i (C_out(s0 + i P) - target[i])^2 over the next `nsteps`
        steps and its gradients by the adjoint kernels (``fm_adjoint_breakthrough``).
        Returns ``(loss, grad_params[3], grad_porosity or None)``; the lattice
        ends `nsteps` further on, its breakthrough series extended."""
        t = np.ascontiguousarray(target, dtype=np.float64).reshape(-1)
        loss = C.c_double(0.0)
        gp = np.zeros(3)
        gpor = np.zeros(self.n) if porosity_grad else None
        check(self._lib.fm_adjoint_breakthrough(
            self.h, int(nsteps), t.ctypes.data if t.size else None, int(t.size), int(checkpoint_every),
            int(max_stored_states), C.byref(loss), gp.ctypes.data, None if gpor is None else gpor.ctypes.data))
        return loss.value, gp, gpor

    def adjoint_stats(self):
        """(forward steps recomputed by the last adjoint call, workspace bytes held)"""
        a, b = C.c_longlong(0), C.c_longlong(0)
        check(self._lib.fm_adjoint_stats(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def adjoint_release(self):
        check(self._lib.fm_adjoint_release(self.h))


def build_tau_field(shape, dx_phys, dt_phys, mask, d_fluid_phys, d_solid_phys):
    """ADUnitConverter<D3Q7>::buildTauField (include/core/io/ADUnitConverter.hpp:63-104):
    the per-cell AD relaxation time, tau(D_solid) where `mask` is set and
    tau(D_fluid) elsewhere, tau = D dt / dx^2 / (1/4) + 1/2 (``fm_build_tau_field``)."""
    nx, ny, nz = shape
    m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    out = np.empty(m.size)
    check(_abi.lib().fm_build_tau_field(int(nx), int(ny), int(nz), float(dx_phys), float(dt_phys), m.ctypes.data,
                                        m.size, float(d_fluid_phys), float(d_solid_phys), out.ctypes.data))
    return out


def from_problem(problem, precision="f32", probe=True, stream=None) -> CoupledLattice:
    """Set up a lattice as src/main.cpp:131-283 does, for `problem`."""
    p = problem
    tau_ad0 = float(p.tau_ad) if np.isscalar(p.tau_ad) else float(np.asarray(p.tau_ad).reshape(-1)[0])
    L = CoupledLattice(p.nx, p.ny, p.nz, rho0=p.rho0, tau=p.tau, tau_ad=tau_ad0, phi0=p.phi0,
                       min_concentration=p.min_conc, periodic=p.periodic, precision=precision, stream=stream)
    solid, region, inlet, outlet = p.masks()
    L.set_collision(p.collision)
    L.set_obstacle_mask(solid)
    if p.collision == "porous":
        L.set_porosity(np.zeros(p.n_cells) if p.porosity is None else p.porosity)
    L.set_coupling(p.coupling)
    if p.ns_inlet == "eq":
        L.add_ns_velocity_eq(inlet, *p.u_in)
    elif p.ns_inlet == "neq":
        L.add_ns_velocity_neq(inlet, *p.u_in)
    if p.ns_outlet == "pressure":
        L.add_ns_pressure(outlet, p.rho_out)
    if p.ns_bounceback:
        L.add_ns_bounceback(solid)
    if not np.isscalar(p.tau_ad):
        L.set_tau_field(p.tau_field())   # a uniform tau_ad is the constructor's
    if p.isotherm == "linear":
        L.set_isotherm_linear(region, p.k_henry, p.k_a)
    elif p.isotherm == "langmuir":
        L.set_isotherm_langmuir(region, p.q_max, p.b_langmuir, p.k_ldf)
    if p.ad_inlet == "dirichlet":
        L.add_ad_dirichlet(inlet, p.c_in)
    elif p.ad_inlet == "pulse":
        pb, pa, pk, pon, poff = p.pulse
        L.add_ad_tanh_pulse(inlet, pb, pa, pon, poff, pk)
    if p.ad_outlet == "neumann":
        L.add_ad_neumann(outlet)
    if probe and p.sample_every > 0:
        L.set_outlet_probe(outlet, p.sample_every)
    L.init_equilibrium()
    return L


def trim_memory(keep_bytes=0):
    """Hand the device memory that closed lattices left in the library's pool
    back to the current device, all but `keep_bytes` of it (fm_trim_memory)."""
    check(_abi.lib().fm_trim_memory(int(keep_bytes)))


def partition_samples(cells, parts):
    """Split samples of the given cell counts into `parts` groups of near-equal
    total cells (largest first, each to the least-loaded group; ties to the
    lower group), for sharding a batch of independent samples across GPUs with
    no exchange between them.  Returns the sample indices of each group, in
    ascending order; deterministic."""
    if parts < 1:
        raise ValueError("partition_samples: parts >= 1")
    groups = [[] for _ in range(parts)]
    load = [0] * parts
    for i in sorted(range(len(cells)), key=lambda j: (-int(cells[j]), j)):
        g = min(range(parts), key=lambda k: (load[k], k))
        groups[g].append(i)
        load[g] += int(cells[i])
    return [sorted(g) for g in groups]


class Batch:
    """Many lattices advanced together by one replayed CUDA graph (fm_batch_*): per
    step one launch over all lattices, or one launch per lattice on forked streams.

    The lattices stay usable on their own (fields, breakthrough, state); the
    batch steps them together, replaying a captured CUDA graph.
    """

    def __init__(self, lattices, stream=None):
        self._lib = _abi.lib()
        self.lattices = list(lattices)
        arr = (C.c_void_p * len(self.lattices))(*[L.h.value for L in self.lattices])
        h = C.c_void_p()
        check(self._lib.fm_batch_create(arr, len(self.lattices), stream, C.byref(h)))
        self.h = h
        for L in self.lattices:
            if not hasattr(L, "_batches"):
                L._batches = weakref.WeakSet()
            L._batches.add(self)

    @property
    def cells(self):
        return int(self._lib.fm_batch_cells(self.h))

    def step(self, nsteps=1):
        check(self._lib.fm_batch_step(self.h, int(nsteps)))

    def synchronize(self):
        check(self._lib.fm_batch_synchronize(self.h))

    def set_config(self, block=256, cells_per_thread=1, prefetch=0, mode=None):
        if mode is None:
            check(self._lib.fm_batch_set_config(self.h, block, cells_per_thread, prefetch))
        else:
            check(self._lib.fm_batch_set_mode(self.h, mode, block, cells_per_thread, prefetch))

    def autotune(self, trial_steps=4):
        m, b, c, p, ms = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_double()
        check(self._lib.fm_batch_autotune(self.h, int(trial_steps), C.byref(m), C.byref(b), C.byref(c), C.byref(p),
                                          C.byref(ms)))
        return {"mode": m.value, "block": b.value, "cells_per_thread": c.value, "prefetch": p.value,
                "ms_per_step": ms.value}

    def close(self):
        if getattr(self, "h", None):
            self._lib.fm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
