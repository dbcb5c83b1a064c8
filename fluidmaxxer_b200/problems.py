"""Problem descriptions for the coupled NS + AD + adsorption step.

A :class:`Problem` holds what the reference's ``main.cpp`` set-up decides
(src/main.cpp:101-303): lattice size and periodicity, the NS collision
operator, boundary conditions, isotherm, relaxation times and the per-cell
masks and fields.  The same object configures the CUDA path
(:mod:`fluidmaxxer_b200.lattice`) and, in tests, the CPU oracle.

The five workloads (lattice units throughout, seeded synthetic geometry):

* :func:`channel_small`   -- 64x32x32 Bernoulli(0.3) channel, linear isotherm, 2000 steps.
* :func:`sphere_pack`     -- 512x256x256 random sphere pack, Langmuir, 10000 steps.
* :func:`sphere_pack_crop`-- 128^3 crop of that pack (precision study).
* :func:`batch_samples`   -- 64 uneven Bernoulli samples with drawn Langmuir parameters.
* :func:`smooth_porous`   -- 128x64x64 continuous solid fraction, porous BGK (adjoint).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

from . import synth

NONE = "none"


def x_plane_mask(nx, ny, nz, x):
    """buildXPlaneMask (include/core/helpers/helpers.hpp:7-14)."""
    m = np.zeros((nz, ny, nx), dtype=np.uint8)
    m[:, :, x] = 1
    return m.reshape(-1)


@dataclasses.dataclass
class Problem:
    nx: int
    ny: int
    nz: int
    solid: np.ndarray                     # uint8 [N], obstacle mask
    periodic: tuple = (False, True, True)
    collision: str = "bgk"                # "bgk" (obstacle bounce-back) | "porous"
    rho0: float = 1.0
    tau: float = 0.8
    tau_ad: object = 0.7                  # scalar or float64 [N]
    phi0: float = 0.0
    min_conc: float = 1e-8
    ns_inlet: str = "neq"                 # "none" | "eq" | "neq"
    u_in: tuple = (0.01, 0.0, 0.0)
    ns_outlet: str = "pressure"           # "none" | "pressure"
    rho_out: float = 1.0
    ns_bounceback: bool = False
    ad_inlet: str = "dirichlet"           # "none" | "dirichlet" | "pulse"
    c_in: float = 1.0
    pulse: tuple = (0.0, 1.0, 10.0, 0, 100)   # base, amp, k, t_on, t_off
    ad_outlet: str = "neumann"            # "none" | "neumann"
    coupling: bool = True
    isotherm: str = "linear"              # "none" | "linear" | "langmuir"
    k_henry: float = 2.0
    k_a: float = 0.01
    q_max: float = 5.0
    b_langmuir: float = 1.5
    k_ldf: float = 0.05
    region: Optional[np.ndarray] = None   # uint8 [N]; None -> solid mask (main.cpp:333)
    inlet: Optional[np.ndarray] = None    # uint8 [N]; None -> x = 0 plane
    outlet: Optional[np.ndarray] = None   # uint8 [N]; None -> x = Nx-1 plane
    porosity: Optional[np.ndarray] = None # float64 [N] for "porous"
    sample_every: int = 20
    steps: int = 2000
    name: str = "custom"
    notes: dict = dataclasses.field(default_factory=dict)

    @property
    def n_cells(self) -> int:
        return self.nx * self.ny * self.nz

    def masks(self):
        """(solid, region, inlet, outlet) as contiguous uint8 [N].  The derived
        x-plane masks are built once per geometry and kept (a 512x256x256 plane
        mask is 33.5 MB)."""
        n = self.n_cells
        key = (self.nx, self.ny, self.nz, id(self.solid), id(self.region), id(self.inlet), id(self.outlet))
        cached = getattr(self, "_masks", None)
        if cached is not None and cached[0] == key:
            return cached[1]
        region = self.solid if self.region is None else self.region
        inlet = x_plane_mask(self.nx, self.ny, self.nz, 0) if self.inlet is None else self.inlet
        outlet = x_plane_mask(self.nx, self.ny, self.nz, self.nx - 1) if self.outlet is None else self.outlet
        for a in (self.solid, region, inlet, outlet):
            if a.shape != (n,):
                raise ValueError("mask size mismatch")
        out = (np.ascontiguousarray(self.solid, np.uint8), np.ascontiguousarray(region, np.uint8),
               np.ascontiguousarray(inlet, np.uint8), np.ascontiguousarray(outlet, np.uint8))
        self._masks = (key, out)
        return out

    def tau_field(self) -> np.ndarray:
        if np.isscalar(self.tau_ad):
            return np.full(self.n_cells, float(self.tau_ad))
        return np.ascontiguousarray(self.tau_ad, dtype=np.float64)

    # -- oracle mapping (tests only) --------------------------------------
    def oracle_config(self) -> dict:
        pb, pa, pk, pon, poff = self.pulse
        return dict(
            nx=self.nx, ny=self.ny, nz=self.nz,
            periodic_x=int(self.periodic[0]), periodic_y=int(self.periodic[1]), periodic_z=int(self.periodic[2]),
            collision={"bgk": 0, "porous": 1}[self.collision],
            rho0=self.rho0, tau=self.tau, phi0=self.phi0, min_conc=self.min_conc,
            ns_inlet={"none": 0, "eq": 1, "neq": 2}[self.ns_inlet], u_in=self.u_in,
            ns_outlet={"none": 0, "pressure": 1}[self.ns_outlet], rho_out=self.rho_out,
            ns_bounceback=int(self.ns_bounceback),
            ad_inlet={"none": 0, "dirichlet": 1, "pulse": 2}[self.ad_inlet], c_in=self.c_in,
            pulse_base=pb, pulse_amp=pa, pulse_k=pk, pulse_on=int(pon), pulse_off=int(poff),
            ad_outlet={"none": 0, "neumann": 1}[self.ad_outlet],
            coupling=int(self.coupling),
            isotherm={"none": 0, "linear": 1, "langmuir": 2}[self.isotherm],
            k_henry=self.k_henry, k_a=self.k_a, q_max=self.q_max, b_langmuir=self.b_langmuir,
            k_ldf=self.k_ldf, sample_every=self.sample_every,
        )

    def oracle_arrays(self) -> dict:
        solid, region, inlet, outlet = self.masks()
        por = None
        if self.collision == "porous":
            por = np.zeros(self.n_cells) if self.porosity is None else np.ascontiguousarray(self.porosity, np.float64)
        return dict(solid=solid, region=region, inlet=inlet, outlet=outlet, porosity=por, tau_ad=self.tau_field())


# ---------------------------------------------------------------------------
# the workloads
# ---------------------------------------------------------------------------

def channel_small(seed: int = 1235, nx=64, ny=32, nz=32, steps=2000) -> Problem:
    """64x32x32 channel: Bernoulli(0.3) solids, x<4 and x>=Nx-4 fluid, solid
    y/z walls, tau 0.8 / 0.7, inlet u = 0.01 and C = 1, linear isotherm
    K_d = 2, k = 0.01, 2000 steps."""
    solid = synth.bernoulli(nx, ny, nz, 0.3, seed, fluid_lo=4, fluid_hi=4, walls=True)
    return Problem(nx=nx, ny=ny, nz=nz, solid=solid, tau=0.8, tau_ad=0.7, u_in=(0.01, 0.0, 0.0),
                   isotherm="linear", k_henry=2.0, k_a=0.01, steps=steps, name=f"channel_{nx}x{ny}x{nz}")


def sphere_pack(seed: int = 1236, nx=512, ny=256, nz=256, steps=10000) -> Problem:
    """512x256x256 random sphere pack (r = 6, RSA to porosity 0.40 or jamming,
    8-voxel fluid buffers, solid y/z walls), Langmuir q_max 5 / K_L 1.5 /
    k 0.05, tau 0.6 / 0.55, inlet u = 0.02 and C = 1, 10000 steps."""
    solid, nsph, por = synth.sphere_pack(nx, ny, nz, 6.0, 0.40, 8, seed, walls=True)
    p = Problem(nx=nx, ny=ny, nz=nz, solid=solid, tau=0.6, tau_ad=0.55, u_in=(0.02, 0.0, 0.0),
                isotherm="langmuir", q_max=5.0, b_langmuir=1.5, k_ldf=0.05, steps=steps,
                name=f"sphere_pack_{nx}x{ny}x{nz}")
    p.notes = {"spheres": nsph, "slab_porosity": por}
    return p


def sphere_pack_crop(seed: int = 1236, edge=128, full=(512, 256, 256), steps=20000) -> Problem:
    """edge^3 crop of the sphere pack (same seed), with its own 8-voxel outlet
    buffer and y/z walls re-applied."""
    nx, ny, nz = full
    solid, _, _ = synth.sphere_pack(nx, ny, nz, 6.0, 0.40, 8, seed, walls=True)
    s = solid.reshape(nz, ny, nx)[:edge, :edge, :edge].copy()
    s[:, :, edge - 8:] = 0
    s[0, :, :] = 1; s[-1, :, :] = 1; s[:, 0, :] = 1; s[:, -1, :] = 1
    return Problem(nx=edge, ny=edge, nz=edge, solid=s.reshape(-1), tau=0.6, tau_ad=0.55,
                   u_in=(0.02, 0.0, 0.0), isotherm="langmuir", q_max=5.0, b_langmuir=1.5,
                   k_ldf=0.05, steps=steps, name=f"sphere_pack_crop_{edge}")


def batch_samples(seed: int = 1237, count=64, edges=(96, 112, 128, 144, 160), steps=5000):
    """`count` independent Bernoulli samples with per-axis edges drawn from
    `edges`, porosity U[0.3,0.5], and q_max, K_L, k_ads log-uniform in
    [1,10], [0.1,5], [0.005,0.1]; tau 0.7 / 0.6, inlet u = 0.01, C = 1."""
    r = synth.uniform(seed, 7 * count).reshape(count, 7)
    out = []
    for i in range(count):
        nx, ny, nz = (edges[min(int(r[i, k] * len(edges)), len(edges) - 1)] for k in range(3))
        por = 0.3 + 0.2 * r[i, 3]
        qm = math.exp(math.log(1.0) + (math.log(10.0) - math.log(1.0)) * r[i, 4])
        kl = math.exp(math.log(0.1) + (math.log(5.0) - math.log(0.1)) * r[i, 5])
        kk = math.exp(math.log(0.005) + (math.log(0.1) - math.log(0.005)) * r[i, 6])
        solid = synth.bernoulli(nx, ny, nz, 1.0 - por, seed * 1000 + i, fluid_lo=4, fluid_hi=4, walls=True)
        out.append(Problem(nx=nx, ny=ny, nz=nz, solid=solid, tau=0.7, tau_ad=0.6, u_in=(0.01, 0.0, 0.0),
                           isotherm="langmuir", q_max=qm, b_langmuir=kl, k_ldf=kk, steps=steps,
                           name=f"sample{i}_{nx}x{ny}x{nz}"))
    return out


def smooth_solid_fraction(nx, ny, nz, seed, sigma=2.0, porosity=0.4):
    """Continuous solid fraction n_s in [0,1]: Gaussian-smoothed (sigma voxels)
    uniform noise s, threshold t at the `porosity` quantile, then
    n_s = 1 / (1 + exp(-(s - t) / (0.25 * std(s))))."""
    s = synth.smooth_noise(nx, ny, nz, sigma, seed)
    t = float(np.quantile(s, porosity))
    w = 0.25 * float(s.std())
    return 1.0 / (1.0 + np.exp(-(s - t) / w))


def smooth_porous(seed: int = 1238, nx=128, ny=64, nz=64, steps=4000, q_max=4.0, b=1.0, k=0.03) -> Problem:
    """128x64x64 porous-BGK problem: porosity 1 - n_s from smoothed noise,
    region n_s > 0.5, Langmuir (4, 1.0, 0.03), tau 0.8 / 0.7, inlet u = 0.01,
    C = 1, breakthrough sampled every 20 steps over 4000."""
    ns = smooth_solid_fraction(nx, ny, nz, seed)
    p = Problem(nx=nx, ny=ny, nz=nz, solid=np.zeros(nx * ny * nz, np.uint8), collision="porous",
                porosity=1.0 - ns, region=(ns > 0.5).astype(np.uint8), tau=0.8, tau_ad=0.7,
                u_in=(0.01, 0.0, 0.0), isotherm="langmuir", q_max=q_max, b_langmuir=b, k_ldf=k,
                steps=steps, sample_every=20, name=f"smooth_porous_{nx}x{ny}x{nz}")
    p.notes = {"n_s": ns}
    return p
