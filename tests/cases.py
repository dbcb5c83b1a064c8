"""Small seeded problem variants covering the reference's operator set.

Each builder returns a fluidmaxxer_b200.problems.Problem; sizes are chosen so
the CPU oracle finishes in well under a second, and some are deliberately not
multiples of 32 cells.
"""
import numpy as np

from fluidmaxxer_b200 import problems, synth


def _pb(nx, ny, nz, p, seed, walls=True, lo=2, hi=2):
    return synth.bernoulli(nx, ny, nz, p, seed, fluid_lo=lo, fluid_hi=hi, walls=walls)


def channel_neq_linear(nx=20, ny=10, nz=8, seed=11):
    return problems.Problem(nx=nx, ny=ny, nz=nz, solid=_pb(nx, ny, nz, 0.3, seed), tau=0.8, tau_ad=0.7,
                            ns_inlet="neq", u_in=(0.02, 0.0, 0.0), isotherm="linear", k_henry=2.0, k_a=0.05,
                            name="channel_neq_linear")


def channel_eq_langmuir(nx=21, ny=9, nz=7, seed=12):
    return problems.Problem(nx=nx, ny=ny, nz=nz, solid=_pb(nx, ny, nz, 0.25, seed), tau=0.6, tau_ad=0.55,
                            ns_inlet="eq", u_in=(0.03, 0.0, 0.0), isotherm="langmuir", q_max=5.0,
                            b_langmuir=1.5, k_ldf=0.05, name="channel_eq_langmuir")


def porous_region(nx=18, ny=8, nz=8, seed=13):
    n = nx * ny * nz
    rng = np.random.default_rng(seed)
    por = rng.uniform(0.2, 1.2, n)       # includes values clamped to [0,1]
    region = (rng.uniform(size=n) < 0.4).astype(np.uint8)
    tau = np.where(region, 0.9, 0.6)     # two-valued tau field as buildTauField makes
    return problems.Problem(nx=nx, ny=ny, nz=nz, solid=np.zeros(n, np.uint8), collision="porous", porosity=por,
                            region=region, tau=0.7, tau_ad=tau, ns_inlet="neq", u_in=(0.02, 0.0, 0.0),
                            isotherm="langmuir", q_max=4.0, b_langmuir=1.0, k_ldf=0.03, name="porous_region")


def pulse_bounceback(nx=16, ny=8, nz=9, seed=14):
    return problems.Problem(nx=nx, ny=ny, nz=nz, solid=_pb(nx, ny, nz, 0.2, seed), tau=0.9, tau_ad=0.8,
                            ns_inlet="eq", u_in=(0.02, 0.0, 0.0), ns_bounceback=True, ad_inlet="pulse",
                            pulse=(0.1, 0.9, 5.0, 5, 30), isotherm="linear", k_henry=1.0, k_a=0.02,
                            name="pulse_bounceback")


def periodic_box(nx=12, ny=10, nz=8, seed=15):
    """Closed periodic box, no boundaries, no reaction: populations are
    conserved exactly up to rounding."""
    n = nx * ny * nz
    return problems.Problem(nx=nx, ny=ny, nz=nz, solid=_pb(nx, ny, nz, 0.2, seed, walls=False, lo=0, hi=0),
                            periodic=(True, True, True), tau=0.7, tau_ad=0.6, ns_inlet="none", ns_outlet="none",
                            ad_inlet="none", ad_outlet="none", isotherm="none", phi0=0.5, name="periodic_box")


def closed_nonperiodic(nx=11, ny=9, nz=7, seed=16):
    """No periodic direction: every face uses the keep-local rule."""
    return problems.Problem(nx=nx, ny=ny, nz=nz, solid=_pb(nx, ny, nz, 0.15, seed, walls=False, lo=0, hi=0),
                            periodic=(False, False, False), tau=0.75, tau_ad=0.65, ns_inlet="neq",
                            u_in=(0.02, 0.0, 0.0), isotherm="linear", k_henry=2.0, k_a=0.01, phi0=0.2,
                            name="closed_nonperiodic")


def uncoupled(nx=14, ny=8, nz=8, seed=17):
    """--coupling off: the AD lattice advects with u = 0 (pure diffusion)."""
    return problems.Problem(nx=nx, ny=ny, nz=nz, solid=_pb(nx, ny, nz, 0.3, seed), coupling=False,
                            isotherm="langmuir", q_max=2.0, b_langmuir=0.5, k_ldf=0.1, name="uncoupled")


ALL = [channel_neq_linear, channel_eq_langmuir, porous_region, pulse_bounceback, periodic_box,
       closed_nonperiodic, uncoupled]
