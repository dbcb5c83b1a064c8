"""Known answers the coupled step must reproduce, independent of any oracle run.

The reference ships no tests, so besides the oracle parity these tests check
the CUDA path against laws of the discretisation itself:

* a closed periodic box conserves the fluid mass sum(rho) and the species
  mass sum(g) + sum(q) exactly, up to rounding (BGK and the LDF exchange only
  move mass between cells and between the fluid and the solid loading);
* a Gaussian concentration pulse in a periodic box at rest spreads with the
  lattice diffusivity D = cs2 (tau_ad - 1/2) = (tau_ad - 1/2) / 4 of D3Q7: once
  the first-order moment has relaxed, its variance grows by exactly 2 D per
  step;
* a uniform batch reactor (no flow, the whole box adsorbing) follows the
  scalar recursion of one cell of src/reaction/LinearLDF.cu:13-48 inside the
  loop of src/main.cpp:319-357, and follows the closed-form linear-driving-
  force uptake q(t) = q* (1 - exp(-k (1 + K) t)), q* = K c0 / (1 + K), to 2%;
* steady flow between two bounce-back walls has the plane-Poiseuille parabolic
  profile;
* the reference's free launchers launch_henry_ldf_source_d3q7 and
  launch_langmuir_ldf_source_d3q7 (include/reaction/LinearLDF.hpp:8-17,
  include/reaction/LangmuirLDF.hpp:7-14) give the same bits as their formula
  evaluated in FP32 in the same order.
"""
import numpy as np
import pytest

from fluidmaxxer_b200 import _abi, lattice, problems, synth

pytestmark = pytest.mark.gpu

W7 = np.array([0.25] + [0.125] * 6)


def _box(nx, ny, nz, precision, solid=None, phi0=0.0, tau=0.7, tau_ad=0.7, region=None, iso=None, coupling=True):
    L = lattice.CoupledLattice(nx, ny, nz, tau=tau, tau_ad=tau_ad, phi0=phi0, periodic=(True, True, True),
                               precision=precision)
    n = nx * ny * nz
    L.set_collision("bgk")
    L.set_obstacle_mask(np.zeros(n, np.uint8) if solid is None else solid)
    L.set_coupling(coupling)
    if iso is not None:
        L.set_isotherm_linear(region, *iso)
    L.init_equilibrium()
    return L


# FP32: the reference's FP32 arithmetic (the FP32 oracle, bit-identical to this
# path) moves the mass by 1.2e-6 in the first steps and the species sum by
# ~1e-6 per 500 steps -- rounding of the collision and of the LDF exchange
@pytest.mark.parametrize("prec, tol", [("f64", 1e-12), ("f32", 1e-5)])
def test_closed_periodic_box_conserves_fluid_and_species_mass(prec, tol):
    nx, ny, nz = 24, 16, 12
    n = nx * ny * nz
    solid = synth.bernoulli(nx, ny, nz, 0.2, 31, fluid_lo=0, fluid_hi=0, walls=False)
    rng = np.random.default_rng(5)
    region = (rng.uniform(size=n) < 0.5).astype(np.uint8)
    L = _box(nx, ny, nz, prec, solid=solid, phi0=0.5, region=region, iso=(2.0, 0.05))
    # a non-uniform start: a density and concentration bump on the fluid
    st = L.get_state()
    bump = np.exp(-((np.arange(n) % nx - nx / 2) ** 2) / 8.0)
    f = st["f"] * (1.0 + 0.05 * bump)
    g = st["g"] * (1.0 + 0.5 * bump)
    L.set_state(f=f, g=g)
    st = L.get_state()
    m_rho0, m_c0 = st["f"].sum(), st["g"].sum() + st["q"].sum()
    for _ in range(4):
        L.step(500)
        st = L.get_state()
        assert abs(st["f"].sum() - m_rho0) <= tol * m_rho0
        assert abs(st["g"].sum() + st["q"].sum() - m_c0) <= tol * m_c0
    assert st["q"].sum() > 0.1 * m_c0          # the exchange did take place
    L.close()


@pytest.mark.parametrize("prec, tol", [("f64", 1e-9), ("f32", 2e-4)])
def test_gaussian_pulse_spreads_at_the_lattice_diffusivity(prec, tol):
    # 256 cells long: the pulse's tails stay ~12 sigma from the periodic seam
    nx, ny, nz, tau_ad, x0, s0, bg = 256, 4, 4, 0.7, 128.0, 4.0, 0.1
    L = _box(nx, ny, nz, prec, tau_ad=tau_ad, coupling=False)
    x = np.arange(nx * ny * nz) % nx
    c = bg + 0.5 * np.exp(-((x - x0) ** 2) / (2.0 * s0 * s0))
    L.set_state(g=W7[:, None] * c[None, :])

    def variance():
        phi = L.field("phi") - bg
        return float(((x - x0) ** 2 * phi).sum() / phi.sum())

    L.step(200)          # the first moment relaxes by (1 - 1/tau_ad)^t
    v0 = variance()
    L.step(800)
    v1 = variance()
    L.close()
    d = (tau_ad - 0.5) / 4.0
    assert abs((v1 - v0) / (2.0 * 800) - d) <= tol * d


def test_batch_reactor_follows_the_ldf_recursion_and_its_closed_form():
    nx, ny, nz, c0, K, k, eps = 8, 4, 4, 1.0, 2.0, 0.01, 1e-8
    n = nx * ny * nz
    L = _box(nx, ny, nz, "f64", phi0=c0, region=np.ones(n, np.uint8), iso=(K, k))
    # one cell of the loop: the LDF source at step s reads phi(s-1) (zero at
    # s = 1, the constructor's buffer), phi(s) is the streamed mass of step s
    phi_prev, m, q = 0.0, c0, 0.0
    got, want = [], []
    for s in range(1, 1001):
        L.step(1)
        dq = k * (K * (max(phi_prev, eps) - eps) - q)
        q += dq
        phi = max(m, eps)
        m = m - dq
        phi_prev = phi
        if s % 20 == 0:
            got.append((L.field("phi").mean(), L.field("q").mean(), np.ptp(L.field("q"))))
            want.append((phi, q))
    L.close()
    got = np.array(got)
    want = np.array(want)
    assert np.all(got[:, 2] == 0.0)                             # uniform stays uniform
    assert np.allclose(got[:, :2], want, rtol=1e-12, atol=1e-14)
    # closed form of the continuous exchange; the loop's source reads the
    # previous step's concentration, so the discrete curve trails it by a step
    t = np.arange(20, 1001, 20)
    q_star = K * c0 / (1.0 + K)
    q_cont = q_star * (1.0 - np.exp(-k * (1.0 + K) * (t - 1)))
    assert np.max(np.abs(got[:, 1] - q_cont)) <= 0.02 * q_star
    assert abs(got[-1, 1] - q_star) <= 1e-6 * q_star            # at equilibrium q = K c
    assert abs(got[-1, 0] + got[-1, 1] - c0) <= 1e-6 * c0


def test_flow_between_walls_has_the_poiseuille_profile():
    nx, ny, nz = 64, 18, 4
    solid = np.zeros((nz, ny, nx), np.uint8)
    solid[:, 0, :] = 1
    solid[:, ny - 1, :] = 1
    p = problems.Problem(nx=nx, ny=ny, nz=nz, solid=solid.reshape(-1), tau=0.8, tau_ad=0.7, u_in=(0.01, 0.0, 0.0),
                         isotherm="none", sample_every=0, steps=8000)
    L = lattice.from_problem(p, "f64")
    L.step(p.steps)
    ux = L.field("ux").reshape(nz, ny, nx)[:, :, nx // 2]
    L.close()
    prof = ux[0, 1:ny - 1]
    assert np.allclose(ux, ux[0:1], rtol=1e-12, atol=1e-15)     # no z dependence
    assert np.allclose(prof, prof[::-1], rtol=1e-9)              # symmetric about the centre
    y = np.arange(1, ny - 1, dtype=np.float64)
    shape = (y - 0.5) * (ny - 1.5 - y)                           # halfway bounce-back walls
    amp = float(prof @ shape / (shape @ shape))
    assert np.max(np.abs(prof - amp * shape)) <= 0.02 * prof.max()


@pytest.mark.parametrize("langmuir", [False, True])
def test_free_ldf_launchers_equal_their_fp32_formula(langmuir):
    import torch

    n, eps = 100_003, np.float32(1e-8)
    rng = np.random.default_rng(9)
    region = (rng.uniform(size=n) < 0.6).astype(np.uint8)
    phi = rng.uniform(-0.1, 1.2, n).astype(np.float32)
    phi[:50] = 0.0
    q0 = rng.uniform(0.0, 2.0, n).astype(np.float32)
    dev = torch.device("cuda:0")
    d_region = torch.from_numpy(region).to(dev)
    d_phi = torch.from_numpy(phi).to(dev)
    d_s = torch.full((n,), 7.0, dtype=torch.float32, device=dev)
    d_q = torch.from_numpy(q0).to(dev)
    torch.cuda.synchronize()
    lib = _abi.lib()
    a, b, k = np.float32(2.5), np.float32(1.5), np.float32(0.05)
    if langmuir:
        rc = lib.fm_launch_langmuir_ldf_source_d3q7(n, d_region.data_ptr(), d_phi.data_ptr(), d_s.data_ptr(),
                                                    d_q.data_ptr(), float(a), float(b), float(k), float(eps), None)
    else:
        rc = lib.fm_launch_henry_ldf_source_d3q7(n, d_region.data_ptr(), d_phi.data_ptr(), d_s.data_ptr(),
                                                 d_q.data_ptr(), float(a), float(k), float(eps), None)
    assert rc == 0, lib.fm_last_error()
    torch.cuda.synchronize()
    # src/reaction/LinearLDF.cu:13-48, src/reaction/LangmuirLDF.cu:7-41, in FP32
    c = np.where(phi < eps, eps, phi).astype(np.float32)
    ce = (c - eps).astype(np.float32)
    if langmuir:
        bc = (b * ce).astype(np.float32)
        qeq = (a * (bc / (np.float32(1) + bc)).astype(np.float32)).astype(np.float32)
    else:
        qeq = (a * ce).astype(np.float32)
    dq = (k * (qeq - q0).astype(np.float32)).astype(np.float32)
    inside = region != 0
    q_want = np.where(inside, (q0 + dq).astype(np.float32), q0)
    s_want = np.where(inside, -dq, np.float32(0))
    assert np.array_equal(d_q.cpu().numpy(), q_want)
    assert np.array_equal(d_s.cpu().numpy(), s_want)
    # no cells: nothing to do; bad arguments are refused before any launch
    assert lib.fm_launch_henry_ldf_source_d3q7(0, None, None, None, None, 1.0, 1.0, 1e-8, None) == 0
    assert lib.fm_launch_henry_ldf_source_d3q7(-1, None, None, None, None, 1.0, 1.0, 1e-8, None) == _abi.FM_ERR_ARG
