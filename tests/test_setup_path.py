"""The set-up path of src/main.cpp:205-251 as one unit.

main.cpp builds its porous run from the geometry mask alone:
``setObstacleMask(mask)``, ``setPorosityFromMask(mask, 0.67, 1.0)``
(include/core/lattice/NSLattice.hpp:88-114), a two-valued AD relaxation time
from ``ADUnitConverter::buildTauField(mask, D_fluid, D_solid)``
(include/core/io/ADUnitConverter.hpp:63-104), the NEQ velocity inlet, the
pressure outlet, ADDirichlet + ADNeumannOutlet and the linear LDF on the
obstacle region.  The CPU tests check ``fm_build_tau_field`` against the
reference's formula and its errors; the GPU test builds that set-up through
the library's own entry points (not through a Problem's precomputed fields)
and compares the run with the oracle, which receives the same fields
restated in numpy.
"""
import numpy as np
import pytest

from fluidmaxxer_b200 import _abi, lattice, synth
from fluidmaxxer_b200._abi import FmError

DX, DT = 2.0e-5, 2.0e-2          # lattice spacing and time step (m, s)
D_FLUID, D_SOLID = 2.0e-9, 6.0e-10


def tau_of(d):
    """tauFromDiffusivityPhys (ADUnitConverter.hpp:45-58) with the D3Q7 cs2 = 1/4."""
    return d * DT / (DX * DX) / 0.25 + 0.5


def test_build_tau_field_is_the_reference_formula():
    nx, ny, nz = 12, 5, 4
    mask = (np.arange(nx * ny * nz) % 3 == 0).astype(np.uint8)
    got = lattice.build_tau_field((nx, ny, nz), DX, DT, mask, D_FLUID, D_SOLID)
    want = np.where(mask != 0, tau_of(D_SOLID), tau_of(D_FLUID))
    assert np.array_equal(got, want)
    assert got.max() == tau_of(D_FLUID) and got.min() == tau_of(D_SOLID)


@pytest.mark.parametrize("args, message", [
    (dict(shape=(1, 4, 4)), b"Nx must be >= 2"),
    (dict(dx=0.0), b"dx_phys must be > 0"),
    (dict(dt=-1.0), b"dt_phys must be > 0"),
    (dict(d_solid=0.0), b"tau_ad <= 0.5 (unstable)"),
    (dict(n=10), b"mask size mismatch"),
])
def test_build_tau_field_raises_the_reference_errors(args, message):
    shape = args.get("shape", (6, 4, 4))
    n = args.get("n", shape[0] * shape[1] * shape[2])
    mask = np.zeros(n, np.uint8)
    with pytest.raises(FmError) as e:
        lattice.build_tau_field(shape, args.get("dx", DX), args.get("dt", DT), mask, D_FLUID,
                                args.get("d_solid", D_SOLID))
    assert e.value.code == _abi.FM_ERR_ARG
    assert message in _abi.lib().fm_last_error()


def _main_cpp_lattice(mask, shape, precision, u_in, k_henry, k_a):
    nx, ny, nz = shape
    L = lattice.CoupledLattice(nx, ny, nz, tau=0.8, tau_ad=0.7, precision=precision)
    inlet = np.zeros((nz, ny, nx), np.uint8); inlet[:, :, 0] = 1
    outlet = np.zeros((nz, ny, nx), np.uint8); outlet[:, :, -1] = 1
    L.set_collision("porous")
    L.set_obstacle_mask(mask)
    L.set_porosity_from_mask(mask, 0.67, 1.0)
    L.add_ns_velocity_neq(inlet.reshape(-1), u_in)
    L.add_ns_pressure(outlet.reshape(-1), 1.0)
    L.set_tau_field(lattice.build_tau_field(shape, DX, DT, mask, D_FLUID, D_SOLID))
    L.set_isotherm_linear(mask, k_henry, k_a)          # region = the obstacle mask (src/main.cpp:333)
    L.add_ad_dirichlet(inlet.reshape(-1), 1.0)
    L.add_ad_neumann(outlet.reshape(-1))
    L.set_outlet_probe(outlet.reshape(-1), 10)
    L.init_equilibrium()
    return L


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_main_cpp_setup_path_matches_the_oracle(prec):
    from fluidmaxxer_b200 import problems
    from oracle.oracle import Oracle

    shape = (32, 12, 10)
    nx, ny, nz = shape
    mask = synth.bernoulli(nx, ny, nz, 0.35, 21, fluid_lo=3, fluid_hi=3, walls=False)
    steps, u_in, k_henry, k_a = 300, 0.02, 2.0, 0.02
    L = _main_cpp_lattice(mask, shape, prec, u_in, k_henry, k_a)
    L.step(steps)
    got = L.fields()
    got_bt = L.breakthrough()
    L.close()

    # the oracle receives the fields the reference's set-up calls produce
    p = problems.Problem(nx=nx, ny=ny, nz=nz, solid=mask, collision="porous",
                         porosity=np.where(mask != 0, 0.67, 1.0), tau=0.8,
                         tau_ad=np.where(mask != 0, tau_of(D_SOLID), tau_of(D_FLUID)), u_in=(u_in, 0.0, 0.0),
                         isotherm="linear", k_henry=k_henry, k_a=k_a, sample_every=10, steps=steps)
    o = Oracle(p, "restated", prec)
    o.step(steps)
    ref = o.get()
    o.close()
    for k in ("rho", "ux", "uy", "uz", "phi", "q"):
        assert np.array_equal(got[k], ref[k]), k
    assert np.allclose(got_bt, ref["c_out"], rtol=1e-12, atol=1e-15)
