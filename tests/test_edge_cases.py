"""Edge cases of the lattice API: invalid and maximal sizes (rejected on the
host, no GPU needed), degenerate lattices, an all-obstacle box, a lone fluid
cell and boundary masks that select no cells (on the GPU, against the oracle:
FP32 and FP64 bit for bit, like the parity variants)."""
import ctypes as C

import numpy as np
import pytest

from fluidmaxxer_b200 import _abi, problems
from fluidmaxxer_b200._abi import FM_ERR_ARG, FM_ERR_UNSUPPORTED


def _create(nx, ny, nz, precision=_abi.FM_F32):
    lib = _abi.lib()
    p = _abi.FmParams(nx, ny, nz, 1.0, 0.8, 0.7, 0.0, 1e-8, 0, 1, 1)
    h = C.c_void_p()
    rc = lib.fm_lattice_create(C.byref(p), precision, None, C.byref(h))
    return rc, lib.fm_last_error().decode()


@pytest.mark.parametrize("dims", [(0, 4, 4), (4, -1, 4), (4, 4, 0)])
def test_invalid_dimensions_are_rejected(dims):
    rc, msg = _create(*dims)
    assert rc == FM_ERR_ARG and "invalid dimensions" in msg


def test_lattices_beyond_the_offset_range_are_rejected():
    # 19 planes of 32-bit offsets: at most 226,050,000 cells
    rc, msg = _create(1024, 1024, 216)
    assert rc == FM_ERR_UNSUPPORTED and "226,050,000" in msg


def test_the_size_limit_is_exact():
    """512x512x862 (225,968,128 cells: 19 planes end below 2^32) passes the size
    check and 512x512x863 does not.  An unknown precision, checked after the
    size, stops the accepted one before anything is allocated."""
    rc, msg = _create(512, 512, 862, precision=17)
    assert rc == FM_ERR_ARG and "precision" in msg
    rc, msg = _create(512, 512, 863, precision=17)
    assert rc == FM_ERR_UNSUPPORTED and "226,050,000" in msg


def test_unknown_precision_is_rejected():
    rc, msg = _create(8, 8, 8, precision=17)
    assert rc == FM_ERR_ARG and "precision" in msg


def _pb(nx, ny, nz, solid, **kw):
    base = dict(nx=nx, ny=ny, nz=nz, solid=np.asarray(solid, np.uint8).reshape(-1), tau=0.8, tau_ad=0.7,
                u_in=(0.02, 0.0, 0.0), isotherm="linear", k_henry=2.0, k_a=0.05, phi0=0.3, name="edge")
    base.update(kw)
    return problems.Problem(**base)


def _tiny(nx, ny, nz, **kw):
    return _pb(nx, ny, nz, np.zeros(nx * ny * nz), **kw)


CASES = {
    "1x1x1_periodic": lambda: _tiny(1, 1, 1, periodic=(True, True, True), ns_inlet="none", ns_outlet="none",
                                    ad_inlet="none", ad_outlet="none"),
    "1x1x1_closed": lambda: _tiny(1, 1, 1, periodic=(False, False, False), ns_inlet="none", ns_outlet="none",
                                  ad_inlet="none", ad_outlet="none"),
    # a one-cell inlet plane is three planes at once, which VelocityDirichletNEQ
    # rejects (as the reference does): these channels use the equilibrium inlet
    "2x1x1_channel": lambda: _tiny(2, 1, 1, ns_inlet="eq"),
    "3x1x1_channel": lambda: _tiny(3, 1, 1, ns_inlet="eq"),
    # nx = 1: the reference's ADNeumannOutlet would read x = -1 (before the
    # array for the first row); neither side applies it there
    "1x5x7_inlet_is_outlet": lambda: _tiny(1, 5, 7, ns_inlet="eq"),
    "2x2x2_langmuir": lambda: _tiny(2, 2, 2, isotherm="langmuir", q_max=3.0, b_langmuir=2.0, k_ldf=0.1,
                                    region=np.ones(8, np.uint8)),
    "all_obstacle": lambda: _pb(6, 4, 4, np.ones(96), collision="bgk"),
    "lone_fluid_cell": lambda: _pb(5, 5, 5, np.where(np.arange(125) == 62, 0, 1), ns_inlet="none",
                                   ns_outlet="none", ad_inlet="none", ad_outlet="none", phi0=0.5),
    "empty_bc_masks": lambda: _tiny(8, 4, 4, inlet=np.zeros(128, np.uint8), outlet=np.zeros(128, np.uint8)),
}


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_edge_lattices_match_oracle(name, prec):
    from tests.test_gpu_parity import run_cuda, run_oracle

    p = CASES[name]()
    steps = 25
    got = run_cuda(p, steps, precision=prec)
    ref = run_oracle(p, steps, prec=prec)
    for k in ("f", "g", "phi", "q"):
        a, b = got["state"][k], ref[k]
        assert np.array_equal(a, b), (k, int(np.count_nonzero(a != b)), float(np.nanmax(np.abs(a - b))))


@pytest.mark.gpu
@pytest.mark.parametrize("dims,msg", [((1, 5, 7), "inferred neighbor out of domain"),
                                      ((2, 1, 1), "exactly one axis-aligned plane")])
def test_neq_inlet_on_a_degenerate_plane_raises_like_the_reference(dims, msg):
    """include/boundary/ns/VelocityDirichletNEQ.hpp:54-107 throws for these planes."""
    from fluidmaxxer_b200 import lattice
    from fluidmaxxer_b200._abi import FmError

    p = _tiny(*dims)
    with pytest.raises(FmError) as e:
        lattice.from_problem(p, "f32")
    assert e.value.code == FM_ERR_ARG and msg in str(e.value)
