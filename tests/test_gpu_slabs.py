"""z-slab decomposition (fluidmaxxer_b200.slabs) on one GPU: the slabs, with
their halos moved every step, reproduce the unsplit lattice bit for bit
(populations and fields in FP32, FP64 and the FP16 pair layout; the
breakthrough series and the domain sums to the order of their FP64 sums).
Lattices whose step is one launch and whose nx*ny is a multiple of 64 step in
parts (boundary planes, halo, interior: fm_step_planes / fm_step_finish); the
others step whole and move the halo after the step."""
import numpy as np
import pytest

from fluidmaxxer_b200 import lattice, problems, slabs
from tests import cases

pytestmark = pytest.mark.gpu


def _cases():
    return {
        "channel_48": lambda: problems.channel_small(nx=48, ny=20, nz=18, steps=80),
        "channel_odd": lambda: problems.channel_small(nx=37, ny=12, nz=13, steps=80),
        "porous_langmuir": lambda: problems.smooth_porous(nx=40, ny=16, nz=12, steps=80),
        "neq_linear_variant": lambda: cases.channel_neq_linear(nz=14),
        "closed_box": lambda: cases.closed_nonperiodic(nz=12),
    }


@pytest.mark.parametrize("prec", ["f32", "f64", "f16"])
@pytest.mark.parametrize("nslabs", [1, 2, 3])
@pytest.mark.parametrize("name", sorted(_cases()))
def test_slabs_reproduce_the_unsplit_lattice(name, nslabs, prec):
    p = _cases()[name]()
    steps = 60
    L = lattice.from_problem(p, prec)
    L.step(steps)
    ref = L.fields()
    bt = L.breakthrough()
    sums = L.reduce()[:3]
    L.close()
    run = slabs.SlabRun(p, nslabs, prec)
    split = run.split_steps
    run.step(steps)
    got = run.fields()
    gbt = run.breakthrough() if p.sample_every > 0 else np.zeros(0)
    gsums = run.reduce()
    run.close()
    assert split == (name in ("channel_48", "porous_langmuir")), split   # nx*ny % 64 and one launch per step
    for k in ref:
        assert np.array_equal(got[k], ref[k]), (k, int(np.count_nonzero(got[k] != ref[k])))
    if p.sample_every > 0:
        assert np.allclose(gbt, bt, rtol=1e-13, atol=0)
    assert np.allclose(gsums, sums, rtol=1e-12, atol=0)


def test_whole_plane_copy_round_trip():
    """fm_pack_zplane / fm_unpack_zplane move all 26 populations of a plane:
    copying plane 3 over plane 5 makes their populations equal (away from the
    x = 0 inlet cells, whose populations the getters take from the inlet's own
    store of every row)."""
    import torch

    p = problems.channel_small(nx=32, ny=16, nz=10, steps=20)
    L = lattice.from_problem(p, "f32")
    L.step(20)
    buf = torch.empty(26 * p.nx * p.ny, dtype=torch.float32, device="cuda")
    assert L._lib.fm_pack_zplane(L.h, 3, buf.data_ptr()) == 0
    assert L._lib.fm_unpack_zplane(L.h, 5, buf.data_ptr()) == 0
    L.synchronize()
    st = L.get_state()
    L.close()
    for k in ("f", "g"):
        a = st[k].reshape(st[k].shape[0], p.nz, p.ny, p.nx)[..., 1:]
        assert np.array_equal(a[:, 3], a[:, 5])
