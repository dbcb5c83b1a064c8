"""z-slab decomposition (fluidmaxxer_b200.slabs) on one GPU: the slabs, stepped
in turn with the halo exchange after every step, reproduce the unsplit lattice
bit for bit (FP32 and FP64 populations, fields; the breakthrough series to the
order of its FP64 block sums)."""
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


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("nslabs", [1, 2, 3])
@pytest.mark.parametrize("name", sorted(_cases()))
def test_slabs_reproduce_the_unsplit_lattice(name, nslabs, prec):
    p = _cases()[name]()
    steps = 60
    L = lattice.from_problem(p, prec)
    L.step(steps)
    ref = L.fields()
    bt = L.breakthrough()
    L.close()
    run = slabs.SlabRun(p, nslabs, prec)
    run.step(steps)
    got = run.fields()
    gbt = run.breakthrough() if p.sample_every > 0 else np.zeros(0)
    run.close()
    for k in ref:
        assert np.array_equal(got[k], ref[k]), (k, int(np.count_nonzero(got[k] != ref[k])))
    if p.sample_every > 0:
        assert np.allclose(gbt, bt, rtol=1e-13, atol=0)
