"""The pair layout of the 16-bit forms (fluidmaxxer_b200/csrc/fm_pair.cuh).

Lattices of the 16-bit forms with nx % 4 == 0 whose boundaries all run inside
the fused step can store each x-row as words of two cells (x, x + nx/2) and
step them with a two-cells-per-thread kernel (opt-in: fm_set_pair_layout);
with nx % 8 == 0 and nx <= 512 the staged variant brings each tile's source
rows into shared memory by bulk copies.  Its arithmetic is the one-cell
deviation-form update's, operation for operation, so the populations, C, q
and the breakthrough series must equal the one-cell kernel's bit for bit
(fm_set_pair_layout(0) forces the one-cell kernel on the natural layout).  The
cases cover the pair kernel's paths: obstacles (bounce-back with mixed
fluid / obstacle pairs), porous BGK, the fused inlet / outlet / AD planes,
periodic x (the fold points wrap) and closed x faces (keep-local), y/z faces
periodic and closed.
"""
import numpy as np
import pytest

from fluidmaxxer_b200 import lattice, problems, synth
from tests import cases

pytestmark = pytest.mark.gpu
FORMS = ["f16", "bf16", "f16q"]


def channel(nx=32, ny=12, nz=10):
    return cases.channel_neq_linear(nx=nx, ny=ny, nz=nz)


def pack(nx=48, ny=20, nz=16):
    """A small sphere pack (r = 3) with y/z walls: many mixed fluid / obstacle pairs."""
    solid, _, _ = synth.sphere_pack(nx, ny, nz, 3.0, 0.45, 4, 1240, walls=True)
    return problems.Problem(nx=nx, ny=ny, nz=nz, solid=solid, tau=0.6, tau_ad=0.55, u_in=(0.02, 0.0, 0.0),
                            isotherm="langmuir", q_max=5.0, b_langmuir=1.5, k_ldf=0.05, steps=120)


def porous(nx=24, ny=12, nz=8):
    return problems.smooth_porous(seed=77, nx=nx, ny=ny, nz=nz, steps=80)


def periodic_x(nx=16, ny=10, nz=8):
    return cases.periodic_box(nx=nx, ny=ny, nz=nz)


def closed(nx=12, ny=9, nz=7):
    p = cases.closed_nonperiodic(nx=nx, ny=ny, nz=nz)
    return p


BUILDERS = [channel, pack, porous, periodic_x, closed]


def run(p, prec, pair, steps, staged=True):
    L = lattice.from_problem(p, prec)
    L.set_pair_layout(pair)
    L.set_pair_kernel(staged)
    layout = L.storage_layout()
    kernel = L.step_kernel()
    L.step(steps)
    st = L.get_state()
    out = dict(f=st["f"], g=st["g"], phi=st["phi"], q=st["q"], bt=L.breakthrough(), fields=L.fields(),
               layout=layout, kernel=kernel, sums=L.reduce(), status=L.step_status())
    L.close()
    return out


def assert_same_run(a, b):
    for k in ("f", "g", "phi", "q", "bt"):
        assert np.array_equal(a[k], b[k]), (k, int(np.count_nonzero(a[k] != b[k])))
    for k in ("rho", "ux", "uy", "uz"):
        assert np.array_equal(a["fields"][k], b["fields"][k]), k
    assert np.allclose(a["sums"], b["sums"], rtol=1e-12, atol=0.0)   # FP64 sums in another order


@pytest.mark.parametrize("prec", FORMS)
@pytest.mark.parametrize("build", BUILDERS, ids=lambda b: b.__name__)
def test_pair_kernels_equal_the_one_cell_kernel(build, prec):
    """Both pair kernels -- the staged one where the shape allows it, and
    k_coupled_pair -- against the one-cell kernel, bit for bit."""
    p = build()
    steps = 97
    ref = run(p, prec, False, steps)
    assert ref["layout"] == "natural" and ref["kernel"] == "one-cell"
    staged = run(p, prec, True, steps)
    direct = run(p, prec, True, steps, staged=False)
    assert staged["layout"] == "pair" and direct["kernel"] == "pair"
    assert staged["kernel"] == ("pair-staged" if p.nx % 8 == 0 else "pair")
    for got in (staged, direct):
        assert got["status"] == 0
        assert_same_run(got, ref)


@pytest.mark.parametrize("prec", ["f16", "f16q"])
def test_staged_kernel_tiles(prec):
    """Shapes of the staged kernel's tiles: many rows per tile with a partial
    last tile (h = 4), one full-width row per tile (h = 256), closed y/z faces
    inside a tile, a tau field and porous BGK (more staged cell arrays)."""
    shapes = [
        problems.Problem(nx=8, ny=5, nz=7, solid=synth.bernoulli(8, 5, 7, 0.2, 3, fluid_lo=1, fluid_hi=1, walls=False),
                         periodic=(False, False, True), u_in=(0.02, 0.0, 0.0), steps=60),
        problems.Problem(nx=512, ny=3, nz=4, solid=synth.bernoulli(512, 3, 4, 0.2, 4, fluid_lo=2, fluid_hi=2),
                         u_in=(0.02, 0.0, 0.0), steps=60),
        cases.porous_region(nx=24, ny=8, nz=8),
    ]
    for p in shapes:
        ref = run(p, prec, False, 61)
        got = run(p, prec, True, 61)
        assert got["kernel"] == "pair-staged", p.nx
        assert got["status"] == 0
        assert_same_run(got, ref)


def test_layout_switches_keep_the_run():
    """Reading the state between steps, turning the pair layout off and on
    again (each a conversion of the stored populations) does not change the
    trajectory."""
    p = channel(nx=40, ny=12, nz=12)
    ref = run(p, "f16q", True, 90)
    L = lattice.from_problem(p, "f16q")
    L.set_pair_layout(True)
    L.step(30)
    L.get_state()                            # read in the pair layout
    L.set_pair_layout(False)
    L.step(30)                               # natural layout, one-cell kernel
    L.fields()
    L.set_pair_layout(True)
    L.step(30)                               # back to the pair layout
    st = L.get_state()
    bt = L.breakthrough()
    L.close()
    for k in ("f", "g", "phi", "q"):
        assert np.array_equal(st[k], ref[k]), k
    assert np.array_equal(bt, ref["bt"])


def test_which_lattices_use_the_pair_layout():
    """The pair layout is opt-in (fm_set_pair_layout): by default every form
    runs the one-cell kernel on the natural layout, which measured faster on
    B200 than both pair kernels."""
    p = channel(nx=32)
    for prec, want in (("f16", "pair"), ("bf16", "pair"), ("f16q", "pair"), ("f32", "natural"), ("f64", "natural")):
        L = lattice.from_problem(p, prec)
        assert L.storage_layout() == "natural" and L.step_kernel() == "one-cell", prec
        L.set_pair_layout(True)
        assert L.storage_layout() == want, prec
        assert L.step_kernel() == ("pair-staged" if want == "pair" else "one-cell"), prec
        L.close()
    # the staged kernel wants nx % 8 == 0 and nx / 2 <= 256 words
    for nx, want in ((12, "pair"), (520, "pair"), (512, "pair-staged"), (8, "pair-staged")):
        L = lattice.from_problem(channel(nx=nx, ny=4, nz=4), "f16")
        L.set_pair_layout(True)
        assert L.step_kernel() == want, nx
        L.close()
    for q, why in ((channel(nx=30), "nx % 4 != 0"), (cases.pulse_bounceback(nx=16), "list-path boundaries")):
        L = lattice.from_problem(q, "f16")
        assert L.storage_layout() == "natural", why
        L.close()


def test_pair_lattices_in_a_batch_step_the_natural_layout():
    ps = problems.batch_samples(seed=31, count=3, edges=(16, 24, 32), steps=40)
    solo = [lattice.from_problem(p, "f16") for p in ps]
    for L in solo:
        L.set_pair_layout(True)
        assert L.storage_layout() == "pair"
        L.step(40)
    bat = [lattice.from_problem(p, "f16") for p in ps]
    for L in bat:
        L.set_pair_layout(True)
        L.step(5)                            # in the pair layout before the batch
    B = lattice.Batch(bat)
    B.step(35)
    B.synchronize()
    for a, b in zip(solo, bat):
        assert b.storage_layout() == "natural"
        sa, sb = a.get_state(), b.get_state()
        for k in ("f", "g", "phi", "q"):
            assert np.array_equal(sa[k], sb[k]), k
    B.close()
    for L in solo + bat:
        L.close()


def test_pull_copy_of_the_pair_layout():
    """fm_bench_pull_copy measures the pair layout's own pattern (32-bit words)."""
    p = channel(nx=64, ny=16, nz=16)
    L = lattice.from_problem(p, "f16")
    L.set_pair_layout(True)
    assert L.storage_layout() == "pair"
    L.step(3)
    ms, nbytes = L.bench_pull_copy(3)
    h = p.nx // 2
    words = p.n_cells // 2 - 2 * (h * p.ny + h + 1)
    assert ms > 0.0 and nbytes == 2 * 26 * 4 * words
    L.close()


def test_a_device_wait_that_gave_up_is_reported():
    """Host-side detection of the staged kernel's bounded waits: with the
    status word set (written from the host, standing in for a wait that ran
    out -- no kernel is made to wait in vain), the getters and fm_reduce
    return FM_ERR_DEVICE; fm_step_status reports the word and clears it, after
    which the lattice steps and reads normally."""
    from fluidmaxxer_b200 import _abi
    from fluidmaxxer_b200._abi import FmError

    p = channel(nx=32)
    L = lattice.from_problem(p, "f16")
    L.set_pair_layout(True)
    L.step(3)
    assert L.step_status() == 0
    assert L._lib.fm_debug_set_status(L.h, 1) == 0
    with pytest.raises(FmError) as e:
        L.fields()
    assert e.value.code == _abi.FM_ERR_DEVICE
    with pytest.raises(FmError) as e:
        L.reduce()
    assert e.value.code == _abi.FM_ERR_DEVICE
    assert L.step_status() == 1
    assert L.step_status() == 0
    L.step(2)
    assert np.isfinite(L.fields()["rho"]).all()
    L.close()
