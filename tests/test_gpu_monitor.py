"""The step monitor (fm_set_monitor / fm_get_monitor): FP64 sums of the mass,
C, q, the outlet flux and a count of diverged cells, reduced inside the fused
step kernel by warp shuffles and block partials (run with -m gpu).

Checked against the separate reductions: fm_reduce after the same step (the
same per-cell values summed in another order), and the outlet flux
sum(C u_x) over x = nx-1 formed on the host from the downloaded fields."""
import numpy as np
import pytest

from fluidmaxxer_b200 import _abi, lattice, problems
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec, tol, ftol", [("f64", 1e-12, 1e-12), ("f32", 1e-9, 1e-6), ("f16", 1e-6, 2e-3),
                                             ("f16q", 1e-6, 2e-3)])
def test_monitor_matches_the_separate_reductions(prec, tol, ftol):
    p = problems.channel_small(nx=48, ny=20, nz=18, steps=60)
    L = lattice.from_problem(p, prec)
    L.set_monitor(1)
    for s in (17, 43):
        L.step(s)
        sums = L.reduce()
        fl = L.fields()
        m = L.monitor()
        assert m["step"][-1] == L.step_count and len(m["step"]) == L.step_count
        for i, k in enumerate(("mass", "C", "q")):
            assert abs(m[k][-1] - sums[i]) <= tol * abs(sums[i]), (k, m[k][-1], sums[i])
        out = np.zeros((p.nz, p.ny, p.nx), bool)
        out[:, :, -1] = True
        flux = float((fl["phi"] * fl["ux"])[out.reshape(-1)].sum())
        assert abs(m["outlet_flux"][-1] - flux) <= ftol * abs(flux) + 1e-15, (m["outlet_flux"][-1], flux)
        assert np.all(m["bad_cells"] == 0)
    L.close()


def test_monitor_period_and_conservation():
    p = cases.periodic_box(nx=16, ny=12, nz=10)
    L = lattice.from_problem(p, "f64")
    L.set_monitor(5)
    L.step(40)
    m = L.monitor()
    L.close()
    assert list(m["step"]) == list(range(5, 41, 5))
    assert np.allclose(m["mass"], m["mass"][0], rtol=1e-13, atol=0)     # a closed periodic box
    assert np.allclose(m["C"] + m["q"], m["C"][0] + m["q"][0], rtol=1e-12, atol=0)


def test_monitor_counts_diverged_cells():
    """A NaN planted in one cell's populations shows in the status count at the
    next monitored step (host-made; no device fault involved)."""
    p = problems.channel_small(nx=32, ny=12, nz=10, steps=10)
    L = lattice.from_problem(p, "f32")
    L.step(5)
    st = L.get_state()
    f = st["f"].copy()
    c = (p.nz // 2 * p.ny + p.ny // 2) * p.nx + p.nx // 2
    f[:, c] = np.nan
    L.set_state(f=f)
    L.set_monitor(1)
    L.step(1)
    m = L.monitor()
    L.close()
    assert m["bad_cells"][-1] >= 1


def test_monitor_needs_a_fused_step():
    L = lattice.from_problem(cases.channel_eq_langmuir(), "f32")   # odd nx: list-path boundaries
    L.set_monitor(1)
    with pytest.raises(_abi.FmError) as e:
        L.step(1)
    assert e.value.code == _abi.FM_ERR_UNSUPPORTED
    L.close()
