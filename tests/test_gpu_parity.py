"""CUDA path vs the oracle on the same seeded inputs (run with -m gpu).

Tolerance: the maximum absolute difference of each field, divided by that
field's max-norm, is at most 1e-5 after the stated step count (FP32 CUDA vs
FP32 and FP64 oracle runs of the same problem).  Domain sums (rho, C, q)
agree to 1e-6 relative.
"""
import numpy as np
import pytest

from fluidmaxxer_b200 import lattice, problems
from oracle.oracle import Oracle, reference_available
from tests import cases
from tests.helpers import field_errors, max_rel

pytestmark = pytest.mark.gpu
TOL = 1e-5
SUM_TOL = 1e-6


def run_cuda(p, steps, precision="f32"):
    L = lattice.from_problem(p, precision)
    L.step(steps)
    out = L.fields()
    out["c_out"] = L.breakthrough()
    out["sums"] = L.reduce()
    out["state"] = L.get_state()
    L.close()
    return out


def run_oracle(p, steps, impl="restated", prec="f32"):
    o = Oracle(p, impl, prec)
    o.step(steps)
    r = o.get(populations=True)
    o.close()
    return r


@pytest.mark.parametrize("build", cases.ALL, ids=lambda b: b.__name__)
def test_variants_match_oracle(build):
    p = build()
    steps = 200
    got = run_cuda(p, steps)
    ref = run_oracle(p, steps)
    errs = field_errors(got, ref)
    assert max(errs.values()) <= TOL, errs
    assert max_rel(got["c_out"], ref["c_out"]) <= TOL
    assert max_rel(got["state"]["f"], ref["f"]) <= TOL
    assert max_rel(got["state"]["g"], ref["g"]) <= TOL
    for i in range(3):
        assert abs(got["sums"][i] - ref["sums"][i]) <= SUM_TOL * max(abs(ref["sums"][i]), 1e-30)


def test_channel_small_2000_steps_vs_fp32_and_fp64():
    """64x32x32 Bernoulli channel, 2000 steps: the stated parity case."""
    p = problems.channel_small()
    got = run_cuda(p, p.steps)
    for prec in ("f32", "f64"):
        ref = run_oracle(p, p.steps, prec=prec)
        errs = field_errors(got, ref)
        assert max(errs.values()) <= TOL, (prec, errs)
        assert max_rel(got["c_out"], ref["c_out"]) <= TOL
        for i in range(3):
            assert abs(got["sums"][i] - ref["sums"][i]) <= SUM_TOL * abs(ref["sums"][i]), (prec, i)


@pytest.mark.skipif(not reference_available("f32"), reason="reference kernels not built")
def test_channel_small_vs_reference_kernels():
    p = problems.channel_small(steps=500)
    got = run_cuda(p, p.steps)
    ref = run_oracle(p, p.steps, impl="reference", prec="f32")
    errs = field_errors(got, ref)
    assert max(errs.values()) <= TOL, errs
