"""The restated oracle agrees bit for bit with the reference's own kernels.

The reference ships no tests or golden vectors, so the restatement
(oracle/fm_oracle.c) is pinned two ways: against the reference kernel bodies
compiled for the host (oracle/_ref, built only where the reference tree is
present), and against golden fixtures generated from them
(tests/golden/make_golden.py), which travel with the repository.
"""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, reference_available
from tests import cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
STEPS = 40


def _run(p, impl, prec, steps=STEPS):
    o = Oracle(p, impl, prec)
    o.step(steps)
    out = o.get(populations=True)
    o.close()
    return out


@pytest.mark.skipif(not reference_available(), reason="reference kernels not built here")
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("build", cases.ALL, ids=lambda b: b.__name__)
def test_restatement_bit_exact_vs_reference_kernels(build, prec):
    p = build()
    a = _run(p, "restated", prec)
    b = _run(p, "reference", prec)
    for k in ("f", "g", "phi", "q", "rho", "ux", "uy", "uz", "c_out"):
        assert np.array_equal(a[k], b[k]), f"{k} differs"


@pytest.mark.parametrize("name", sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz")))
def test_restatement_matches_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    build = getattr(cases, str(z["case"]))
    steps = int(z["steps"])
    prec = str(z["precision"])
    a = _run(build(), "restated", prec, steps)
    for k in ("rho", "ux", "uy", "uz", "phi", "q", "c_out"):
        assert np.array_equal(a[k], z[k]), f"{k} differs from golden"
    assert np.array_equal(a["f"].sum(axis=1), z["f_plane_sums"])
