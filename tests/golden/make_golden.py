"""Generate the golden fixtures from the reference's own kernels.

Runs the reference kernel bodies compiled for the host (oracle/_ref, built by
oracle/build_oracle.py from the reference tree) on the small seeded cases of
tests/cases.py and stores the macroscopic fields, the breakthrough series and
per-direction population sums.  Re-run in the container that holds the
reference tree:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle  # noqa: E402
from tests import cases  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
PLAN = [("channel_neq_linear", "f64", 60), ("channel_neq_linear", "f32", 60), ("channel_eq_langmuir", "f32", 60),
        ("porous_region", "f64", 50), ("pulse_bounceback", "f32", 50), ("closed_nonperiodic", "f64", 50)]


def main():
    for case, prec, steps in PLAN:
        o = Oracle(getattr(cases, case)(), "reference", prec)
        o.step(steps)
        r = o.get(populations=True)
        np.savez_compressed(os.path.join(OUT, f"{case}_{prec}.npz"), case=case, precision=prec, steps=steps,
                            rho=r["rho"], ux=r["ux"], uy=r["uy"], uz=r["uz"], phi=r["phi"], q=r["q"],
                            c_out=r["c_out"], f_plane_sums=r["f"].sum(axis=1))
        print("wrote", case, prec, steps)


if __name__ == "__main__":
    main()
