"""Digest of the FP64 oracle's fields after 20000 steps of the 128^3 sphere-pack crop.

Runs the plain-C restatement (oracle/fm_oracle.c, FP64, OpenMP over the host
threads; about 45 minutes on 16 threads) on problems.sphere_pack_crop() and
writes crop128_f64_digest.json: the SHA-256 of each output field's float64
bytes (rho, ux, uy, uz, phi, q over all 2,097,152 cells), the field max-norms,
and the breakthrough series C_out (every 20 steps).  The GPU test compares the
CUDA FP64 path's fields with these hashes, i.e. bit for bit.

Usage: python tests/golden/make_crop_digest.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fluidmaxxer_b200 import problems  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

STEPS = 20000
FIELDS = ("rho", "ux", "uy", "uz", "phi", "q")


def digest(fields, c_out):
    out = {"steps": STEPS, "problem": "sphere_pack_crop_128", "sha256": {}, "max_abs": {}}
    for k in FIELDS:
        a = np.ascontiguousarray(fields[k], dtype="<f8")
        out["sha256"][k] = hashlib.sha256(a.tobytes()).hexdigest()
        out["max_abs"][k] = float(np.abs(a).max())
    out["c_out"] = [float(v) for v in c_out]
    return out


def main():
    p = problems.sphere_pack_crop()
    o = Oracle(p, "restated", "f64")
    for _ in range(STEPS // 1000):
        o.step(1000)
    r = o.get(max_samples=2000)
    o.close()
    with open(os.path.join(HERE, "crop128_f64_digest.json"), "w") as fh:
        json.dump(digest(r, r["c_out"]), fh, indent=1)


if __name__ == "__main__":
    main()
