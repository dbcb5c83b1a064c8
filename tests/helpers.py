"""Comparison helpers shared by the parity tests."""
import numpy as np


def max_rel(a, b):
    """max |a - b| normalised by the max-norm of b (the field scale)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = float(np.abs(b).max())
    if scale == 0.0:
        return float(np.abs(a).max())
    return float(np.abs(a - b).max()) / scale


def field_errors(got, ref, keys=("rho", "ux", "uy", "uz", "phi", "q")):
    return {k: max_rel(got[k], ref[k]) for k in keys}
