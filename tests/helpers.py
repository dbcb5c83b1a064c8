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


def vec_rel(got, ref):
    """max over cells and components of |u_got - u_ref| over max |u_ref|: the
    velocity is one vector field, so every component is measured against the
    field's max-norm (the small transverse components would otherwise turn
    rounding noise of ~1e-9 into a large per-component relative error)."""
    a = np.stack([np.asarray(got[k], np.float64) for k in ("ux", "uy", "uz")])
    b = np.stack([np.asarray(ref[k], np.float64) for k in ("ux", "uy", "uz")])
    scale = float(np.abs(b).max())
    return float(np.abs(a - b).max()) / scale if scale else float(np.abs(a).max())


def field_errors(got, ref):
    """Relative errors of rho, u (vector max-norm), C and q."""
    return {"rho": max_rel(got["rho"], ref["rho"]), "u": vec_rel(got, ref),
            "phi": max_rel(got["phi"], ref["phi"]), "q": max_rel(got["q"], ref["q"])}
