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


def revolve_cost(l, c):
    """Forward steps needed to reverse l steps from a held start state with c
    state buffers (binomial checkpointing): t(l, c) = r l - C(c + r, r - 1),
    r the least repetition number with C(c + r, c) >= l; l(l-1)/2 for c = 1."""
    from math import comb

    if l <= 1:
        return 0
    if c == 1:
        return l * (l - 1) // 2
    r = 1
    while comb(c + r, c) < l:
        r += 1
    return r * l - comb(c + r, r - 1)
