"""ctypes access to the oracle libraries (TEST INFRASTRUCTURE ONLY).

``Oracle(problem, impl="restated"|"reference", precision="f64"|"f32")`` runs
FluidMaxxer's coupled time step on the CPU:

* ``restated``  -- ``oracle/fm_oracle.c``, the plain-C restatement;
* ``reference`` -- the reference's own kernel bodies compiled for the host
  (``oracle/_ref``), driven in the reference loop order.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline arm use
this module; the product path never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class FmoConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("periodic_x", C.c_int), ("periodic_y", C.c_int), ("periodic_z", C.c_int),
        ("collision", C.c_int),
        ("rho0", C.c_double), ("tau", C.c_double),
        ("phi0", C.c_double), ("min_conc", C.c_double),
        ("ns_inlet", C.c_int), ("u_in", C.c_double * 3),
        ("ns_outlet", C.c_int), ("rho_out", C.c_double),
        ("ns_bounceback", C.c_int),
        ("ad_inlet", C.c_int), ("c_in", C.c_double),
        ("pulse_base", C.c_double), ("pulse_amp", C.c_double), ("pulse_k", C.c_double),
        ("pulse_on", C.c_int), ("pulse_off", C.c_int),
        ("ad_outlet", C.c_int),
        ("coupling", C.c_int),
        ("isotherm", C.c_int),
        ("k_henry", C.c_double), ("k_a", C.c_double),
        ("q_max", C.c_double), ("b_langmuir", C.c_double), ("k_ldf", C.c_double),
        ("sample_every", C.c_int),
    ]


class FmoInputs(C.Structure):
    _fields_ = [
        ("solid", C.c_void_p), ("porosity", C.c_void_p), ("tau_ad", C.c_void_p),
        ("region", C.c_void_p), ("inlet", C.c_void_p), ("outlet", C.c_void_p),
    ]


class FmoOutputs(C.Structure):
    _fields_ = [
        ("rho", C.c_void_p), ("ux", C.c_void_p), ("uy", C.c_void_p), ("uz", C.c_void_p),
        ("phi", C.c_void_p), ("q", C.c_void_p), ("sphi", C.c_void_p),
        ("f", C.c_void_p), ("g", C.c_void_p),
        ("c_out", C.c_void_p), ("c_out_cap", C.c_int), ("n_samples", C.c_int),
        ("sums", C.c_double * 4),
    ]


_LIBS: dict = {}


def _lib(impl: str, precision: str):
    key = (impl, precision)
    if key in _LIBS:
        return _LIBS[key]
    if impl == "restated":
        path, pre = os.path.join(HERE, f"libfmoracle_{precision}.so"), "fmo_"
    elif impl == "reference":
        path, pre = os.path.join(HERE, "_ref", f"libfmref_{precision}.so"), "fmo_ref_"
    else:
        raise ValueError(impl)
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library missing: {path} (run oracle/build_oracle.py)")
    lib = C.CDLL(path)
    fns = {}
    for name, res, args in (
        ("create", C.c_void_p, [C.POINTER(FmoConfig), C.POINTER(FmoInputs)]),
        ("set_state", C.c_int, [C.c_void_p] + [C.c_void_p] * 4),
        ("step", C.c_int, [C.c_void_p, C.c_int]),
        ("get", C.c_int, [C.c_void_p, C.POINTER(FmoOutputs)]),
        ("precision_bytes", C.c_int, []),
        ("destroy", None, [C.c_void_p]),
    ):
        fn = getattr(lib, pre + name)
        fn.restype = res
        fn.argtypes = args
        fns[name] = fn
    if impl == "reference":
        fn = lib.fmo_ref_threads
        fn.restype = C.c_int
        fns["threads"] = fn
    _LIBS[key] = fns
    return fns


def reference_available(precision: str = "f64") -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libfmref_{precision}.so"))


def _ptr(a):
    return None if a is None else a.ctypes.data


class Oracle:
    """One CPU lattice pair (NS + AD) advanced in the reference loop order."""

    def __init__(self, problem, impl: str = "restated", precision: str = "f64"):
        self.p = problem
        self.fn = _lib(impl, precision)
        cfg = FmoConfig()
        for k, v in problem.oracle_config().items():
            if k == "u_in":
                for i in range(3):
                    cfg.u_in[i] = float(v[i])
            else:
                setattr(cfg, k, v)
        self._keep = problem.oracle_arrays()
        a = self._keep
        ins = FmoInputs(_ptr(a["solid"]), _ptr(a["porosity"]), _ptr(a["tau_ad"]),
                        _ptr(a["region"]), _ptr(a["inlet"]), _ptr(a["outlet"]))
        self.h = self.fn["create"](C.byref(cfg), C.byref(ins))
        if not self.h:
            raise ValueError("oracle rejected the problem set-up")
        self.n = problem.n_cells

    def step(self, nsteps: int):
        if self.fn["step"](self.h, int(nsteps)) != 0:
            raise RuntimeError("oracle step failed")

    def set_state(self, f=None, g=None, phi=None, q=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (f, g, phi, q)]
        self.fn["set_state"](self.h, *[_ptr(a) for a in arrs])

    def get(self, populations: bool = False, max_samples: int = 1 << 16):
        n = self.n
        out = {k: np.empty(n) for k in ("rho", "ux", "uy", "uz", "phi", "q", "sphi")}
        if populations:
            out["f"] = np.empty(19 * n)
            out["g"] = np.empty(7 * n)
        c_out = np.empty(max_samples)
        o = FmoOutputs()
        for k in ("rho", "ux", "uy", "uz", "phi", "q", "sphi"):
            setattr(o, k, out[k].ctypes.data)
        if populations:
            o.f, o.g = out["f"].ctypes.data, out["g"].ctypes.data
        o.c_out, o.c_out_cap = c_out.ctypes.data, max_samples
        self.fn["get"](self.h, C.byref(o))
        out["c_out"] = c_out[: min(o.n_samples, max_samples)].copy()
        out["sums"] = np.array(list(o.sums))
        if populations:
            out["f"] = out["f"].reshape(19, n)
            out["g"] = out["g"].reshape(7, n)
        return out

    def close(self):
        if self.h:
            self.fn["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def reference_threads() -> int:
    return int(_lib("reference", "f32")["threads"]())
