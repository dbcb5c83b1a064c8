"""Differentiable breakthrough curve: a thin ``torch.autograd.Function`` over
``fm_adjoint_breakthrough``.

:func:`breakthrough_loss` maps the isotherm parameters ``(q_max, b, k_ldf)``
(Langmuir; ``(K_henry, 0, k_ldf)`` for the linear isotherm) and the per-cell
solid fraction ``n_s`` (porosity ``1 - n_s``, porous collision) to the loss
``sum_i (C_out(i P) - target_i)^2`` of a problem run from equilibrium.  The
forward pass runs the CUDA forward step with checkpoints and the hand-written
adjoint kernels in one library call, so ``backward`` only scales the cached
gradients by the incoming gradient.  The region mask (``n_s > 0.5`` in the
smooth porous problem) is a fixed input: it is not differentiated.
"""
from __future__ import annotations

import numpy as np

from . import lattice as _lattice


def _set_parameters(L, problem, params, n_s):
    solid, region, _, _ = problem.masks()
    if problem.isotherm == "langmuir":
        L.set_isotherm_langmuir(region, float(params[0]), float(params[1]), float(params[2]))
    elif problem.isotherm == "linear":
        L.set_isotherm_linear(region, float(params[0]), float(params[2]))
    else:
        raise ValueError("breakthrough_loss: the problem has no isotherm")
    if n_s is not None:
        if problem.collision != "porous":
            raise ValueError("breakthrough_loss: n_s needs the porous collision")
        L.set_porosity(1.0 - np.asarray(n_s, dtype=np.float64).reshape(-1))
    L.init_equilibrium()


def breakthrough_loss_np(L, problem, params, n_s, target, nsteps=None, checkpoint_every=0, max_stored_states=0):
    """NumPy form: returns ``(loss, dL/dparams[3], dL/dn_s or None)``."""
    _set_parameters(L, problem, params, n_s)
    steps = problem.steps if nsteps is None else nsteps
    loss, gp, gpor = L.adjoint_breakthrough(steps, target, checkpoint_every, max_stored_states,
                                            porosity_grad=n_s is not None)
    return loss, gp, (None if gpor is None else -gpor)


def _function():
    import torch

    class BreakthroughLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params, n_s, L, problem, target, nsteps, checkpoint_every, max_stored_states):
            ns_np = None if n_s is None else n_s.detach().cpu().double().numpy()
            loss, gp, gns = breakthrough_loss_np(L, problem, params.detach().cpu().double().numpy(), ns_np,
                                                 target, nsteps, checkpoint_every, max_stored_states)
            ctx.gp = torch.as_tensor(gp, dtype=params.dtype, device=params.device)
            ctx.gns = None if gns is None else torch.as_tensor(gns, dtype=n_s.dtype, device=n_s.device).view_as(n_s)
            return torch.tensor(loss, dtype=params.dtype, device=params.device)

        @staticmethod
        def backward(ctx, g):
            gns = None if ctx.gns is None else g * ctx.gns
            return g * ctx.gp, gns, None, None, None, None, None, None

    return BreakthroughLoss


_FN = None


def breakthrough_loss(params, n_s, problem, target, lattice=None, precision="f64", nsteps=None, checkpoint_every=200,
                      max_stored_states=0):
    """Differentiable loss of `problem`'s breakthrough curve against `target`.

    params: tensor [3]; n_s: tensor [N] or None; target: array of the sampled
    outlet means C_out(P), C_out(2P), ...  `lattice` (from
    :func:`fluidmaxxer_b200.lattice.from_problem`) is reused when given."""
    global _FN
    if _FN is None:
        _FN = _function()
    L = lattice if lattice is not None else _lattice.from_problem(problem, precision)
    return _FN.apply(params, n_s, L, problem, np.asarray(target, dtype=np.float64), nsteps, checkpoint_every,
                     max_stored_states)
