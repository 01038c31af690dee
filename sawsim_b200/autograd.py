"""PyTorch surface of the adjoint: Y11 as a differentiable function of cell parameters.

``y11(params, model, freqs)`` returns the admittance Y11 of the cell
``model.build(params)`` at ``freqs`` (Hz): -i w Q / V for the 2D Q9 cells
(src/sawsim/solver.py:128), +i w Q / V / aperture for the Hex27 slabs
(src/sawsim/hex_solver.py:103)
as a complex128 tensor; its backward pass returns dL/dparams from the adjoint
gradient computed with the same factorisation (``ss_adjoint_gradient``).  Torch is
only the autograd surface: the sweep and the gradient run in libsawsim_b200.so.
"""
from __future__ import annotations

import numpy as np
import torch


def y11_and_jacobian(model, params, freqs, precision='fp64', V=1.0, device=0, stats=None):
    """(Y[n_f], dY/dp[n_f, n_params], status) at parameters ``params`` of a
    ``params.Q9Model`` or ``params.HexModel`` (the model fixes the Y11 sign and
    normalisation of its pipeline).  A dict passed as ``stats`` receives the
    engine's counters (``FrequencySolver.stats``) of the run."""
    p = np.asarray(params, dtype=float)
    case = model.build(p)
    eng = model.engine(case, device=device)
    try:
        w = 2 * np.pi * np.asarray(freqs, dtype=float)
        Q, dQ, st = eng.gradient(w, model.seeds(p), V, precision)
        if stats is not None:
            stats.update(eng.stats())
    finally:
        eng.close()
    Y = model.y11(w, Q, V, case)
    dY = model.y11(w[:, None], dQ, V, case)
    return Y, dY, st


def y11_only(model, params, freqs, precision='fp64', V=1.0, device=0):
    """(Y[n_f], status) at parameters ``params``: the sweep alone, no adjoint."""
    p = np.asarray(params, dtype=float)
    case = model.build(p)
    eng = model.engine(case, device=device)
    try:
        w = 2 * np.pi * np.asarray(freqs, dtype=float)
        Q, st, _ = eng.charges(w, V, precision)
    finally:
        eng.close()
    return model.y11(w, Q, V, case), st


class Y11Sweep(torch.autograd.Function):
    """Forward: Y11 at every frequency; backward: the adjoint Jacobian product."""

    @staticmethod
    def forward(ctx, params, model, freqs, precision):
        p = params.detach().cpu().numpy()
        if ctx.needs_input_grad[0]:
            Y, dY, st = y11_and_jacobian(model, p, freqs, precision)
        else:               # no backward can follow: the sweep alone
            (Y, st), dY = y11_only(model, p, freqs, precision), None
        if (st != 0).any():
            raise RuntimeError(f'sweep did not converge at {int((st != 0).sum())} points')
        ctx.save_for_backward(torch.from_numpy(dY) if dY is not None else torch.empty(0))
        ctx.param_dtype = params.dtype
        return torch.from_numpy(Y)

    @staticmethod
    def backward(ctx, grad_y):
        (dY,) = ctx.saved_tensors
        # real parameters, complex outputs: dL/dp = Re(sum_f conj(g_f) dY_f/dp)
        g = (grad_y.conj().unsqueeze(1) * dY).real.sum(0)
        return g.to(ctx.param_dtype), None, None, None


def y11(params: torch.Tensor, model, freqs, precision: str = 'fp64') -> torch.Tensor:
    """Differentiable Y11(params) of a ``params.Q9Model`` at ``freqs`` (Hz)."""
    return Y11Sweep.apply(params, model, freqs, precision)
