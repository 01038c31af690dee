"""PyTorch surface of the adjoint: Y11 as a differentiable function of cell parameters.

``y11(params, model, freqs)`` returns the 2D admittance Y11 = -i w Q / V
(src/sawsim/solver.py:128) of the cell ``model.build(params)`` at ``freqs`` (Hz)
as a complex128 tensor; its backward pass returns dL/dparams from the adjoint
gradient computed with the same factorisation (``ss_adjoint_gradient``).  Torch is
only the autograd surface: the sweep and the gradient run in libsawsim_b200.so.
"""
from __future__ import annotations

import numpy as np
import torch

from . import cases


def y11_and_jacobian(model, params, freqs, precision='fp64', V=1.0, device=0):
    """(Y[n_f], dY/dp[n_f, n_params], status) at parameters ``params``."""
    p = np.asarray(params, dtype=float)
    case = model.build(p)
    eng = cases.engine_for(case, device=device)
    try:
        w = 2 * np.pi * np.asarray(freqs, dtype=float)
        Q, dQ, st = eng.gradient(w, model.seeds(p), V, precision)
    finally:
        eng.close()
    Y = -1j * w * Q / V
    dY = -1j * w[:, None] * dQ / V
    return Y, dY, st


class Y11Sweep(torch.autograd.Function):
    """Forward: Y11 at every frequency; backward: the adjoint Jacobian product."""

    @staticmethod
    def forward(ctx, params, model, freqs, precision):
        Y, dY, st = y11_and_jacobian(model, params.detach().cpu().numpy(), freqs, precision)
        if (st != 0).any():
            raise RuntimeError(f'sweep did not converge at {int((st != 0).sum())} points')
        ctx.save_for_backward(torch.from_numpy(dY))
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
