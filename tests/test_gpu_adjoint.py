"""Adjoint gradient dY11/dp on the GPU (marked gpu).

The ME1 two-layer cell at 8x16 elements, parameters: pitch, the three layer
thicknesses, the film's Euler angle theta and its six stiffness constants.
Bars: the adjoint Jacobian agrees with central finite differences of the GPU
sweep (relative step 1e-5) to 1e-4 of each parameter's largest entry, and with
central differences (relative step 1e-4) of the oracle's FP64 SuperLU sweep
(the reference's algorithm on the CPU) to 1e-4; the torch autograd surface returns
Re(sum_f conj(g_f) dY_f/dp).
"""
import numpy as np
import pytest

from helpers import oracle_engine
from sawsim_b200 import cases, params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def jac(built_lib):
    from sawsim_b200.autograd import y11_and_jacobian
    model = params.Q9Model(8, 16)
    v = model.defaults()
    f = np.linspace(1.6e9, 2.0e9, 5)
    Y, dY, st = y11_and_jacobian(model, v, f, 'fp64')
    assert (st == 0).all()
    return model, v, f, Y, dY


def _y_gpu(model, v, f):
    eng = cases.engine_for(model.build(v))
    try:
        Q, st, _ = eng.charges(2 * np.pi * f, 1.0, 'fp64')
    finally:
        eng.close()
    return -1j * 2 * np.pi * f * Q


def _y_oracle(model, v, f):
    _, _, o = oracle_engine(model.build(v))
    return -1j * 2 * np.pi * f * o.sweep(f)


def _fd(fn, model, v, f, i, rel=1e-5):
    h = rel * abs(v[i])
    vp, vm = v.copy(), v.copy()
    vp[i] += h
    vm[i] -= h
    return (fn(model, vp, f) - fn(model, vm, f)) / (2 * h)


@pytest.mark.parametrize('i', range(11), ids=params.GEOMETRY + params.MATERIAL)
def test_adjoint_matches_finite_differences(jac, i):
    model, v, f, Y, dY = jac
    fd = _fd(_y_gpu, model, v, f, i)
    assert np.max(np.abs(dY[:, i] - fd)) <= 1e-4 * np.max(np.abs(fd))


@pytest.mark.parametrize('i', [0, 1, 4, 5], ids=['pitch_um', 't_film_um', 'euler_theta_deg', 'C11'])
def test_adjoint_matches_oracle_fp64_gradient(jac, i):
    model, v, f, Y, dY = jac
    # the oracle's SuperLU solutions carry ~1e-9 relative noise at this
    # conditioning (independent factorisations at p +- h), which a 1e-5 step
    # amplifies to ~1e-4 of the derivative; a 1e-4 step keeps that noise and the
    # O(h^2) truncation both below 1e-5
    fd = _fd(_y_oracle, model, v, f, i, rel=1e-4)
    assert np.max(np.abs(dY[:, i] - fd)) <= 1e-4 * np.max(np.abs(fd))


def test_mixed_gradient_matches_fp64(jac):
    from sawsim_b200.autograd import y11_and_jacobian
    model, v, f, Y, dY = jac
    Y32, dY32, st = y11_and_jacobian(model, v, f, 'mixed')
    assert (st == 0).all()
    assert np.max(np.abs(dY32 - dY)) <= 1e-6 * np.max(np.abs(dY))


def test_torch_backward(jac):
    import torch
    from sawsim_b200.autograd import y11
    model, v, f, Y, dY = jac
    p = torch.tensor(v, dtype=torch.float64, requires_grad=True)
    y = y11(p, model, f)
    loss = (y.abs() ** 2).sum()
    loss.backward()
    expect = (2 * np.conj(Y)[:, None] * dY).real.sum(0)
    assert np.allclose(p.grad.numpy(), expect, rtol=1e-10, atol=0)


@pytest.fixture(scope='module')
def hex_jac(built_lib):
    from sawsim_b200.autograd import y11_and_jacobian
    model = params.HexModel(8, 2, 12, stack='double')
    v = model.defaults()
    f = np.linspace(1.6e9, 2.0e9, 4)
    Y, dY, st = y11_and_jacobian(model, v, f, 'fp64')
    assert (st == 0).all()
    return model, v, f, Y, dY


def _y_hex(model, v, f):
    case = model.build(v)
    eng = model.engine(case)
    try:
        Q, st, _ = eng.charges(2 * np.pi * f, 1.0, 'fp64')
    finally:
        eng.close()
    return model.y11(2 * np.pi * f, Q, 1.0, case)


@pytest.mark.parametrize('i', [0, 1], ids=['pitch_um', 't_film_um'])
def test_hex_adjoint_matches_finite_differences(hex_jac, i):
    """Hex27 slab (the parameters of the four-layer slab's gradient workload: pitch
    and film thickness): the adjoint
    Jacobian of Y11 = +i w Q / V / aperture against central differences."""
    model, v, f, Y, dY = hex_jac
    fd = _fd(_y_hex, model, v, f, i)
    assert np.max(np.abs(dY[:, i] - fd)) <= 1e-4 * np.max(np.abs(fd))


def test_hex_mixed_gradient_matches_fp64(hex_jac):
    from sawsim_b200.autograd import y11_and_jacobian
    model, v, f, Y, dY = hex_jac
    Y32, dY32, st = y11_and_jacobian(model, v, f, 'mixed')
    assert (st == 0).all()
    assert np.max(np.abs(dY32 - dY)) <= 1e-6 * np.max(np.abs(dY))
