"""The backend's drop-in classes on the GPU (marked gpu): the reference pipeline's
calls (``sweep.FrequencySolver(K, M, *bc)``, ``set_damping``, ``charge_stream``,
``solve`` at the peak, ``sweep`` returning ``(Q, |Y|)``; ``FrequencySolver3D(K, M,
boundary, t_fb, t_lr)`` with ``solve(omega, voltage=...)``) on the oracle's
assembled matrices, against the oracle's SuperLU route (bars as the matrix-input
tests: Q within 1e-7 in 2D, 2e-5 for Hex27)."""
import numpy as np
import pytest

from helpers import oracle_engine
from oracle import hex27 as oh, q9 as oq9, solver as osol
from sawsim_b200 import backend, cases

pytestmark = pytest.mark.gpu


def test_q9_pipeline_calls(built_lib):
    case = cases.make_case('me1_64x256', cols=8, rows=16, points=5)
    K, M, o = oracle_engine(case)
    m = oq9.build_model(case.cell.msh())
    bc = osol.bc_periodic(m, case.cell.LINES3, ndisp=3)
    eng = backend.FrequencySolver(K, M, *bc)
    try:
        assert eng.n_active == o.n_active and eng.precision == 'fp64'
        fre = case.freqs
        with backend.charge_stream(eng, fre, 1.0) as results:
            Q = np.array([next(results) for _ in fre])
        Qo = o.sweep(fre)
        assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < 1e-7
        Qs, Ys = eng.sweep(fre, 1.0, n_jobs=8, progress=False)
        assert np.array_equal(Qs, Q)
        assert np.allclose(Ys, np.abs(1j * 2 * np.pi * fre * Q))
        peak = int(np.argmax(Ys))
        disp, q, y = eng.solve(2 * np.pi * fre[peak], V=1.0)
        assert disp.shape == (K.shape[0],)
        assert abs(q - Q[peak]) <= 1e-12 * abs(Q[peak])
    finally:
        eng.close()


def test_hex_pipeline_calls(built_lib):
    from test_gpu_hex import _oracle
    c = cases.make_hex_case('hex_8x4x48', nx=8, ny=2, nz=12, points=3)
    K, M, o = _oracle(c)
    mach, elec = oh.boundary_idx_vect_3ds(c.cell.sets, c.pos_m, 3 * c.N)
    t_fb = oh._fold(np.concatenate([mach['period_B'], elec['period_B']]),
                    np.concatenate([mach['period_F'], elec['period_F']]), K.shape[0])
    t_lr = oh._fold(np.concatenate([mach['period_R'], elec['period_R']]),
                    np.concatenate([mach['period_L'], elec['period_L']]), K.shape[0])
    eng = backend.FrequencySolver3D(K, M, (mach, elec), t_fb, t_lr)
    try:
        assert eng.n_act == o.n_active
        with backend.charge_stream(eng, c.freqs, 1.0, is_hex=True) as results:
            Q = np.array([next(results) for _ in c.freqs])
        Qo = o.sweep(c.freqs)
        assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < 2e-5
        _, q, _ = eng.solve(2 * np.pi * c.freqs[1], voltage=1.0)
        assert abs(q - Q[1]) <= 1e-12 * abs(Q[1])
    finally:
        eng.close()
