"""Parity at the full sizes of the benchmarked configurations (marked gpu).

* ME0 16x64 (12.8k DOF, the CPU-runnable configuration): Q at 7 points of the
  101-point band within 1e-7 of the oracle's SuperLU solve (sweep.py:352-353),
  and the FP64 solution's normwise backward error in the oracle's own system
  below 1e-12 at three points.
* ME1 two-layer 64x256 (262k DOF, the benchmarked cell): backward error of the
  FP64 solution and of the FP64 adjoint in the oracle's own assembled and
  condensed system below 1e-12 at the band's first, middle and last points.  A
  SuperLU solve of this system takes minutes per point, and two backward-stable
  solvers of a system this ill-conditioned differ in Q well above 1e-7, so the
  size-independent backward error is the bar (sweep.py:335-364).
* Hex27 8x4x48 (49.7k DOF): the same backward-error bar at three points
  (bc_solve.py:154-175).
"""
import numpy as np
import pytest

from helpers import oracle_engine
from oracle import hex27 as oh
from sawsim_b200 import cases

pytestmark = pytest.mark.gpu


def backward_error(A, x, b):
    r = A @ x - b
    normA = abs(A).sum(axis=1).max()
    return np.linalg.norm(r, np.inf) / (normA * np.linalg.norm(x, np.inf) + np.linalg.norm(b, np.inf))


def test_me0_full_charges_and_backward_error(built_lib):
    case = cases.make_case('me0_16x64')
    _, _, o = oracle_engine(case)
    g = cases.engine_for(case)
    try:
        f = case.freqs[np.linspace(0, len(case.freqs) - 1, 7).astype(int)]
        Q, st, _ = g.charges(2 * np.pi * f, 1.0, 'fp64')
        assert (st == 0).all()
        Qo = o.sweep(f)
        assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < 1e-7
        for fi in f[[0, 3, 6]]:
            w = 2 * np.pi * fi
            A, rhs = o.system(w)
            disp, q, _ = g.solve(w)
            assert backward_error(A, disp[o.active], rhs) < 1e-12
            assert abs(q - Q[list(f).index(fi)]) <= 1e-12 * abs(q)
    finally:
        g.close()


@pytest.fixture(scope='module')
def me1_full(built_lib):
    case = cases.make_case('me1_64x256')
    _, _, o = oracle_engine(case)
    g = cases.engine_for(case)
    yield case, o, g
    g.close()


def test_me1_full_backward_error(me1_full):
    case, o, g = me1_full
    assert g.n_active == o.n_active == 262664
    f = case.freqs[[0, len(case.freqs) // 2, -1]]
    Q, st, _ = g.charges(2 * np.pi * f, 1.0, 'fp64')
    assert (st == 0).all()
    for i, fi in enumerate(f):
        w = 2 * np.pi * fi
        A, rhs = o.system(w)
        disp, q, _ = g.solve(w)
        assert backward_error(A, disp[o.active], rhs) < 1e-12, fi
        # the charge is the reference's kts . disp of the same solution
        _, Qo = o.charge(disp[o.active])
        assert abs(q - Qo) <= 1e-9 * abs(Qo)
        assert abs(Q[i] - q) <= 1e-9 * abs(q)


def test_me1_full_adjoint_backward_error(me1_full):
    case, o, g = me1_full
    w = 2 * np.pi * case.freqs[len(case.freqs) // 2]
    A, _ = o.system(w)
    kq = (o._T.T @ o.kts)[o.active]
    lam = g.solve_adjoint(w, 'fp64')
    assert backward_error(A.T.tocsr(), lam, kq) < 1e-12


def _hex_oracle(c):
    pml_mask = c.cell.hex_tag == c.cell.pml_tag
    mats = [dict(rho=m.rho, C=m.C, e=m.e, eps=m.eps, indx=np.where((c.mat_idx == i) & ~pml_mask)[0])
            for i, m in enumerate(c.materials)]
    pm = c.materials[c.cell.tag_map[c.cell.pml_tag]]
    p = c.pml[0]
    pml = [dict(region=3, indx=np.where(pml_mask)[0], za=p.za, zp=p.zp, xa=0.0, xp=0.0, dmax=p.dmax, n=p.n,
                rho=pm.rho, C=pm.C, e=pm.e, eps=pm.eps)]
    M, K = oh.form_stiffness_mass_3d(c.hexas, c.pos_m, mats, pml, c.omega_top)
    return oh.FrequencySolver3D(K, M, oh.boundary_idx_vect_3ds(c.cell.sets, c.pos_m, 3 * c.N))


def test_hex_full_backward_error(built_lib):
    c = cases.make_hex_case('hex_8x4x48')
    o = _hex_oracle(c)
    g = cases.hex_engine_for(c)
    try:
        assert g.n_active == o.n_active
        for fi in c.freqs[[0, len(c.freqs) // 2, -1]]:
            w = 2 * np.pi * fi
            A, rhs = o.system(w)
            disp, _, _ = g.solve(w)
            assert backward_error(A, disp[o.active], rhs) < 1e-12, fi
    finally:
        g.close()


def test_me1_full_thin_panel_tiles(me1_full, monkeypatch):
    """The benchmarked cell's tail panels (its 36-pivot leaves factor a 32-wide
    panel, then 4 pivots whose panel-step GEMMs are 4 columns wide / 4 rows high)
    with those GEMMs in thin SIMT 128x8 / 8x128 tiles beside the DMMA tiles: a
    backward error below 1e-12 in the oracle's system, and the charges of the
    DMMA-only panel GEMMs within 1e-8 (the same pivots, other rounding)."""
    case, o, _ = me1_full
    f = case.freqs[[0, len(case.freqs) // 2, -1]]
    monkeypatch.setenv('SS_SCHUR_TILE', '3')    # tuner off: C-staged DMMA Schur and panel tiles
    out = {}
    for thin in ('0', '1'):
        monkeypatch.setenv('SS_PANEL_THIN', thin)
        e = cases.engine_for(case)
        try:
            Q, st, _ = e.charges(2 * np.pi * f, 1.0, 'fp64')
            s = e.stats()
            if thin == '1':
                w = 2 * np.pi * f[1]
                A, rhs = o.system(w)
                disp, _, _ = e.solve(w)
        finally:
            e.close()
        assert (st == 0).all()
        assert s['panel_gemm_dmma'] == 3
        out[thin] = (Q, s['panel_thin_tiles'])
    assert out['0'][1] == 0 and out['1'][1] > 0
    assert backward_error(A, disp[o.active], rhs) < 1e-12
    assert np.max(np.abs(out['1'][0] - out['0'][0]) / np.abs(out['0'][0])) < 1e-8
