"""Assembled-matrix input on the GPU (marked gpu): the reference engine's own
constructor arguments, ``sweep.FrequencySolver(K, M, fix, zheng, fu,
merge_groups)`` (src/sawsim/saw2d/sweep.py:283-314) and ``FrequencySolver3D(K, M,
boundary, t_fb, t_lr)`` (saw3d/bc_solve.py:108-136), fed with the oracle's
assembled matrices (pinned to the reference's own K and M).

Bars: Q within 1e-7 (2D) / 2e-5 (Hex27, as the mesh path; 1e-4 for the
finite-device variant, conditioned worse) of the oracle's
SuperLU solve and a normwise backward error below 1e-12 in the oracle's system,
with the graph nested dissection (no geometry) and with the node map and
coordinates (the mesh path's geometric ordering); with the mesh engine's own
matrices, node map and coordinates the sweep reproduces the mesh engine bit for
bit; Rayleigh damping by ``set_damping(D, beta)`` as the oracle's; new values
through ``update_matrices`` keep the analysis and equal a fresh engine's.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from helpers import oracle_engine
from oracle import hex27 as oh, q9 as oq9, solver as osol
from sawsim_b200 import _lib as L, cases
from sawsim_b200.engine import FrequencySolver

pytestmark = pytest.mark.gpu


def _backward_error(A, x, b):
    r = A @ x - b
    normA = abs(A).sum(axis=1).max()
    return np.linalg.norm(r, np.inf) / (normA * np.linalg.norm(x, np.inf) + np.linalg.norm(b, np.inf))


def _bc(case):
    m = oq9.build_model(case.cell.msh())
    return osol.bc_periodic(m, case.cell.LINES3, ndisp=3 if case.mode_extension else 2)


def _layout(case, K):
    N = case.mesh.pos_m.shape[0]
    return dict(dof_node=np.arange(K.shape[0]) % N, node_xyz=case.mesh.pos_m[:, :2])


@pytest.fixture(scope='module', params=['me1_64x256', 'me0_16x64'])
def q9(request, built_lib):
    case = cases.make_case(request.param, cols=8, rows=20, points=5)
    K, M, o = oracle_engine(case)
    return case, K, M, o


@pytest.mark.parametrize('ordering', ['graph', 'geometric'])
def test_matrix_input_matches_oracle(q9, ordering):
    case, K, M, o = q9
    lay = _layout(case, K) if ordering == 'geometric' else {}
    e = FrequencySolver.from_matrices(K, M, *_bc(case), **lay)
    try:
        assert e.n_active == o.n_active
        Q, st, _ = e.charges(2 * np.pi * case.freqs, 1.0, 'fp64')
        assert (st == 0).all()
        Qo = o.sweep(case.freqs)
        assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < 1e-7
        w = 2 * np.pi * case.freqs[2]
        A, rhs = o.system(w)
        disp, q, _ = e.solve(w)
        assert _backward_error(A, disp[o.active], rhs) < 1e-12
        # disp carries the prescribed potentials and the slaves' master values
        fix, zheng, fu, _ = _bc(case)
        assert np.allclose(disp[zheng], 1.0) and np.allclose(disp[fu], 0.0)
        Qm, stm, _ = e.charges(2 * np.pi * case.freqs, 1.0, 'mixed')
        assert (stm == 0).all()
        assert np.max(np.abs(Qm - Q) / np.abs(Q)) < 1e-6
    finally:
        e.close()


def test_graph_ordering_is_reported(q9):
    case, K, M, o = q9
    e = FrequencySolver.from_matrices(K, M, *_bc(case))
    g = FrequencySolver.from_matrices(K, M, *_bc(case), **_layout(case, K))
    try:
        fg, fm = e.stats()['factor_flops_per_point'], g.stats()['factor_flops_per_point']
        # the graph ordering costs more flops than the geometric one, within 1.6x
        assert fm <= fg < 1.6 * fm
    finally:
        e.close()
        g.close()


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
def test_mesh_engine_matrices_reproduce_mesh_engine(built_lib, precision, monkeypatch):
    monkeypatch.setenv('SS_SCHUR_TILE', '2')
    monkeypatch.setenv('SS_SCHUR_TILE_C64', '0')
    case = cases.make_case('me1_64x256', cols=8, rows=20, points=5)
    g = cases.engine_for(case)
    try:
        Kg, Mg = g.export(L.SS_MAT_K), g.export(L.SS_MAT_M)
        e = FrequencySolver.from_matrices(Kg, Mg, *case.bc, **_layout(case, Kg))
        try:
            w = 2 * np.pi * case.freqs
            Qg, _, _ = g.charges(w, 1.0, precision)
            Qe, st, _ = e.charges(w, 1.0, precision)
            assert (st == 0).all()
            assert np.array_equal(Qg, Qe)
            assert e.stats()['factor_flops_per_point'] == g.stats()['factor_flops_per_point']
        finally:
            e.close()
    finally:
        g.close()


BETA = 2e-12


def test_matrix_damping_matches_oracle(built_lib):
    from test_gpu_loss import _damping_materials
    case = cases.make_case('me1_64x256', cols=8, rows=16, points=5)
    K, M, o = oracle_engine(case)
    m = oq9.build_model(case.cell.msh())
    pml = [oq9.PMLRegion(tag=p.tag, kind=p.kind, ya=p.ya, yp=p.yp) for p in case.pml]
    D, _ = oq9.assemble(m, _damping_materials(case.materials), case.mat_idx, pml, case.omega_top)
    o.set_damping(D, BETA)
    e = FrequencySolver.from_matrices(K, M, *_bc(case))
    try:
        Q0, _, _ = e.charges(2 * np.pi * case.freqs, 1.0, 'fp64')
        e.set_damping(D, BETA)
        Q, st, _ = e.charges(2 * np.pi * case.freqs, 1.0, 'fp64')
        assert (st == 0).all()
        Qo = o.sweep(case.freqs)
        assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < 1e-7
        assert np.max(np.abs(Q0 - Qo) / np.abs(Qo)) > 1e-6      # the damping is visible
    finally:
        e.close()


def test_update_matrices_keeps_analysis(built_lib):
    """New K, M on the same pattern (the PML frozen at another top frequency) give
    the charges of a fresh engine built from them, with the analysis kept."""
    case = cases.make_case('me1_64x256', cols=8, rows=16, points=5)
    K, M, _ = oracle_engine(case)
    case2 = cases.make_case('me1_64x256', cols=8, rows=16, points=5, f1=1.1 * case.freqs[-1])
    K2, M2, o2 = oracle_engine(case2)
    e = FrequencySolver.from_matrices(K, M, *_bc(case))
    f = FrequencySolver.from_matrices(K2, M2, *_bc(case))
    try:
        w = 2 * np.pi * case.freqs
        e.charges(w, 1.0, 'fp64')
        t_an = e.stats()['analyze_s']
        e.update_matrices(K2, M2)
        assert e.stats()['analyze_s'] == t_an
        Qe, st, _ = e.charges(w, 1.0, 'fp64')
        Qf, _, _ = f.charges(w, 1.0, 'fp64')
        assert (st == 0).all()
        assert np.max(np.abs(Qe - Qf) / np.abs(Qf)) < 1e-12
        assert np.max(np.abs(Qe - o2.sweep(case.freqs)) / np.abs(Qe)) < 1e-7
        with pytest.raises(ValueError):
            e.update_matrices(K=K2 + sp.eye(K2.shape[0], k=K2.shape[0] - 1, dtype=complex))   # outside the pattern
    finally:
        e.close()
        f.close()


@pytest.mark.parametrize('ordering', ['graph', 'geometric'])
def test_hex_matrix_input_matches_oracle(built_lib, ordering):
    from test_gpu_hex import _oracle
    c = cases.make_hex_case('hex_8x4x48', nx=8, ny=2, nz=12, points=5)
    K, M, o = _oracle(c)
    m, e = oh.boundary_idx_vect_3ds(c.cell.sets, c.pos_m, 3 * c.N)
    t_fb = oh._fold(np.concatenate([m['period_B'], e['period_B']]), np.concatenate([m['period_F'], e['period_F']]),
                    K.shape[0])
    t_lr = oh._fold(np.concatenate([m['period_R'], e['period_R']]), np.concatenate([m['period_L'], e['period_L']]),
                    K.shape[0])
    n = np.arange(K.shape[0])
    lay = dict(dof_node=np.where(n < 3 * c.N, n // 3, n - 3 * c.N), node_xyz=c.pos_m) if ordering == 'geometric' else {}
    g = FrequencySolver.from_matrices_3d(K, M, (m, e), t_fb, t_lr, **lay)
    try:
        assert g.n_active == o.n_active
        Q, st, _ = g.charges(2 * np.pi * c.freqs, 1.0, 'fp64')
        assert (st == 0).all()
        Qo = o.sweep(c.freqs)
        assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < 2e-5
        w = 2 * np.pi * c.freqs[2]
        A, rhs = o.system(w)
        disp, _, _ = g.solve(w)
        assert _backward_error(A, disp[o.active], rhs) < 1e-12
    finally:
        g.close()


def test_hex_finite_device_matrix_input_matches_oracle(built_lib):
    """``FrequencySolver3D_FP(K, M, boundary, t_fb, t_float)`` (bc_solve.py:214-335): the
    finite-device variant, front/back periodic only, with two floating electrodes whose
    potentials fold onto one DOF each.  Its fold operators go to ``from_matrices_3d``
    unchanged.  The floating strips are the reference fixture's (surface nodes beside
    the driven pair: a synthetic finite device on the slab mesh, ref_hex_fp_8x2x12.npz)."""
    from conftest import GOLDEN
    from test_gpu_hex import _oracle
    c = cases.make_hex_case('hex_8x4x48', nx=8, ny=2, nz=12, points=3)
    ref = np.load(GOLDEN / 'ref_hex_fp_8x2x12.npz')
    K, M, _ = _oracle(c)
    m, e = oh.boundary_idx_vect_3ds(c.cell.sets, c.pos_m, 3 * c.N)
    e = dict(e, XFL=ref['XFL'], XFR=ref['XFR'])
    o = oh.FrequencySolver3DFP(K, M, (m, e))
    t_fb = oh._fold(np.concatenate([m['period_B'], e['period_B']]), np.concatenate([m['period_F'], e['period_F']]),
                    K.shape[0])
    t_float = oh.float_fold(e, K.shape[0])
    g = FrequencySolver.from_matrices_3d(K, M, (m, e), t_fb, t_float)
    try:
        assert g.n_active == o.n_active
        Q, st, _ = g.charges(2 * np.pi * c.freqs, 1.0, 'fp64')
        assert (st == 0).all()
        # without the left/right fold the system is conditioned worse than the
        # periodic slab's: two backward-stable solvers (this one, SuperLU) differ in Q
        # by up to ~3e-5 here; the backward error below is the exact bar
        Qo = o.sweep(c.freqs)
        assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < 1e-4
        assert np.max(np.abs(Q - ref['Q']) / np.abs(ref['Q'])) < 1e-4      # the reference's own solver
        w0 = 2 * np.pi * c.freqs[1]
        A, rhs = o.system(w0)
        disp, _, _ = g.solve(w0)
        assert _backward_error(A, disp[o.active], rhs) < 1e-12
        # the floating electrodes are equipotential
        for xs in (e['XFL'], e['XFR']):
            assert np.allclose(disp[xs], disp[xs[0]], rtol=0, atol=0)
    finally:
        g.close()
