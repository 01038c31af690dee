"""GPU parity against the oracle, through the C ABI (marked gpu).

Bars: global K/M pattern bit-exact and values within 1e-12 of each component
block's max; condensed Km_aa/Mm_aa within 1e-12 per block (absent oracle entries
= 0); charges Q within 1e-7 relative (FP64) and 1e-6 relative (mixed precision
with FP64 refinement) of the oracle's SuperLU solve.
"""
import numpy as np
import pytest

from conftest import GOLDEN
from helpers import block_rel_err, oracle_engine
from sawsim_b200 import _lib as L, cases, cells
from sawsim_b200.engine import FrequencySolver
from sawsim_b200.materials import Material

pytestmark = pytest.mark.gpu

SMALL = [('me0_16x64', 8, 16), ('me1_64x256', 8, 16), ('me1_128x512', 8, 20)]


@pytest.fixture(scope='module', params=SMALL, ids=lambda p: f'{p[0]}_{p[1]}x{p[2]}')
def pair(request, built_lib):
    name, cols, rows = request.param
    case = cases.make_case(name, cols=cols, rows=rows)
    K, M, oeng = oracle_engine(case)
    geng = cases.engine_for(case)
    yield case, K, M, oeng, geng
    geng.close()


def _comp(case, n):
    return np.arange(n) // case.mesh.N


def test_global_pattern_and_values(pair):
    case, K, M, _, g = pair
    nc = 4 if case.mode_extension else 3
    comp = _comp(case, K.shape[0])
    for which, ref in ((L.SS_MAT_K, K), (L.SS_MAT_M, M)):
        A = g.export(which)
        ref = ref.tocsr()
        ref.sort_indices()
        assert np.array_equal(A.indptr, ref.indptr)
        assert np.array_equal(A.indices, ref.indices)
        assert block_rel_err(A, ref, comp, comp, nc) <= 1e-12


def test_condensed_matrices(pair):
    case, _, _, o, g = pair
    nc = 4 if case.mode_extension else 3
    comp = o.active // case.mesh.N
    for which, ref in ((L.SS_MAT_KC, o.Km_aa), (L.SS_MAT_MC, o.Mm_aa)):
        A = g.export(which)
        assert A.shape == ref.shape
        assert block_rel_err(A, ref.tocsr(), comp, comp, nc) <= 1e-12
    assert g.n_active == o.n_active


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-7), ('mixed', 1e-6)])
def test_charges_match_oracle(pair, precision, tol):
    case, _, _, o, g = pair
    f = np.linspace(case.freqs[0], case.freqs[-1], 7)
    Qo = o.sweep(f)
    Q, st, it = g.charges(2 * np.pi * f, 1.0, precision)
    assert (st == 0).all(), st
    assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < tol


def test_repeat_is_bitwise_identical(pair):
    case, _, _, _, g = pair
    w = 2 * np.pi * case.freqs[[0, -1]]
    Q1, _, _ = g.charges(w, 1.0, 'fp64')
    Q2, _, _ = g.charges(w, 1.0, 'fp64')
    assert np.array_equal(Q1, Q2)


def test_fields_match_oracle(pair):
    case, _, _, o, g = pair
    w = 2 * np.pi * case.freqs[len(case.freqs) // 2]
    d_o, Q_o, Y_o = o.solve(w, 1.0)
    d_g, Q_g, Y_g = g.solve(w, 1.0)
    assert np.max(np.abs(d_g - d_o)) <= 1e-7 * np.max(np.abs(d_o))
    assert abs(Y_g - Y_o) <= 1e-7 * abs(Y_o)


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-7), ('mixed', 1e-6)])
def test_adjoint_solves_transposed_system(pair, precision, tol):
    """A_aa^T lambda = kq (the folded charge row) on the oracle's own matrices, and
    lambda agrees with a SuperLU solve of the transposed system."""
    import scipy.sparse.linalg as spla
    case, _, _, o, g = pair
    w = 2 * np.pi * case.freqs[len(case.freqs) // 3]
    A, _ = o.system(w)
    kq = (o._T.T @ o.kts)[o.active]
    g.set_option('krylov_tol', 1e-10)         # the adjoint alone, at a tight Krylov target
    try:
        lam = g.solve_adjoint(w, precision)
    finally:
        g.set_option('krylov_tol', 1e-8)
    At = A.T.tocsr()
    eta = np.linalg.norm(At @ lam - kq, np.inf) / (abs(At).sum(axis=1).max() * np.linalg.norm(lam, np.inf) +
                                                   np.linalg.norm(kq, np.inf))
    # normwise backward error: FP64 direct + refinement, or the mixed Krylov target
    assert eta <= (1e-12 if precision == 'fp64' else 1e-10)
    ref = spla.splu(A.T.tocsc()).solve(kq)
    assert np.max(np.abs(lam - ref)) <= tol * np.max(np.abs(ref))


@pytest.mark.parametrize('name', ['sp_double_layer', 'sp_quad_layer'])
def test_template_published_curve(built_lib, name):
    """The rebuilt sp_double_layer and sp_quad_layer templates reproduce the
    reference's published curves at their 5 test frequencies on the GPU FP64 path."""
    gl = np.load(GOLDEN / f'{name}.npz')
    cell = {'sp_double_layer': cells.sp_double_layer_cell, 'sp_quad_layer': cells.sp_quad_layer_cell}[name]()
    mesh = cases.mesh_from_msh(cell.msh())
    mats = [Material(gl['rho'][i], gl['C'][i], gl['e'][i], gl['eps'][i]) for i in range(len(gl['rho']))]
    idx = np.array([cell.tag_map[t] for t in mesh.elem_tag])
    bottom = mesh.pos_m[:, 1].min()
    pml = [cases.PML(tag=cell.pml_tag, kind='y', yp=bottom, ya=bottom + 2 * float(gl['pitch_um']) * 1e-6)]
    f = gl['frequency_hz']
    eng = FrequencySolver.from_q9(mesh, mats, idx, pml, 2 * np.pi * f[-1], cases.bc_periodic(mesh, cell.LINES3, 3))
    Y = -1j * 2 * np.pi * f * eng.sweep(f)
    pub = gl['published_magnitude']
    assert np.max(np.abs(np.abs(Y) - pub) / pub) < 1e-8
    eng.close()


def test_auto_precision_picks_a_converging_mode(pair):
    """SS_PREC_AUTO probes the mixed path; whichever it keeps, Q matches FP64."""
    case, _, _, _, g = pair
    w = 2 * np.pi * np.linspace(case.freqs[0], case.freqs[-1], 5)
    Q64, _, _ = g.charges(w, 1.0, 'fp64')
    Qa, st, _ = g.charges(w, 1.0, 'auto')
    assert (st == 0).all()
    assert int(g.stats()['precision_used']) in (0, 1)
    assert np.max(np.abs(Qa - Q64) / np.abs(Q64)) < 1e-6
    # the decision is kept for the same band: a repeated AUTO sweep runs the same
    # mode without probing (fewer launches) and gives the same charges
    used, launches = int(g.stats()['precision_used']), g.stats()['launches']
    Qb, st, _ = g.charges(w, 1.0, 'auto')
    assert (st == 0).all()
    assert int(g.stats()['precision_used']) == used
    assert g.stats()['launches'] < launches
    assert np.max(np.abs(Qa - Qb) / np.abs(Qa)) < 1e-12
    # another band probes again
    g.charges(w[:3], 1.0, 'auto')
    assert int(g.stats()['precision_used']) in (0, 1)
