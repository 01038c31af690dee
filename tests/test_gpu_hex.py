"""Hex27 slab on the GPU against the Hex27 oracle (marked gpu).

Bars: global K/M pattern bit-exact and values within 1e-12 of each component
block's max; condensed k_aa/m_aa within 1e-12 (absent oracle entries = 0); the
FP64 solution's normwise backward error in the oracle's own system < 1e-12 and
Q within 2e-5 of the oracle's SuperLU solve (the unscaled 3D systems have
condition numbers near 3e15, so rounding-level differences in K move Q by up
to ~5e-6); mixed precision within 1e-6 of FP64.
"""
import numpy as np
import pytest

from helpers import block_rel_err
from oracle import hex27 as oh
from sawsim_b200 import _lib as L, cases

pytestmark = pytest.mark.gpu

SMALL = [(8, 1, 6), (8, 2, 12)]


def _oracle(c):
    pml_mask = c.cell.hex_tag == c.cell.pml_tag
    mats = [dict(rho=m.rho, C=m.C, e=m.e, eps=m.eps, indx=np.where((c.mat_idx == i) & ~pml_mask)[0])
            for i, m in enumerate(c.materials)]
    pm = c.materials[c.cell.tag_map[c.cell.pml_tag]]
    p = c.pml[0]
    pml = [dict(region=3, indx=np.where(pml_mask)[0], za=p.za, zp=p.zp, xa=0.0, xp=0.0, dmax=p.dmax, n=p.n,
                rho=pm.rho, C=pm.C, e=pm.e, eps=pm.eps)]
    M, K = oh.form_stiffness_mass_3d(c.hexas, c.pos_m, mats, pml, c.omega_top)
    return K, M, oh.FrequencySolver3D(K, M, oh.boundary_idx_vect_3ds(c.cell.sets, c.pos_m, 3 * c.N))


@pytest.fixture(scope='module', params=SMALL, ids=lambda s: f'{s[0]}x{s[1]}x{s[2]}')
def hexpair(request, built_lib):
    nx, ny, nz = request.param
    c = cases.make_hex_case('hex_8x4x48', nx=nx, ny=ny, nz=nz, points=5)
    K, M, o = _oracle(c)
    g = cases.hex_engine_for(c)
    yield c, K, M, o, g
    g.close()


def _comp(n, N):
    n = np.asarray(n)
    return np.where(n < 3 * N, n % 3, 3)


def test_hex_global_pattern_and_values(hexpair):
    c, K, M, _, g = hexpair
    comp = _comp(np.arange(4 * c.N), c.N)
    for which, ref in ((L.SS_MAT_K, K), (L.SS_MAT_M, M)):
        A = g.export(which)
        ref = ref.tocsr()
        ref.sort_indices()
        assert np.array_equal(A.indptr, ref.indptr)
        assert np.array_equal(A.indices, ref.indices)
        assert block_rel_err(A, ref, comp, comp, 4) <= 1e-12


def test_hex_condensed(hexpair):
    c, _, _, o, g = hexpair
    comp = _comp(o.active, c.N)
    for which, ref in ((L.SS_MAT_KC, o.k_aa), (L.SS_MAT_MC, o.m_aa)):
        A = g.export(which)
        assert A.shape == ref.shape
        assert block_rel_err(A, ref.tocsr(), comp, comp, 4) <= 1e-12
    assert g.n_active == o.n_active


def test_hex_fp64_backward_error_and_charges(hexpair):
    c, _, _, o, g = hexpair
    Qo = o.sweep(c.freqs)
    Q, st, _ = g.charges(2 * np.pi * c.freqs, 1.0, 'fp64')
    assert (st == 0).all()
    assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < 2e-5
    w = 2 * np.pi * c.freqs[2]
    A, rhs = o.system(w)
    disp, _, _ = g.solve(w)
    x = disp[o.active]
    r = A @ x - rhs
    eta = np.linalg.norm(r, np.inf) / (abs(A).sum(axis=1).max() * np.linalg.norm(x, np.inf) + np.linalg.norm(rhs, np.inf))
    assert eta < 1e-12


def test_hex_mixed_matches_fp64(hexpair):
    c, _, _, _, g = hexpair
    w = 2 * np.pi * c.freqs
    Q64, _, _ = g.charges(w, 1.0, 'fp64')
    Q32, st, _ = g.charges(w, 1.0, 'mixed')
    assert (st == 0).all(), st
    assert g.stats()['fp64_resolved'] == 0
    assert np.max(np.abs(Q32 - Q64) / np.abs(Q64)) < 1e-6
