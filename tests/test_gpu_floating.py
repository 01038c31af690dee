"""Finite-device boundary sets with floating electrodes (sweep.bc_floating,
sweep.py:75-91) through the GPU engine, against the oracle (marked gpu).

The structured cell's line sets stand in for a finite device: the left and right
edge nodes become the two floating electrodes (each one equipotential group of
phi DOFs, folded into its first node), the bottom is clamped, the + and -
electrodes are driven as usual.  Without the Bloch pairs the clamped cell with
free sides is ill-conditioned: two backward-stable solvers (this library's and
SciPy SuperLU) differ in Q by about 1e-5 relative.  Bars: the condensed system's
size equals the oracle's; the FP64 solution's normwise backward error in the
oracle's own system below 1e-12; Q within 1e-4 of the oracle's SuperLU solve;
mixed within 1e-6 of FP64.
"""
import numpy as np
import pytest

from oracle import q9 as oq9, solver as osol
from sawsim_b200 import cases
from sawsim_b200.engine import FrequencySolver

pytestmark = pytest.mark.gpu


def test_floating_electrodes_match_oracle(built_lib):
    case = cases.make_case('me1_64x256', cols=8, rows=16, points=5)
    bc = cases.bc_floating(case.mesh, case.cell.LINES3, 3, tag_bottom=21, tag_xfl=19, tag_xfr=20, tag_zheng=17,
                           tag_fu=18)
    assert all(g.size > 2 for g in bc[3])
    m = oq9.build_model(case.cell.msh())
    pml = [oq9.PMLRegion(tag=p.tag, kind=p.kind, ya=p.ya, yp=p.yp) for p in case.pml]
    K, M = oq9.assemble(m, case.materials, case.mat_idx, pml, case.omega_top)
    o = osol.FrequencySolver(K, M, *bc)
    g = FrequencySolver.from_q9(case.mesh, case.materials, case.mat_idx, case.pml, case.omega_top, bc)
    try:
        assert g.n_active == o.n_active
        w = 2 * np.pi * case.freqs
        Q, st, _ = g.charges(w, 1.0, 'fp64')
        assert (st == 0).all()
        Qo = o.sweep(case.freqs)
        assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < 1e-4
        for wi in w[[0, -1]]:
            A, rhs = o.system(wi)
            disp, q, _ = g.solve(wi)
            x = disp[o.active]
            r = A @ x - rhs
            eta = np.linalg.norm(r, np.inf) / (abs(A).sum(axis=1).max() * np.linalg.norm(x, np.inf) +
                                               np.linalg.norm(rhs, np.inf))
            assert eta < 1e-12
        Qm, stm, _ = g.charges(w, 1.0, 'mixed')
        assert (stm == 0).all() and g.stats()['fp64_resolved'] == 0
        assert np.max(np.abs(Qm - Q) / np.abs(Q)) < 1e-6
    finally:
        g.close()
