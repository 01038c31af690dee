"""Loss path on the GPU against the oracle (marked gpu): Rayleigh stiffness
damping A = K + i w beta D - w^2 M with D the elastic K_uu of the piezo material
only (solver.py:109-115, sweep.py:316-323), and dielectric loss eps (1 - i eta)
on the piezo material (models.py:68-70).  Bars: Q within 1e-7 of the oracle's
SuperLU solve (FP64) and mixed within 1e-6 of FP64, on small ME1 and ME0 cells.
"""
import numpy as np
import pytest

from helpers import oracle_engine
from oracle import q9 as oq9
from sawsim_b200 import cases
from sawsim_b200.engine import FrequencySolver
from sawsim_b200.materials import Material

pytestmark = pytest.mark.gpu

BETA = 2e-12


def _damping_materials(mats):
    """The reference's damping set: the piezo material's C only (solver.py:111-113)."""
    return [Material(m.rho, m.C, 0 * m.e, 0 * m.eps) if i == 0 else Material(m.rho, 0 * m.C, 0 * m.e, 0 * m.eps)
            for i, m in enumerate(mats)]


@pytest.mark.parametrize('name', ['me1_64x256', 'me0_16x64'])
def test_rayleigh_damping_matches_oracle(built_lib, name):
    case = cases.make_case(name, cols=8, rows=16, points=5)
    _, _, o = oracle_engine(case)
    m = oq9.build_model(case.cell.msh())
    pml = [oq9.PMLRegion(tag=p.tag, kind=p.kind, ya=p.ya, yp=p.yp) for p in case.pml]
    asm = oq9.assemble if case.mode_extension else oq9.assemble_me0
    D, _ = asm(m, _damping_materials(case.materials), case.mat_idx, pml, case.omega_top)
    o.set_damping(D, BETA)
    g = FrequencySolver.from_q9(case.mesh, case.materials, case.mat_idx, case.pml, case.omega_top, case.bc,
                                mode_extension=case.mode_extension,
                                damping_materials=_damping_materials(case.materials), beta=BETA)
    try:
        w = 2 * np.pi * case.freqs
        Q, st, _ = g.charges(w, 1.0, 'fp64')
        assert (st == 0).all()
        Qo = o.sweep(case.freqs)
        assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < 1e-7
        # the loss is visible: undamped charges differ
        _, _, o0 = oracle_engine(case)
        assert np.max(np.abs(o0.sweep(case.freqs[:2]) - Qo[:2]) / np.abs(Qo[:2])) > 1e-6
        Qm, stm, _ = g.charges(w, 1.0, 'mixed')
        assert (stm == 0).all()
        assert np.max(np.abs(Qm - Q) / np.abs(Q)) < 1e-6
    finally:
        g.close()


def test_dielectric_loss_matches_oracle(built_lib):
    case = cases.make_case('me1_64x256', cols=8, rows=16, points=5)
    eta = 0.01
    p = case.materials[0]
    case.materials[0] = Material(p.rho, p.C, p.e, p.eps * (1 - 1j * eta))
    _, _, o = oracle_engine(case)
    g = cases.engine_for(case)
    try:
        Q, st, _ = g.charges(2 * np.pi * case.freqs, 1.0, 'fp64')
        assert (st == 0).all()
        Qo = o.sweep(case.freqs)
        assert np.max(np.abs(Q - Qo) / np.abs(Qo)) < 1e-7
    finally:
        g.close()
