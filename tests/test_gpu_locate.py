"""Batched locate on the GPU engine (marked gpu): one engine serves every sweep
of a locate (agent.py:406-477) and its zoomed result equals what a fresh
engine, assembled for the zoom band as the reference's ``run`` would be, gives;
on a damped engine the Q stage's windows agree with the oracle's sweep of the
same windows."""
import numpy as np
import pytest

from helpers import oracle_engine
from oracle import q9 as oq9
from sawsim_b200 import cases
from sawsim_b200.engine import FrequencySolver
from sawsim_b200.locate import locate
from sawsim_b200.materials import Material
from sawsim_b200.metrics import peak_quality_extrapolated, resonances

pytestmark = pytest.mark.gpu


def test_locate_reuses_the_analysis_and_matches_a_fresh_engine(built_lib):
    case = cases.make_case('me1_64x256', cols=8, rows=16)
    g = cases.engine_for(case)
    try:
        s0 = g.stats()
        r = locate(g, 1.6, 2.0, 101, (1.5, 2.2), zoom_points=61, precision='fp64')
        assert r['ok'], r
        s1 = g.stats()
        assert r['sweeps'] >= 2
        # no new analysis: the symbolic counters are those of the construction
        assert s1['analyze_s'] == s0['analyze_s'] and s1['n_fronts'] == s0['n_fronts']
        zs, ze = r['band_ghz']
        fresh_case = cases.make_case('me1_64x256', cols=8, rows=16, points=61, f0=zs * 1e9, f1=ze * 1e9)
        fresh = cases.engine_for(fresh_case)
        try:
            w = 2 * np.pi * fresh_case.freqs
            Qf, st, _ = fresh.charges(w, 1.0, 'fp64')
            Qg, st2, _ = g.charges(w, 1.0, 'fp64')
        finally:
            fresh.close()
        assert (st == 0).all() and (st2 == 0).all()
        assert np.max(np.abs(Qg - Qf) / np.abs(Qf)) < 1e-10
        rf = resonances(fresh_case.freqs, -1j * w * Qf)
        assert rf['fr_ghz'] == r['fr_ghz'] and rf['fa_ghz'] == r['fa_ghz']
    finally:
        g.close()


BETA = 1e-13        # the reference's lossy test setting (tests/test_quality.py:38)


def _damping_materials(mats):
    """The reference's damping set: the piezo material's C only (solver.py:111-113)."""
    return [Material(m.rho, m.C, 0 * m.e, 0 * m.eps) if i == 0 else Material(m.rho, 0 * m.C, 0 * m.e, 0 * m.eps)
            for i, m in enumerate(mats)]


def _oracle_window(cols, rows, lo_ghz, hi_ghz, points):
    """The oracle's damped sweep of one window, assembled with the PML frozen at the
    window's top as the reference's run does (solver.py:104-115)."""
    c = cases.make_case('me1_64x256', cols=cols, rows=rows, points=points, f0=lo_ghz * 1e9, f1=hi_ghz * 1e9)
    _, _, o = oracle_engine(c)
    m = oq9.build_model(c.cell.msh())
    pml = [oq9.PMLRegion(tag=p.tag, kind=p.kind, ya=p.ya, yp=p.yp) for p in c.pml]
    D, _ = oq9.assemble(m, _damping_materials(c.materials), c.mat_idx, pml, c.omega_top)
    o.set_damping(D, BETA)
    return c.freqs, o.sweep(c.freqs)


def test_lossy_locate_with_q_matches_the_oracle(built_lib):
    """Locate with the Q stage (agent.py:386-403, :332-383) on a damped GPU engine:
    q_r and q_a resolved, and the final window of each Q stage, swept again by the
    oracle (SuperLU with the reference's set_damping), gives the same Q (1e-5) and
    peak frequency (1 Hz)."""
    case = cases.make_case('me1_64x256', cols=8, rows=16)
    g = FrequencySolver.from_q9(case.mesh, case.materials, case.mat_idx, case.pml, case.omega_top, case.bc,
                                mode_extension=case.mode_extension,
                                damping_materials=_damping_materials(case.materials), beta=BETA)
    try:
        r = locate(g, 1.6, 2.0, 101, (1.5, 2.2), zoom_points=61, precision='fp64', with_q=True)
    finally:
        g.close()
    assert r['ok'] and r.get('q_r') and r.get('q_a'), r
    for part, kind in (('resonance', 'r'), ('antiresonance', 'a')):
        q = r['quality'][part]
        assert q['q'] is not None, q
        h = q['history'][-1]
        f, Qo = _oracle_window(8, 16, h['window_ghz'][0], h['window_ghz'][1], h['points'])
        mag2 = np.abs(-1j * 2 * np.pi * f * Qo) ** 2
        pq = peak_quality_extrapolated(f, mag2 if kind == 'r' else 1.0 / np.maximum(mag2, 1e-300))
        assert abs(pq['q'] - q['q']) <= 1e-5 * q['q'], (part, pq['q'], q['q'])
        assert abs(pq['f0_hz'] * 1e-9 - q['f_ghz']) < 1e-9
