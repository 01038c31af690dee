"""Batched locate on the GPU engine (marked gpu): one engine serves every sweep
of a locate (agent.py:406-477) and its zoomed result equals what a fresh
engine, assembled for the zoom band as the reference's ``run`` would be, gives."""
import numpy as np
import pytest

from sawsim_b200 import cases
from sawsim_b200.locate import locate
from sawsim_b200.metrics import resonances

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
