"""fr/fa extraction (sawsim_b200.metrics) against the reference's own extractor
(src/sawsim/metrics.py:98-171) on its stored template curves and synthetic
resonators (tests/golden/metrics_curves.npz, made by make_metrics_golden.py).
CPU only."""
import json
import math

import numpy as np
import pytest

from conftest import GOLDEN
from sawsim_b200.metrics import compare, resonances

_G = np.load(GOLDEN / 'metrics_curves.npz')
_META = json.loads(str(_G['meta']))
# the warning codes this restatement keeps (Q and mode-list warnings are not restated)
_KEPT = {'peak_at_band_edge', 'no_resonance_found', 'antiresonance_not_found', 'coarse_sampling',
         'stronger_response_at_band_edge'}


@pytest.mark.parametrize('i', range(len(_META)), ids=[m['name'] for m in _META])
def test_matches_reference_extractor(i):
    ref = _META[i]
    r = resonances(_G[f'f{i}'], _G[f'y{i}'])
    assert r['fr_ghz'] == ref['fr_ghz']
    assert r['fa_ghz'] == ref['fa_ghz']
    assert r['k2eff'] == ref['k2eff']
    assert set(r['warnings']) == {w for w in ref['warnings'] if w in _KEPT}


def test_subgrid_lossless_pair():
    """Sub-sample fr/fa of a lossless pole/zero pair (tests/test_agent.py:22-28)."""
    f = np.linspace(1.6e9, 2.0e9, 201)
    fr, fa = 1.7512345e9, 1.8123456e9
    r = resonances(f, np.abs(f * (f ** 2 - fa ** 2) / (f ** 2 - fr ** 2)))
    assert abs(r['fr_ghz'] - fr * 1e-9) < r['uncertainty_mhz'] * 1e-3
    assert abs(r['fa_ghz'] - fa * 1e-9) < r['uncertainty_mhz'] * 1e-3
    assert r['k2eff'] == pytest.approx(math.pi ** 2 / 4 * (fa - fr) / fa, rel=1e-2)


def test_compare_is_zero_on_identical_curves():
    f = _G['f0']
    r = resonances(f, _G['y0'])
    d = compare(r, r)
    assert d['fr_diff_mhz'] == 0.0 and d['fa_diff_mhz'] == 0.0 and d['k2eff_diff_pct_points'] == 0.0
