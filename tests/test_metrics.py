"""fr/fa extraction (sawsim_b200.metrics) against the reference's own extractor
(src/sawsim/metrics.py:84-171) on its stored template curves and synthetic
lossless and lossy resonators (tests/golden/metrics_curves.npz, made by
make_metrics_golden.py).  CPU only."""
import json
import math

import numpy as np
import pytest

from conftest import GOLDEN
from sawsim_b200.metrics import compare, resonances

_G = np.load(GOLDEN / 'metrics_curves.npz')
_META = json.loads(str(_G['meta']))


@pytest.mark.parametrize('i', range(len(_META)), ids=[m['name'] for m in _META])
def test_matches_reference_extractor(i):
    """The whole result: fr / fa / k2eff, the coarse q_r / q_a, the mode list,
    warning codes and notes."""
    ref = dict(_META[i])
    ref.pop('name')
    assert resonances(_G[f'f{i}'], _G[f'y{i}']) == ref


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
