"""Q extraction and the Q stage of a lossy locate (CPU).

* ``metrics.peak_quality`` / ``peak_quality_extrapolated`` against the
  reference's own functions (src/sawsim/metrics.py:38-81) on stored lossy
  resonator curves: identical results;
* ``locate.quality`` / ``add_quality`` against the reference's
  ``agent.quality`` / ``_add_quality`` (src/sawsim/agent.py:332-403), recorded on
  analytic lossy resonators by tests/golden/make_quality_golden.py: the same
  windows, Q and refined peaks (the stand-in engine below returns charges, so Y
  goes through Q = Y / (-i w) and back: agreement to rounding);
* the known answer of the reference's tests/test_quality.py:18-25: the
  extrapolated Q recovers the resonator's Q within 4e-3;
* ``locate(..., with_q=True)`` / ``converge`` end to end on the stand-in.
"""
import json
import math

import numpy as np
import pytest

from conftest import GOLDEN
from sawsim_b200.locate import add_quality, converge, locate, quality
from sawsim_b200.metrics import peak_quality, peak_quality_extrapolated

_G = json.loads((GOLDEN / 'quality_cases.json').read_text())


def resonator(f, fr, qr, fa, qa):
    """Lossy admittance with poles / zeros at fr (1 + i / 2 Qr), fa (1 + i / 2 Qa)."""
    pr, pa = fr * (1 + 0.5j / qr), fa * (1 + 0.5j / qa)
    return 1j * f * (f ** 2 - pa ** 2) / (f ** 2 - pr ** 2)


class Lossy:
    """Stand-in engine: charges whose passive-sign admittance -i w Q is the model's Y."""

    def __init__(self, *model):
        self.model = model
        self.sweeps = []

    def set_freeze_frequency(self, w):
        pass

    def charges(self, w, V=1.0, precision='auto'):
        f = w / (2 * np.pi)
        self.sweeps.append((f[0], f[-1], f.size))
        return resonator(f, *self.model) / (-1j * w) * V, np.zeros(f.size, np.int32), np.zeros(f.size, np.int32)

    def stats(self):
        return dict(sweep_device_ms=1.0, precision_used=0.0)


@pytest.mark.parametrize('c', _G['curves'], ids=[c['name'] for c in _G['curves']])
def test_peak_quality_matches_reference(c):
    f, p = np.array(c['f']), np.array(c['power'])
    assert peak_quality(f, p) == c['peak_quality']
    assert peak_quality_extrapolated(f, p) == c['peak_quality_extrapolated']


def _close_history(mine, ref):
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        assert a['window_ghz'] == pytest.approx(b['window_ghz'], abs=1e-9) and a['points'] == b['points']
        assert a['samples_in_linewidth'] == b['samples_in_linewidth']
        assert (a['q'] is None) == (b['q'] is None)
        if a['q'] is not None:
            assert a['q'] == pytest.approx(b['q'], rel=1e-9, abs=1e-3)


@pytest.mark.parametrize('c', _G['quality'], ids=[c['name'] for c in _G['quality']])
def test_quality_windows_match_reference(c):
    ref = c['result']
    r = quality(Lossy(*c['model']), c['f_ghz'], c['kind'], c['width'], tuple(c['limits']))
    _close_history(r['history'], ref['history'])
    assert r['ok'] == ref['ok'] and r['converged'] == ref['converged'] and r.get('note') == ref.get('note')
    assert r['f_ghz'] == pytest.approx(ref['f_ghz'], abs=1e-12)
    if ref['q'] is None:
        assert r['q'] is None
    else:
        assert r['q'] == pytest.approx(ref['q'], rel=1e-9)
        assert r['samples_in_linewidth'] == ref['samples_in_linewidth']
        assert r['linewidth_mhz'] == pytest.approx(ref['linewidth_mhz'], rel=1e-9)


@pytest.mark.parametrize('c', _G['add_quality'], ids=[c['name'] for c in _G['add_quality']])
def test_add_quality_matches_reference(c):
    ref = c['result']
    r = add_quality(dict(fr_ghz=c['fr_ghz'], fa_ghz=c['fa_ghz']), Lossy(*c['model']), tuple(c['limits']))
    assert r['q_r'] == pytest.approx(ref['q_r'], abs=0.01) and r['q_a'] == pytest.approx(ref['q_a'], abs=0.01)
    assert r['fr_ghz'] == pytest.approx(ref['fr_ghz'], abs=1e-7)
    assert r['fa_ghz'] == pytest.approx(ref['fa_ghz'], abs=1e-7)
    assert r['k2eff'] == pytest.approx(ref['k2eff'], abs=1e-6)
    _close_history(r['quality']['resonance']['history'], ref['resonance']['history'])
    _close_history(r['quality']['antiresonance']['history'], ref['antiresonance']['history'])


@pytest.mark.parametrize('per_linewidth', [13, 26, 45])
def test_extrapolated_q_recovers_the_resonator_q(per_linewidth):
    fr, q = 1.75e9, 900.0
    lw = fr / q
    f = np.linspace(fr - 1.5 * lw, fr + 1.5 * lw, 3 * per_linewidth + 1)
    r = peak_quality_extrapolated(f, np.abs(resonator(f, fr, q, 1.82e9, 900.0)) ** 2)
    assert abs(r['q'] / q - 1) < 4e-3 and abs(r['f0_hz'] / fr - 1) < 1e-5
    assert abs(r['q'] - q) <= abs(r['q_linear'] - q) + 1e-9


def test_peak_quality_needs_both_half_power_points():
    f = np.linspace(1.7e9, 1.71e9, 41)
    assert peak_quality(f, np.abs(resonator(f, 1.7097e9, 900, 1.8e9, 900)) ** 2) is None


def test_lossy_locate_and_converge_with_q():
    model = (1.7512345e9, 1200.0, 1.8123456e9, 1500.0)
    e = Lossy(*model)
    r = locate(e, 1.6, 2.0, 201, (1.0, 3.0), zoom_points=101, with_q=True)
    assert r['ok'] and r['quality']['resonance']['converged'] and r['quality']['antiresonance']['converged']
    assert abs(r['q_r'] / 1200 - 1) < 1e-2 and abs(r['q_a'] / 1500 - 1) < 1e-2
    assert abs(r['fr_ghz'] - 1.7512345) < 2e-5 and abs(r['fa_ghz'] - 1.8123456) < 2e-5
    assert r['k2eff'] == pytest.approx(math.pi ** 2 / 4 * (r['fa_ghz'] - r['fr_ghz']) / r['fa_ghz'], abs=1e-6)
    # every Q window is one more sweep of the same engine
    n_q = len(r['quality']['resonance']['history']) + len(r['quality']['antiresonance']['history'])
    assert r['sweeps'] == len(r['history']) + n_q == len(e.sweeps)
    fine = Lossy(model[0] * 0.9995, 1250.0, model[2] * 0.9995, 1550.0)
    c = converge(Lossy(*model), fine, 1.6, 2.0, 201, (1.0, 3.0), with_q=True)
    assert c['ok'] and c['fine']['q_r'] and c['shift']['q_r_rel_change'] == pytest.approx(50 / 1200, abs=1e-2)
    assert c['shift']['q_a_rel_change'] == pytest.approx(50 / 1500, abs=1e-2)
