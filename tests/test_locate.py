"""Batched locate / converge decision rules (agent.py:406-477, :492-525) on a
stand-in engine whose charges follow an analytic lossless resonator
Y = -i w Q = i w C0 (f^2 - fa^2 + i d) / (f^2 - fr^2 + i d) with a small loss d (CPU; the GPU engine is
exercised in test_gpu_locate.py)."""
import numpy as np
import pytest

from sawsim_b200.locate import converge, locate


class Resonator:
    def __init__(self, fr, fa):
        self.fr, self.fa = fr, fa
        self.sweeps = []
        self.omega_top = None
        self._ms = 0.0

    def set_freeze_frequency(self, w):
        self.omega_top = w

    def charges(self, w, V=1.0, precision='auto'):
        f = w / (2 * np.pi)
        self.sweeps.append((f[0], f[-1], f.size))
        Y = 1j * w * 1e-12 * (f ** 2 - self.fa ** 2 + 1e14j) / (f ** 2 - self.fr ** 2 + 1e14j)
        return Y / (-1j * w) * V, np.zeros(f.size, dtype=np.int32), np.zeros(f.size, dtype=np.int32)

    def stats(self):
        return dict(sweep_device_ms=1.0, precision_used=0.0)


def test_locate_zooms_to_the_pair():
    e = Resonator(1.7512345e9, 1.8123456e9)
    r = locate(e, 1.6, 2.0, 201, (1.0, 3.0), zoom_points=101)
    assert r['ok'] and r['sweeps'] == 2
    # the zoom band is [fr - (fa - fr), fa + (fa - fr)] around the coarse fr/fa
    zs, ze = r['band_ghz']
    assert zs < 1.7512345 < 1.8123456 < ze and ze - zs < 0.2
    step_ghz = r['frequency_step_mhz'] * 1e-3
    assert abs(r['fr_ghz'] - 1.7512345) < step_ghz and abs(r['fa_ghz'] - 1.8123456) < step_ghz
    # the PML freeze frequency follows each sweep's top
    assert e.omega_top == pytest.approx(2 * np.pi * ze * 1e9)


def test_locate_widens_towards_a_rising_edge():
    e = Resonator(1.9012e9, 1.9512e9)
    r = locate(e, 1.6, 1.8, 101, (1.0, 3.0))
    assert r['ok']
    bands = [h['band_ghz'] for h in r['history']]
    assert bands[0] == [1.6, 1.8] and bands[1] == [1.6, 1.9]      # stop raised by half the span
    assert abs(r['fr_ghz'] - 1.9012) < 1e-3 and abs(r['fa_ghz'] - 1.9512) < 1e-3


def test_locate_extends_the_top_for_a_missing_antiresonance():
    e = Resonator(1.9512e9, 2.0512e9)
    r = locate(e, 1.6, 2.0, 201, (1.0, 3.0))
    assert r['ok'] and r['history'][1]['band_ghz'] == [1.6, 2.2]


def test_locate_fails_cleanly_without_a_pair():
    class Rising(Resonator):
        # |Y|/f rises across the whole template band: no pair, peak at the edge
        def charges(self, w, V=1.0, precision='auto'):
            self.sweeps.append(w.size)
            Q = -(w / (2 * np.pi)) * 1e-21 + 0j
            return Q, np.zeros(w.size, dtype=np.int32), np.zeros(w.size, dtype=np.int32)
    e = Rising(0, 0)
    r = locate(e, 1.6, 2.0, 101, (1.6, 2.0))
    # more points at every retry (203, 401), then give up
    assert not r['ok'] and e.sweeps == [101, 203, 401]


def test_converge_sweeps_the_fine_engine_on_the_zoom_band():
    coarse = Resonator(1.7512345e9, 1.8123456e9)
    fine = Resonator(1.7502345e9, 1.8113456e9)       # 1 MHz lower on the finer mesh
    r = converge(coarse, fine, 1.6, 2.0, 201, (1.0, 3.0))
    assert r['ok'] and len(fine.sweeps) == 1
    assert fine.sweeps[0][2] == r['points']
    assert r['shift']['fr_diff_mhz'] == pytest.approx(-1.0, abs=r['frequency_step_mhz'])
