"""Resonance / antiresonance extraction from a swept admittance curve (host side).

Restates the reference's figure-of-merit module (``src/sawsim/metrics.py``),
which judges the sweep's fr/fa criterion:

* ``resonances`` :98-171 -- |Y|/f removes the static-capacitance slope; every
  local maximum of |Y|/f (``_local_extrema`` :33-35) is paired with the lowest
  |Y|/f sample before the next maximum; pairs whose minimum lies more than 15 %
  above the peak frequency are bulk-wave humps and are dropped; the main pair is
  the one with the largest relative dip (capped at 0.5), ties broken by the
  highest peak;
* ``_vfit`` :18-27 -- sub-sample refinement: vertex of a V through the extreme
  sample and its neighbours, clipped to half a step (fr is fitted on 1/(|Y|/f),
  fa on |Y|/f);
* ``compare`` :188-199 -- fr/fa deviation in MHz and ppm, k2eff in %-points;
* ``_rounded`` :174-185 -- GHz and MHz rounded to 0.1 kHz, other floats to 6
  significant digits;
* ``peak_quality`` :38-64 and ``peak_quality_extrapolated`` :67-81 -- Q of a
  peak of |Y|^2 (fr) or |Z|^2 (fa) from its 3 dB width, with the linear
  interpolation bias removed by Richardson extrapolation; the Q windows of a
  lossy locate (``sawsim_b200.locate.quality``) use them;
* ``_half_power_q`` :84-95 -- the coarse q_r / q_a of one sweep: the 3 dB width
  of |Y| (|Z| for fa) between the neighbouring extrema, only when it spans at
  least ``MIN_SAMPLES_IN_LINEWIDTH`` samples; and the mode list of
  ``resonances`` :160-170 (every pair, strongest first, then by frequency).

Warnings are the reference's codes (the text before its colon).
"""
from __future__ import annotations

import math

import numpy as np

K2_FORMULA = 'k2eff = pi^2/4 * (fa - fr) / fa'
MIN_SAMPLES_IN_LINEWIDTH = 8      # a 3 dB width over fewer samples is a sampling artefact
Q_NOTE = ('Q not resolved at this frequency step (3 dB width spans < %d samples); q_r/q_a are null - locate '
          'with beta_dk/eta_eps > 0 resolves Q' % MIN_SAMPLES_IN_LINEWIDTH)


def _vertex(f, g, i):
    """Frequency of the vertex of the V through samples i-1, i, i+1 of g (minimum at i)."""
    if i <= 0 or i >= len(g) - 1:
        return float(f[i])
    half = 0.5 * (f[i + 1] - f[i - 1])
    slope = max(g[i - 1] - g[i], g[i + 1] - g[i]) / half
    if not slope > 0:
        return float(f[i])
    shift = (g[i - 1] - g[i + 1]) / (2.0 * slope)
    return float(f[i] + min(max(shift, -half / 2), half / 2))


def _maxima(y):
    """Interior indices i with y[i] > y[i-1] and y[i] >= y[i+1]."""
    mid = y[1:-1]
    return np.flatnonzero((mid > y[:-2]) & (mid >= y[2:])) + 1


def _minima(y):
    return _maxima(-y)


def _round(key, v):
    """GHz and MHz to 0.1 kHz, other floats to 6 significant digits, through nested
    dicts and lists (a list's items take the list's key)."""
    if isinstance(v, float):
        if key.endswith('_ghz'):
            return round(v, 7)
        if key.endswith('_mhz'):
            return round(v, 4)
        return float('%.6g' % v)
    if isinstance(v, dict):
        return {k: _round(k, x) for k, x in v.items()}
    if isinstance(v, list):
        return [_round(key, x) for x in v]
    return v


def _half_power_q(f, mag, i, lo, hi):
    """Q = f[i] / 3 dB width of the peak of ``mag`` at sample i, the half-power
    samples searched outwards within [lo, hi]; None unless both exist and the
    width spans at least MIN_SAMPLES_IN_LINEWIDTH samples."""
    p = mag ** 2
    half = p[i] / 2
    a = next((j for j in range(i - 1, lo - 1, -1) if p[j] <= half), None)
    b = next((j for j in range(i + 1, hi + 1) if p[j] <= half), None)
    if a is None or b is None or b - a < MIN_SAMPLES_IN_LINEWIDTH:
        return None
    fl = np.interp(half, [p[a], p[a + 1]], [f[a], f[a + 1]])
    fh = np.interp(half, [p[b], p[b - 1]], [f[b], f[b - 1]])
    return float(f[i] / (fh - fl)) if fh > fl else None


def resonances(frequency_hz, admittance, max_modes: int = 5) -> dict:
    """fr / fa (GHz), k2eff, the coarse q_r / q_a, the in-band modes (at most
    ``max_modes``), warnings and notes of a sampled admittance (complex Y or |Y|)."""
    f = np.asarray(frequency_hz, dtype=float)
    mag = np.abs(np.asarray(admittance))
    n = f.size
    out = dict(fr_ghz=None, fa_ghz=None, k2eff=None, k2_formula=K2_FORMULA, q_r=None, q_a=None,
               frequency_step_mhz=None, uncertainty_mhz=None, points_between_fr_fa=None, modes=[], warnings=[],
               notes=[])
    if n < 5 or not np.all(np.isfinite(mag)):
        out['warnings'].append('curve too short or contains non-finite values')
        return out
    step = float(np.max(np.diff(f)))
    out['frequency_step_mhz'] = step * 1e-6
    out['uncertainty_mhz'] = step * 0.5e-6
    g = mag / f
    inv = 1.0 / np.maximum(g, np.finfo(float).tiny)
    peaks = _maxima(g)
    pairs = []
    for j, p in enumerate(peaks):
        stop = int(peaks[j + 1]) if j + 1 < len(peaks) else n - 1
        a = int(p) + int(np.argmin(g[p:stop + 1]))
        if a == p:
            continue
        if a != n - 1 and f[a] - f[p] > 0.15 * f[p]:
            continue
        pairs.append(((g[p] - g[a]) / g[p], int(p), a, stop))
    if not pairs:
        if int(np.argmax(g)) in (0, n - 1):
            out['warnings'].append('peak_at_band_edge')
        else:
            out['warnings'].append('no_resonance_found')
        return _round('', out)
    rank = lambda t: (min(t[0], 0.5), g[t[1]])      # noqa: E731
    score, r, a, stop = max(pairs, key=rank)
    fr = _vertex(f, inv, r)
    out['fr_ghz'] = fr * 1e-9
    minima = _minima(g)
    before = minima[minima < r]
    out['q_r'] = _half_power_q(f, mag, r, int(before[-1]) if before.size else 0, a)
    if a == n - 1:
        out['warnings'].append('antiresonance_not_found')
    else:
        fa = _vertex(f, g, a)
        out['fa_ghz'] = fa * 1e-9
        out['k2eff'] = math.pi ** 2 / 4 * (fa - fr) / fa
        out['points_between_fr_fa'] = int(a - r - 1)
        out['q_a'] = _half_power_q(f, 1.0 / np.maximum(mag, np.finfo(float).tiny), a, r, stop)
        if a - r < 6:
            out['warnings'].append('coarse_sampling')
    if max(g[0], g[-1]) > 3 * g[r]:
        out['warnings'].append('stronger_response_at_band_edge')
    if out['q_r'] is None:
        out['notes'].append(Q_NOTE)
    for st, p, q, _ in sorted(pairs, key=rank, reverse=True)[:max_modes]:
        out['modes'].append(dict(fr_ghz=_vertex(f, inv, p) * 1e-9, fa_ghz=_vertex(f, g, q) * 1e-9 if q != n - 1 else None,
                                 peak_abs_y=float(mag[p]), strength=float(st), is_main=bool(p == r)))
    out['modes'].sort(key=lambda m: m['fr_ghz'])
    strong = [m for m in out['modes'] if m['strength'] > 0.5 * min(score, 0.5) and m['peak_abs_y'] > 0.1 * mag[r]]
    if len(strong) > 1:
        out['warnings'].append('multiple_modes')
    return _round('', out)


def compare(reference: dict, candidate: dict) -> dict:
    """fr/fa/k2eff deviation of ``candidate`` from ``reference`` (both from ``resonances``)."""
    d = {}
    for key in ('fr_ghz', 'fa_ghz'):
        a, b = reference.get(key), candidate.get(key)
        ok = a is not None and b is not None
        d[key.replace('_ghz', '_diff_mhz')] = _round('_mhz', (b - a) * 1e3) if ok else None
        d[key.replace('_ghz', '_diff_ppm')] = _round('', (b - a) / a * 1e6) if ok else None
    a, b = reference.get('k2eff'), candidate.get('k2eff')
    d['k2eff_diff_pct_points'] = _round('', (b - a) * 100) if a is not None and b is not None else None
    return d


def peak_quality(f, power):
    """Q of the highest peak of ``power`` (|Y|^2 for fr, |Z|^2 = 1/|Y|^2 for fa),
    or None when the peak is a window edge or a half-power crossing lies outside
    the window (metrics.py:38-64).

    The peak is the vertex of the parabola through the top sample and its two
    neighbours (shift clipped to half a step); the half-power frequencies are
    linear interpolations of ``power`` between the samples that straddle half the
    vertex value, nearest the peak on each side; Q = f0 / (fh - fl)."""
    f = np.asarray(f, dtype=float)
    p = np.asarray(power, dtype=float)
    n = p.size
    i = int(np.argmax(p))
    if i == 0 or i == n - 1:
        return None
    pl, pc, pr = p[i - 1], p[i], p[i + 1]
    curv = pl - 2 * pc + pr
    s = 0.5 * (pl - pr) / curv if curv < 0 else 0.0
    s = min(max(s, -0.5), 0.5)
    step = f[i + 1] - f[i]
    f0 = f[i] + s * step
    half = (pc - 0.25 * (pl - pr) * s) / 2
    a = next((j for j in range(i, 0, -1) if p[j - 1] <= half < p[j]), None)
    b = next((j for j in range(i, n - 1) if p[j + 1] <= half < p[j]), None)
    if a is None or b is None:
        return None
    fl = f[a - 1] + (half - p[a - 1]) / (p[a] - p[a - 1]) * (f[a] - f[a - 1])
    fh = f[b] + (p[b] - half) / (p[b] - p[b + 1]) * (f[b + 1] - f[b])
    return dict(f0_hz=float(f0), fl_hz=float(fl), fh_hz=float(fh), q=float(f0 / (fh - fl)),
                samples_in_linewidth=int(b - a + 1), step_hz=float(step))


def peak_quality_extrapolated(f, power):
    """``peak_quality`` with the half-power interpolation bias removed
    (metrics.py:67-81): the bias falls as 1/n^2 in the samples per linewidth, so
    with Q_n from every sample and Q_n/2 the mean over the two every-other-sample
    subsets, Q = Q_n + (Q_n - Q_n/2) / 3.  Adds ``q_linear`` (Q_n) and ``q_half``
    (Q_n/2, None when neither subset resolves the peak)."""
    full = peak_quality(f, power)
    if full is None:
        return None
    f = np.asarray(f)
    power = np.asarray(power)
    sub = [peak_quality(f[k::2], power[k::2]) for k in (0, 1)]
    qs = [r['q'] for r in sub if r]
    if not qs:
        return dict(full, q_linear=full['q'], q_half=None)
    q_half = float(np.mean(qs))
    return dict(full, q=full['q'] + (full['q'] - q_half) / 3, q_linear=full['q'], q_half=q_half)
