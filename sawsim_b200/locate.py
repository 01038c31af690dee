"""Batched locate / converge on one engine.

The reference's ``agent.locate`` (src/sawsim/agent.py:406-477) finds fr/fa with
2-9 sweeps: a coarse sweep of the template band, repeated while the pair is not
bracketed (more points when no pair is found, the band widened by half its span
towards a rising edge, the top extended when fa is missing), then up to three
zoomed sweeps around [fr - (fa - fr), fa + (fa - fr)] until fewer than five
samples between fr and fa no longer occur.  ``agent.converge`` (:492-525)
locates on one mesh and sweeps a finer mesh on the same zoomed band.

Every ``run`` of the reference rebuilds the mesh, reassembles K and M with the
PML frozen at the sweep's top frequency (solver.py:106-107), and refactors each
point with a fresh symbolic analysis.  Here one engine serves every sweep of a
locate: a new band top reassembles the values on the GPU
(``FrequencySolver.set_freeze_frequency``, which keeps the condensation maps, the
nested-dissection ordering, the symbolic analysis, the factorisation plans and
their autotuner picks), and each sweep is one batched ``ss_sweep``.  The
decision rules and the fr/fa extractor (``metrics.resonances``) are the
reference's.

For a lossy system (Rayleigh damping or dielectric loss: the reference's
``beta_dk`` / ``eta_eps`` > 0) ``locate(..., with_q=True)`` adds the reference's
Q stage (``agent._add_quality`` :386-403, ``agent.quality`` :332-383): around fr
(peak of |Y|^2) and fa (peak of |Z|^2) windows of +/-3 linewidths re-centre and
size the line until it spans at least 8 samples, then a window of +/-1.5
linewidths gives Q by ``metrics.peak_quality_extrapolated``; the refined peaks
replace fr / fa.  Every window is one more batched sweep on the same engine.
"""
from __future__ import annotations

import math

import numpy as np

from .metrics import compare, peak_quality, peak_quality_extrapolated, resonances


def y11_2d(w, Q, V=1.0):
    """Passive-sign 2D admittance Y = -i w Q / V (solver.py:128)."""
    return -1j * w * Q / V


def _sweep(eng, start_ghz, stop_ghz, points, precision, y11, V, refreeze):
    f = np.linspace(start_ghz * 1e9, stop_ghz * 1e9, int(points))
    w = 2 * np.pi * f
    if refreeze:
        eng.set_freeze_frequency(float(w[-1]))
    Q, st, _ = eng.charges(w, V, precision)
    if (st != 0).any():
        raise RuntimeError(f'sweep {start_ghz}-{stop_ghz} GHz: {int(np.sum(st != 0))} points failed')
    s = eng.stats()
    Y = y11(w, Q, V)
    r = resonances(f, Y)
    r.update(band_ghz=[float(start_ghz), float(stop_ghz)], points=int(points), device_ms=s['sweep_device_ms'],
             precision_used='mixed' if int(s['precision_used']) == 1 else 'fp64')
    return r, f, Y


def quality(eng, f_ghz, kind='r', width_ghz=None, band_limits_ghz=(0.0, math.inf), *, points=61,
            final_points=121, max_sweeps=6, precision='auto', V=1.0, y11=y11_2d, refreeze=True) -> dict:
    """Q at the resonance (``kind`` 'r': peak of |Y|^2) or the antiresonance ('a':
    peak of |Z|^2 = 1/|Y|^2) near ``f_ghz`` (agent.py:332-383).

    Windows of +/-3 linewidths (``points`` samples) re-centre on the peak and take
    its 3 dB width as the next linewidth, widening threefold when a half-power
    point falls outside, until the line spans at least 8 samples (at most
    ``max_sweeps`` windows); a final window of +/-1.5 linewidths
    (``final_points``) gives Q by ``peak_quality_extrapolated``.  Windows are
    clipped to ``band_limits_ghz``.  Returns ``ok``, ``q`` (None when not
    resolved), ``f_ghz``, ``converged`` (the full and half samplings agree within
    1 %), ``history`` and ``device_ms``."""
    f_lo, f_hi = band_limits_ghz
    f0, width = float(f_ghz), float(width_ghz or f_ghz * 2e-3)
    history = []
    spent = [0.0]

    def window(half, n, extrapolate=False):
        lo, hi = round(max(f_lo, f0 - half), 7), round(min(f_hi, f0 + half), 7)
        r, f, Y = _sweep(eng, lo, hi, n, precision, y11, V, refreeze)
        spent[0] += r['device_ms']
        mag2 = np.abs(Y) ** 2
        power = mag2 if kind == 'r' else 1.0 / np.maximum(mag2, 1e-300)
        pq = (peak_quality_extrapolated if extrapolate else peak_quality)(f, power)
        history.append(dict(window_ghz=[lo, hi], points=int(n), q=pq and round(pq['q'], 3),
                            samples_in_linewidth=pq and pq['samples_in_linewidth']))
        return pq

    def unresolved(note):
        return dict(ok=True, q=None, f_ghz=f0, converged=False, note=note, history=history, device_ms=spent[0])

    for _ in range(max_sweeps):
        pq = window(3 * width, points)
        if pq is None:                      # a half-power point outside the window: widen
            width *= 3
            continue
        f0, width = pq['f0_hz'] * 1e-9, (pq['fh_hz'] - pq['fl_hz']) * 1e-9
        if f0 / width > 1e6:
            return unresolved('Q > 1e6: no resolvable loss (lossless model or radiation-limited only)')
        if pq['samples_in_linewidth'] >= 8:
            break
    else:
        return unresolved(f'linewidth not resolved within {max_sweeps} windows')
    pq = window(1.5 * width, final_points, extrapolate=True)
    if pq is None:
        return unresolved('final window failed')
    spread = abs(pq['q_linear'] - pq['q_half']) / pq['q'] if pq.get('q_half') else None
    return dict(ok=True, q=pq['q'], f_ghz=pq['f0_hz'] * 1e-9, linewidth_mhz=(pq['fh_hz'] - pq['fl_hz']) * 1e-6,
                samples_in_linewidth=pq['samples_in_linewidth'], q_linear=pq['q_linear'], q_half=pq.get('q_half'),
                converged=spread is not None and spread < 0.01, history=history, device_ms=spent[0])


def add_quality(result, eng, band_limits_ghz, **kw) -> dict:
    """Refine fr / fa of a located ``result`` and add q_r / q_a (agent.py:386-403):
    ``quality`` at fr and at fa with a first linewidth of 3 % of fa - fr; a
    resolved Q replaces q_r / q_a and its refined peak fr / fa, and k2eff follows
    the refined pair.  ``kw`` goes to ``quality``."""
    width = (result['fa_ghz'] - result['fr_ghz']) * 0.03
    qr = quality(eng, result['fr_ghz'], 'r', width, band_limits_ghz, **kw)
    qa = quality(eng, result['fa_ghz'], 'a', width, band_limits_ghz, **kw)
    for key, q in (('r', qr), ('a', qa)):
        if q.get('ok') and q.get('q'):
            result['q_' + key] = round(q['q'], 2)
            result[f'f{key}_ghz'] = round(q['f_ghz'], 7)
    if result.get('fr_ghz') and result.get('fa_ghz'):
        result['k2eff'] = round(math.pi ** 2 / 4 * (result['fa_ghz'] - result['fr_ghz']) / result['fa_ghz'], 6)
    result['notes'] = [n for n in result.get('notes', []) if not n.startswith('Q not resolved')]
    result['quality'] = dict(method='Q = f_peak / 3 dB width of |Y|^2 (fr) and |Z|^2 (fa); final window +/-1.5 '
                                    'linewidths, interpolation bias removed by Richardson extrapolation; fr/fa '
                                    'are the refined peaks', resonance=qr, antiresonance=qa)
    result['device_ms'] = result.get('device_ms', 0.0) + qr['device_ms'] + qa['device_ms']
    result['sweeps'] = result.get('sweeps', 0) + len(qr['history']) + len(qa['history'])
    return result


def locate(eng, start_ghz, stop_ghz, points, band_limits_ghz, *, zoom_points=101, precision='auto', V=1.0,
           y11=y11_2d, refreeze=True, with_q=False) -> dict:
    """fr / fa of the main resonance with the reference's coarse -> widen -> zoom
    rules (agent.py:406-477) on one engine.  ``band_limits_ghz`` = the template's
    (start min, stop max).  Returns the zoomed sweep's ``resonances`` plus
    ``coarse``, ``history``, ``sweeps`` and ``device_ms`` (all sweeps).
    ``with_q`` adds the Q stage (``add_quality``); the reference turns it on when
    its config has ``beta_dk`` or ``eta_eps`` > 0 (agent.py:473-476)."""
    f_lo, f_hi = band_limits_ghz
    start, stop, pts = float(start_ghz), float(stop_ghz), int(points)
    history = []
    total_ms = 0.0
    s = None
    for _ in range(6):
        s, f, Y = _sweep(eng, start, stop, pts, precision, y11, V, refreeze)
        total_ms += s['device_ms']
        history.append(dict(band_ghz=[start, stop], points=pts, fr_ghz=s['fr_ghz'], fa_ghz=s['fa_ghz']))
        w = ' '.join(s['warnings'])
        span = stop - start
        at_limits = start <= f_lo and stop >= f_hi
        if 'no_resonance_found' in w or ('peak_at_band_edge' in w and at_limits):
            if pts >= 401:
                break
            pts = min(401, 2 * pts + 1)        # weak coupling: sample the fr..fa gap
            continue
        if 'peak_at_band_edge' in w:
            g = np.abs(Y) / f
            at_low = int(np.argmax(g)) == 0
            start = round(max(f_lo, start - span / 2), 4) if at_low else start
            stop = round(min(f_hi, stop + span / 2), 4) if not at_low else stop
            continue
        if 'antiresonance_not_found' in w and stop < f_hi:
            stop = round(min(f_hi, stop + span / 2), 4)
            continue
        break
    if s['fr_ghz'] is None or s['fa_ghz'] is None:
        return dict(ok=False, error=f'could not bracket fr and fa within the band {f_lo}..{f_hi} GHz',
                    history=history, last=s, sweeps=len(history), device_ms=total_ms)
    coarse = dict(fr_ghz=s['fr_ghz'], fa_ghz=s['fa_ghz'], band_ghz=[start, stop], points=pts)
    z = s
    for _ in range(3):      # zoom; again while the fr..fa gap is under-sampled
        fr, fa = z['fr_ghz'], z['fa_ghz']
        half = max(fa - fr, 2e-3 * z['frequency_step_mhz'])
        zs, ze = round(max(f_lo, fr - half), 6), round(min(f_hi, fa + half), 6)
        nz, _, _ = _sweep(eng, zs, ze, zoom_points, precision, y11, V, refreeze)
        total_ms += nz['device_ms']
        if nz['fr_ghz'] is None or nz['fa_ghz'] is None:
            break
        z = nz
        history.append(dict(band_ghz=[zs, ze], points=int(zoom_points), fr_ghz=z['fr_ghz'], fa_ghz=z['fa_ghz']))
        if 'coarse_sampling' not in z['warnings']:
            break
    if z is s:
        return dict(ok=False, error='zoomed sweep lost the resonance; inspect the coarse result', coarse=coarse,
                    history=history, sweeps=len(history), device_ms=total_ms)
    out = dict(z, ok=True, coarse=coarse, history=history, sweeps=len(history), device_ms=total_ms)
    if with_q:
        out = add_quality(out, eng, band_limits_ghz, precision=precision, V=V, y11=y11, refreeze=refreeze)
    return out


def converge(coarse_eng, fine_eng, start_ghz, stop_ghz, points, band_limits_ghz, *, zoom_points=101,
             precision='auto', V=1.0, y11=y11_2d, refreeze=True, with_q=False) -> dict:
    """Locate on the coarse mesh, sweep the fine mesh on the same zoomed band and
    report the fr / fa shift (agent.py:492-525); with the Q stage on, the fine
    sweep gets it too and the shift carries the relative change of q_r / q_a."""
    base = locate(coarse_eng, start_ghz, stop_ghz, points, band_limits_ghz, zoom_points=zoom_points,
                  precision=precision, V=V, y11=y11, refreeze=refreeze, with_q=with_q)
    if not base.get('ok'):
        return base
    (zs, ze), pts = base['band_ghz'], base['points']
    fine, _, _ = _sweep(fine_eng, zs, ze, pts, precision, y11, V, refreeze)
    sweeps = base['sweeps'] + 1
    if base.get('quality'):
        fine = add_quality(fine, fine_eng, band_limits_ghz, precision=precision, V=V, y11=y11, refreeze=refreeze)
        sweeps += fine['sweeps']
    d = compare(base, fine)
    for key in ('q_r', 'q_a'):
        if base.get(key) and fine.get(key):
            d[key + '_rel_change'] = round((fine[key] - base[key]) / base[key], 5)
    step = base['frequency_step_mhz']
    shift = max(abs(d['fr_diff_mhz'] or 0), abs(d['fa_diff_mhz'] or 0))
    return dict(ok=True, coarse=dict(fr_ghz=base['fr_ghz'], fa_ghz=base['fa_ghz'], k2eff=base['k2eff'],
                                     q_r=base.get('q_r'), q_a=base.get('q_a')),
                fine=dict(fr_ghz=fine['fr_ghz'], fa_ghz=fine['fa_ghz'], k2eff=fine['k2eff'], q_r=fine.get('q_r'),
                          q_a=fine.get('q_a')), shift=d,
                frequency_step_mhz=step, uncertainty_mhz=base['uncertainty_mhz'], shift_mhz=shift,
                band_ghz=[zs, ze], points=pts, sweeps=sweeps,
                device_ms=base['device_ms'] + fine['device_ms'])
