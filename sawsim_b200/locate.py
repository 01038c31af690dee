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
"""
from __future__ import annotations

import numpy as np

from .metrics import compare, resonances


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


def locate(eng, start_ghz, stop_ghz, points, band_limits_ghz, *, zoom_points=101, precision='auto', V=1.0,
           y11=y11_2d, refreeze=True) -> dict:
    """fr / fa of the main resonance with the reference's coarse -> widen -> zoom
    rules (agent.py:406-477) on one engine.  ``band_limits_ghz`` = the template's
    (start min, stop max).  Returns the zoomed sweep's ``resonances`` plus
    ``coarse``, ``history``, ``sweeps`` and ``device_ms`` (all sweeps)."""
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
    return out


def converge(coarse_eng, fine_eng, start_ghz, stop_ghz, points, band_limits_ghz, *, zoom_points=101,
             precision='auto', V=1.0, y11=y11_2d, refreeze=True) -> dict:
    """Locate on the coarse mesh, sweep the fine mesh on the same zoomed band and
    report the fr / fa shift (agent.py:492-525)."""
    base = locate(coarse_eng, start_ghz, stop_ghz, points, band_limits_ghz, zoom_points=zoom_points,
                  precision=precision, V=V, y11=y11, refreeze=refreeze)
    if not base.get('ok'):
        return base
    (zs, ze), pts = base['band_ghz'], base['points']
    fine, _, _ = _sweep(fine_eng, zs, ze, pts, precision, y11, V, refreeze)
    d = compare(base, fine)
    step = base['frequency_step_mhz']
    shift = max(abs(d['fr_diff_mhz'] or 0), abs(d['fa_diff_mhz'] or 0))
    return dict(ok=True, coarse=dict(fr_ghz=base['fr_ghz'], fa_ghz=base['fa_ghz'], k2eff=base['k2eff']),
                fine=dict(fr_ghz=fine['fr_ghz'], fa_ghz=fine['fa_ghz'], k2eff=fine['k2eff']), shift=d,
                frequency_step_mhz=step, uncertainty_mhz=base['uncertainty_mhz'], shift_mhz=shift,
                band_ghz=[zs, ze], points=pts, sweeps=base['sweeps'] + 1,
                device_ms=base['device_ms'] + fine['device_ms'])
