"""Generate tests/golden/quality_cases.json from the reference's own Q stage.

Run in the build container, where the reference (Duane245/sawsim 2.1.0) is
mounted read-only at /root/reference (SAWSIM_REFERENCE overrides):

    python tests/golden/make_quality_golden.py

It records, on analytic lossy resonators Y(f) = i f (f^2 - pa^2) / (f^2 - pr^2)
with poles and zeros pr = fr (1 + i / 2 Qr), pa = fa (1 + i / 2 Qa) (the form of
the reference's tests/test_quality.py):

* ``sawsim.metrics.peak_quality`` and ``peak_quality_extrapolated``
  (src/sawsim/metrics.py:38-81) on sampled |Y|^2 and |Z|^2 curves, with the
  curves themselves;
* ``sawsim.agent.quality`` (src/sawsim/agent.py:332-383) and ``_add_quality``
  (:386-403), driven through a stand-in for the reference's ``run`` /
  ``load_curve`` that samples the analytic resonator on each window the
  reference asks for (f = linspace(start 1e9, stop 1e9, points), as
  solver.py:104 builds it), with the template band limits patched in.

The tests read the fixture, never the reference checkout.
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get('SAWSIM_REFERENCE', '/root/reference'))
sys.path.insert(0, str(REF / 'src'))

from sawsim import agent  # noqa: E402
from sawsim.metrics import peak_quality, peak_quality_extrapolated  # noqa: E402


def resonator(f, fr, qr, fa, qa):
    pr, pa = fr * (1 + 0.5j / qr), fa * (1 + 0.5j / qa)
    return 1j * f * (f ** 2 - pa ** 2) / (f ** 2 - pr ** 2)


def curve_cases():
    out = []
    rng = np.random.default_rng(11)
    for i in range(24):
        fr = rng.uniform(1.6e9, 1.9e9)
        q = float(rng.choice([150.0, 900.0, 3000.0]))
        lw = fr / q
        n = int(rng.integers(9, 160))
        lo, hi = fr - rng.uniform(0.4, 3.0) * lw, fr + rng.uniform(0.4, 3.0) * lw
        kind = 'r' if i % 2 == 0 else 'a'
        model = (fr, q, fr * 1.035, q * 1.2) if kind == 'r' else (fr / 1.035, q / 1.2, fr, q)
        out.append(dict(name=f'curve_{i}', kind=kind, lo=lo, hi=hi, n=n, model=model))
    return out


def power_of(y, kind):
    m2 = np.abs(y) ** 2
    return m2 if kind == 'r' else 1.0 / np.maximum(m2, 1e-300)


def drive(model, limits):
    """Point the reference's run / load_curve / band limits at the analytic model."""
    def run(config, on_progress=None):
        return dict(ok=True, output_dir=json.dumps([config['start_ghz'], config['stop_ghz'], config['points']]))

    def load_curve(path):
        start, stop, points = json.loads(path)
        f = np.linspace(start * 1e9, stop * 1e9, points)
        return f, resonator(f, *model), 'analytic'

    agent.run, agent.load_curve = run, load_curve
    agent._band_limits = lambda model_id: limits


def quality_cases():
    return [dict(name='fr_q900', model=(1.75e9, 900.0, 1.82e9, 1100.0), f_ghz=1.7503, kind='r', width=None,
                 limits=(0.5, 5.0)),
            dict(name='fa_q1100', model=(1.75e9, 900.0, 1.82e9, 1100.0), f_ghz=1.8197, kind='a', width=None,
                 limits=(0.5, 5.0)),
            dict(name='fr_q5000_offcentre', model=(1.7512e9, 5000.0, 1.8123e9, 5000.0), f_ghz=1.7530, kind='r',
                 width=0.0018, limits=(0.5, 5.0)),
            dict(name='fr_q150_widen', model=(1.70e9, 150.0, 1.80e9, 150.0), f_ghz=1.7004, kind='r', width=0.0005,
                 limits=(0.5, 5.0)),
            dict(name='fa_q150', model=(1.70e9, 150.0, 1.80e9, 150.0), f_ghz=1.8010, kind='a', width=0.003,
                 limits=(0.5, 5.0)),
            dict(name='lossless', model=(1.75e9, 1e8, 1.82e9, 1e8), f_ghz=1.75, kind='r', width=None,
                 limits=(0.5, 5.0)),
            dict(name='band_clipped', model=(1.6010e9, 400.0, 1.66e9, 400.0), f_ghz=1.601, kind='r', width=None,
                 limits=(1.6, 2.0))]


def add_quality_cases():
    return [dict(name='located_q900', model=(1.75e9, 900.0, 1.82e9, 1100.0), fr_ghz=1.75021, fa_ghz=1.81987,
                 limits=(0.5, 5.0)),
            dict(name='located_q3000', model=(1.7312e9, 3000.0, 1.7935e9, 2500.0), fr_ghz=1.7311, fa_ghz=1.7937,
                 limits=(0.5, 5.0))]


def main():
    curves = []
    for c in curve_cases():
        f = np.linspace(c['lo'], c['hi'], c['n'])
        p = power_of(resonator(f, *c['model']), c['kind'])
        curves.append(dict(c, f=f.tolist(), power=p.tolist(), peak_quality=peak_quality(f, p),
                           peak_quality_extrapolated=peak_quality_extrapolated(f, p)))
    qual = []
    for c in quality_cases():
        drive(c['model'], c['limits'])
        r = agent.quality(dict(model_id='sp_double_layer'), c['f_ghz'], c['kind'], c['width'])
        for h in r['history']:
            h.pop('output_dir', None)
        qual.append(dict(c, result=r))
    addq = []
    for c in add_quality_cases():
        drive(c['model'], c['limits'])
        res = dict(fr_ghz=c['fr_ghz'], fa_ghz=c['fa_ghz'], notes=[])
        r = agent._add_quality(res, dict(model_id='sp_double_layer'), None)
        for part in ('resonance', 'antiresonance'):
            for h in r['quality'][part]['history']:
                h.pop('output_dir', None)
        addq.append(dict(c, result=dict(fr_ghz=r['fr_ghz'], fa_ghz=r['fa_ghz'], q_r=r.get('q_r'), q_a=r.get('q_a'),
                                        k2eff=r['k2eff'], resonance=r['quality']['resonance'],
                                        antiresonance=r['quality']['antiresonance'])))
    (HERE / 'quality_cases.json').write_text(json.dumps(dict(curves=curves, quality=qual, add_quality=addq)))
    print(len(curves), 'curves,', len(qual), 'quality cases,', len(addq), 'add_quality cases')


if __name__ == '__main__':
    main()
