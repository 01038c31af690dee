"""Generate tests/golden/metrics_curves.npz from the reference's own fr/fa extractor.

Run in the build container, where the reference (Duane245/sawsim 2.1.0) is
mounted read-only at /root/reference:

    python tests/golden/make_metrics_golden.py

It feeds ``sawsim.metrics.resonances`` (src/sawsim/metrics.py:98-171) with

* the stored solver and independent-FEM curves of every template in the
  reference's tests/data/*.npz (801-point sweeps);
* the synthetic lossless resonator curves its tests build
  (tests/test_agent.py:16-52), at seeded random fr/fa, with and without a
  capacitive background, plus band-edge and missing-antiresonance cases;

and records the curves with the reference's fr_ghz / fa_ghz / k2eff / warning
codes.  The tests read the fixture, never the reference checkout.
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# the reference checkout: SAWSIM_REFERENCE, else where the build container mounts it
REF = Path(os.environ.get('SAWSIM_REFERENCE', '/root/reference'))
sys.path.insert(0, str(REF / 'src'))

from sawsim.metrics import resonances  # noqa: E402


def curves():
    out = []
    for p in sorted((REF / 'tests/data').glob('*.npz')):
        d = np.load(p)
        for key in ('sawsim_magnitude', 'reference_magnitude'):
            out.append((f'{p.stem}:{key}', d['frequency_hz'], d[key]))
    rng = np.random.default_rng(7)
    for i in range(12):
        lo, hi = 1.6e9, 2.0e9
        fr = rng.uniform(1.62e9, 1.9e9)
        fa = fr * (1 + rng.uniform(0.005, 0.06))
        n = int(rng.choice([101, 201, 401]))
        f = np.linspace(lo, hi, n)
        y = f * (f ** 2 - fa ** 2) / (f ** 2 - fr ** 2)
        if i % 2:
            y = 2j * np.pi * f * 1e-12 * (fa ** 2 - f ** 2) / (fr ** 2 - f ** 2)
        out.append((f'lossless_{i}', f, np.abs(y)))
    f = np.linspace(1.6e9, 2.0e9, 201)
    out.append(('band_edge', f, np.abs(f * (f ** 2 - 1.62e9 ** 2) / (f ** 2 - 1.55e9 ** 2))))
    out.append(('no_antiresonance', f, np.abs(f * (f ** 2 - 2.2e9 ** 2) / (f ** 2 - 1.9511e9 ** 2))))
    return out


def main():
    arrays, meta = {}, []
    for i, (name, f, y) in enumerate(curves()):
        r = resonances(f, y)
        arrays[f'f{i}'] = np.asarray(f, dtype=float)
        arrays[f'y{i}'] = np.asarray(y, dtype=float)
        meta.append(dict(name=name, fr_ghz=r['fr_ghz'], fa_ghz=r['fa_ghz'], k2eff=r['k2eff'],
                         warnings=[w.split(':')[0] for w in r['warnings']]))
    arrays['meta'] = np.array(json.dumps(meta))
    np.savez_compressed(HERE / 'metrics_curves.npz', **arrays)
    print(len(meta), 'curves')


if __name__ == '__main__':
    main()
