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
* seeded lossy curves with one to three resonators (poles and zeros at
  fr (1 + i / 2Q), as tests/test_quality.py builds them) on a capacitive
  background, so that the coarse q_r / q_a and the mode list are exercised;

and records the curves with the reference's whole ``resonances`` result
(warnings as their codes, the text before the colon).  The tests read the
fixture, never the reference checkout.
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
    rng = np.random.default_rng(3)
    for i in range(16):
        n = int(rng.choice([201, 401, 801]))
        f = np.linspace(1.6e9, 2.0e9, n)
        y = 2j * np.pi * f * 1e-13 + 0j
        for _ in range(int(rng.integers(1, 4))):
            fr = rng.uniform(1.6e9, 1.95e9)
            fa = fr * (1 + rng.uniform(0.003, 0.06))
            q = float(rng.choice([50.0, 150.0, 400.0, 3000.0]))
            pr, pa = fr * (1 + 0.5j / q), fa * (1 + 0.5j / (1.1 * q))
            y = y + rng.uniform(0.2, 1) * 1e-12 * 1j * f * (f ** 2 - pa ** 2) / (f ** 2 - pr ** 2)
        out.append((f'lossy_{i}', f, y))
    f = np.linspace(1.6e9, 2.0e9, 801)
    for i, (fr, q) in enumerate([(1.70e9, 60.0), (1.75e9, 100.0), (1.80e9, 200.0), (1.72e9, 300.0)]):
        pr, pa = fr * (1 + 0.5j / q), 1.04 * fr * (1 + 0.5j / (1.2 * q))
        y = 2j * np.pi * f * 1e-13 + 1e-12 * 1j * f * (f ** 2 - pa ** 2) / (f ** 2 - pr ** 2)
        out.append((f'lossy_single_{i}', f, y))
    return out


def main():
    arrays, meta = {}, []
    for i, (name, f, y) in enumerate(curves()):
        r = resonances(f, y)
        arrays[f'f{i}'] = np.asarray(f, dtype=float)
        arrays[f'y{i}'] = np.asarray(y)
        r['warnings'] = [w.split(':')[0] for w in r['warnings']]
        meta.append(dict(r, name=name))
    arrays['meta'] = np.array(json.dumps(meta))
    np.savez_compressed(HERE / 'metrics_curves.npz', **arrays)
    print(len(meta), 'curves')


if __name__ == '__main__':
    main()
