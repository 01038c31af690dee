"""Measured ceilings of the Schur-update kernels (``ss_measure_gemm_ceiling``).

    python -m sawsim_b200.ceiling [--kernel K ...] [--m M] [--k K] [--fronts N] [--reps R]

prints one JSON line per kernel: the median algorithmic rate (8 real flops per
complex multiply-add) on ``fronts`` dense synthetic fronts of ``m`` rows with
``k`` pivots.  Kernels: 0 FP64 DMMA 64x64, 1 FP64 SIMT 128x64, 2 / 3 complex64
TMA + tcgen05 3xTF32 with 128 / 64-column tiles, 4 complex64 SIMT FP32 128x64,
5 FP64 DMMA 64x64 with three real products per complex block, 6 the same with
the C tile staged in shared memory.  These are the roofline denominators the benchmark reports beside the live rates.
"""
from __future__ import annotations

import argparse
import json

from .engine import Handle

NAMES = {0: 'FP64 DMMA 64x64', 1: 'FP64 SIMT 128x64', 2: 'complex64 TMA + tcgen05 3xTF32, 128-column tiles',
         3: 'complex64 TMA + tcgen05 3xTF32, 64-column tiles', 4: 'complex64 SIMT FP32 128x64',
         5: 'FP64 DMMA 64x64, three real products per complex block',
         6: 'FP64 DMMA 64x64, three real products per complex block, C staged in shared memory'}


def main(argv=None):
    import ctypes as C
    p = argparse.ArgumentParser()
    p.add_argument('--kernel', type=int, nargs='+', default=[0, 1, 2, 3, 4, 5, 6])
    p.add_argument('--m', type=int, default=2560)
    p.add_argument('--k', type=int, default=512)
    p.add_argument('--fronts', type=int, default=8)
    p.add_argument('--reps', type=int, default=5)
    p.add_argument('--device', type=int, default=0)
    a = p.parse_args(argv)
    h = Handle(a.device)
    try:
        for kern in a.kernel:
            out = C.c_double()
            h('ss_measure_gemm_ceiling', kern, a.m, a.k, a.fronts, a.reps, C.byref(out))
            print(json.dumps(dict(kernel=kern, name=NAMES.get(kern), m=a.m, k=a.k, fronts=a.fronts, reps=a.reps,
                                  tflops=out.value)), flush=True)
    finally:
        h.close()


if __name__ == '__main__':
    main()
