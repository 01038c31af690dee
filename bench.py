#!/usr/bin/env python
"""Benchmark: Y11 frequency points per second on one B200.

Workload: the seeded ME1 two-layer Q9 cell (3m film 0.6p / SiO2 0.3p / Si 3p /
PML 1p, 64x256 elements, 264,708 DOF, 262k active) swept over 201 frequencies
in 1.6-2.0 GHz.  One step = one whole sweep (all 201 points: batched
factorisation of every point, solves, refinement, charges).  K/M assembly,
condensation, ordering and symbolic analysis are host/device setup, done once
before timing and reported separately.

``--impl reference`` times the reference's CPU algorithm (the oracle port of
src/sawsim/saw2d/sweep.py: real-block SciPy SuperLU per point, the route the
reference takes without PARDISO) on this host's cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

PEAKS = REPO / 'MEASURED_PEAKS.json'
# bounded CPU samples: the same cell family at two reduced sizes (one full-size point
# takes minutes to hours of SuperLU on one core); the full-size points/s is
# extrapolated with the DOF exponent fitted between the two
CPU_SAMPLE = {'me0_16x64': [dict(cols=8, rows=32), dict(cols=16, rows=64)],
              'me1_64x256': [dict(cols=16, rows=64), dict(cols=32, rows=128)],
              'me1_128x512': [dict(cols=16, rows=64), dict(cols=32, rows=128)],
              'hex_8x4x48': [dict(nx=8, ny=1, nz=12), dict(nx=8, ny=2, nz=24)]}
SCHUR_DRAM_BYTES_PER_POINT = {'me1_64x256': 6.16e9}
FULL_POINT_LIMIT_S = 300.0     # the measured full-size CPU point gives up after this (a lower bound)
METRIC = 'Y11 points/s, 1 B200: batched FP32-TC+refine vs FP64 sweep, fr/fa within 1 kHz'


def parse():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=3)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    p.add_argument('--precision', default='auto', choices=['auto', 'mixed', 'fp64'])
    p.add_argument('--case', default='me1_64x256')
    p.add_argument('--points', type=int, default=None)
    p.add_argument('--no-cpu-baseline', action='store_true')
    p.add_argument('--no-modes', action='store_true', help='skip the untimed FP64-vs-mixed comparison')
    p.add_argument('--gradient', action='store_true',
                   help='time Y11 and dY11/dp by the adjoint on a parametrised cell instead of the sweep')
    p.add_argument('--no-full-point', action='store_true',
                   help='reference arm: skip the one measured full-size CPU point')
    return p.parse_args()


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        q = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
             'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
             'clocks_event_reasons.sw_power_cap')
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), f'--query-gpu={q}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None
            return self

        def reader():
            for line in self.proc.stdout:
                self.samples.append([x.strip() for x in line.split(',')])
        self._t = threading.Thread(target=reader, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.samples:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=['unsampled'])
        sm = [float(s[0]) for s in self.samples if s[0].replace('.', '').isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and s[3 + i] == 'Active'})
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                    reasons=reasons, samples=len(self.samples))


def peaks():
    try:
        d = json.loads(PEAKS.read_text())
        return d, 'measured'
    except Exception:
        return dict(hbm_gbs=6650.0, bf16_tflops=1590.0, bf16_tflops_sustained=1400.0), 'fallback'


# ----------------------------------------------------------------------------- CPU side
def _cpu_point(args):
    """One frequency point of the reference algorithm (oracle port), in a worker process."""
    case_name, size, f = args
    os.environ.setdefault('OMP_NUM_THREADS', '1')
    from helpers_cpu import oracle_solver_for
    eng = oracle_solver_for(case_name, **size)
    t = time.perf_counter()
    if case_name.startswith('hex'):
        eng.solve(2 * np.pi * f, 1.0)
    else:
        eng.solve(2 * np.pi * f, 1.0, route='realblock')
    return time.perf_counter() - t


def _dofs(c):
    return 4 * c.N if c.name.startswith('hex') else c.mesh.N * (4 if c.mode_extension else 3)


def cpu_sweep_sample(case_name, npoints, workers):
    """Full-size points/s of the reference route, extrapolated from two bounded samples.

    At each of two reduced sizes of the same cell family, ``npoints`` points run on
    ``workers`` spawn processes (one BLAS thread each); the per-point cost is fitted
    as a power of the DOF count and evaluated at the full size."""
    import multiprocessing as mp
    full = make(case_name)
    meas = []
    ctx = mp.get_context('spawn')
    with ctx.Pool(workers, initializer=_cpu_init) as pool:
        for size in CPU_SAMPLE[case_name]:
            c = make(case_name, **size)
            fs = np.linspace(c.freqs[0], c.freqs[-1], npoints)
            pool.map(_cpu_point, [(case_name, size, fs[0])] * workers)      # build per-worker engines
            t = time.perf_counter()
            pool.map(_cpu_point, [(case_name, size, f) for f in fs], chunksize=1)
            meas.append((_dofs(c), npoints / (time.perf_counter() - t)))
    (n0, v0), (n1, v1) = meas
    alpha = float(np.log(v0 / v1) / np.log(n1 / n0))
    nf = _dofs(full)
    value = v1 * (n1 / nf) ** alpha
    route = ('complex SciPy SuperLU per point (the Hex27 fallback of saw3d/bc_solve.py:166-167)'
             if case_name.startswith('hex') else 'real-block SciPy SuperLU per point as the reference without PARDISO')
    sample = (f'{npoints} points each at {n0} and {n1} DOF of the {case_name} family ({v0:.4g} and {v1:.4g} points/s), '
              f'{route}, {workers} spawn workers x 1 BLAS thread; per-point cost ~ DOF^{alpha:.2f} extrapolated '
              f'to the full {nf} DOF')
    return value, sample


def _cpu_init():
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REPO / 'oracle'))


def _full_point(case_name, out):
    """One frequency point of the reference route at the full size (spawned
    process, one BLAS thread): build seconds, solve seconds, peak RSS."""
    os.environ['OMP_NUM_THREADS'] = '1'
    _cpu_init()
    import resource
    from helpers_cpu import oracle_solver_for
    t = time.perf_counter()
    eng = oracle_solver_for(case_name)
    build = time.perf_counter() - t
    c = make(case_name)
    f = c.freqs[len(c.freqs) // 2]
    t = time.perf_counter()
    if case_name.startswith('hex'):
        eng.solve(2 * np.pi * f, 1.0)
    else:
        eng.solve(2 * np.pi * f, 1.0, route='realblock')
    out.put(dict(solve_s=time.perf_counter() - t, build_s=build, f_ghz=f / 1e9, n_active=int(eng.n_active),
                 peak_rss_gb=resource.getrusage(resource.RUSAGE_SELF).ru_maxrss / 1e6))


def full_point_start(case_name):
    import multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    p = ctx.Process(target=_full_point, args=(case_name, q), daemon=True)
    p.start()
    return p, q, time.perf_counter()


def full_point_finish(handle, limit_s):
    """The measured full-size point, waiting at most until `limit_s` after its start."""
    import queue
    p, q, t0 = handle
    try:
        res = q.get(timeout=max(1.0, limit_s - (time.perf_counter() - t0)))
    except queue.Empty:
        res = dict(unfinished_after_s=round(time.perf_counter() - t0, 1))
    if p.is_alive():
        p.terminate()
    p.join(5)
    return res


def reference_arm(a, rank, world):
    """Reference CPU implementation (oracle port) on this host, rank 0 only."""
    if rank != 0:
        return
    workers = min(8, os.cpu_count() or 1)
    # one full-size point of the same route, measured once on a core beside the
    # sampling workers (it takes minutes: it overlaps the sampled steps)
    full = full_point_start(a.case) if not a.no_full_point else None
    res = []
    for i in range(a.warmup + a.steps):
        v, sample = cpu_sweep_sample(a.case, 2 * workers, workers)
        if i >= a.warmup:
            res.append(v)
    value = float(np.mean(res))
    measured = full_point_finish(full, FULL_POINT_LIMIT_S) if full else None
    if measured and 'solve_s' in measured:
        measured['extrapolated_point_s'] = workers / value
        measured['extrapolated_over_measured'] = (workers / value) / measured['solve_s']
    print(json.dumps(dict(impl='reference', metric=METRIC, value=value, unit='points/s', n_gpus=a.gpus,
                          steps=a.steps, warmup=a.warmup, higher_is_better=True, scaling='weak', vs_baseline=None,
                          dtype='f64', data='synthetic',
                          config=dict(workload=workload_name(make(a.case, a.points)),
                                      route='oracle port of the reference route, bounded sample, extrapolated'),
                          cpu_baseline=dict(value=value, unit='points/s', cores=workers, kind='port', sample=sample,
                                            measured_full_point=measured),
                          e2e=dict(value=value, unit='points/s', h2d_bytes_per_step=0, d2h_bytes_per_step=0))),
          flush=True)


# ----------------------------------------------------------------------------- GPU side
def make(case_name, points=None, **size):
    from sawsim_b200 import cases
    if case_name.startswith('hex'):
        return cases.make_hex_case(case_name, points=points, **size)
    return cases.make_case(case_name, points=points, **size)


def workload_name(c):
    if c.name.startswith('hex'):
        i = c.info
        return (f'{c.name}: double-layer Hex27 slab {i["nx"]}x{i["ny"]}x{i["nz"]} ({4 * c.N} DOF), '
                f'{c.freqs.size} points {c.freqs[0] / 1e9:.1f}-{c.freqs[-1] / 1e9:.1f} GHz, seed {i["seed"]}')
    i = c.info
    kind = 'ME1 two-layer' if c.name == 'me1_64x256' else ('ME0' if c.name.startswith('me0') else 'ME1 four-layer')
    return (f'{c.name}: {kind} Q9 cell {i["cols"]}x{i["rows"]}, {c.freqs.size} points '
            f'{c.freqs[0] / 1e9:.1f}-{c.freqs[-1] / 1e9:.1f} GHz, seed {i["seed"]}')


def schur_kernel_name(s, used):
    """The Schur-update kernels the plan's autotuner picked, with their level counts."""
    if used == 'mixed':
        names = ['tc::pack_kernel + tc::tma_gemm_kernel<128,2> (TMA + tcgen05 3xTF32, 128x128 complex tiles)',
                 'tc::pack_kernel + tc::tma_gemm_kernel<64,3> (TMA + tcgen05 3xTF32, 128x64 complex tiles)',
                 'front_gemm_kernel<float> (SIMT FP32 128x64)']
    else:
        names = ['front_gemm_kernel<double> SIMT 128x64',
                 'front_dmma3_kernel (FP64 DMMA 64x64, three real products per complex block)',
                 'front_dmma_kernel<2,2> (FP64 DMMA 64x64)',
                 'front_dmma3_kernel<2,2,CST> (the same with the C tile staged in shared memory)']
    keys = ['schur_candidate0', 'schur_candidate1', 'schur_candidate2', 'schur_candidate3']
    parts = [f'{n} on {int(s[k])} levels' for n, k in zip(names, keys) if s.get(k, 0) > 0]
    return 'Schur update F22 -= F21 F12: ' + ', '.join(parts)


def _sweep_stats(eng, w, precision, reps):
    """Device time of `reps` sweeps after one untimed sweep (plan, tuner, graphs)."""
    eng.charges(w, 1.0, precision)
    ms, out = [], None
    for _ in range(reps):
        Q, st, it = eng.charges(w, 1.0, precision)
        s = eng.stats()
        ms.append(s['sweep_device_ms'])
        out = (Q, st, it, s)
    return float(np.median(ms)), out


def mode_comparison(eng, f, w, reps):
    """FP64 and mixed sweeps of the same points: rates, refinement and the mixed
    sweep's Y11 / fr / fa error against FP64 (the metric's comparison).  The mixed
    mode runs at the library's default Krylov target and once more at 1e-6 (the
    metric's Y11 accuracy), each with the FP64 re-solve of unconverged points."""
    from sawsim_b200.metrics import compare, resonances
    res = {}
    Ys = {}
    for mode, prec, tol in (('fp64', 'fp64', None), ('mixed', 'mixed', None), ('mixed_tol_1e-6', 'mixed', 1e-6)):
        if tol is not None:
            eng.set_option('krylov_tol', tol)
        try:
            ms, (Q, st, it, s) = _sweep_stats(eng, w, prec, reps)
        finally:
            if tol is not None:
                eng.set_option('krylov_tol', 1e-8)
        Ys[mode] = -1j * w * Q
        res[mode] = dict(points_per_s=w.size / (ms * 1e-3), ms_per_sweep=ms, chunk=int(s['chunk']),
                         points_not_ok=int(np.sum(st != 0)))
        if prec == 'mixed':
            d = compare(resonances(f, Ys['fp64']), resonances(f, Ys[mode]))
            res[mode].update(krylov_steps_per_point=(s['krylov_steps_primal'] + s['krylov_steps_adjoint']) / w.size,
                             refinement_not_converged=int(s['mixed_not_converged']),
                             points_resolved_in_fp64=int(s['fp64_resolved']), fp64_resolve_ms=s['fp64_resolve_ms'],
                             y11_max_rel_err_vs_fp64=float(np.max(np.abs(Ys[mode] - Ys['fp64']) / np.abs(Ys['fp64']))),
                             y11_median_rel_err_vs_fp64=float(np.median(np.abs(Ys[mode] - Ys['fp64']) /
                                                                        np.abs(Ys['fp64']))),
                             fr_diff_khz_vs_fp64=None if d['fr_diff_mhz'] is None else d['fr_diff_mhz'] * 1e3,
                             fa_diff_khz_vs_fp64=None if d['fa_diff_mhz'] is None else d['fa_diff_mhz'] * 1e3,
                             ratio_over_fp64=None)
            res[mode]['ratio_over_fp64'] = res[mode]['points_per_s'] / res['fp64']['points_per_s']
    res['ratio_mixed_over_fp64'] = res['mixed']['points_per_s'] / res['fp64']['points_per_s']
    return res


def rooflines(eng, c, s, st0, used, schur_ms, nf, pk, pk_kind, ceilings):
    """Roofline entries: the Schur update (tensor), the triangular solves and the
    assembly (HBM), each from this run's CUDA-event times and the algorithmic work
    of the project's symbolic analysis."""
    out = []
    launches = max(1.0, s['schur_launches'])
    flops_launch = s['schur_gemm_flops'] / launches
    ms_launch = float(np.mean(schur_ms)) / launches
    achieved = flops_launch / (ms_launch * 1e-3) / 1e12 if ms_launch > 0 else None
    traffic, traffic_note = None, None
    if used == 'fp64' and c.name in SCHUR_DRAM_BYTES_PER_POINT:
        traffic = SCHUR_DRAM_BYTES_PER_POINT[c.name] * nf / launches
        traffic_note = ('dram__bytes_read.sum + dram__bytes_write.sum of the Schur launches in an ncu capture of '
                        '1 and 2 points of this cell (bytes grow in proportion to the points), scaled to this '
                        "run's points per launch; not measured in this run")
    if used == 'mixed':
        peak = pk.get('bf16_tflops', 1590.0) / 2
        peak_note = (f'TF32 dense = half the {pk_kind} cuBLAS bf16 burst; achieved counts the algorithmic complex '
                     f'flops over the per-level mix of tcgen05 3xTF32 tiles (three MMA passes each) and SIMT FP32 '
                     f'tiles; own-kernel ceilings on dense 2560-row fronts: {ceilings}')
    else:
        peak = max(ceilings.get('fp64_dmma', 0.0), ceilings.get('fp64_dmma_3m', 0.0),
                   ceilings.get('fp64_dmma_3m_cst', 0.0)) or None
        peak_note = ('measured ceiling of this library\'s fastest FP64 Schur tile on 8 dense fronts of 2560 rows '
                     'with 512 pivots (ss_measure_gemm_ceiling, median of 5 launches; DMMA with three real products '
                     'per complex block counts the algorithmic complex flops, so it can exceed the nominal FP64 '
                     'tensor peak of 37-40 TFLOP/s)')
    out.append(dict(kernel=schur_kernel_name(s, used), bound='tensor', achieved=achieved, peak=peak, unit='TFLOP/s',
                    frac=(achieved / peak) if achieved and peak else None, traffic=traffic,
                    traffic_unit='bytes per launch', traffic_note=traffic_note, peak_note=peak_note,
                    flops_per_launch=flops_launch))
    hbm = pk.get('hbm_gbs', 6650.0)
    # triangular solves: the first solve of every chunk (forward + backward over all
    # fronts), algorithmic bytes nnz(L+U) x scalar + 2 n x 16 per point
    scal = 8 if used == 'mixed' else 16
    n = st0['n_active']
    sb = nf * (st0['nnz_lu'] * scal + 2 * n * 16)
    if s['solve_ms'] > 0:
        ach = sb / (s['solve_ms'] * 1e-3) / 1e9
        out.append(dict(kernel='front_fwd* / front_bwd* (batched forward + backward triangular solves, first solve '
                               'of every chunk)', bound='hbm', achieved=ach, peak=hbm, unit='GB/s', frac=ach / hbm,
                        traffic=None, bytes_per_point=sb / nf,
                        peak_note=f'{pk_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)'))
    # assembly: K and M written on the CSR pattern + coordinates + connectivity +
    # gather map, element kernel + scatter kernel times of the setup's ss_assemble
    t_asm = st0['element_kernel_ms'] + st0['scatter_kernel_ms']
    if t_asm > 0:
        K = eng.export(0)
        Mx = eng.export(1)
        npe = 27 if c.name.startswith('hex') else 9
        ne = c.hexas.shape[0] if c.name.startswith('hex') else c.mesh.ne
        N = c.N if c.name.startswith('hex') else c.mesh.N
        dim = 3 if c.name.startswith('hex') else 2
        ab = 16 * (K.nnz + Mx.nnz) + 8 * dim * N + 8 * npe * ne + 8 * npe * npe * ne
        ach = ab / (t_asm * 1e-3) / 1e9
        out.append(dict(kernel='q9/hex27 element kernel + gather_pairs_kernel (GPU assembly of K and M, once per '
                               'engine)', bound='hbm', achieved=ach, peak=hbm, unit='GB/s', frac=ach / hbm, traffic=None,
                        bytes=ab, ms=t_asm,
                        bytes_note='16 (nnz K + nnz M) written + coordinates + connectivity + 8-byte gather map '
                                   'entries; the element-matrix scratch round trip is not algorithmic',
                        peak_note=f'{pk_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)'))
    return out


def b200_arm(a, rank, world, local):
    import torch
    import torch.distributed as dist
    from sawsim_b200 import cases
    torch.cuda.set_device(local)
    c = make(a.case, a.points)
    t0 = time.perf_counter()
    eng = cases.hex_engine_for(c, device=local) if a.case.startswith('hex') else cases.engine_for(c, device=local)
    setup_s = time.perf_counter() - t0
    st0 = eng.stats()
    from sawsim_b200.shard import gather_charges, shard
    # N GPUs sweep an N-times denser grid of the same band, interleaved shards of
    # c.freqs.size points per rank (weak scaling); the charges are gathered once per sweep
    n_total = world * c.freqs.size
    f_all = np.linspace(c.freqs[0], c.freqs[-1], n_total)
    mine = shard(n_total, rank, world)
    w = 2 * np.pi * f_all[mine]
    nf = w.size
    first_sweep_ms = None
    for i in range(a.warmup):
        Q, status, iters = eng.charges(w, 1.0, a.precision)
        if i == 0:
            first_sweep_ms = eng.stats()['sweep_device_ms']
    probe_ms = eng.stats()['auto_probe_ms'] if a.precision == 'auto' else None

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    dev_ms, wall_s, schur_ms, launches = [], [], [], 0
    barrier()
    # the timed steps form the NVTX range "timed", so that a profiler can be told
    # to record only their launches (ncu --nvtx --nvtx-include "timed/")
    torch.cuda.nvtx.range_push('timed')
    with Clocks(local) as clk:
        for _ in range(a.steps):
            t = time.perf_counter()
            Q, status, iters = eng.charges(w, 1.0, a.precision)      # host buffers in, host Q out
            if world > 1:
                Q_all = gather_charges(Q, n_total, rank, world)
            wall_s.append(time.perf_counter() - t)
            s = eng.stats()
            s_timed = s
            dev_ms.append(s['sweep_device_ms'])
            schur_ms.append(s['schur_gemm_ms'])
            launches += int(s['launches'])
        barrier()
    torch.cuda.nvtx.range_pop()
    dev = float(np.sum(dev_ms)) / 1e3
    wall = float(np.sum(wall_s))
    used = 'mixed' if int(s_timed['precision_used']) == 1 else 'fp64'
    # accuracy of the timed sweep: fr/fa of Y11 = -i w Q / V (solver.py:128)
    from sawsim_b200.metrics import resonances
    if world > 1:
        Q_all = gather_charges(Q, n_total, rank, world)
    else:
        Q_all = Q
    w_all = 2 * np.pi * f_all
    Y = -1j * w_all * Q_all
    res = resonances(f_all, Y)
    acc = dict(fr_ghz=res['fr_ghz'], fa_ghz=res['fa_ghz'], k2eff=res['k2eff'])
    if world > 1:
        t = torch.tensor([dev, wall], device='cuda', dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev, wall = t.tolist()
    s = s_timed           # counters of the last timed sweep
    # untimed: both precision modes on this rank's points, and the measured ceilings
    modes = None if a.no_modes else mode_comparison(eng, f_all[mine], w, 2)
    ceilings = {'fp64_dmma': eng.gemm_ceiling(0), 'fp64_dmma_3m': eng.gemm_ceiling(5),
                'fp64_dmma_3m_cst': eng.gemm_ceiling(6)}
    if used == 'mixed' or modes is not None:
        ceilings.update(c64_tma_tcgen05_128=eng.gemm_ceiling(2), c64_tma_tcgen05_64=eng.gemm_ceiling(3),
                        c64_simt=eng.gemm_ceiling(4))
    pk, pk_kind = peaks()
    roof = rooflines(eng, c, s, st0, used, schur_ms, nf, pk, pk_kind, ceilings)
    line = None
    if rank == 0:
        cpu = None
        if not a.no_cpu_baseline:
            workers = min(8, os.cpu_count() or 1)
            v, sample = cpu_sweep_sample(a.case, 2 * workers, workers)
            cpu = dict(value=v, unit='points/s', cores=workers, kind='port', sample=sample)
            acc.update(oracle_check(c, eng, a.case))
        bad = int(np.sum(status != 0))
        line = dict(metric=METRIC, value=world * nf * a.steps / dev, unit='points/s', n_gpus=world,
                    steps=a.steps, warmup=a.warmup, ms_per_step=dev * 1e3 / a.steps, higher_is_better=True,
                    scaling='weak', vs_baseline=None, dtype='c64+f64' if used == 'mixed' else 'c128',
                    data='synthetic',
                    config=dict(workload=workload_name(c),
                                precision=a.precision, precision_used=used, accuracy=acc,
                                auto_probe_ms=probe_ms, first_sweep_ms=first_sweep_ms,
                                auto_note=('SS_PREC_AUTO probes the mixed path on the band ends in the first sweep '
                                           '(first_sweep_ms includes it, auto_probe_ms is its share); the timed '
                                           'sweeps keep the decision' if a.precision == 'auto' else None),
                                modes=modes,
                                n_active=int(st0['n_active']), fronts=int(st0['n_fronts']),
                                factor_gflop_per_point=st0['factor_flops_per_point'] / 1e9,
                                setup_s=setup_s, analyze_s=st0['analyze_s'], assemble_ms=st0['assemble_ms'],
                                l2='inputs larger than L2 (front arena of GBs per chunk)',
                                chunk=int(s['chunk']), points_not_converged=bad,
                                panel_gemm=dict(tiles=int(s['panel_gemm_dmma']),
                                                thin_tiles_per_point=int(s['panel_thin_tiles']),
                                                note='0 SIMT, 1 DMMA, 2 DMMA three products, 3 the same with C '
                                                     'staged, 4 SIMT with C staged; thin: tasks <= 8 wide in '
                                                     'SIMT 128x8 / 8x128 tiles beside the DMMA ones'),
                                mean_refinement_steps=float(np.mean(iters)),
                                parallelism=f'interleaved frequency shards x{world}' if world > 1 else 'one GPU'),
                    e2e=dict(value=world * nf * a.steps / wall, unit='points/s', h2d_bytes_per_step=8 * nf,
                             d2h_bytes_per_step=16 * nf + 8 * nf),
                    gpu_launches=launches,
                    roofline=roof[0], rooflines=roof, gemm_ceilings_tflops=ceilings,
                    clocks=clk.summary(), cpu_baseline=cpu)
    return line


def oracle_check(c, eng, case_name):
    """Part of the CPU-baseline leg: the oracle (the CPU restatement of the
    reference) assembles and condenses the same cell, and the GPU FP64 solutions
    at two sampled points are checked in the oracle's own system (normwise
    backward error)."""
    sys.path.insert(0, str(REPO / 'oracle'))
    from helpers_cpu import oracle_solver_for
    o = oracle_solver_for(case_name)
    out = []
    for fi in c.freqs[[len(c.freqs) // 3, 2 * len(c.freqs) // 3]]:
        wi = 2 * np.pi * fi
        A, rhs = o.system(wi)
        disp, _, _ = eng.solve(wi)
        x = disp[o.active]
        r = A @ x - rhs
        eta = np.linalg.norm(r, np.inf) / (abs(A).sum(axis=1).max() * np.linalg.norm(x, np.inf) +
                                           np.linalg.norm(rhs, np.inf))
        out.append(dict(f_ghz=fi / 1e9, backward_error=float(eta)))
    return dict(fp64_backward_error_in_oracle_system=out)


def gradient_arm(a):
    """Y11 and dY11/dp by the adjoint (``autograd.y11_and_jacobian``) at points
    spanning fr..fa of a parametrised cell, with a central-difference check of
    two parameters at two points (the four-layer ME1 128x512 cell and the
    four-layer Hex27 12x6x80 slab)."""
    from sawsim_b200 import autograd, params
    from sawsim_b200.metrics import resonances
    models = {'me1_64x256': lambda: params.Q9Model(64, 256),
              'me1_128x512': lambda: params.Q9Model(128, 512, stack='four_layer'),
              'hex_8x4x48': lambda: params.HexModel(8, 4, 48),
              'hex_12x6x80': lambda: params.HexModel(12, 6, 80, stack='four', f0=1.5e9, f1=2.1e9)}
    model = models[a.case]()
    v = model.defaults()
    # the band around the resonance pair: a coarse FP64 sweep of the model's band
    case = model.build(v)
    eng = model.engine(case)
    try:
        fc = np.linspace(model.f0, model.f1, 41)
        Q, _, _ = eng.charges(2 * np.pi * fc, 1.0, 'fp64')
        r = resonances(fc, model.y11(2 * np.pi * fc, Q, 1.0, case))
    finally:
        eng.close()
    fr, fa = r['fr_ghz'] * 1e9, r['fa_ghz'] * 1e9
    d = fa - fr
    f = np.linspace(fr - 0.25 * d, fa + 0.25 * d, a.points or 64)
    t = time.perf_counter()
    es = {}
    Y, dY, st = autograd.y11_and_jacobian(model, v, f, a.precision, stats=es)
    wall = time.perf_counter() - t
    used = 'mixed' if int(es.get('precision_used', 0)) == 1 else 'fp64'
    # central differences (relative step 1e-5, FP64 sweeps) of two parameters at two points
    idx = [int(np.argmin(np.abs(f - fr))), int(np.argmin(np.abs(f - fa)))]
    checks = []
    for j in (0, 1):
        hstep = 1e-5 * abs(v[j])
        vp, vm = v.copy(), v.copy()
        vp[j] += hstep
        vm[j] -= hstep
        yp, _ = autograd.y11_only(model, vp, f[idx], 'fp64')
        ym, _ = autograd.y11_only(model, vm, f[idx], 'fp64')
        fd = (yp - ym) / (2 * hstep)
        checks.append(dict(param=model.names[j], rel_err=[float(abs(dY[i, j] - fd[q]) / abs(fd[q]))
                                                          for q, i in enumerate(idx)]))
    return dict(metric='Y11 and dY11/dp points/s (adjoint)', value=f.size / wall, unit='points/s', n_gpus=1,
                steps=1, warmup=0, higher_is_better=True, scaling='weak', vs_baseline=None,
                dtype='c64+f64' if used == 'mixed' else 'c128', data='synthetic',
                config=dict(workload=f'{a.case} parametrised ({type(model).__name__}), {f.size} points spanning fr..fa',
                            n_params=len(model.names), params=model.names, precision=a.precision,
                            precision_used=used,
                            fr_ghz=r['fr_ghz'], fa_ghz=r['fa_ghz'], points_not_converged=int(np.sum(st != 0)),
                            wall_s_including_engine_build=wall, fd_checks=checks))


def main():
    a = parse()
    if a.gradient:
        print(json.dumps(gradient_arm(a)), flush=True)
        return
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if a.impl == 'reference':
        reference_arm(a, rank, world)
        return
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=timedelta(seconds=600))
    line = b200_arm(a, rank, world, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
