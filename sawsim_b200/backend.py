"""Drop-in engine classes for SawSim's own pipeline, and the switch that installs them.

The reference's pipelines build their per-frequency engine from the assembled
matrices and drive it point by point:

* ``src/sawsim/solver.py:108`` ``sweep.FrequencySolver(K, M, *bc)`` (with
  ``set_damping(D, beta)`` at :109-115), then ``charge_stream(engine, fre, V)``
  (:116-126) and ``engine.solve(omega, V)`` at the peak (:132);
* ``src/sawsim/hex_solver.py:92`` ``FrequencySolver3D(K, M, boundary, t_fb, t_lr)``
  and ``charge_stream(..., is_hex=True)``, which calls ``solve(omega, voltage=V)``;
* ``src/sawsim/saw2d/saw3d/bc_solve.py:262`` ``FrequencySolver3D_FP(K, M, boundary,
  t_fb, t_float)``.

The classes below take the same constructor arguments and answer the same
methods (``solve`` returns ``(disp, Q, |Y|)``, ``sweep`` returns ``(Q, |Y|)``), backed
by :class:`sawsim_b200.engine.FrequencySolver` (fold, condensation, ordering and
every point's factorisation on the GPU).  :func:`charge_stream` replaces
``frequency_tasks.charge_stream`` (``frequency_tasks.py:33-55``): one batched sweep
of all the frequencies instead of a fork pool of per-point solves, yielding the
charges in frequency order.  :func:`install` points a loaded reference package at
them, so that its ``run_simulation`` runs on the GPU unchanged.
"""
from __future__ import annotations

import os
import sys
from contextlib import contextmanager
from pathlib import Path

import numpy as np

from .engine import FrequencySolver as _Engine


def _precision(precision):
    """The sweep precision: the argument, else ``SAWSIM_B200_PRECISION``, else FP64
    (the drop-in; 'auto' and 'mixed' as in ``ss_sweep``)."""
    return precision or os.environ.get('SAWSIM_B200_PRECISION', 'fp64')


class FrequencySolver:
    """``sweep.FrequencySolver(K, M, fix, zheng, fu, merge_groups)`` (sweep.py:275-393)."""

    def __init__(self, K, M, fix, zheng, fu, merge_groups, precision=None, device: int = 0, **layout):
        self._e = _Engine.from_matrices(K, M, fix, zheng, fu, merge_groups, device=device, **layout)
        self.precision = _precision(precision)
        self.gdof = int(K.shape[0])
        self.n_active = self._e.n_active

    def set_damping(self, D, beta):
        """Rayleigh stiffness damping A = K + i w beta D - w^2 M (sweep.py:316-323)."""
        self._e.set_damping(D, beta)

    def solve(self, omega: float, V: float = 1.0):
        """``(disp, Q, |Y|)`` at one angular frequency (sweep.py:335-364)."""
        return self._e.solve(omega, V)

    def charges(self, fre, V: float = 1.0):
        """Charges at frequencies ``fre`` (Hz), all points in batched GPU sweeps."""
        return self._e.sweep(fre, V, self.precision)

    def sweep(self, fre, V: float = 1.0, n_jobs: int = 1, progress: bool = True):
        """``(Q, |Y|)`` over ``fre`` (Hz) (sweep.py:366-393); ``n_jobs`` and ``progress``
        are accepted for the signature: every point goes into one batched sweep."""
        fre = np.asarray(fre, dtype=float)
        Q = self.charges(fre, V)
        return Q, np.abs(1j * 2 * np.pi * fre * Q / V)

    def close(self):
        self._e.close()


class FrequencySolver3D:
    """``FrequencySolver3D(K, M, boundary, t_fb, t_lr)`` (bc_solve.py:108-202) and, with the
    floating-electrode fold as the second operator, ``FrequencySolver3D_FP(K, M,
    boundary, t_fb, t_float)`` (bc_solve.py:262-345)."""

    def __init__(self, K, M, boundary, t_fb, t_second, precision=None, device: int = 0, **layout):
        self._e = _Engine.from_matrices_3d(K, M, boundary, t_fb, t_second, device=device, **layout)
        self.precision = _precision(precision)
        self.boundary = boundary
        self.gdof = int(K.shape[0])
        self.n_act = self._e.n_active

    def solve(self, omega: float, voltage: float = 1.0):
        """``(disp, Q, |Y|)`` at one angular frequency (bc_solve.py:154-175)."""
        return self._e.solve(omega, voltage)

    def charges(self, fre, voltage: float = 1.0):
        return self._e.sweep(fre, voltage, self.precision)

    def sweep(self, fre, voltage: float = 1.0, n_jobs: int = 1, progress: bool = True):
        """``(Q, |Y|)`` over ``fre`` (Hz) (bc_solve.py:177-202), one batched sweep."""
        fre = np.asarray(fre, dtype=float)
        Q = self.charges(fre, voltage)
        return Q, np.abs(1j * 2 * np.pi * fre * Q / voltage)

    def close(self):
        self._e.close()


FrequencySolver3D_FP = FrequencySolver3D


@contextmanager
def charge_stream(engine, frequencies, voltage, *, is_hex=False):
    """``frequency_tasks.charge_stream`` (frequency_tasks.py:33-55): the charges at
    ``frequencies`` (Hz) in order.  For the engines of this module they come from one
    batched GPU sweep; any other engine is solved point by point, as the reference's
    single-worker path does."""
    f = np.asarray(frequencies, dtype=float)
    if isinstance(engine, (FrequencySolver, FrequencySolver3D)):
        Q = engine.charges(f, voltage)
        yield (complex(q) for q in Q)
        return
    kwargs = {'voltage': voltage} if is_hex else {'V': voltage}
    yield (complex(engine.solve(2 * np.pi * x, **kwargs)[1]) for x in f)


# (module, attribute, replacement) of every reference name the pipelines look up
_PATCHES = [('sawsim.saw2d.sweep', 'FrequencySolver', FrequencySolver),
            ('sawsim.saw2d.saw3d.bc_solve', 'FrequencySolver3D', FrequencySolver3D),
            ('sawsim.saw2d.saw3d.bc_solve', 'FrequencySolver3D_FP', FrequencySolver3D_FP),
            ('sawsim.saw2d.saw3d', 'FrequencySolver3D', FrequencySolver3D),
            ('sawsim.frequency_tasks', 'charge_stream', charge_stream),
            ('sawsim.solver', 'charge_stream', charge_stream),
            ('sawsim.hex_solver', 'charge_stream', charge_stream),
            ('sawsim.hex_solver', 'FrequencySolver3D', FrequencySolver3D)]


def _metadata_writer(write):
    """The pipelines' ``atomic_json`` (solver.py:28-32) with ``metadata.json``
    naming this backend.  The reference writes ``backend`` as 'PARDISO' or 'SciPy
    SuperLU' from whether pypardiso imports (solver.py:146, hex_solver.py:74) and
    ``frequency_workers`` from its fork-pool size (solver.py:146), neither of which
    says what solved a sweep that ran here; every other file passes unchanged."""
    if getattr(write, 'sawsim_b200', False):
        return write

    def atomic_json(path, data):
        if Path(path).name == 'metadata.json' and isinstance(data, dict) and 'backend' in data:
            data = dict(data, backend=f'B200 (sawsim_b200, {_precision(None)})')
            if 'frequency_workers' in data:
                data['frequency_workers'] = 1
        return write(path, data)

    atomic_json.sawsim_b200 = True
    return atomic_json


def install(modules=None):
    """Point the reference's already imported modules at this backend.

    ``modules`` maps module names to module objects (default ``sys.modules``);
    the names of ``_PATCHES`` that a loaded module defines are replaced, and the
    pipelines' ``atomic_json`` is wrapped so that their ``metadata.json`` names
    this backend.  Returns the list of ``module.attribute`` names replaced, so
    that a caller can check that the pipeline it runs was reached."""
    mods = sys.modules if modules is None else modules
    done = []
    for mod, attr, new in _PATCHES:
        m = mods.get(mod)
        if m is not None and hasattr(m, attr):
            setattr(m, attr, new)
            done.append(f'{mod}.{attr}')
    m = mods.get('sawsim.solver')
    if m is not None and hasattr(m, 'atomic_json'):
        m.atomic_json = _metadata_writer(m.atomic_json)
        done.append('sawsim.solver.atomic_json')
    return done


def install_from_env(modules=None):
    """``install`` when the environment selects this backend (``SAWSIM_BACKEND=b200``)."""
    if os.environ.get('SAWSIM_BACKEND', '').lower() == 'b200':
        return install(modules)
    return []
