"""The backend switch on CPU: which reference names ``install`` replaces, the
environment selection, the metadata the pipelines write through the wrapped
``atomic_json``, and ``charge_stream``'s point-by-point path for engines that are
not this backend's (the reference's own, here a stand-in)."""
import types

import numpy as np

from sawsim_b200 import backend


def _fake_reference():
    names = {'sawsim.saw2d.sweep': ['FrequencySolver'],
             'sawsim.saw2d.saw3d.bc_solve': ['FrequencySolver3D', 'FrequencySolver3D_FP'],
             'sawsim.saw2d.saw3d': ['FrequencySolver3D'],
             'sawsim.frequency_tasks': ['charge_stream'],
             'sawsim.solver': ['charge_stream'],
             'sawsim.hex_solver': ['charge_stream', 'FrequencySolver3D']}
    mods = {}
    for mod, attrs in names.items():
        m = types.ModuleType(mod)
        for a in attrs:
            setattr(m, a, object())
        mods[mod] = m
    return mods


def test_install_replaces_every_pipeline_name():
    mods = _fake_reference()
    done = backend.install(mods)
    assert len(done) == 8
    assert mods['sawsim.saw2d.sweep'].FrequencySolver is backend.FrequencySolver
    assert mods['sawsim.solver'].charge_stream is backend.charge_stream
    assert mods['sawsim.hex_solver'].FrequencySolver3D is backend.FrequencySolver3D
    assert mods['sawsim.saw2d.saw3d.bc_solve'].FrequencySolver3D_FP is backend.FrequencySolver3D


def test_install_touches_only_loaded_modules():
    mods = {'sawsim.solver': types.ModuleType('sawsim.solver')}
    mods['sawsim.solver'].charge_stream = None
    assert backend.install(mods) == ['sawsim.solver.charge_stream']


def test_install_from_env(monkeypatch):
    mods = _fake_reference()
    monkeypatch.delenv('SAWSIM_BACKEND', raising=False)
    assert backend.install_from_env(mods) == []
    monkeypatch.setenv('SAWSIM_BACKEND', 'b200')
    assert len(backend.install_from_env(mods)) == 8


class _PointEngine:
    """Stand-in for the reference's engine: Q = omega * V."""

    def __init__(self, hex_kw):
        self.hex_kw = hex_kw

    def solve(self, omega, V=None, voltage=None):
        v = voltage if self.hex_kw else V
        assert v is not None
        return None, complex(omega * v), None


def test_charge_stream_point_by_point_for_other_engines():
    f = np.array([1e9, 2e9, 3e9])
    for is_hex in (False, True):
        with backend.charge_stream(_PointEngine(is_hex), f, 2.0, is_hex=is_hex) as res:
            q = [next(res) for _ in f]
        assert np.allclose(q, 2 * np.pi * f * 2.0)


def test_install_names_the_backend_in_the_metadata(monkeypatch):
    monkeypatch.delenv('SAWSIM_B200_PRECISION', raising=False)
    written = []
    m = types.ModuleType('sawsim.solver')
    m.atomic_json = lambda path, data: written.append((str(path), data))
    mods = {'sawsim.solver': m}
    assert backend.install(mods) == ['sawsim.solver.atomic_json']
    first = m.atomic_json
    backend.install(mods)                      # a second install does not wrap twice
    assert m.atomic_json is first
    meta = dict(backend='SciPy SuperLU', frequency_workers=8, nodes=12)
    m.atomic_json('out/metadata.json', meta)
    m.atomic_json('out/curve.json', dict(backend='left alone'))
    assert written[0] == ('out/metadata.json', dict(backend='B200 (sawsim_b200, fp64)', frequency_workers=1,
                                                    nodes=12))
    assert meta['backend'] == 'SciPy SuperLU'  # the caller's dict is not modified
    assert written[1] == ('out/curve.json', dict(backend='left alone'))
