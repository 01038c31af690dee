"""Error paths through the C ABI (marked gpu: a handle needs a CUDA device).

Every failure is made on the host (out-of-order calls, bad sizes, non-finite
inputs, a refinement budget too small to converge); none faults the GPU.
"""
import ctypes as C

import numpy as np
import pytest

from sawsim_b200 import _lib as L, cases
from sawsim_b200.engine import FrequencySolver, Handle
from sawsim_b200.materials import pack

pytestmark = pytest.mark.gpu


def _rc(h, name, *args):
    return getattr(h.lib, name)(h.h, *args)


def test_calls_out_of_order(built_lib):
    h = Handle(0)
    try:
        om = L.f64([1e10])
        Q = np.zeros(2)
        st = np.zeros(1, dtype=np.int32)
        assert _rc(h, 'ss_sweep', 1, L.ptr(om, C.c_double), 1.0, 0, L.ptr(Q, C.c_double), L.ptr(st, C.c_int),
                   None) == L.SS_ESTATE
        assert _rc(h, 'ss_analyze') == L.SS_ESTATE
        assert _rc(h, 'ss_assemble') == L.SS_ESTATE
        assert b'analyze' in h.lib.ss_last_error(h.h) or b'mesh' in h.lib.ss_last_error(h.h)
    finally:
        h.close()


@pytest.fixture(scope='module')
def small(built_lib):
    case = cases.make_case('me1_64x256', cols=8, rows=16)
    g = cases.engine_for(case)
    yield case, g
    g.close()


def test_bad_sweep_arguments(small):
    case, g = small
    h = g._h
    Q = np.zeros(4)
    st = np.zeros(2, dtype=np.int32)
    pq, ps = L.ptr(Q, C.c_double), L.ptr(st, C.c_int)
    good = L.f64(2 * np.pi * case.freqs[:2])
    assert _rc(h, 'ss_sweep', -1, L.ptr(good, C.c_double), 1.0, 0, pq, ps, None) == L.SS_EINVAL
    assert _rc(h, 'ss_sweep', 2, None, 1.0, 0, pq, ps, None) == L.SS_EINVAL
    assert _rc(h, 'ss_sweep', 2, L.ptr(good, C.c_double), 0.0, 0, pq, ps, None) == L.SS_EINVAL
    assert _rc(h, 'ss_sweep', 2, L.ptr(good, C.c_double), 1.0, 7, pq, ps, None) == L.SS_EINVAL
    for bad in ([-1.0, 1e10], [np.nan, 1e10], [np.inf, 1e10]):
        om = L.f64(bad)
        assert _rc(h, 'ss_sweep', 2, L.ptr(om, C.c_double), 1.0, 0, pq, ps, None) == L.SS_EINVAL
    # the handle stays usable after rejected calls
    Qg, stg, _ = g.charges(good, 1.0, 'fp64')
    assert (stg == 0).all() and np.isfinite(Qg).all()


def test_non_finite_inputs_rejected(small):
    case, g = small
    h = g._h
    mats = list(case.materials)
    rho, Cm, em, epsm = pack(mats, 3)
    Cm = Cm.copy()
    Cm[0, 0, 0, 0] = np.nan
    assert _rc(h, 'ss_set_materials', L.SS_MAT_K, len(rho), L.ptr(rho, C.c_double), L.ptr(Cm, C.c_double),
               L.ptr(em, C.c_double), L.ptr(epsm, C.c_double)) == L.SS_EINVAL
    assert _rc(h, 'ss_set_damping', float('nan')) == L.SS_EINVAL
    assert _rc(h, 'ss_set_damping', -1.0) == L.SS_EINVAL
    # a positive beta without damping materials is a call out of order
    assert _rc(h, 'ss_set_damping', 1e-12) == L.SS_ESTATE


def test_options_validated(small):
    _, g = small
    for name, value in (('krylov_restart', 0), ('krylov_restart', 2.5), ('krylov_tol', 1.5), ('fp64_fallback', 2),
                        ('no_such_option', 1)):
        with pytest.raises(L.SawsimError) as e:
            g.set_option(name, value)
        assert e.value.code == L.SS_EINVAL
    with pytest.raises(L.SawsimError) as e:
        g.gemm_ceiling(9)
    assert e.value.code == L.SS_EINVAL


def test_unconverged_mixed_points_reported_then_resolved_in_fp64(built_lib):
    """A one-step Krylov budget cannot reach the 1e-10 target on the 16.5k-DOF
    cell (3-7 steps are needed): without the FP64 re-solve those points come back
    SS_ENOCONV; with it (the default) every point is SS_OK and carries the FP64
    charge."""
    case = cases.make_case('me1_64x256', cols=16, rows=64)
    g = cases.engine_for(case)
    try:
        w = 2 * np.pi * np.linspace(case.freqs[0], case.freqs[-1], 9)
        Q64, st64, _ = g.charges(w, 1.0, 'fp64')
        assert (st64 == 0).all()
        g.set_option('krylov_restart', 1)
        g.set_option('krylov_cycles', 1)
        g.set_option('fp64_fallback', 0)
        _, st, _ = g.charges(w, 1.0, 'mixed')
        s = g.stats()
        assert (st == L.SS_ENOCONV).any()
        assert s['mixed_not_converged'] == int(np.sum(st == L.SS_ENOCONV)) and s['fp64_resolved'] == 0
        g.set_option('fp64_fallback', 1)
        Q, st, _ = g.charges(w, 1.0, 'mixed')
        s = g.stats()
        assert (st == 0).all()
        assert s['fp64_resolved'] == s['mixed_not_converged'] > 0
        bad = s['fp64_resolved']
        assert bad > 0
        # re-solved points carry the FP64 charge of the same point
        assert np.max(np.abs(Q - Q64) / np.abs(Q64)) < 1e-6
    finally:
        g.close()


def test_auto_decision_kept_until_an_option_changes(small):
    case, g = small
    w = 2 * np.pi * case.freqs[:5]
    g.charges(w, 1.0, 'auto')
    probe = g.stats()['auto_probe_ms']
    assert probe > 0
    g.charges(w, 1.0, 'auto')
    assert g.stats()['auto_probe_ms'] == probe            # no new probe for the same band
    # a changed option drops the decision: the next AUTO sweep probes again, and
    # its device time includes the probe
    g.set_option('auto_probe_steps', 12)
    g.charges(w, 1.0, 'auto')
    s = g.stats()
    assert s['auto_probe_ms'] > 0 and s['sweep_device_ms'] >= s['auto_probe_ms']


def test_matrix_input_errors(built_lib):
    """ss_set_csr / ss_set_values reject bad patterns and out-of-order calls; a
    matrix handle has no mesh to assemble or differentiate."""
    h = Handle(0)
    try:
        v = np.zeros(2 * 3)
        assert _rc(h, 'ss_set_values', L.SS_MAT_K, L.ptr(v, C.c_double)) == L.SS_ESTATE     # no pattern yet
        ip, ix = L.i64([0, 2, 3]), L.i64([1, 0, 1])                                          # row 0 not ascending
        assert _rc(h, 'ss_set_csr', 2, L.ptr(ip, C.c_int64), L.ptr(ix, C.c_int64), 0, 0, None, None) == L.SS_EINVAL
        ix = L.i64([0, 2, 1])                                                                 # column out of range
        assert _rc(h, 'ss_set_csr', 2, L.ptr(ip, C.c_int64), L.ptr(ix, C.c_int64), 0, 0, None, None) == L.SS_EINVAL
        ix = L.i64([0, 1, 1])
        xyz = L.f64([[0.0, 0.0]])
        assert _rc(h, 'ss_set_csr', 2, L.ptr(ip, C.c_int64), L.ptr(ix, C.c_int64), 1, 2, None,
                   L.ptr(xyz, C.c_double)) == L.SS_EINVAL                                     # coordinates need dof_node
        dn = L.i64([0, 1])
        assert _rc(h, 'ss_set_csr', 2, L.ptr(ip, C.c_int64), L.ptr(ix, C.c_int64), 1, 0, L.ptr(dn, C.c_int64),
                   None) == L.SS_EINVAL                                                       # node id out of range
        assert _rc(h, 'ss_set_csr', 2, L.ptr(ip, C.c_int64), L.ptr(ix, C.c_int64), 0, 0, None, None) == L.SS_OK
        assert _rc(h, 'ss_set_values', 7, L.ptr(v, C.c_double)) == L.SS_EINVAL
        bad = np.array([1.0, 0.0, np.nan, 0.0, 1.0, 0.0])
        assert _rc(h, 'ss_set_values', L.SS_MAT_K, L.ptr(bad, C.c_double)) == L.SS_EINVAL
        assert _rc(h, 'ss_assemble') == L.SS_ESTATE
        assert _rc(h, 'ss_analyze') == L.SS_ESTATE                                            # no values yet
    finally:
        h.close()
    case = cases.make_case('me1_64x256', cols=8, rows=16, points=3)
    g = cases.engine_for(case)
    try:
        e = FrequencySolver.from_matrices(g.export(L.SS_MAT_K), g.export(L.SS_MAT_M), *case.bc)
        try:
            with pytest.raises(L.SawsimError) as ex:
                e.gradient(2 * np.pi * case.freqs[:1], [dict(drho=np.ones(2))])
            assert ex.value.code == L.SS_ESTATE
        finally:
            e.close()
        with pytest.raises(ValueError):
            g.update_matrices(K=None)                       # a mesh engine assembles its own matrices
    finally:
        g.close()
