"""The oracle is pinned before it is trusted (CPU only).

* against the reference's published sp_double_layer and sp_quad_layer curves
  (tests/data of the reference, copied into tests/golden/<name>.npz with their
  materials);
* against the reference's own matrices and charges on small seeded cells
  (tests/golden/ref_me*.npz, produced by tests/golden/make_golden.py).
"""
import hashlib

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import oracle_engine
from oracle import q9 as oq9, solver as osol
from sawsim_b200 import cases, cells
from sawsim_b200.materials import Material


def _hash(A):
    A = A.tocsr()
    A.sort_indices()
    h = hashlib.sha256()
    h.update(np.asarray(A.indptr, dtype=np.int64).tobytes())
    h.update(np.asarray(A.indices, dtype=np.int64).tobytes())
    return h.hexdigest()


def template_oracle(name='sp_double_layer'):
    g = np.load(GOLDEN / f'{name}.npz')
    cell = {'sp_double_layer': cells.sp_double_layer_cell, 'sp_quad_layer': cells.sp_quad_layer_cell}[name]()
    m = oq9.build_model(cell.msh())
    mats = [Material(g['rho'][i], g['C'][i], g['e'][i], g['eps'][i]) for i in range(len(g['rho']))]
    idx = oq9.material_index(m, cell.tag_map)
    bottom = m.pos_m[:, 1].min()
    pml = [oq9.PMLRegion(tag=cell.pml_tag, kind='y', yp=bottom, ya=bottom + 2 * float(g['pitch_um']) * 1e-6)]
    f = g['frequency_hz']
    K, M = oq9.assemble(m, mats, idx, pml, 2 * np.pi * f[-1])
    eng = osol.FrequencySolver(K, M, *osol.bc_periodic(m, cell.LINES3, ndisp=3))
    return g, eng


@pytest.mark.parametrize('name', ['sp_double_layer', 'sp_quad_layer'])
def test_template_published_curve(name):
    """Structured templates rebuilt without Gmsh: the oracle reproduces the
    reference's published curve at its test frequencies."""
    g, eng = template_oracle(name)
    f = g['frequency_hz']
    Y = osol.admittance_2d(f, eng.sweep(f))
    pub = g['published_magnitude']
    assert np.max(np.abs(np.abs(Y) - pub) / pub) < 1e-8
    # and the reference's own run on the same rebuilt mesh (summation-order noise
    # of COO->CSR is amplified by the conditioning to ~1e-8, piezo_fem.py:383-387)
    assert np.max(np.abs(Y - g['reference_run_admittance']) / np.abs(g['reference_run_admittance'])) < 5e-8


def test_double_layer_realblock_route():
    g, eng = template_oracle()
    f = g['frequency_hz'][:2]
    Qc = eng.sweep(f, route='complex')
    Qr = eng.sweep(f, route='realblock')
    assert np.max(np.abs(Qc - Qr) / np.abs(Qr)) < 5e-8


@pytest.mark.parametrize('path', sorted(p.name for p in GOLDEN.glob('ref_me*.npz')))
def test_oracle_matches_reference_run(path):
    g = np.load(GOLDEN / path)
    name = path[4:].rsplit('_', 1)[0]
    case = cases.make_case(name, cols=int(g['cols']), rows=int(g['rows']))
    K, M, eng = oracle_engine(case)
    assert _hash(K) == str(g['K_pattern_sha256'])
    assert _hash(M) == str(g['M_pattern_sha256'])
    for A, key in ((K, 'Kv'), (M, 'Mv')):
        ref = g[key]
        assert np.max(np.abs(A @ g['v'] - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.array_equal(eng.active, g['active'])
    for A, key in ((eng.Km_aa, 'Kaa_w'), (eng.Mm_aa, 'Maa_w')):
        ref = g[key]
        assert np.max(np.abs(A @ g['w'] - ref)) <= 1e-12 * np.max(np.abs(ref))
    Q = eng.sweep(g['frequency_hz'])
    assert np.max(np.abs(Q - g['Q']) / np.abs(g['Q'])) < 5e-8
