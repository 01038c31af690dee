"""Material builders pinned to the reference's own outputs (CPU).

The fixture ``golden/materials.npz`` was written by ``golden/make_materials_golden.py``
with the reference's ``crystal.tensors`` (src/sawsim/crystal.py:30-78),
``oula_transfer`` / ``rotation_matrix`` / ``project_xy_plane_strain`` /
``project_xz_plane_strain``
(src/sawsim/saw2d/materials.py:28-71, :250-265, :281-290, :303-308) and central
differences of ``oula_transfer`` in the second Euler angle.  These tests check
``sawsim_b200.materials`` (which feeds both the GPU path and the oracle) and the
d/dtheta tangent of ``sawsim_b200.params`` against them.
"""
from pathlib import Path

import numpy as np
import pytest

from sawsim_b200 import materials as mt
from sawsim_b200.params import rotation_tangent

G = np.load(Path(__file__).resolve().parent / 'golden' / 'materials.npz')
KEYS = ['C11', 'C12', 'C13', 'C14', 'C33', 'C44', 'e15', 'e22', 'e31', 'e33', 'eps11', 'eps33']


def _crystal(consts):
    k = dict(zip(KEYS, consts))
    for x in ('C11', 'C12', 'C13', 'C14', 'C33', 'C44'):
        k[x] = k[x] * 1e9
    return mt.trigonal_3m(k, 4700.0)


def test_eps0_matches_crystal_builder():
    assert mt.EPS0 == float(G['EPS0'])


@pytest.mark.parametrize('seed', range(4))
def test_trigonal_3m_matches_reference(seed):
    m = _crystal(G[f's{seed}_consts'])
    np.testing.assert_allclose(m.C, G[f's{seed}_C'], rtol=1e-15, atol=0)
    np.testing.assert_array_equal(m.e, G[f's{seed}_e'])
    np.testing.assert_allclose(m.eps, G[f's{seed}_eps'], rtol=1e-15, atol=0)


def test_trigonal_3m_reproduces_literature_record():
    """The reference's own known answer (tests/test_stack_materials.py:64-72):
    rebuilding LiNbO3 from its independent constants gives the library record."""
    m = _crystal(G['linbo3_consts'])
    built = G['linbo3_built']
    np.testing.assert_allclose(m.C.ravel(), built[:36], rtol=1e-15, atol=0)
    np.testing.assert_allclose(m.e.ravel(), built[36:54], rtol=0, atol=0)
    np.testing.assert_allclose(m.eps.ravel(), built[54:], rtol=1e-15, atol=0)
    rec = G['linbo3_record']
    np.testing.assert_allclose(m.C.ravel(), rec[:36], rtol=0, atol=1e-3)
    np.testing.assert_allclose(m.e.ravel(), rec[36:54])
    np.testing.assert_allclose(m.eps.ravel(), rec[54:])


@pytest.mark.parametrize('name,mat', [('al', mt.al()), ('sio2', mt.sio2()), ('polysi', mt.poly_si()),
                                      ('si', mt.si_cubic())])
def test_isotropic_and_cubic_match_reference(name, mat):
    ref = G['cubic_si' if name == 'si' else f'iso_{name}']
    np.testing.assert_allclose(mat.C.ravel(), ref[:36], rtol=1e-15, atol=0)
    np.testing.assert_array_equal(mat.e.ravel(), ref[36:54])
    np.testing.assert_allclose(mat.eps.ravel(), ref[54:], rtol=1e-15, atol=0)


@pytest.mark.parametrize('seed', range(4))
def test_rotation_and_projection_match_oula_transfer(seed):
    """ZXZ rotation, Bond transform and plane-strain projection at the seeded
    Euler triple and four fixed ones: equal to the reference bit for bit."""
    m = _crystal(G[f's{seed}_consts'])
    for t, ref in zip(G[f's{seed}_triples'], G[f's{seed}_rot']):
        a = mt.rotation_matrix(t)
        r = mt.rotate(m, t)
        p = mt.project_xy_plane_strain(r)
        ours = np.concatenate([a.ravel(), r.C.ravel(), r.e.ravel(), r.eps.ravel(), p.C.ravel(), p.e.ravel(),
                               p.eps.ravel()])
        np.testing.assert_array_equal(ours, ref, err_msg=str(t))


@pytest.mark.parametrize('seed', range(4))
def test_tc_projection_matches_reference(seed):
    """The TC-SAW xz-plane projection of the rotated tensors: equal to the
    reference's project_xz_plane_strain bit for bit."""
    m = _crystal(G[f's{seed}_consts'])
    for t, ref in zip(G[f's{seed}_triples'], G[f's{seed}_xz']):
        q = mt.project_xz_plane_strain(mt.rotate(m, t))
        np.testing.assert_array_equal(np.concatenate([q.C.ravel(), q.e.ravel(), q.eps.ravel()]), ref, err_msg=str(t))


@pytest.mark.parametrize('seed', range(4))
def test_theta_tangent_matches_reference_differences(seed):
    """d(rotated C, e, eps)/d theta of the adjoint seeds against central
    differences (step 1e-4 degrees) of the reference's oula_transfer."""
    m = _crystal(G[f's{seed}_consts'])
    t = rotation_tangent(m, G[f's{seed}_euler'])
    ours = np.concatenate([t.C.ravel(), t.e.ravel(), t.eps.ravel()])
    ref = G[f's{seed}_dtheta']
    for lo, hi in ((0, 36), (36, 54), (54, 63)):      # per tensor, relative to its largest entry
        scale = np.abs(ref[lo:hi]).max()
        assert np.abs(ours[lo:hi] - ref[lo:hi]).max() <= 1e-7 * scale
