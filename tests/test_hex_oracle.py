"""The Hex27 oracle and the host-side 3D boundary builder are pinned against the
reference's own 2.5D slab path (tests/golden/ref_hex_*.npz, made by
make_hex_golden.py from saw3d/assembly.py, boundary.py and bc_solve.py).  CPU only."""
import numpy as np
import pytest

from conftest import GOLDEN
from oracle import hex27 as oh
from sawsim_b200 import cases

SMALL = [(8, 1, 6, 4), (8, 2, 12, 3)]


def _inputs(c):
    pml_mask = c.cell.hex_tag == c.cell.pml_tag
    mats = [dict(rho=m.rho, C=m.C, e=m.e, eps=m.eps, indx=np.where((c.mat_idx == i) & ~pml_mask)[0])
            for i, m in enumerate(c.materials)]
    pm = c.materials[c.cell.tag_map[c.cell.pml_tag]]
    p = c.pml[0]
    pml = [dict(region=3, indx=np.where(pml_mask)[0], za=p.za, zp=p.zp, xa=0.0, xp=0.0, dmax=p.dmax, n=p.n,
                rho=pm.rho, C=pm.C, e=pm.e, eps=pm.eps)]
    return mats, pml


@pytest.fixture(scope='module', params=SMALL, ids=lambda s: f'{s[0]}x{s[1]}x{s[2]}')
def slab(request):
    nx, ny, nz, nf = request.param
    c = cases.make_hex_case('hex_8x4x48', nx=nx, ny=ny, nz=nz, points=nf)
    g = np.load(GOLDEN / f'ref_hex_{nx}x{ny}x{nz}.npz')
    mats, pml = _inputs(c)
    M, K = oh.form_stiffness_mass_3d(c.hexas, c.pos_m, mats, pml, c.omega_top)
    bnd = oh.boundary_idx_vect_3ds(c.cell.sets, c.pos_m, 3 * c.N)
    return c, g, K, M, bnd


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def test_assembly_matches_reference(slab):
    c, g, K, M, _ = slab
    N = c.N
    # u rows/cols carry the 6.7e-11 scale, phi rows do not: compare per row block
    for rows in (slice(0, 3 * N), slice(3 * N, 4 * N)):
        assert _rel((K @ g['v'])[rows], g['Kv'][rows]) < 1e-12
    assert _rel(M @ g['v'], g['Mv']) < 1e-12


def test_boundary_lists_match_reference(slab):
    c, g, _, _, (m, e) = slab
    for k, x in m.items():
        assert np.array_equal(x, g[f'm_{k}']), k
    for k, x in e.items():
        assert np.array_equal(x, g[f'e_{k}']), k


def test_host_fold_groups_match_reference(slab):
    """cases.bc_periodic_3d gives the same master/slave pairs, in the same two stages."""
    c, g, _, _, _ = slab
    fix, zheng, fu, groups, two = c.bc
    fb = np.array(groups[:two])
    lr = np.array(groups[two:])
    assert np.array_equal(fb[:, 0], np.concatenate([g['m_period_F'], g['e_period_F']]))
    assert np.array_equal(fb[:, 1], np.concatenate([g['m_period_B'], g['e_period_B']]))
    assert np.array_equal(lr[:, 0], np.concatenate([g['m_period_L'], g['e_period_L']]))
    assert np.array_equal(lr[:, 1], np.concatenate([g['m_period_R'], g['e_period_R']]))
    assert np.array_equal(fix, g['m_fix']) and np.array_equal(zheng, g['e_zheng']) and np.array_equal(fu, g['e_fu'])


def test_solver_matches_reference(slab):
    c, g, K, M, bnd = slab
    eng = oh.FrequencySolver3D(K, M, bnd)
    assert np.array_equal(eng.active, g['active'])
    assert _rel(eng.k_aa @ g['w'], g['kaa_w']) < 1e-11
    # The unscaled 3D systems have 2-norm condition numbers near 3e15: K from the
    # oracle's element-wise Grams and from the reference's global B^T D B products
    # differ at 1e-16, which moves Q by up to ~5e-6 relative.  Given the
    # reference's own K and M, the oracle's solve reproduces its Q exactly.
    Q = eng.sweep(g['frequency_hz'])
    assert np.max(np.abs(Q - g['Q']) / np.abs(g['Q'])) < 2e-5


def test_four_layer_slab_pairs_match_coordinates():
    """The four-layer slab's front/back and left/right pairs sit at equal (x, z) /
    (y, z) and one aperture / one period apart (the checks of hex_models.py:34-45)."""
    c = cases.make_hex_case('hex_12x6x80', nx=12, ny=2, nz=16)
    fix, zheng, fu, groups, two = c.bc
    N = c.N
    node = lambda d: d // 3 if d < 3 * N else d - 3 * N          # noqa: E731
    g = np.array(groups)
    m = np.array([node(d) for d in g[:, 0]])
    s = np.array([node(d) for d in g[:, 1]])
    P = c.pos_m
    fb, lr = slice(0, two), slice(two, None)
    assert np.allclose(P[m[fb]][:, [0, 2]], P[s[fb]][:, [0, 2]], atol=1e-13)
    assert np.allclose(P[s[fb], 1] - P[m[fb], 1], c.cell.aperture_um * 1e-6, atol=1e-13)
    assert np.allclose(P[m[lr]][:, [1, 2]], P[s[lr]][:, [1, 2]], atol=1e-13)
    assert np.allclose(P[s[lr], 0] - P[m[lr], 0], c.cell.period_um * 1e-6, atol=1e-13)


def test_finite_device_solver_matches_reference():
    """The oracle's finite-device solver (front/back fold, then the floating
    electrodes' equipotential fold) against the reference's FrequencySolver3D_FP
    (bc_solve.py:214-335) on the 8x2x12 slab with two floating strips
    (ref_hex_fp_8x2x12.npz)."""
    c = cases.make_hex_case('hex_8x4x48', nx=8, ny=2, nz=12, points=3)
    g = np.load(GOLDEN / 'ref_hex_fp_8x2x12.npz')
    mats, pml = _inputs(c)
    M, K = oh.form_stiffness_mass_3d(c.hexas, c.pos_m, mats, pml, c.omega_top)
    m, e = oh.boundary_idx_vect_3ds(c.cell.sets, c.pos_m, 3 * c.N)
    e = dict(e, XFL=g['XFL'], XFR=g['XFR'])
    eng = oh.FrequencySolver3DFP(K, M, (m, e))
    assert np.array_equal(eng.active, g['active'])
    Q = eng.sweep(g['frequency_hz'])
    assert np.max(np.abs(Q - g['Q']) / np.abs(g['Q'])) < 2e-5
