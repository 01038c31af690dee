"""The adjoint's parameter seeds on CPU (sawsim_b200.params): the geometry seeds
(node coordinates and PML bounds per unit of pitch or layer thickness) are the
exact derivatives of the cell builders, which are affine in those parameters,
and the stiffness seeds are the derivatives of the rotated 3m stiffness, which
is linear in its constants.  Checked against central differences at a step
10^4 times smaller than the seeds' own."""
import numpy as np
import pytest

from sawsim_b200 import materials as mt
from sawsim_b200.params import MATERIAL, HexModel, Q9Model


def _fd_cell(model, v, i, rel):
    h = rel * v[i]
    vp, vm = v.copy(), v.copy()
    vp[i] += h
    vm[i] -= h
    cp, cm = model._cell(vp), model._cell(vm)
    return cp, cm, h


@pytest.mark.parametrize('stack', ['two_layer', 'four_layer'])
def test_q9_geometry_seeds_are_exact(stack):
    model = Q9Model(8, 16, stack=stack)
    v = model.defaults()
    seeds = model.seeds(v)
    n = model._cell(v).POS.shape[0]
    for i, name in enumerate(model.geometry):
        cp, cm, h = _fd_cell(model, v, i, 5e-6)
        assert cp.POS.shape[0] == cm.POS.shape[0] == n          # same topology
        fd = (cp.POS[:, :2] - cm.POS[:, :2]) * 1e-6 / (2 * h)
        s = seeds[i]['dpos']
        assert np.max(np.abs(s - fd)) <= 1e-7 * max(np.max(np.abs(s)), 1e-6), name
        assert np.abs(s).max() > 0, name
        assert seeds[i]['dinner'][0, 1] == pytest.approx((cp.pml_top_um - cm.pml_top_um) * 1e-6 / (2 * h), rel=1e-7)
        assert seeds[i]['douter'][0, 1] == pytest.approx((cp.pml_bottom_um - cm.pml_bottom_um) * 1e-6 / (2 * h),
                                                          rel=1e-7, abs=1e-15)


def test_q9_stiffness_seeds_are_exact():
    model = Q9Model(8, 16)
    v = model.defaults()
    seeds = model.seeds(v)
    it = len(model.geometry)
    angles = np.array([model.euler[0], v[it], model.euler[2]])
    for j, name in enumerate(MATERIAL[1:], start=it + 1):
        h = 1e-3 * abs(v[j])
        vp, vm = v.copy(), v.copy()
        vp[j] += h
        vm[j] -= h
        fd = (mt.rotate(model._crystal_at(vp), angles).C - mt.rotate(model._crystal_at(vm), angles).C) / (2 * h)
        dC = seeds[j]['dC']
        assert np.max(np.abs(dC[0] - fd)) <= 1e-8 * np.max(np.abs(fd)), name
        assert not np.any(dC[1:]) and not np.any(seeds[j]['de']) and not np.any(seeds[j]['deps'])


def test_q9_theta_seed_matches_the_rotation():
    model = Q9Model(8, 16)
    v = model.defaults()
    it = len(model.geometry)
    s = model.seeds(v)[it]
    h = 1e-4
    out = []
    for d in (h, -h):
        angles = np.array([model.euler[0], v[it] + d, model.euler[2]])
        out.append(mt.rotate(model._crystal_at(v), angles))
    for key in ('C', 'e', 'eps'):
        fd = (getattr(out[0], key) - getattr(out[1], key)) / (2 * h)
        got = s['dC' if key == 'C' else 'de' if key == 'e' else 'deps'][0]
        assert np.max(np.abs(got - fd)) <= 1e-6 * np.max(np.abs(fd)), key


def test_hex_geometry_seeds_are_exact():
    model = HexModel(8, 2, 12)
    v = model.defaults()
    seeds = model.seeds(v)
    n = model._cell(v).POS.shape[0]
    for i, name in enumerate(model.names):
        cp, cm, h = _fd_cell(model, v, i, 5e-6)
        assert cp.POS.shape[0] == cm.POS.shape[0] == n
        fd = (cp.POS - cm.POS) * 1e-6 / (2 * h)
        s = seeds[i]['dpos']
        assert np.max(np.abs(s - fd)) <= 1e-7 * np.max(np.abs(s)), name
        assert seeds[i]['dinner'][0, 2] == pytest.approx((cp.pml_top_um - cm.pml_top_um) * 1e-6 / (2 * h),
                                                          rel=1e-7, abs=1e-15)
