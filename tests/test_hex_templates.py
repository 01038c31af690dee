"""The reference's 2.5D Hex27 templates rebuilt without Gmsh
(cells.sp_2p5d_template_cell), run through the oracle on CPU at the test
frequencies of the reference's own template test (tests/test_templates.py:14-39):

* |Y| (the raw slice admittance, i w Q / V) against the published curve within
  5e-4 (the reference's regression tolerance is 2e-3; the published curves come
  from PARDISO and the oracle solves with SuperLU, which differ by about 1e-4 on
  these systems, docs/validation.en.md:41-43);
* and against the independent FEM curve within the template's own
  ``reference_rtol``.
"""
import json

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import hex27 as oh
from sawsim_b200 import cells

_G = json.loads((GOLDEN / 'hex_templates.json').read_text())


@pytest.mark.parametrize('t', _G, ids=[t['kind'] for t in _G])
def test_hex_template_reproduces_published_curves(t):
    cfg = t['config']
    cell = cells.sp_2p5d_template_cell(t['kind'], cfg['pitch_um'], cfg['electrode_um'], cfg['substrate_um'],
                                       [layer['thickness_um'] for layer in cfg['layers']], cfg['metal_ratio'],
                                       cfg['mesh_um'], cfg['aperture_um'])
    pos_m = cell.POS * 1e-6
    idx = np.array([cell.tag_map[int(tag)] for tag in cell.hex_tag])
    pml_mask = cell.hex_tag == cell.pml_tag
    mats = [dict(rho=m['rho'], C=np.array(m['C']), e=np.array(m['e']), eps=np.array(m['eps'])) for m in t['materials']]
    regions = [dict(mats[i], indx=np.where((idx == i) & ~pml_mask)[0]) for i in range(len(mats))]
    bottom = float(pos_m[:, 2].min())
    pml = [dict(region=3, indx=np.where(pml_mask)[0], za=bottom + 2 * cfg['pitch_um'] * 1e-6, zp=bottom, xa=0.0,
                xp=0.0, dmax=1e11, n=3, **mats[cell.tag_map[cell.pml_tag]])]
    M, K = oh.form_stiffness_mass_3d(cell.HEXAS27, pos_m, regions, pml, 2 * np.pi * t['freeze_hz'])
    o = oh.FrequencySolver3D(K, M, oh.boundary_idx_vect_3ds(cell.sets, pos_m, 3 * cell.POS.shape[0]))
    f = np.array(t['frequency_hz'])
    Y = np.abs(1j * 2 * np.pi * f * o.sweep(f) / cfg['voltage'])
    pub, fem = np.array(t['published']), np.array(t['independent_fem'])
    assert np.max(np.abs(Y - pub) / pub) < 5e-4
    assert np.max(np.abs(Y - fem) / fem) < t['reference_rtol']


@pytest.mark.parametrize('t', _G, ids=[t['kind'] for t in _G])
def test_hex_template_through_the_product_host_path(t):
    """The rebuilt templates through the product's own host path (the Bloch / front-back
    sets of cases.bc_periodic_3d, the host analysis): the oracle's active DOFs and a
    complete front tree, so the GPU engine takes them like the slab cells."""
    from sawsim_b200 import cases
    from sawsim_b200.analysis import analyze_hex27
    cfg = t['config']
    cell = cells.sp_2p5d_template_cell(t['kind'], cfg['pitch_um'], cfg['electrode_um'], cfg['substrate_um'],
                                       [layer['thickness_um'] for layer in cfg['layers']], cfg['metal_ratio'],
                                       cfg['mesh_um'], cfg['aperture_um'])
    pos_m = cell.POS * 1e-6
    N = cell.POS.shape[0]
    a = analyze_hex27(pos_m, cell.HEXAS27, cases.bc_periodic_3d(cell.sets, pos_m, N))
    mach, elec = oh.boundary_idx_vect_3ds(cell.sets, pos_m, 3 * N)
    presc = np.unique(np.concatenate([mach['fix'], mach['period_B'], mach['period_R'], elec['period_R'],
                                      elec['period_B'], elec['zheng'], elec['fu']]))
    assert np.array_equal(a.active, np.setdiff1d(np.arange(4 * N), presc))
    assert int(a.k.sum()) == a.n_active
