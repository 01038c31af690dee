"""Template cases from configuration fields (sawsim_b200.templates), on CPU:
the sp_double_layer default configuration's case through the oracle reproduces
the published curve (1e-8, as the cell itself does); the wiring of materials,
PML, Bloch sets, loss and projections follows the reference's builders
(models.py:27-140, hex_models.py:57-107); unsupported requests are refused."""
import json

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import oracle_engine
from oracle import solver as osol
from sawsim_b200 import cases, cells, templates
from sawsim_b200.materials import Material

DOUBLE = dict(model_id='sp_double_layer', mode_extension=1, substrate_material='sp_baseline', electrode_material='al',
              layers=[dict(material_id='si_isotropic', thickness_um=8.33)], pitch_um=1.085, electrode_um=0.17,
              substrate_um=0.6, metal_ratio=0.5, mesh_um=0.5, start_ghz=1.5, stop_ghz=2.7, points=5, voltage=1.0)


def _double_materials():
    g = np.load(GOLDEN / 'sp_double_layer.npz')
    return g, [Material(g['rho'][i], g['C'][i], g['e'][i], g['eps'][i]) for i in range(len(g['rho']))]


def test_double_layer_config_reproduces_the_published_curve():
    g, mats = _double_materials()
    case, loss = templates.case_for(DOUBLE, mats)
    assert loss.beta_dk == 0 and loss.eta_eps == 0
    assert np.allclose(case.freqs, g['frequency_hz'])
    _, _, o = oracle_engine(case)
    Y = osol.admittance_2d(case.freqs, o.sweep(case.freqs))
    assert np.max(np.abs(np.abs(Y) - g['published_magnitude']) / g['published_magnitude']) < 1e-8


def test_q9_wiring_follows_the_reference_builder():
    _, mats = _double_materials()
    cfg = dict(DOUBLE, model_id='sp_stack', layers=[dict(material_id='sio2', thickness_um=0.5),
                                                     dict(material_id='si', thickness_um=7.0)],
               coatings=[dict(material_id='sio2', thickness_um=0.4)], eta_eps=0.01, beta_dk=1e-13)
    mats4 = mats + [mats[2], mats[2]]
    case, loss = templates.case_for(cfg, mats4)
    cell = case.cell
    # tags 16 piezo, 15 electrode, 22/23 backings, 24 coating, 25 PML with the last backing's material
    assert cell.tag_map == {16: 0, 15: 1, 22: 2, 23: 3, 24: 4, 25: 3}
    assert np.array_equal(case.mat_idx, [cell.tag_map[int(t)] for t in case.mesh.elem_tag])
    p = case.pml[0]
    assert p.tag == 25 and p.kind == 'y' and p.ya - p.yp == pytest.approx(2 * cfg['pitch_um'] * 1e-6)
    assert p.yp == pytest.approx(case.mesh.pos_m[:, 1].min())
    # dielectric loss on the piezo only; Rayleigh damping on its stiffness only
    assert np.allclose(case.materials[0].eps, mats4[0].eps * (1 - 0.01j))
    assert all(np.array_equal(a.eps, b.eps) for a, b in zip(case.materials[1:], mats4[1:]))
    assert loss.beta_dk == 1e-13
    d = templates.damping_materials(case.materials)
    assert np.array_equal(d[0].C, case.materials[0].C) and not np.any(d[0].e) and not np.any(d[1].C)
    # plane strain: xy projection, xz for the TC-SAW substrate
    me0, _ = templates.case_for(dict(cfg, mode_extension=0), mats4)
    assert me0.materials[0].C.shape == (3, 3) and me0.materials[0].C[2, 2] == mats4[0].C[5, 5]
    tc, _ = templates.case_for(dict(cfg, mode_extension=0, substrate_material='linbo3_tc'), mats4)
    assert tc.materials[0].C[1, 1] == mats4[0].C[2, 2] and tc.materials[0].C[2, 2] == mats4[0].C[4, 4]
    assert len(me0.bc[0]) < len(case.bc[0])                     # two displacement components


def test_hex_template_config():
    t = json.loads((GOLDEN / 'hex_templates.json').read_text())[1]
    mats = [Material(m['rho'], np.array(m['C']), np.array(m['e']), np.array(m['eps'])) for m in t['materials']]
    case, loss = templates.case_for(dict(t['config'], start_ghz=1.75, stop_ghz=2.0, points=251), mats)
    assert isinstance(case, cases.HexCase) and case.freqs[-1] == pytest.approx(t['freeze_hz'])
    assert case.cell.pml_tag == 10 and case.cell.tag_map[10] == 2
    p = case.pml[0]
    assert p.kind == 'z' and p.za - p.zp == pytest.approx(2 * t['config']['pitch_um'] * 1e-6)
    ref = cells.sp_2p5d_template_cell('double', substrate_um=0.6, layers_um=[6.51])
    assert np.array_equal(case.hexas, ref.HEXAS27)


def test_unsupported_requests_are_refused():
    _, mats = _double_materials()
    with pytest.raises(ValueError, match='default geometry'):
        templates.case_for(dict(DOUBLE, pitch_um=1.2), mats)
    with pytest.raises(ValueError, match='materials expected'):
        templates.case_for(DOUBLE, mats[:2])
    with pytest.raises(ValueError, match='no Gmsh-free rebuild'):
        templates.case_for(dict(DOUBLE, model_id='sp_tcsaw'), mats)


def test_config_objects_are_accepted():
    """A configuration object with ``model_dump`` (the reference's SimulationConfig)
    gives the same case as its dict."""
    _, mats = _double_materials()

    class Config:
        def model_dump(self):
            return dict(DOUBLE)

    a, _ = templates.case_for(Config(), mats)
    b, _ = templates.case_for(DOUBLE, mats)
    assert np.array_equal(a.mat_idx, b.mat_idx) and np.array_equal(a.freqs, b.freqs)
