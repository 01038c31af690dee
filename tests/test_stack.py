"""The generic sp_stack template rebuilt without Gmsh (cells.sp_stack_cell), on CPU:

* its layout equals what the reference's own builder (src/sawsim/sp_meshes/
  stack.py:GM, run against a recording stand-in for gmsh by
  tests/golden/make_stack_golden.py) lays out, on five stacks: band levels,
  strip cuts, rows and columns, the tag of every (band, strip) surface, the
  electrode lines;
* the reference's cross-template test (tests/test_stack_materials.py:54-63):
  sp_stack with no layers at the sp_single_layer configuration, located by the
  oracle, gives fr / fa within 1 MHz of the independent FEM curve of
  sp_single_layer, and the same fr / fa as the reference's own assembly and
  solve on the rebuilt mesh.
"""
import json

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import q9 as oq9, solver as osol
from sawsim_b200 import cells
from sawsim_b200.locate import locate
from sawsim_b200.materials import Material

_G = json.loads((GOLDEN / 'sp_stack.json').read_text())


@pytest.mark.parametrize('case', _G['layouts'], ids=[f'layout{i}' for i in range(len(_G['layouts']))])
def test_layout_matches_reference_builder(case):
    ref = case['layout']
    c = cells.sp_stack_cell(case['pitch'], case['mr'], case['d'], case['h_piezo'], case['backings'],
                            case['coatings'], case['mesh_um'])
    info = c.info
    assert info['rows'] == ref['rows'] and info['cols'] == ref['cols']
    assert info['h_near'] == ref['h_near'] and info['h_deep'] == ref['h_deep']
    assert info['tag_backing'] == ref['tag_backing'] and info['tag_coating'] == ref['tag_coating']
    assert c.pml_tag == ref['tag_pml'] and info['pml_thickness_um'] == pytest.approx(ref['pml_thickness_um'])
    levels, cuts = np.array(ref['levels']), np.array(ref['cuts'])
    assert np.allclose(info['levels'], levels, rtol=0, atol=1e-12) and np.allclose(info['cuts'], cuts, rtol=0,
                                                                                  atol=1e-12)
    # every element lies in a (band, strip) surface of the reference, with its tag, and every surface is filled
    ctr = c.POS[c.QUADS9[:, 8].astype(int) - 1]
    band = np.searchsorted(levels, ctr[:, 1]) - 1
    strip = np.searchsorted(cuts, ctr[:, 0]) - 1
    mine = {(int(b), int(s), int(t)) for b, s, t in zip(band, strip, c.QUADS9[:, 9])}
    assert mine == {tuple(x) for x in ref['surfaces']}
    counts = {}
    for b, s in zip(band, strip):
        counts[(b, s)] = counts.get((b, s), 0) + 1
    for (b, s), n in counts.items():
        assert n == ref['rows'][b] * ref['cols'][s]
    # electrode lines: contact and top of the two strips, and the two outer flanks
    e_band = len(ref['rows']) - 1 - len(ref['tag_coating'])
    seg = 2 * (ref['cols'][1] + ref['cols'][2]) + 2 * ref['rows'][e_band]
    for tag in (17, 18):
        assert int(np.sum(c.LINES3[:, 3] == tag)) == seg
    # the cell is periodic: left and right line nodes pair by height
    lt, rt = (np.unique(c.LINES3[c.LINES3[:, 3] == t, :3].astype(int).ravel()) - 1 for t in (19, 20))
    assert np.allclose(np.sort(c.POS[lt, 1]), np.sort(c.POS[rt, 1])) and np.allclose(c.POS[lt, 0], 0)


class _OracleRun:
    """Oracle assembly and SuperLU solve on a cell, assembled with the PML frozen at
    each sweep's top frequency, as the reference's run does (solver.py:104-108)."""

    def __init__(self, cell, mats, pitch_um):
        self.m = oq9.build_model(cell.msh())
        self.mats = mats
        self.idx = oq9.material_index(self.m, cell.tag_map)
        bottom = float(self.m.pos_m[:, 1].min())
        self.pml = [oq9.PMLRegion(tag=cell.pml_tag, kind='y', yp=bottom, ya=bottom + 2 * pitch_um * 1e-6)]
        self.bc = osol.bc_periodic(self.m, cell.LINES3, ndisp=3)
        self.eng, self.top = None, None

    def set_freeze_frequency(self, w):
        if w != self.top:
            K, M = oq9.assemble(self.m, self.mats, self.idx, self.pml, w)
            self.eng, self.top = osol.FrequencySolver(K, M, *self.bc), w

    def charges(self, w, V=1.0, precision='fp64'):
        return self.eng.sweep(w / (2 * np.pi)) * V, np.zeros(w.size, np.int32), np.zeros(w.size, np.int32)

    def stats(self):
        return dict(sweep_device_ms=0.0, precision_used=0.0)


def test_single_layer_stack_matches_the_independent_fem():
    s = _G['single_layer']
    cfg = s['config']
    mats = [Material(s['rho'][i], np.array(s['C'][i]), np.array(s['e'][i]), np.array(s['eps'][i]))
            for i in range(len(s['rho']))]
    cell = cells.sp_stack_cell(cfg['pitch_um'], cfg['metal_ratio'], cfg['electrode_um'], cfg['substrate_um'], [], [],
                               cfg['mesh_um'])
    r = locate(_OracleRun(cell, mats, cfg['pitch_um']), cfg['start_ghz'], cfg['stop_ghz'], 41,
               tuple(s['band_limits_ghz']), zoom_points=101, precision='fp64')
    assert r['ok']
    fem, ref = s['independent_fem'], s['reference_on_rebuilt_mesh']
    assert abs(r['fr_ghz'] - fem['fr_ghz']) < 1e-3 and abs(r['fa_ghz'] - fem['fa_ghz']) < 1e-3
    assert abs(r['fr_ghz'] - ref['fr_ghz']) <= 1e-6 and abs(r['fa_ghz'] - ref['fa_ghz']) <= 1e-6
    assert r['band_ghz'] == ref['band_ghz'] and r['sweeps'] == ref['sweeps']


@pytest.mark.parametrize('t', _G['layered'], ids=[t['name'] for t in _G['layered']])
def test_stack_reproduces_the_layered_templates(t):
    """The same cross-template bar on the layered templates: sp_stack with their
    backings at their configurations, located by the oracle, within 1 MHz of their
    independent FEM fr / fa (sp_triple_layer is meshed unstructured by Gmsh and
    has no rebuild of its own)."""
    cfg = t['config']
    mats = [Material(t['rho'][i], np.array(t['C'][i]), np.array(t['e'][i]), np.array(t['eps'][i]))
            for i in range(len(t['rho']))]
    cell = cells.sp_stack_cell(cfg['pitch_um'], cfg['metal_ratio'], cfg['electrode_um'], cfg['substrate_um'],
                               [layer['thickness_um'] for layer in cfg['layers']], [], cfg['mesh_um'])
    r = locate(_OracleRun(cell, mats, cfg['pitch_um']), cfg['start_ghz'], cfg['stop_ghz'], 41,
               tuple(_G['single_layer']['band_limits_ghz']), zoom_points=101, precision='fp64')
    fem = t['independent_fem']
    assert r['ok'] and abs(r['fr_ghz'] - fem['fr_ghz']) < 1e-3 and abs(r['fa_ghz'] - fem['fa_ghz']) < 1e-3


@pytest.mark.parametrize('case', _G['layouts'][:2], ids=['no_layers', 'layers_and_coatings'])
def test_stack_through_the_product_host_path(case):
    """The rebuilt stack through the product's own host path (mesh, Bloch sets,
    host analysis): the active DOFs are the oracle's (its bc_periodic and fold) and
    the front tree is complete, so the GPU engine takes the cell like any Q9 cell."""
    from sawsim_b200 import cases
    from sawsim_b200.analysis import analyze_q9
    c = cells.sp_stack_cell(case['pitch'], case['mr'], case['d'], case['h_piezo'], case['backings'],
                            case['coatings'], case['mesh_um'])
    mesh = cases.mesh_from_msh(c.msh())
    a = analyze_q9(mesh.pos_m, mesh.quads, cases.bc_periodic(mesh, c.LINES3, 3))
    m = oq9.build_model(c.msh())
    fix, zheng, fu, groups = osol.bc_periodic(m, c.LINES3, ndisp=3)
    _, slaves, _ = osol.merge_transform(4 * m.N, groups)
    presc = np.unique(np.concatenate([np.asarray(fix, int), slaves, np.asarray(zheng, int), np.asarray(fu, int)]))
    assert np.array_equal(a.active, np.setdiff1d(np.arange(4 * m.N), presc))
    assert int(a.k.sum()) == a.n_active
