"""Generate tests/golden/sp_stack.json from the reference's sp_stack template.

Run in the build container, where the reference (Duane245/sawsim 2.1.0) is
mounted read-only at /root/reference (SAWSIM_REFERENCE overrides):

    python tests/golden/make_stack_golden.py

It records, with no Gmsh (the reference's builder runs against a recording
stand-in for the gmsh module):

* for several stacks (no layers; the quad-layer stack with two coatings; six
  backings; three coatings; finer and coarser meshes; other pitch and metal
  ratio), what the reference's ``sp_meshes/stack.py:GM`` lays out: the band
  levels and strip cuts (its geometry points), rows and columns per band and
  strip, the physical tag of every (band, strip) surface, its tag lists;
* the layered templates' configurations (sp_double_layer, sp_triple_layer,
  sp_quad_layer: their tests/data records), resolved materials and the fr / fa
  of their independent FEM and published curves;
* the single-layer configuration of the reference's own cross-template test
  (tests/test_stack_materials.py:54-63, ``sp_stack`` with no layers against the
  ``sp_single_layer`` data): the resolved materials (records of its material
  library, the substrate rotated by ``oula_transfer``), the band limits of the
  template, fr / fa of the independent FEM curve (``reference_magnitude``) and
  of the reference's own published curve, both by the reference's
  ``resonances``, and fr / fa located on the rebuilt mesh by the reference's
  assembly and SciPy solve (``piezo_fem.assemble``, ``sweep.FrequencySolver``)
  with the PML frozen at each sweep's top, through the locate rules of
  ``sawsim_b200.locate`` (those of agent.py:406-477).

The tests read the fixture, never the reference checkout.
"""
from __future__ import annotations

import json
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
REF = Path(os.environ.get('SAWSIM_REFERENCE', '/root/reference'))
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REF / 'src'))


class _Recorder:
    """Stand-in for the gmsh module: records the points, the surfaces' corner
    points and the physical groups that stack.GM asks for."""

    def __init__(self):
        self.points, self.lines, self.loops, self.surfaces, self.groups = [], [], [], [], []
        rec = self

        class Geo:
            def addPoint(self, x, y, z, lc):
                rec.points.append((x, y))
                return len(rec.points)

            def addLine(self, a, b):
                rec.lines.append((a, b))
                return len(rec.lines)

            def addCurveLoop(self, ls):
                rec.loops.append(ls)
                return len(rec.loops)

            def addPlaneSurface(self, loops):
                rec.surfaces.append(loops[0])
                return len(rec.surfaces)

            def synchronize(self):
                pass

            class mesh:
                @staticmethod
                def setTransfiniteCurve(*a):
                    pass

                @staticmethod
                def setTransfiniteSurface(*a):
                    pass

                @staticmethod
                def setRecombine(*a):
                    pass

        class Model:
            geo = Geo()

            def add(self, name):
                pass

            def addPhysicalGroup(self, dim, items, tag):
                rec.groups.append((dim, list(items), tag))

            class mesh:
                @staticmethod
                def generate(*a):
                    pass

                @staticmethod
                def setOrder(*a):
                    pass

        self.model = Model()
        self.option = types.SimpleNamespace(setNumber=lambda *a: None)

    def initialize(self):
        pass


def gm_layout(pitch, mr, d, h_piezo, backings, coatings, mesh_um):
    rec = _Recorder()
    sys.modules['gmsh'] = rec
    import importlib
    import sawsim.sp_meshes.stack as stack
    importlib.reload(stack)
    out = stack.GM(pitch, mr, d, h_piezo, list(backings), list(coatings), mesh_um)
    # each surface's corner points -> (level index, strip index) of its bottom-left corner
    ys = sorted({y for _, y in rec.points})
    xs = sorted({x for x, _ in rec.points})
    cells = []
    for loop in rec.surfaces:
        first = rec.loops[loop - 1][0]                   # bottom line, left to right
        a, b = rec.lines[abs(first) - 1]
        x0, y0 = rec.points[a - 1]
        cells.append([ys.index(y0), xs.index(x0)])
    surf_tag = {}
    for dim, items, tag in rec.groups:
        if dim == 2:
            for s in items:
                surf_tag[s] = tag
    return dict(levels=ys, cuts=xs, rows=out['rows'], cols=out['cols'], h_near=out['h_near'], h_deep=out['h_deep'],
                tag_backing=out['tag_backing'], tag_coating=out['tag_coating'], tag_pml=out['tag_pml'],
                pml_thickness_um=out['pml_thickness_um'],
                surfaces=[[c[0], c[1], surf_tag[i + 1]] for i, c in enumerate(cells)])


LAYOUTS = [dict(pitch=1.085, mr=0.5, d=0.17, h_piezo=8.0, backings=[], coatings=[], mesh_um=0.5),
           dict(pitch=1.085, mr=0.5, d=0.17, h_piezo=0.6, backings=[0.5, 1.0, 7.83], coatings=[0.4, 0.05],
                mesh_um=0.25),
           dict(pitch=2.0, mr=0.4, d=0.2, h_piezo=0.5, backings=[0.3, 0.3, 0.4, 1.0, 2.0, 5.0], coatings=[],
                mesh_um=0.3),
           dict(pitch=0.9968, mr=0.46, d=0.16633, h_piezo=15.9488, backings=[], coatings=[0.72144, 0.04, 0.1],
                mesh_um=0.1),
           dict(pitch=1.5, mr=0.6, d=0.1, h_piezo=3.0, backings=[10.0], coatings=[0.3], mesh_um=0.8)]


def single_layer():
    from sawsim.material_library import get_record
    from sawsim.material_runtime import from_record
    from sawsim.metrics import resonances
    from sawsim.saw2d import piezo_fem, sweep
    from sawsim.saw2d.materials import Material, oula_transfer
    from sawsim.sp_specs import MODEL_SPECS
    from sawsim_b200 import cells
    from sawsim_b200.locate import locate

    meta = json.loads((REF / 'tests/data/sp_single_layer.json').read_text())
    data = np.load(REF / 'tests/data/sp_single_layer.npz')
    cfg = meta['config']
    sub = from_record(get_record(cfg['substrate_material']))
    el = from_record(get_record(cfg['electrode_material']))
    C, e, eps = oula_transfer([cfg['euler_phi_deg'], cfg['euler_theta_deg'], cfg['euler_psi_deg']], sub.C, sub.e,
                              sub.eps)
    mats = [Material(sub.rho, C, e, eps), el]
    lim = {f['key']: (f['min'], f['max']) for f in MODEL_SPECS['sp_stack']['numeric_fields']}
    limits = (lim['start_ghz'][0], lim['stop_ghz'][1])
    cell = cells.sp_stack_cell(cfg['pitch_um'], cfg['metal_ratio'], cfg['electrode_um'], cfg['substrate_um'], [],
                               [], cfg['mesh_um'])
    model = piezo_fem.build_model(type('M', (), cell.msh())())
    mi = piezo_fem.material_index(model, cell.tag_map)
    bottom = float(model.pos_m[model.nodes_with_tag(21, cell.LINES3), 1].min())
    pml = [piezo_fem.PMLRegion(tag=cell.pml_tag, kind='y', yp=bottom, ya=bottom + 2 * cfg['pitch_um'] * 1e-6)]
    bc = sweep.bc_periodic(model, cell.LINES3, ndisp=3)

    class ReferenceRun:
        """The reference's assembly and solve on the rebuilt mesh, assembled with the
        PML frozen at each sweep's top frequency as its run does (solver.py:104-108)."""

        def __init__(self):
            self.eng, self.top = None, None

        def set_freeze_frequency(self, w):
            if w != self.top:
                K, M = piezo_fem.assemble(model, mats, mi, pml, w)
                self.eng, self.top = sweep.FrequencySolver(K, M, *bc), w

        def charges(self, w, V=1.0, precision='fp64'):
            Q = np.array([self.eng.solve(x, V)[1] for x in w])
            return Q, np.zeros(w.size, np.int32), np.zeros(w.size, np.int32)

        def stats(self):
            return dict(sweep_device_ms=0.0, precision_used=0.0)

    r = locate(ReferenceRun(), cfg['start_ghz'], cfg['stop_ghz'], 41, limits, zoom_points=101, precision='fp64')
    fem = resonances(data['frequency_hz'], data['reference_magnitude'])
    pub = resonances(data['frequency_hz'], data['sawsim_magnitude'])
    return dict(config={k: v for k, v in cfg.items() if k != 'material_snapshots'}, band_limits_ghz=list(limits),
                rho=[m.rho for m in mats], C=[np.asarray(m.C).tolist() for m in mats],
                e=[np.asarray(m.e).tolist() for m in mats], eps=[np.asarray(m.eps).tolist() for m in mats],
                independent_fem=dict(fr_ghz=fem['fr_ghz'], fa_ghz=fem['fa_ghz']),
                published=dict(fr_ghz=pub['fr_ghz'], fa_ghz=pub['fa_ghz']),
                reference_on_rebuilt_mesh=dict(fr_ghz=r['fr_ghz'], fa_ghz=r['fa_ghz'], band_ghz=r['band_ghz'],
                                               sweeps=r['sweeps']))


def layered_templates():
    """The layered templates' configurations (their tests/data records), resolved
    materials and the fr / fa of their independent FEM and published curves."""
    from sawsim.material_library import get_record
    from sawsim.material_runtime import from_record
    from sawsim.metrics import resonances
    from sawsim.saw2d.materials import oula_transfer
    out = []
    for name in ('sp_double_layer', 'sp_triple_layer', 'sp_quad_layer'):
        meta = json.loads((REF / f'tests/data/{name}.json').read_text())
        data = np.load(REF / f'tests/data/{name}.npz')
        cfg = {k: v for k, v in meta['config'].items() if k != 'material_snapshots'}
        sub = from_record(get_record(cfg['substrate_material']))
        el = from_record(get_record(cfg['electrode_material']))
        lays = [from_record(get_record(layer['material_id'])) for layer in cfg['layers']]
        C, e, eps = oula_transfer([cfg['euler_phi_deg'], cfg['euler_theta_deg'], cfg['euler_psi_deg']], sub.C,
                                  sub.e, sub.eps)
        rho = [sub.rho, el.rho] + [m.rho for m in lays]
        Cs = [C, el.C] + [m.C for m in lays]
        es = [e, el.e] + [m.e for m in lays]
        epss = [eps, el.eps] + [m.eps for m in lays]
        fem = resonances(data['frequency_hz'], data['reference_magnitude'])
        pub = resonances(data['frequency_hz'], data['sawsim_magnitude'])
        out.append(dict(name=name, config=cfg, rho=rho, C=[np.asarray(x).tolist() for x in Cs],
                        e=[np.asarray(x).tolist() for x in es], eps=[np.asarray(x).tolist() for x in epss],
                        independent_fem=dict(fr_ghz=fem['fr_ghz'], fa_ghz=fem['fa_ghz']),
                        published=dict(fr_ghz=pub['fr_ghz'], fa_ghz=pub['fa_ghz'])))
    return out


def main():
    layouts = [dict(args, layout=gm_layout(**args)) for args in LAYOUTS]
    sys.modules.pop('gmsh', None)
    out = dict(layouts=layouts, single_layer=single_layer(), layered=layered_templates())
    (HERE / 'sp_stack.json').write_text(json.dumps(out))
    s = out['single_layer']
    print(len(layouts), 'layouts; single layer: independent FEM', s['independent_fem'], 'reference on the rebuilt mesh',
          s['reference_on_rebuilt_mesh'])


if __name__ == '__main__':
    main()
