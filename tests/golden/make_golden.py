"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in the build container, where the reference (Duane245/sawsim 2.1.0) is
mounted read-only at /root/reference:

    python tests/golden/make_golden.py

It imports the reference's own modules (``sawsim.saw2d.piezo_fem``,
``sawsim.saw2d.sweep``, the material library) and records, for meshes built by
``sawsim_b200.cells`` without Gmsh:

* ``sp_double_layer.npz``, ``sp_quad_layer.npz`` — each template's published
  curve at its 5 test frequencies (``tests/data/<name>.npz['sawsim_magnitude']``),
  the resolved material tensors of the template, and the reference's own |Y|
  there on the rebuilt mesh;
* ``ref_<case>.npz`` — for small seeded synthetic cells (ME0 and ME1): a hash of
  the reference's global K pattern, K @ v and M @ v for a seeded v, the condensed
  Km_aa @ w, Mm_aa @ w, the active DOF list and the reference's Q at a few
  frequencies (SciPy SuperLU route, sweep.py:352-353).

The fixtures are small; the tests read them, never the reference checkout.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
# the reference checkout: SAWSIM_REFERENCE, else where the build container mounts it
REF = Path(os.environ.get('SAWSIM_REFERENCE', '/root/reference'))
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REF / 'src'))

from sawsim.material_library import get_record            # noqa: E402
from sawsim.material_runtime import from_record           # noqa: E402
from sawsim.saw2d import piezo_fem, sweep                 # noqa: E402
from sawsim.saw2d.materials import Material, oula_transfer  # noqa: E402

from sawsim_b200 import cases, cells                      # noqa: E402

SMALL = [('me0_16x64', 8, 16, 5), ('me1_64x256', 8, 16, 5), ('me1_128x512', 8, 20, 4)]


def pattern_hash(A) -> str:
    A = A.tocsr()
    A.sort_indices()
    h = hashlib.sha256()
    h.update(np.asarray(A.indptr, dtype=np.int64).tobytes())
    h.update(np.asarray(A.indices, dtype=np.int64).tobytes())
    return h.hexdigest()


def template(name, cell):
    """A structured template's published curve at its test frequencies, its
    resolved materials and the reference's own run on the rebuilt mesh."""
    meta = json.loads((REF / f'tests/data/{name}.json').read_text())
    d = np.load(REF / f'tests/data/{name}.npz')
    idx = np.array(meta['test_indices'])
    cfg = meta['config']
    sub = from_record(get_record(cfg['substrate_material']))
    el = from_record(get_record(cfg['electrode_material']))
    lays = [from_record(get_record(layer['material_id'])) for layer in cfg['layers']]
    C, e, eps = oula_transfer([cfg['euler_phi_deg'], cfg['euler_theta_deg'], cfg['euler_psi_deg']],
                              sub.C, sub.e, sub.eps)
    mats = [Material(sub.rho, C, e, eps), el] + lays
    model = piezo_fem.build_model(type('M', (), cell.msh())())
    tag_map = cell.tag_map
    mi = piezo_fem.material_index(model, tag_map)
    bottom = float(model.pos_m[model.nodes_with_tag(21, cell.LINES3), 1].min())
    pml = [piezo_fem.PMLRegion(tag=cell.pml_tag, kind='y', yp=bottom, ya=bottom + 2 * cfg['pitch_um'] * 1e-6)]
    f = d['frequency_hz'][idx]
    fre = np.linspace(f[0], f[-1], len(idx))
    K, M = piezo_fem.assemble(model, mats, mi, pml, 2 * np.pi * fre[-1])
    eng = sweep.FrequencySolver(K, M, *sweep.bc_periodic(model, cell.LINES3, ndisp=3))
    Q = np.array([eng.solve(2 * np.pi * x, 1.0)[1] for x in fre])
    Y = -1j * 2 * np.pi * fre * Q
    np.savez_compressed(HERE / f'{name}.npz', frequency_hz=fre, published_magnitude=d['sawsim_magnitude'][idx],
                        reference_fem_magnitude=d['reference_magnitude'][idx], reference_run_admittance=Y,
                        rho=np.array([m.rho for m in mats]), C=np.stack([m.C for m in mats]),
                        e=np.stack([m.e for m in mats]), eps=np.stack([m.eps for m in mats]),
                        pitch_um=cfg['pitch_um'])
    err = np.max(np.abs(np.abs(Y) - d['sawsim_magnitude'][idx]) / d['sawsim_magnitude'][idx])
    print(name, ': reference run vs published curve', err)


def small(name, cols, rows, nf):
    c = cases.make_case(name, cols=cols, rows=rows)
    model = piezo_fem.Model(pos_m=c.mesh.pos_m, quads=c.mesh.quads, elem_tag=c.mesh.elem_tag, N=c.mesh.N)
    mats = [Material(m.rho, m.C, m.e, m.eps) for m in c.materials]
    pml = [piezo_fem.PMLRegion(tag=p.tag, kind=p.kind, ya=p.ya, yp=p.yp) for p in c.pml]
    asm = piezo_fem.assemble if c.mode_extension else piezo_fem.assemble_ME0
    K, M = asm(model, mats, c.mat_idx, pml, c.omega_top)
    ndisp = 3 if c.mode_extension else 2
    bc = sweep.bc_periodic(model, c.cell.LINES3, ndisp=ndisp)
    eng = sweep.FrequencySolver(K, M, *bc)
    rng = np.random.default_rng(1234)
    v = rng.standard_normal(K.shape[0]) + 1j * rng.standard_normal(K.shape[0])
    w = rng.standard_normal(eng.n_active) + 1j * rng.standard_normal(eng.n_active)
    fre = np.linspace(c.freqs[0], c.freqs[-1], nf)
    Q = np.array([eng.solve(2 * np.pi * x, 1.0)[1] for x in fre])
    np.savez_compressed(HERE / f'ref_{name}_{cols}x{rows}.npz', K_pattern_sha256=pattern_hash(K),
                        M_pattern_sha256=pattern_hash(M), K_nnz=K.nnz, M_nnz=M.nnz, v=v, Kv=K @ v, Mv=M @ v, w=w,
                        Kaa_w=eng.Km_aa @ w, Maa_w=eng.Mm_aa @ w, active=eng.active, frequency_hz=fre, Q=Q,
                        cols=cols, rows=rows)
    print(name, cols, rows, 'K nnz', K.nnz, 'active', eng.n_active)


if __name__ == '__main__':
    template('sp_double_layer', cells.sp_double_layer_cell())
    template('sp_quad_layer', cells.sp_quad_layer_cell())
    for args in SMALL:
        small(*args)
