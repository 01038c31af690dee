"""Generate tests/golden/hex_templates.json from the reference's 2.5D Hex27 templates.

Run in the build container, where the reference (Duane245/sawsim 2.1.0) is
mounted read-only at /root/reference (SAWSIM_REFERENCE overrides):

    python tests/golden/make_hex_templates_golden.py

For each of sp_2p5d_{single,double,triple,quad}_layer it records, from the
reference's tests/data/<template>.json / .npz: the configuration, the materials
resolved as the reference resolves them (its material library records; the
substrate and any rotated layer through ``oula_transfer``,
src/sawsim/material_runtime.py:12-24), the test frequencies of its template test
(tests/test_templates.py:14-39), the published curve (``sawsim_magnitude``) and
the independent FEM curve (``reference_magnitude``) there, the frequency the PML
is frozen at (the band's top) and the two tolerances of that test.  The tests
read the fixture, never the reference checkout.
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get('SAWSIM_REFERENCE', '/root/reference'))
sys.path.insert(0, str(REF / 'src'))

from sawsim.material_library import get_record  # noqa: E402
from sawsim.material_runtime import from_record  # noqa: E402
from sawsim.saw2d.materials import oula_transfer  # noqa: E402


def template(kind):
    name = f'sp_2p5d_{kind}_layer'
    meta = json.loads((REF / f'tests/data/{name}.json').read_text())
    data = np.load(REF / f'tests/data/{name}.npz')
    cfg = {k: v for k, v in meta['config'].items() if k != 'material_snapshots'}
    ids = [cfg['substrate_material'], cfg['electrode_material']] + [layer['material_id'] for layer in cfg['layers']]
    angles = [[cfg['euler_phi_deg'], cfg['euler_theta_deg'], cfg['euler_psi_deg']], [0.0, 0.0, 0.0]]
    angles += [[layer.get('euler_phi_deg', 0.0), layer.get('euler_theta_deg', 0.0), layer.get('euler_psi_deg', 0.0)]
               for layer in cfg['layers']]
    mats = []
    for i, (mid, ang) in enumerate(zip(ids, angles)):
        m = from_record(get_record(mid))
        C, e, eps = oula_transfer(ang, m.C, m.e, m.eps) if i == 0 or any(ang) else (m.C, m.e, m.eps)
        mats.append(dict(rho=float(m.rho), C=np.asarray(C).tolist(), e=np.asarray(e).tolist(),
                         eps=np.asarray(eps).tolist()))
    idx = np.array(meta['test_indices'])
    return dict(kind=kind, config=cfg, materials=mats, frequency_hz=data['frequency_hz'][idx].tolist(),
                freeze_hz=float(data['frequency_hz'][-1]), published=data['sawsim_magnitude'][idx].tolist(),
                independent_fem=data['reference_magnitude'][idx].tolist(), regression_rtol=meta['regression_rtol'],
                reference_rtol=meta['reference_rtol'])


def main():
    out = [template(k) for k in ('single', 'double', 'triple', 'quad')]
    (HERE / 'hex_templates.json').write_text(json.dumps(out))
    print(len(out), 'templates')


if __name__ == '__main__':
    main()
