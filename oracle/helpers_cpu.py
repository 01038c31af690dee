"""CPU-baseline helper (test/benchmark infrastructure): an oracle engine per case,
cached per process."""
import sys

import numpy as np
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

_cache = {}


def oracle_solver_for(case_name, **size):
    key = (case_name, tuple(sorted(size.items())))
    if key not in _cache:
        from sawsim_b200 import cases
        if case_name.startswith('hex'):
            from oracle import hex27
            c = cases.make_hex_case(case_name, **size)
            mask = c.cell.hex_tag == c.cell.pml_tag
            mats = [dict(rho=m.rho, C=m.C, e=m.e, eps=m.eps, indx=np.where((c.mat_idx == i) & ~mask)[0])
                    for i, m in enumerate(c.materials)]
            pm, p = c.materials[c.cell.tag_map[c.cell.pml_tag]], c.pml[0]
            pml = [dict(region=3, indx=np.where(mask)[0], za=p.za, zp=p.zp, xa=0.0, xp=0.0, dmax=p.dmax, n=p.n,
                        rho=pm.rho, C=pm.C, e=pm.e, eps=pm.eps)]
            M, K = hex27.form_stiffness_mass_3d(c.hexas, c.pos_m, mats, pml, c.omega_top)
            _cache[key] = hex27.FrequencySolver3D(K, M, hex27.boundary_idx_vect_3ds(c.cell.sets, c.pos_m, 3 * c.N))
        else:
            from oracle import q9, solver
            c = cases.make_case(case_name, **size)
            m = q9.build_model(c.cell.msh())
            pml = [q9.PMLRegion(tag=p.tag, kind=p.kind, ya=p.ya, yp=p.yp) for p in c.pml]
            asm = q9.assemble if c.mode_extension else q9.assemble_me0
            K, M = asm(m, c.materials, c.mat_idx, pml, c.omega_top)
            ndisp = 3 if c.mode_extension else 2
            _cache[key] = solver.FrequencySolver(K, M, *solver.bc_periodic(m, c.cell.LINES3, ndisp=ndisp))
    return _cache[key]
