"""Generate tests/golden/ref_hex_<nx>x<ny>x<nz>.npz from the reference's own Hex27 path.

Run in the build container, where the reference (Duane245/sawsim 2.1.0) is
mounted read-only at /root/reference:

    python tests/golden/make_hex_golden.py

For small seeded slabs built by ``sawsim_b200.cells.hex_double_layer_slab``
(no Gmsh) it calls the reference's ``form_stiffness_mass_3d``
(saw3d/assembly.py:230), ``boundary_idx_vect_3ds`` (saw3d/boundary.py:84),
``build_periodic_operators`` and ``FrequencySolver3D`` (saw3d/bc_solve.py:36, :108;
SciPy route) and records K @ v, M @ v for a seeded v, the periodic / prescribed
DOF lists, the active set, k_aa @ w, m_aa @ w and Q at a few frequencies.  The
reference's ``saw3d`` package imports gmsh at import time; a placeholder module
stands in for it (no Gmsh call is made on this path).  The tests read the
fixtures, never the reference checkout.
"""
from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
# the reference checkout: SAWSIM_REFERENCE, else where the build container mounts it
sys.path.insert(0, str(Path(os.environ.get('SAWSIM_REFERENCE', '/root/reference')) / 'src'))
sys.modules.setdefault('gmsh', types.ModuleType('gmsh'))

from sawsim.saw2d.saw3d.assembly import form_stiffness_mass_3d          # noqa: E402
from sawsim.saw2d.saw3d.bc_solve import (FrequencySolver3D, FrequencySolver3D_FP,  # noqa: E402
                                         build_periodic_operators, build_periodic_operators_fp)
from sawsim.saw2d.saw3d.boundary import boundary_idx_vect_3ds            # noqa: E402

from sawsim_b200 import cases                                            # noqa: E402

SMALL = [(8, 1, 6, 4), (8, 2, 12, 3)]
FP = (8, 2, 12, 3)      # slab of the finite-device fixture


def floating_strips(c):
    """Synthetic floating electrodes on the slab: the substrate-surface nodes (z = 0)
    outside the driven pair and the front/back faces, in the outer tenth of the cell
    on either side (XFL, XFR); phi DOFs at 3N + node, ascending."""
    P, S = c.pos_m, c.cell.sets
    surf = np.where(np.isclose(P[:, 2], 0.0))[0]
    free = np.setdiff1d(surf, np.concatenate([S['zheng'], S['fu'], S['front'], S['back']]))
    w = P[:, 0].max()
    gu = 3 * c.N
    return np.sort(free[P[free, 0] < 0.1 * w]) + gu, np.sort(free[P[free, 0] > 0.9 * w]) + gu


def reference_inputs(c):
    pml_mask = c.cell.hex_tag == c.cell.pml_tag
    mats = []
    for mi, m in enumerate(c.materials):
        ids = np.where((c.mat_idx == mi) & ~pml_mask)[0]
        mats.append(dict(rho=m.rho, C=m.C, e=m.e, eps=m.eps, indx=ids))
    pm = c.materials[c.cell.tag_map[c.cell.pml_tag]]
    p = c.pml[0]
    pml = [dict(region=1, indx=np.array([], dtype=np.int64)), dict(region=2, indx=np.array([], dtype=np.int64)),
           dict(region=3, indx=np.where(pml_mask)[0], za=p.za, zp=p.zp, xa=0.0, xp=0.0, dmax=p.dmax, n=p.n,
                rho=pm.rho, C=pm.C, e=pm.e, eps=pm.eps)]
    return mats, pml


def main():
    for nx, ny, nz, nf in SMALL:
        c = cases.make_hex_case('hex_8x4x48', nx=nx, ny=ny, nz=nz, points=nf)
        mats, pml = reference_inputs(c)
        M, K = form_stiffness_mass_3d(c.hexas, c.pos_m, mats, pml, c.omega_top)
        bnd = boundary_idx_vect_3ds(c.cell.sets, c.pos_m, 3 * c.N)
        tfb, tlr = build_periodic_operators(bnd, 4 * c.N)
        eng = FrequencySolver3D(K, M, bnd, tfb, tlr)
        rng = np.random.default_rng(4321)
        v = rng.standard_normal(K.shape[0]) + 1j * rng.standard_normal(K.shape[0])
        w = rng.standard_normal(eng.n_act) + 1j * rng.standard_normal(eng.n_act)
        Q = np.array([eng.solve(2 * np.pi * f, 1.0)[1] for f in c.freqs])
        lists = {f'm_{k}': np.asarray(x) for k, x in bnd.machine.items()}
        lists.update({f'e_{k}': np.asarray(x) for k, x in bnd.electric.items()})
        np.savez_compressed(HERE / f'ref_hex_{nx}x{ny}x{nz}.npz', v=v, Kv=K @ v, Mv=M @ v, K_nnz=K.nnz, w=w,
                            kaa_w=eng.k_aa @ w, maa_w=eng.m_aa @ w, active=eng.active, frequency_hz=c.freqs, Q=Q,
                            **lists)
        print(nx, ny, nz, 'nodes', c.N, 'K nnz', K.nnz, 'active', eng.n_act)
        if (nx, ny, nz, nf) == FP:
            # the finite-device solver (bc_solve.py:214-335) on the same slab with two
            # floating strips added to the electric sets
            xfl, xfr = floating_strips(c)
            bnd.electric['XFL'], bnd.electric['XFR'] = xfl, xfr
            tfb, tfl = build_periodic_operators_fp(bnd, 4 * c.N)
            fp = FrequencySolver3D_FP(K, M, bnd, tfb, tfl)
            Qfp = np.array([fp.solve(2 * np.pi * f, 1.0)[1] for f in c.freqs])
            np.savez_compressed(HERE / f'ref_hex_fp_{nx}x{ny}x{nz}.npz', XFL=xfl, XFR=xfr, active=fp.active,
                                frequency_hz=c.freqs, Q=Qfp)
            print('finite device: active', fp.n_act)


if __name__ == '__main__':
    main()
