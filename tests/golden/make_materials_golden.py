"""Generate tests/golden/materials.npz from the reference's own material code.

Run in the build container, where the reference (Duane245/sawsim 2.1.0) is
checked out (SAWSIM_REFERENCE, default /root/reference):

    python tests/golden/make_materials_golden.py

It records, with the reference's functions only:

* ``crystal.tensors`` (src/sawsim/crystal.py:30-78) for the seeded synthetic 3m
  crystals of seeds 0-3 (constants drawn by ``sawsim_b200.materials.seeded_3m``,
  whose draws are inputs here, not outputs under test), for the literature
  LiNbO3 record the reference's own known-answer test uses
  (tests/test_stack_materials.py:64-72), and for the isotropic Al / SiO2 /
  poly-Si and cubic Si constants of the synthetic cells;
* ``rotation_matrix`` and ``oula_transfer`` (src/sawsim/saw2d/materials.py:28-71,
  :250-265) of each seeded crystal at its own seeded Euler triple and at four
  fixed triples, and ``project_xy_plane_strain`` (:281-290) and
  ``project_xz_plane_strain`` (:303-308) of the results;
* central differences (step 1e-4 degrees) of ``oula_transfer`` in the second
  Euler angle at the seeded triples, the reference value of the d/dtheta
  tangent that the adjoint gradient seeds.

The fixture is small; the tests read it, never the reference checkout.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
REF = Path(os.environ.get('SAWSIM_REFERENCE', '/root/reference'))
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REF / 'src'))

from sawsim.crystal import EPS0, tensors                                     # noqa: E402
from sawsim.material_library import get_record                                # noqa: E402
from sawsim.saw2d.materials import (Material, oula_transfer, project_xy_plane_strain, project_xz_plane_strain,  # noqa: E402
                                    rotation_matrix)

from sawsim_b200 import materials as mt                                       # noqa: E402

FIXED = np.array([[0.0, -42.0, 0.0], [0.0, 48.0, 0.0], [30.0, 127.5, -60.0], [-179.0, 0.25, 89.0]])
H = 1e-4


def consts_of(seed):
    """The seeded crystal's independent constants (GPa, C/m^2, relative eps)."""
    m, euler = mt.seeded_3m(seed)
    C, e, eps = m.C, m.e, m.eps
    k = dict(C11=C[0, 0] / 1e9, C12=C[0, 1] / 1e9, C13=C[0, 2] / 1e9, C14=C[0, 3] / 1e9, C33=C[2, 2] / 1e9,
             C44=C[3, 3] / 1e9, e15=e[0, 4], e22=e[1, 1], e31=e[2, 0], e33=e[2, 2],
             eps11=eps[0, 0] / EPS0, eps33=eps[2, 2] / EPS0)
    return k, euler


def main():
    out = {}
    keys = ['C11', 'C12', 'C13', 'C14', 'C33', 'C44', 'e15', 'e22', 'e31', 'e33', 'eps11', 'eps33']
    for seed in range(4):
        k, euler = consts_of(seed)
        out[f's{seed}_consts'] = np.array([k[x] for x in keys])
        out[f's{seed}_euler'] = euler
        C, e, eps = (np.array(x, dtype=float) for x in tensors('trigonal_3m', k))
        out[f's{seed}_C'], out[f's{seed}_e'], out[f's{seed}_eps'] = C, e, eps
        triples = np.vstack([euler[None, :], FIXED])
        out[f's{seed}_triples'] = triples
        rot, xz = [], []
        for t in triples:
            a = rotation_matrix(t)
            Cr, er, epsr = oula_transfer(t, C, e, eps)
            p = project_xy_plane_strain(Material(4700.0, Cr, er, epsr))
            rot.append(np.concatenate([a.ravel(), Cr.ravel(), er.ravel(), epsr.ravel(), p.C.ravel(), p.e.ravel(),
                                       p.eps.ravel()]))
            q = project_xz_plane_strain(Material(4700.0, Cr, er, epsr))
            xz.append(np.concatenate([q.C.ravel(), q.e.ravel(), q.eps.ravel()]))
        out[f's{seed}_rot'] = np.array(rot)
        out[f's{seed}_xz'] = np.array(xz)
        tp, tm = euler.copy(), euler.copy()
        tp[1] += H
        tm[1] -= H
        fp = oula_transfer(tp, C, e, eps)
        fm = oula_transfer(tm, C, e, eps)
        out[f's{seed}_dtheta'] = np.concatenate([((np.asarray(x) - np.asarray(y)) / (2 * H)).ravel()
                                                 for x, y in zip(fp, fm)])
    r = get_record('linbo3_bouchy_2022')
    Cl, el, epsl = np.array(r['C_pa']), np.array(r['e_c_m2']), np.array(r['eps_f_m'])
    kl = dict(C11=Cl[0, 0] / 1e9, C12=Cl[0, 1] / 1e9, C13=Cl[0, 2] / 1e9, C14=Cl[0, 3] / 1e9, C33=Cl[2, 2] / 1e9,
              C44=Cl[3, 3] / 1e9, e15=el[0, 4], e22=el[1, 1], e31=el[2, 0], e33=el[2, 2],
              eps11=epsl[0, 0] / EPS0, eps33=epsl[2, 2] / EPS0)
    out['linbo3_consts'] = np.array([kl[x] for x in keys])
    out['linbo3_record'] = np.concatenate([Cl.ravel(), el.ravel(), epsl.ravel()])
    C, e, eps = tensors('trigonal_3m', kl)
    out['linbo3_built'] = np.concatenate([np.ravel(C), np.ravel(e), np.ravel(eps)])
    iso = {'al': dict(E_gpa=70, nu=0.35), 'sio2': dict(E_gpa=72, nu=0.17, eps_r=3.9),
           'polysi': dict(E_gpa=169, nu=0.22, eps_r=4.5)}
    for name, k in iso.items():
        C, e, eps = tensors('isotropic', k)
        out[f'iso_{name}'] = np.concatenate([np.ravel(C), np.ravel(e), np.ravel(eps)])
    C, e, eps = tensors('cubic', dict(C11=165.7, C12=63.9, C44=79.6, eps_r=11.7))
    out['cubic_si'] = np.concatenate([np.ravel(C), np.ravel(e), np.ravel(eps)])
    out['EPS0'] = np.array(EPS0)
    np.savez_compressed(HERE / 'materials.npz', **out)
    print('wrote', HERE / 'materials.npz', len(out), 'arrays')


if __name__ == '__main__':
    main()
