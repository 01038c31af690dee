"""Parametrised Q9 cells for the adjoint gradient (host setup).

A ``Q9Model`` maps a parameter vector to the inputs of the GPU assembly
(``FrequencySolver.from_q9``: mesh, materials, PML region, Bloch sets) and to
the derivative seeds of ``ss_adjoint_gradient``:

* geometry (``pitch_um`` and one thickness per layer band): node coordinates
  and PML bounds are affine in these for fixed element counts, so a central
  difference of the cell builder is their exact derivative;
* the piezo film's Euler angle ``euler_theta_deg`` (second ZXZ angle,
  src/sawsim/saw2d/materials.py:250-265): derivative of the Bond rotation
  C' = M C M^T, e' = a e M^T, eps' = a eps a^T (materials.py:28-71) through
  da/dtheta, with dM from a complex step of the (quadratic) Bond matrix;
* the piezo film's stiffness constants ``C11 C12 C13 C14 C33 C44`` (the 3m
  tensor builder, crystal.py:55-77): C is linear in them.

The reference exposes these parameters through its templates (pitch_um,
layer thickness_um, euler angles, material records); it has no derivative.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import cases, cells, materials as mt

MATERIAL = ['euler_theta_deg', 'C11', 'C12', 'C13', 'C14', 'C33', 'C44']
# layer stacks below the film: (name, tag, thickness in pitches, row fraction numerator /32)
STACKS = {
    'two_layer': dict(layers=[('film', 16, 0.6, 6), ('sio2', 22, 0.3, 3), ('si', 23, 3.0, None)], pml=(24, 6),
                      materials=['sio2', 'si_cubic']),
    'four_layer': dict(layers=[('film', 16, 0.5, 5), ('sio2', 22, 0.25, 3), ('polysi', 23, 0.5, 5), ('si', 24, 3.0, None)],
                       pml=(25, 5), materials=['sio2', 'poly_si', 'si_cubic']),
}
GEOMETRY = ['pitch_um', 't_film_um', 't_sio2_um', 't_si_um']


def _rx_derivative(angles_deg):
    """d a / d beta (per radian) of a = Rz(alpha) Rx(beta) Rz(gamma)."""
    al, be, ga = np.asarray(angles_deg, dtype=float) * np.pi / 180.0

    def rz(t):
        c, s = np.cos(t), np.sin(t)
        return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1.0]])

    c, s = np.cos(be), np.sin(be)
    drx = np.array([[0, 0, 0], [0, -s, -c], [0, c, -s]])
    return rz(al) @ drx @ rz(ga)


def rotation_tangent(crystal: mt.Material, angles_deg) -> mt.Material:
    """d(rotated tensors)/d(theta in degrees) of ``materials.rotate(crystal, angles)``."""
    a = mt.rotation_matrix(angles_deg)
    da = _rx_derivative(angles_deg) * (np.pi / 180.0)
    M = mt.bond_matrix(a)
    h = 1e-30
    dM = np.imag(mt.bond_matrix(a + 1j * h * da)) / h
    C, e, eps = crystal.C, crystal.e, crystal.eps
    return mt.Material(0.0, dM @ C @ M.T + M @ C @ dM.T, da @ e @ M.T + a @ e @ dM.T,
                       da @ eps @ a.T + a @ eps @ da.T)


@dataclass
class Q9Model:
    """An ME1 Q9 cell as a function of its geometry (pitch and every layer
    thickness, um) and MATERIAL parameters.  ``stack='two_layer'``: the cell of
    ``cells.me1_two_layer_cell`` (film 0.6p, SiO2 0.3p, Si 3p); ``'four_layer'``:
    ``cells.me1_four_layer_cell`` (film 0.5p, SiO2 0.25p, poly-Si 0.5p, Si 3p).
    PML thickness = pitch; electrodes 0.08 p0 thick."""

    cols: int = 64
    rows: int = 256
    seed: int = 0
    stack: str = 'two_layer'
    f0: float = 1.6e9
    f1: float = 2.0e9
    crystal: mt.Material = field(init=False)
    euler: np.ndarray = field(init=False)
    k3m: dict = field(init=False)

    def __post_init__(self):
        self.crystal, self.euler = mt.seeded_3m(self.seed)
        self.k3m = self._constants(self.crystal)

    @staticmethod
    def _constants(x):
        C = x.C
        return dict(C11=C[0, 0], C12=C[0, 1], C13=C[0, 2], C14=C[0, 3], C33=C[2, 2], C44=C[3, 3])

    @property
    def geometry(self):
        return ['pitch_um'] + [f't_{name}_um' for name, *_ in STACKS[self.stack]['layers']]

    @property
    def names(self):
        return self.geometry + MATERIAL

    def defaults(self) -> np.ndarray:
        p = 1.085
        k = self.k3m
        th = [t * p for _, _, t, _ in STACKS[self.stack]['layers']]
        return np.array([p] + th + [float(self.euler[1]), k['C11'], k['C12'], k['C13'], k['C14'], k['C33'],
                                    k['C44']])

    # ------------------------------------------------------------------ build
    def _cell(self, v):
        st = STACKS[self.stack]
        ng = len(self.geometry)
        p, th = v[0], v[1:ng]
        pml_tag, pml_frac = st['pml']
        r_pml = self.rows * pml_frac // 32
        bands, used = [], r_pml
        for (name, tag, _, frac), t in zip(st['layers'], th):
            r = self.rows * frac // 32 if frac else None
            bands.append([tag, t, r])
            used += r or 0
        for b in bands:
            if b[2] is None:
                b[2] = self.rows - used
        return cells.q9_cell(p, self.cols, [cells.Band(*b) for b in bands] + [cells.Band(pml_tag, p, r_pml)],
                             cells.Band(cells.TAG_ELECTRODE, 0.08 * 1.085, 1))

    def _crystal_at(self, v):
        k = dict(zip(MATERIAL[1:], v[len(self.geometry) + 1:]))
        x = self.crystal
        C = mt.trigonal_3m(dict(k, e15=0, e22=0, e31=0, e33=0, eps11=1, eps33=1), x.rho).C
        return mt.Material(x.rho, C, x.e, x.eps)

    def build(self, v):
        """(case, materials) at parameters ``v``."""
        v = np.asarray(v, dtype=float)
        cell = self._cell(v)
        mesh = cases.mesh_from_msh(cell.msh())
        angles = np.array([self.euler[0], v[len(self.geometry)], self.euler[2]])
        piezo = mt.rotate(self._crystal_at(v), angles)
        mats = [piezo, mt.al()] + [getattr(mt, m)() for m in STACKS[self.stack]['materials']]
        idx = np.array([cell.tag_map[t] for t in mesh.elem_tag], dtype=np.int64)
        bottom = float(mesh.pos_m[:, 1].min())
        pml = [cases.PML(tag=cell.pml_tag, kind='y', yp=bottom, ya=cell.pml_top_um * 1e-6)]
        bc = cases.bc_periodic(mesh, cell.LINES3, 3)
        freqs = np.linspace(self.f0, self.f1, 5)
        case = cases.Case('me1_param', cell, mesh, mats, idx, pml, bc, freqs, 1,
                          dict(seed=self.seed, cols=self.cols, rows=self.rows))
        return case

    def engine(self, case, device=0):
        return cases.engine_for(case, device=device)

    @staticmethod
    def y11(w, Q, V, case):
        """-i w Q / V (src/sawsim/solver.py:128)."""
        return -1j * w * Q / V

    def seeds(self, v):
        """Derivative seeds of every parameter at ``v`` (one dict per parameter)."""
        v = np.asarray(v, dtype=float)
        out = []
        n_mat = 2 + len(STACKS[self.stack]['materials'])
        it = len(self.geometry)
        for i, name in enumerate(self.names):
            s = dict(dpos=None, dC=None, de=None, deps=None, drho=None, dinner=None, douter=None)
            if name in self.geometry:
                h = 0.05 * v[i]
                vp, vm = v.copy(), v.copy()
                vp[i] += h
                vm[i] -= h
                cp, cm = self._cell(vp), self._cell(vm)
                s['dpos'] = (cp.POS[:, :2] - cm.POS[:, :2]) * 1e-6 / (2 * h)
                yp = lambda c: np.array([[0.0, c.pml_bottom_um * 1e-6, 0.0]])        # noqa: E731
                ya = lambda c: np.array([[0.0, c.pml_top_um * 1e-6, 0.0]])           # noqa: E731
                s['douter'] = (yp(cp) - yp(cm)) / (2 * h)
                s['dinner'] = (ya(cp) - ya(cm)) / (2 * h)
            else:
                dC = np.zeros((n_mat, 6, 6), complex)
                de = np.zeros((n_mat, 3, 6), complex)
                deps = np.zeros((n_mat, 3, 3), complex)
                angles = np.array([self.euler[0], v[it], self.euler[2]])
                if name == 'euler_theta_deg':
                    t = rotation_tangent(self._crystal_at(v), angles)
                    dC[0], de[0], deps[0] = t.C, t.e, t.eps
                else:
                    j = MATERIAL.index(name) - 1
                    k = dict(zip(MATERIAL[1:], np.eye(6)[j]))
                    unit = mt.trigonal_3m(dict(k, e15=0, e22=0, e31=0, e33=0, eps11=1, eps33=1), 1.0)
                    a = mt.rotation_matrix(angles)
                    M = mt.bond_matrix(a)
                    dC[0] = M @ unit.C @ M.T
                s['dC'], s['de'], s['deps'] = dC, de, deps
            out.append(s)
        return out


@dataclass
class HexModel:
    """A Hex27 slab (``cells.hex_double_layer_slab`` or ``hex_four_layer_slab``) as a
    function of ``pitch_um`` (the period: x scales, aperture, depths and electrode
    height stay) and ``t_film_um`` (the piezo film thickness: the film stretches,
    everything below it moves down, PML bounds included)."""

    nx: int = 8
    ny: int = 4
    nz: int = 48
    seed: int = 0
    stack: str = 'double'
    f0: float = 1.6e9        # band (Hz); the PML is frozen at its top
    f1: float = 2.0e9
    crystal: mt.Material = field(init=False)
    euler: np.ndarray = field(init=False)

    def __post_init__(self):
        self.crystal, self.euler = mt.seeded_3m(self.seed)

    names = ['pitch_um', 't_film_um']

    def _layers(self):
        p = 1.085
        if self.stack == 'double':
            nz = self.nz
            r = [nz // 6, nz // 3]
            return [(cells.HEX_TAG_PIEZO, 0.6 * p, r[0]), (cells.HEX_TAG_LAYER, 1.4 * p, r[1]),
                    (10, 2 * p, nz - sum(r))], 0.5, ['sio2']
        nz = self.nz
        r = [nz // 8, nz // 16, nz // 8]
        r_pml = nz // 4
        return [(cells.HEX_TAG_PIEZO, 0.5 * p, r[0]), (cells.HEX_TAG_LAYER, 0.25 * p, r[1]), (11, 0.5 * p, r[2]),
                (12, 1.75 * p, nz - sum(r) - r_pml), (13, p, r_pml)], 1.0 / 3.0, ['sio2', 'poly_si', 'si_cubic']

    def defaults(self) -> np.ndarray:
        return np.array([1.085, self._layers()[0][0][1]])

    def _cell(self, v):
        p0 = 1.085
        layers, ratio, _ = self._layers()
        bands = [cells.Band(tag, v[1] if i == 0 else t, rows) for i, (tag, t, rows) in enumerate(layers)]
        return cells.hex_slab_cell(v[0], self.nx, self.ny, bands, cells.Band(cells.HEX_TAG_ELECTRODE, 0.08 * p0, 1),
                                   0.5 * p0, metal_ratio=ratio)

    def build(self, v):
        v = np.asarray(v, dtype=float)
        cell = self._cell(v)
        piezo = mt.rotate(self.crystal, self.euler)
        mats = [piezo, mt.al()] + [getattr(mt, m)() for m in self._layers()[2]]
        idx = np.array([cell.tag_map[int(t)] for t in cell.hex_tag], dtype=np.int64)
        pos_m = cell.POS * 1e-6
        bottom = float(pos_m[:, 2].min())
        pml = [cases.PML(tag=cell.pml_tag, kind='z', za=cell.pml_top_um * 1e-6, zp=bottom)]
        bc = cases.bc_periodic_3d(cell.sets, pos_m, pos_m.shape[0])
        return cases.HexCase('hex_param', cell, pos_m, cell.HEXAS27, mats, idx, pml, bc, np.linspace(self.f0, self.f1, 5),
                             dict(seed=self.seed, nx=self.nx, ny=self.ny, nz=self.nz))

    def engine(self, case, device=0):
        return cases.hex_engine_for(case, device=device)

    @staticmethod
    def y11(w, Q, V, case):
        """+i w Q / V / aperture (src/sawsim/hex_solver.py:103)."""
        return 1j * w * Q / V / (case.cell.aperture_um * 1e-6)

    def seeds(self, v):
        v = np.asarray(v, dtype=float)
        out = []
        for i in range(len(self.names)):
            h = 0.05 * v[i]
            vp, vm = v.copy(), v.copy()
            vp[i] += h
            vm[i] -= h
            cp, cm = self._cell(vp), self._cell(vm)
            s = dict(dpos=(cp.POS - cm.POS) * 1e-6 / (2 * h))
            zb = lambda c: np.array([[0.0, 0.0, c.pml_bottom_um * 1e-6]])     # noqa: E731
            zt = lambda c: np.array([[0.0, 0.0, c.pml_top_um * 1e-6]])        # noqa: E731
            s['douter'] = (zb(cp) - zb(cm)) / (2 * h)
            s['dinner'] = (zt(cp) - zt(cm)) / (2 * h)
            out.append(s)
        return out
