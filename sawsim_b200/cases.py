"""Host setup for the sweep: mesh container, PML regions, Bloch boundary sets,
and the seeded synthetic cells the benchmarks and tests run on.

* ``Mesh`` holds what ``piezo_fem.build_model`` returns (src/sawsim/saw2d/piezo_fem.py:161-186):
  coordinates in metres, 0-based Q9 connectivity and the element tag.
* ``PML`` is one complex-stretched region (piezo_fem.py:192-208).
* ``bc_periodic`` returns ``(fix, zheng, fu, merge_groups)`` for the two-pitch cell
  (src/sawsim/saw2d/sweep.py:41-72): left/right Bloch pairs sorted by y with the
  bottom corners paired only in phi, bottom u fixed, + and - electrode phi.
* ``make_case`` builds the named synthetic cells: seeded 3m crystal rotated by a
  seeded ZXZ triple, isotropic Al electrodes, SiO2 / cubic Si / poly-Si layers,
  a 1p bottom PML frozen at the top frequency.  No dataset is involved.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import cells, materials as mt


@dataclass
class Mesh:
    pos_m: np.ndarray
    quads: np.ndarray
    elem_tag: np.ndarray

    @property
    def N(self) -> int:
        return int(self.pos_m.shape[0])

    @property
    def ne(self) -> int:
        return int(self.quads.shape[0])

    def nodes_with_tag(self, tag: int, lines: np.ndarray) -> np.ndarray:
        return np.unique(lines[lines[:, 3] == tag][:, :3].astype(np.int64) - 1)


def mesh_from_msh(msh) -> Mesh:
    return Mesh(np.asarray(msh['POS'])[:, :2] * 1e-6, np.asarray(msh['QUADS9'])[:, :9].astype(np.int64) - 1,
                np.asarray(msh['QUADS9'])[:, 9].astype(np.int64))


@dataclass
class PML:
    tag: int
    kind: str
    dmax: float = 1e11
    n: int = 3
    xa: float = 0.0
    xp: float = 0.0
    ya: float = 0.0
    yp: float = 0.0


def bc_periodic(mesh: Mesh, lines, ndisp: int = 3, tag_bottom=21, tag_left=19, tag_right=20,
                tag_zheng=17, tag_fu=18):
    N = mesh.N
    bottom = mesh.nodes_with_tag(tag_bottom, lines)
    left = mesh.nodes_with_tag(tag_left, lines)
    right = mesh.nodes_with_tag(tag_right, lines)
    zheng = mesh.nodes_with_tag(tag_zheng, lines)
    fu = mesh.nodes_with_tag(tag_fu, lines)
    cl = np.intersect1d(bottom, left)
    cr = np.intersect1d(bottom, right)
    Lft = np.setdiff1d(left, cl)
    Rgt = np.setdiff1d(right, cr)
    Lft = Lft[np.argsort(mesh.pos_m[Lft, 1], kind='stable')]
    Rgt = Rgt[np.argsort(mesh.pos_m[Rgt, 1], kind='stable')]
    if Lft.size != Rgt.size:
        raise ValueError('left/right periodic node counts differ')
    m = np.concatenate([Lft + a * N for a in range(ndisp)] + [Lft + ndisp * N, cl + ndisp * N])
    s = np.concatenate([Rgt + a * N for a in range(ndisp)] + [Rgt + ndisp * N, cr + ndisp * N])
    groups = [np.array([a, b]) for a, b in zip(m, s)]
    fix = np.concatenate([bottom + a * N for a in range(ndisp)])
    return fix, zheng + ndisp * N, fu + ndisp * N, groups


@dataclass
class Case:
    name: str
    cell: object
    mesh: Mesh
    materials: list
    mat_idx: np.ndarray
    pml: list
    bc: tuple
    freqs: np.ndarray
    mode_extension: int
    info: dict = field(default_factory=dict)

    @property
    def omega_top(self) -> float:
        return 2 * np.pi * float(self.freqs[-1])


def _crystal(seed):
    xtal, euler = mt.seeded_3m(seed)
    return mt.rotate(xtal, euler), euler


CASES = {
    # name: (cell builder, default cols, rows, ME, f0, f1, npoints)
    'me0_16x64': ('me0', 16, 64, 0, 1.6e9, 2.0e9, 101),
    'me1_64x256': ('me1_2', 64, 256, 1, 1.6e9, 2.0e9, 201),
    'me1_128x512': ('me1_4', 128, 512, 1, 1.6e9, 2.0e9, 64),
}


def make_case(name: str, seed: int = 0, cols=None, rows=None, points=None, f0=None, f1=None) -> Case:
    """Seeded synthetic cell ``name`` (see ``CASES``), optionally resized."""
    kind, c0, r0, me, fa, fb, npt = CASES[name]
    cols = cols or c0
    rows = rows or r0
    piezo, euler = _crystal(seed)
    if kind == 'me0':
        cell = cells.me0_cell(cols, rows)
        mats = [mt.project_xy_plane_strain(piezo), mt.project_xy_plane_strain(mt.al())]
    elif kind == 'me1_2':
        cell = cells.me1_two_layer_cell(cols, rows)
        mats = [piezo, mt.al(), mt.sio2(), mt.si_cubic()]
    else:
        cell = cells.me1_four_layer_cell(cols, rows)
        mats = [piezo, mt.al(), mt.sio2(), mt.poly_si(), mt.si_cubic()]
    mesh = mesh_from_msh(cell.msh())
    idx = np.full(mesh.ne, -1, dtype=np.int64)
    for tag, mi in cell.tag_map.items():
        idx[mesh.elem_tag == tag] = mi
    assert (idx >= 0).all()
    bottom = float(mesh.pos_m[:, 1].min())
    pml = [PML(tag=cell.pml_tag, kind='y', yp=bottom, ya=cell.pml_top_um * 1e-6)]
    ndisp = 3 if me else 2
    bc = bc_periodic(mesh, cell.LINES3, ndisp)
    freqs = np.linspace(f0 or fa, f1 or fb, points or npt)
    return Case(name, cell, mesh, mats, idx, pml, bc, freqs, me, dict(seed=seed, euler_deg=list(map(float, euler)),
                                                                   cols=cols, rows=rows))


def engine_for(case: Case, device: int = 0):
    """GPU engine for a case (assembly, condensation and analysis on the device)."""
    from .engine import FrequencySolver
    return FrequencySolver.from_q9(case.mesh, case.materials, case.mat_idx, case.pml, case.omega_top, case.bc,
                                   mode_extension=case.mode_extension, device=device)
