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
    za: float = 0.0
    zp: float = 0.0


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


def bc_floating(mesh: Mesh, lines, ndisp: int = 3, tag_bottom=7, tag_xfl=3, tag_xfr=4, tag_zheng=5, tag_fu=6):
    """Finite-device boundary sets with floating electrodes (sweep.py:75-91): the
    bottom u fixed, the + and - electrode phi prescribed, and the phi DOFs of each
    floating electrode merged into one equipotential group (its first node the
    master)."""
    N = mesh.N
    bottom = mesh.nodes_with_tag(tag_bottom, lines)
    xfl = mesh.nodes_with_tag(tag_xfl, lines)
    xfr = mesh.nodes_with_tag(tag_xfr, lines)
    zheng = mesh.nodes_with_tag(tag_zheng, lines)
    fu = mesh.nodes_with_tag(tag_fu, lines)
    fix = np.concatenate([bottom + a * N for a in range(ndisp)])
    groups = [xfl + ndisp * N, xfr + ndisp * N]
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


# ---------------------------------------------------------------------------- Hex27 slabs
def bc_periodic_3d(sets, pos_m, N: int):
    """(fix, zheng, fu, groups, two_stage) for ss_set_bc from the slab's boundary node
    sets, following boundary_idx_vect_3ds (src/sawsim/saw2d/saw3d/boundary.py:84-148)
    and the two-stage fold of bc_solve.py:36-44: electrode nodes leave the
    front/back sets (their u DOFs stay front/back periodic, their phi is
    prescribed), bottom nodes leave front/back/L/R (their phi pairs are kept
    separately), L/R lose the back edge; pairs are matched by coordinates rounded
    to 0.1 nm (y then z for L/R, x then z for front/back).  Groups are
    [master, slave]: the front/back pairs first (``two_stage`` of them), then
    the left/right pairs.  DOFs: u interleaved 3n + c, phi at 3N + n."""
    I, D = np.intersect1d, np.setdiff1d
    g2, L, R, front, back, zheng, fu = (np.asarray(sets[k], dtype=np.int64) for k in
                                        ('bottom', 'L', 'R', 'front', 'back', 'zheng', 'fu'))
    cor = np.round(np.asarray(pos_m) * 1e9, 1)

    def lr(a, b):
        return a[np.lexsort((cor[a, 2], cor[a, 1]))], b[np.lexsort((cor[b, 2], cor[b, 1]))]

    def fb(a, b):
        return a[np.lexsort((cor[a, 2], cor[a, 0]))], b[np.lexsort((cor[b, 2], cor[b, 0]))]

    def mach(n):
        return np.concatenate([3 * n, 3 * n + 1, 3 * n + 2])

    fz, bz, ff, bf = I(front, zheng), I(back, zheng), I(front, fu), I(back, fu)
    front = D(front, np.concatenate([fz, ff]))
    back = D(back, np.concatenate([bz, bf]))
    g2F, g2b, g2L, g2R = I(g2, front), I(g2, back), I(g2, L), I(g2, R)
    g2Le, g2Re = D(g2L, I(g2, I(L, back))), D(g2R, I(g2, I(R, back)))
    front, back, L, R = D(front, g2F), D(back, g2b), D(L, g2L), D(R, g2R)
    L, R = D(L, I(L, back)), D(R, I(R, back))
    L, R = lr(L, R)
    front, back = fb(front, back)
    g2F, g2b = fb(g2F, g2b)
    g2Le, g2Re = lr(g2Le, g2Re)
    fz, bz = fb(fz, bz)
    ff, bf = fb(ff, bf)
    gu = 3 * N
    F = np.concatenate([mach(front), mach(fz), mach(ff), front + gu, g2F + gu])
    B = np.concatenate([mach(back), mach(bz), mach(bf), back + gu, g2b + gu])
    Lm = np.concatenate([mach(L), L + gu, g2Le + gu])
    Rs = np.concatenate([mach(R), R + gu, g2Re + gu])
    if F.size != B.size or Lm.size != Rs.size:
        raise ValueError('periodic node sets do not pair up')
    groups = [np.array([a, b]) for a, b in zip(F, B)] + [np.array([a, b]) for a, b in zip(Lm, Rs)]
    return mach(g2), zheng + gu, fu + gu, groups, int(F.size)


@dataclass
class HexCase:
    name: str
    cell: object
    pos_m: np.ndarray
    hexas: np.ndarray
    materials: list
    mat_idx: np.ndarray
    pml: list
    bc: tuple
    freqs: np.ndarray
    info: dict = field(default_factory=dict)

    @property
    def omega_top(self) -> float:
        return 2 * np.pi * float(self.freqs[-1])

    @property
    def N(self) -> int:
        return int(self.pos_m.shape[0])


HEX_CASES = {
    # name: (cell builder, nx, ny, nz, f0, f1, npoints)
    'hex_8x4x48': ('double', 8, 4, 48, 1.6e9, 2.0e9, 101),
    'hex_12x6x80': ('four', 12, 6, 80, 1.5e9, 2.1e9, 401),
}


def make_hex_case(name: str, seed: int = 0, nx=None, ny=None, nz=None, points=None) -> HexCase:
    """Seeded synthetic Hex27 slab: ``hex_8x4x48`` the double layer of
    ``cells.hex_double_layer_slab`` (film / SiO2 / SiO2 PML), ``hex_12x6x80`` the four
    layers of ``cells.hex_four_layer_slab`` (film / SiO2 / poly-Si / Si / Si PML); Al
    electrodes; bottom PML z-stretch frozen at the top frequency, dmax 1e11, n 3, as
    src/sawsim/hex_models.py:75-77."""
    kind, x0, y0, z0, fa, fb, npt = HEX_CASES[name]
    piezo, euler = _crystal(seed)
    if kind == 'double':
        cell = cells.hex_double_layer_slab(nx or x0, ny or y0, nz or z0)
        mats = [piezo, mt.al(), mt.sio2()]
    else:
        cell = cells.hex_four_layer_slab(nx or x0, ny or y0, nz or z0)
        mats = [piezo, mt.al(), mt.sio2(), mt.poly_si(), mt.si_cubic()]
    idx = np.array([cell.tag_map[int(t)] for t in cell.hex_tag], dtype=np.int64)
    pos_m = cell.POS * 1e-6
    bottom = float(pos_m[:, 2].min())
    pml = [PML(tag=cell.pml_tag, kind='z', za=cell.pml_top_um * 1e-6, zp=bottom)]
    bc = bc_periodic_3d(cell.sets, pos_m, pos_m.shape[0])
    freqs = np.linspace(fa, fb, points or npt)
    return HexCase(name, cell, pos_m, cell.HEXAS27, mats, idx, pml, bc, freqs,
                   dict(seed=seed, euler_deg=list(map(float, euler)), nx=cell.info['nx'], ny=cell.info['ny'],
                        nz=cell.info['nz']))


def hex_engine_for(case: HexCase, device: int = 0):
    """GPU engine for a Hex27 slab (assembly, two-stage fold and analysis on the device)."""
    from .engine import FrequencySolver
    return FrequencySolver.from_hex27(case.pos_m, case.hexas, case.cell.hex_tag, case.materials, case.mat_idx,
                                      case.pml, case.omega_top, case.bc, device=device)
