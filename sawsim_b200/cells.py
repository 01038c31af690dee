"""Gmsh-free structured unit cells (host setup).

The reference meshes its templates with Gmsh (``src/sawsim/sp_meshes/*.py``),
which needs an OpenGL stack that is unavailable here.  The structured
templates are plain tensor-product grids, so this module builds them directly
in the reference's ``Msh`` layout (``src/sawsim/saw2d/mmesh.py:7-11``):

* ``POS``    (N, 3) float, micrometres, z = 0 for 2D;
* ``QUADS9`` (ne, 10) float, 1-based Q9 node ids + physical tag column;
* ``LINES3`` (nl, 4) float, 1-based Line3 node ids + physical tag column.

Q9 node order is corners counter-clockwise from bottom-left, then the edge
mid-nodes (bottom, right, top, left), then the centre, which is the order of
``piezo_fem._q9_shapes`` (``src/sawsim/saw2d/piezo_fem.py:70-80``).  Elements
are counter-clockwise, so the signed Jacobian determinant is positive.

Physical tags follow ``src/sawsim/sp_meshes/double.py:150-172``: 15 electrode
(Al), 16 piezo film, 22.. backing layers, the PML tag after the last layer;
lines 17 (+ electrode), 18 (- electrode), 19 left, 20 right, 21 bottom.
The unit cell is two pitches wide with one + and one - electrode
(``src/sawsim/models.py:41``), Bloch phase 0 left/right.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

TAG_ELECTRODE = 15
TAG_PIEZO = 16
TAG_ZHENG = 17
TAG_FU = 18
TAG_LEFT = 19
TAG_RIGHT = 20
TAG_BOTTOM = 21


@dataclass
class Band:
    """One horizontal layer of the cell: physical tag, thickness (um), element rows."""

    tag: int
    thickness_um: float
    rows: int


@dataclass
class Q9Cell:
    """A structured Q9 cell in ``Msh`` layout plus the bookkeeping the builders need."""

    POS: np.ndarray
    QUADS9: np.ndarray
    LINES3: np.ndarray
    tag_map: dict
    pml_tag: int
    pml_top_um: float
    pml_bottom_um: float
    period_um: float
    info: dict = field(default_factory=dict)

    @property
    def nbNod(self) -> int:
        return int(self.POS.shape[0])

    def msh(self) -> dict:
        return dict(nbNod=self.nbNod, POS=self.POS, QUADS9=self.QUADS9, LINES3=self.LINES3)


def _clean13(x: np.ndarray) -> np.ndarray:
    """Round to 13 significant digits, the precision of the reference's mesh harvest
    (``src/sawsim/saw2d/gmsh_io.py:57-62``)."""
    flat = np.asarray(x, dtype=float).ravel()
    return np.array([float(f"{v:.13g}") for v in flat]).reshape(np.shape(x))


def _band_levels(top: float, bands) -> tuple[list, list]:
    """Element-edge y levels from ``top`` downward through ``bands``; returns
    (levels listed bottom->top, band index per element row bottom->top)."""
    levels = [top]
    owner = []
    y = top
    for bi, b in enumerate(bands):
        y0 = y
        y1 = y - b.thickness_um
        for r in range(1, b.rows + 1):
            levels.append(y0 + (y1 - y0) * r / b.rows)
            owner.append(bi)
        y = y1
    return levels[::-1], owner[::-1]


def q9_cell(pitch_um: float, columns: int, bands, electrode: Band | None,
            metal_ratio: float = 0.5, x_cuts=None) -> Q9Cell:
    """Build a two-pitch-wide structured Q9 cell.

    ``bands`` lists the layers from the surface downward; the last band is the
    PML.  ``electrode`` is the tooth band above y = 0 (tag 15), two teeth of width
    ``metal_ratio * pitch`` centred at p/2 and 3p/2.  ``x_cuts`` optionally gives
    the element-edge x positions (um) explicitly; otherwise ``columns`` uniform
    columns span [0, 2p] and the tooth edges must fall on column edges.
    """
    p = float(pitch_um)
    w = 2 * p
    if x_cuts is None:
        xs = [w * i / columns for i in range(columns + 1)]
    else:
        xs = list(map(float, x_cuts))
        columns = len(xs) - 1
    edges = [p * (1 - metal_ratio) / 2, p * (1 + metal_ratio) / 2,
             p * (3 - metal_ratio) / 2, p * (3 + metal_ratio) / 2]
    tooth_cols = []
    for a, b in ((edges[0], edges[1]), (edges[2], edges[3])):
        ia = int(np.argmin(np.abs(np.array(xs) - a)))
        ib = int(np.argmin(np.abs(np.array(xs) - b)))
        if abs(xs[ia] - a) > 1e-9 * w or abs(xs[ib] - b) > 1e-9 * w or ib <= ia:
            raise ValueError('electrode edges must fall on column edges')
        tooth_cols.append((ia, ib))

    levels, owner = _band_levels(0.0, bands)               # bottom -> top
    nrows = len(owner)
    nx = 2 * columns + 1
    ny = 2 * nrows + 1
    # node x positions: element edges plus mid-points
    xn = np.empty(nx)
    xn[0::2] = xs
    xn[1::2] = 0.5 * (np.array(xs[:-1]) + np.array(xs[1:]))
    yn = np.empty(ny)
    yn[0::2] = levels
    yn[1::2] = 0.5 * (np.array(levels[:-1]) + np.array(levels[1:]))

    gid = np.arange(nx * ny).reshape(ny, nx)               # [row j, col i]
    pos = [np.column_stack([np.tile(xn, ny), np.repeat(yn, nx)])]
    n_next = nx * ny

    quads, tags = [], []

    def q9(g, i, j):
        return [g[j, i], g[j, i + 2], g[j + 2, i + 2], g[j + 2, i],
                g[j, i + 1], g[j + 1, i + 2], g[j + 2, i + 1], g[j + 1, i], g[j + 1, i + 1]]

    for er in range(nrows):
        tag = bands[owner[er]].tag
        for ec in range(columns):
            quads.append(q9(gid, 2 * ec, 2 * er))
            tags.append(tag)

    lines = []

    def add_line(nodes, tag):
        for k in range(0, len(nodes) - 2, 2):
            lines.append([nodes[k], nodes[k + 2], nodes[k + 1], tag])

    add_line(list(gid[0, :]), TAG_BOTTOM)
    add_line(list(gid[:, 0]), TAG_LEFT)
    add_line(list(gid[:, -1]), TAG_RIGHT)

    if electrode is not None:
        trows = electrode.rows
        tl = [0.0 + electrode.thickness_um * r / trows for r in range(trows + 1)]
        ty = np.empty(2 * trows + 1)
        ty[0::2] = tl
        ty[1::2] = 0.5 * (np.array(tl[:-1]) + np.array(tl[1:]))
        for (ia, ib), ltag in zip(tooth_cols, (TAG_ZHENG, TAG_FU)):
            ci0, ci1 = 2 * ia, 2 * ib
            tw = ci1 - ci0 + 1
            g = np.empty((2 * trows + 1, tw), dtype=np.int64)
            g[0, :] = gid[-1, ci0:ci1 + 1]                 # shared with the surface row
            cnt = (2 * trows) * tw
            g[1:, :] = (n_next + np.arange(cnt)).reshape(2 * trows, tw)
            n_next += cnt
            pos.append(np.column_stack([np.tile(xn[ci0:ci1 + 1], 2 * trows),
                                        np.repeat(ty[1:], tw)]))
            for er in range(trows):
                for ec in range((tw - 1) // 2):
                    quads.append(q9(g, 2 * ec, 2 * er))
                    tags.append(electrode.tag)
            add_line(list(g[0, :]), ltag)                  # contact with the film
            add_line(list(g[:, 0]), ltag)                  # left flank
            add_line(list(g[:, -1]), ltag)                 # right flank
            add_line(list(g[-1, :]), ltag)                 # top
    P = np.vstack(pos)
    POS = _clean13(np.column_stack([P, np.zeros(P.shape[0])]))
    QUADS9 = np.column_stack([np.array(quads, dtype=float) + 1, np.array(tags, dtype=float)])
    L = np.array(lines, dtype=float)
    L[:, :3] += 1
    pml = bands[-1]
    bottom = float(POS[:, 1].min())
    layer_tags = [b.tag for b in bands[1:-1]]
    tag_map = {TAG_PIEZO: 0, TAG_ELECTRODE: 1}
    tag_map.update({t: i + 2 for i, t in enumerate(layer_tags)})
    tag_map[pml.tag] = len(layer_tags) + 1 if layer_tags else 0
    return Q9Cell(POS=POS, QUADS9=QUADS9, LINES3=L, tag_map=tag_map, pml_tag=pml.tag,
                  pml_top_um=bottom + pml.thickness_um, pml_bottom_um=bottom, period_um=w,
                  info=dict(columns=columns, rows=nrows, tooth_cols=tooth_cols))


def sp_double_layer_cell() -> Q9Cell:
    """The reference's ``sp_double_layer`` template at its defaults, rebuilt without Gmsh.

    Geometry of ``src/sawsim/sp_meshes/double.py:21-185`` with pitch 1.085 um,
    Al 0.17 um (1 row), LT film 0.6 um (3 rows), Si 8.33 um (31 rows), PML 2p
    (8 rows), 8 columns of p/4: 340 elements, 1465 nodes.
    """
    p = 1.085
    return q9_cell(p, 8, [Band(TAG_PIEZO, 0.6, 3), Band(22, 8.33, 31), Band(23, 2 * p, 8)],
                   Band(TAG_ELECTRODE, 0.17, 1))


def me0_cell(columns: int = 16, rows: int = 64, pitch_um: float = 1.085) -> Q9Cell:
    """Plane-strain single-crystal cell: 3p piezo substrate over a 1p PML.

    ``rows`` element rows split 3:1 between substrate and PML; electrode teeth of
    thickness 0.08p (one element row) and metal ratio 0.5 on top.
    """
    p = pitch_um
    r_pml = rows // 4
    return q9_cell(p, columns, [Band(TAG_PIEZO, 3 * p, rows - r_pml), Band(22, p, r_pml)],
                   Band(TAG_ELECTRODE, 0.08 * p, 1))


def me1_two_layer_cell(columns: int = 64, rows: int = 256, pitch_um: float = 1.085) -> Q9Cell:
    """ME1 two-layer cell: 3m film 0.6p / SiO2 0.3p / Si 3p / PML 1p.

    Element rows 3/16 film, 3/32 SiO2, 17/32 Si, 3/16 PML (48/24/136/48 at 256).
    Material order: 0 piezo, 1 Al, 2 SiO2, 3 Si (the PML continues the Si).
    """
    p = pitch_um
    r_film = rows * 3 // 16
    r_ox = rows * 3 // 32
    r_pml = rows * 3 // 16
    r_si = rows - r_film - r_ox - r_pml
    return q9_cell(p, columns, [Band(TAG_PIEZO, 0.6 * p, r_film), Band(22, 0.3 * p, r_ox),
                                Band(23, 3 * p, r_si), Band(24, p, r_pml)],
                   Band(TAG_ELECTRODE, 0.08 * p, 1))


def me1_four_layer_cell(columns: int = 128, rows: int = 512, pitch_um: float = 1.085) -> Q9Cell:
    """Four-layer Q9 stack: piezo 0.5p / SiO2 0.25p / poly-Si 0.5p / Si 3p / PML 1p.

    Material order: 0 piezo, 1 Al, 2 SiO2, 3 poly-Si, 4 Si.
    """
    p = pitch_um
    r_film = rows * 5 // 32
    r_ox = rows * 3 // 32
    r_poly = rows * 5 // 32
    r_pml = rows * 5 // 32
    r_si = rows - r_film - r_ox - r_poly - r_pml
    return q9_cell(p, columns, [Band(TAG_PIEZO, 0.5 * p, r_film), Band(22, 0.25 * p, r_ox),
                                Band(23, 0.5 * p, r_poly), Band(24, 3 * p, r_si),
                                Band(25, p, r_pml)],
                   Band(TAG_ELECTRODE, 0.08 * p, 1))
