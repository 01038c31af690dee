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

import math
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


def sp_quad_layer_cell() -> Q9Cell:
    """The reference's ``sp_quad_layer`` template at its defaults, rebuilt without Gmsh.

    Geometry of ``src/sawsim/sp_meshes/quad.py:26-160`` with pitch 1.085 um,
    MR 0.5, Al 0.17 um (1 row), LT 0.6 um (3 rows, tag 16), SiO2 0.5 um (2 rows,
    tag 22), poly-Si 1.0 um (4 rows, tag 23), Si 7.83 um (29 rows, tag 24), PML
    2.17 um (8 rows, tag 25, the Si material), 8 columns of p/4: 372 elements,
    1601 nodes.  Material order: 0 piezo, 1 Al, 2 SiO2, 3 poly-Si, 4 Si.
    """
    p = 1.085
    return q9_cell(p, 8, [Band(TAG_PIEZO, 0.6, 3), Band(22, 0.5, 2), Band(23, 1.0, 4), Band(24, 7.83, 29),
                          Band(25, 2.17, 8)], Band(TAG_ELECTRODE, 0.17, 1))


def _stack_bands(pitch_um, electrode_um, substrate_um, backings, coatings, mesh_um, pml_pitches):
    """Element bands of the generic stack, bottom first: (tag, y_bottom, y_top, rows),
    with 'E' for the electrode band, following src/sawsim/sp_meshes/stack.py:27-68:
    mesh_um near the surface (depth <= 2p), max(h, min(4h, p/2)) deeper, a band
    that crosses depth 2p split there; the PML (2p, at least 8 rows, deep
    spacing) below the last backing; above y = 0 the electrode band, then the
    coatings (the first measured from the piezo surface)."""
    p, h, d = float(pitch_um), float(mesh_um), float(electrode_um)
    h_deep = max(h, min(4 * h, p / 2))
    near = 2 * p
    nb, nc = len(backings), len(coatings)
    depth = [(TAG_PIEZO, 0.0, float(substrate_um))]
    z = float(substrate_um)
    for i, t in enumerate(backings):
        depth.append((22 + i, z, z + t))
        z += t
    split = []
    for tag, top, bot in depth:
        split += [(tag, top, near), (tag, near, bot)] if top < near < bot - 1e-12 else [(tag, top, bot)]

    def nrows(span, step):
        return max(1, math.ceil(span / step - 1e-9))

    below = [(tag, -bot, -top, nrows(bot - top, h if bot <= near + 1e-12 else h_deep)) for tag, top, bot in split]
    pml_h = pml_pitches * p
    tag_pml = 22 + nb + nc
    below.append((tag_pml, -(z + pml_h), -z, max(8, nrows(pml_h, h_deep))))
    below.sort(key=lambda b: b[1])
    above = [('E', 0.0, d, nrows(d, h))]
    if nc:
        top = float(coatings[0])
        if not top > d:
            raise ValueError('the first coating is measured from the piezo surface and must exceed the electrode')
        above.append((22 + nb, d, top, nrows(top - d, h)))
        for j, t in enumerate(coatings[1:], start=1):
            above.append((22 + nb + j, top, top + t, nrows(t, h)))
            top += t
    return below, above, dict(h_near=h, h_deep=h_deep, pml_thickness_um=pml_h, tag_pml=tag_pml,
                              tag_backing=[22 + i for i in range(nb)], tag_coating=[22 + nb + j for j in range(nc)])


def sp_stack_cell(pitch_um: float = 1.085, metal_ratio: float = 0.5, electrode_um: float = 0.17,
                  substrate_um: float = 8.0, backings=(), coatings=(), mesh_um: float = 0.5,
                  pml_pitches: float = 2.0) -> Q9Cell:
    """The reference's generic ``sp_stack`` template (``src/sawsim/sp_meshes/stack.py``),
    rebuilt without Gmsh: a two-pitch cell with one + and one - electrode, from the
    bottom: PML | backings (last .. first) | piezo substrate | electrodes, embedded
    in the first coating when there is one | further coatings.

    Across, 9 cuts at the electrode edges and centres make 8 strips of
    ceil(width / mesh_um) uniform columns each, the same on every level; down,
    every band has the rows of ``_stack_bands``, uniform inside the band.  Without
    coatings the electrode band holds only the four electrode strips (free
    surface between them).  ``backings`` and ``coatings`` are thicknesses in um
    (0-6 and 0-3 of them); tags 16 piezo, 15 electrode, 22.. backings, then
    coatings, then the PML; lines 17 / 18 (the electrodes' contact, flanks and
    top), 19 left, 20 right, 21 bottom.  Material order (the reference's
    ``build_mesh`` for sp_stack): 0 piezo, 1 electrode, then backings and
    coatings; the PML takes the last backing's material, or the piezo's.
    """
    p = float(pitch_um)
    w = 2 * p
    below, above, meta = _stack_bands(pitch_um, electrode_um, substrate_um, list(backings), list(coatings),
                                      mesh_um, pml_pitches)
    mr = float(metal_ratio)
    cuts = [0.0, p * (1 - mr) / 2, p / 2, p * (1 + mr) / 2, p, p * (3 - mr) / 2, 1.5 * p, p * (3 + mr) / 2, w]
    cols = [max(1, math.ceil((cuts[i + 1] - cuts[i]) / mesh_um - 1e-9)) for i in range(8)]
    # element edges and the strip / band of every element column / row
    xe, strip_of = [], []
    for i in range(8):
        xe += [cuts[i] + (cuts[i + 1] - cuts[i]) * j / cols[i] for j in range(cols[i])]
        strip_of += [i] * cols[i]
    xe.append(w)
    bands = below + above
    ye, band_of = [], []
    for bi, (_, y0, y1, nr) in enumerate(bands):
        ye += [y0 + (y1 - y0) * r / nr for r in range(nr)]
        band_of += [bi] * nr
    ye.append(bands[-1][2])
    ncol, nrow = len(xe) - 1, len(ye) - 1
    e_band = len(below)                                     # the band between y = 0 and y = d
    teeth = {1: TAG_ZHENG, 2: TAG_ZHENG, 5: TAG_FU, 6: TAG_FU}
    coated = bool(meta['tag_coating'])

    def elem_tag(r, c):
        bi = band_of[r]
        if bi != e_band:
            return bands[bi][0]
        if strip_of[c] in teeth:
            return TAG_ELECTRODE
        return meta['tag_coating'][0] if coated else None  # free surface between bare electrodes

    tags = np.array([[elem_tag(r, c) or 0 for c in range(ncol)] for r in range(nrow)])
    # candidate node grid (element edges and mid-points), then only the used nodes
    xn = np.empty(2 * ncol + 1)
    xn[0::2] = xe
    xn[1::2] = 0.5 * (np.array(xe[:-1]) + np.array(xe[1:]))
    yn = np.empty(2 * nrow + 1)
    yn[0::2] = ye
    yn[1::2] = 0.5 * (np.array(ye[:-1]) + np.array(ye[1:]))
    grid = np.arange(yn.size * xn.size).reshape(yn.size, xn.size)

    def q9(r, c):
        j, i = 2 * r, 2 * c
        g = grid
        return [g[j, i], g[j, i + 2], g[j + 2, i + 2], g[j + 2, i],
                g[j, i + 1], g[j + 1, i + 2], g[j + 2, i + 1], g[j + 1, i], g[j + 1, i + 1]]

    quads, qtags = [], []
    for r in range(nrow):
        for c in range(ncol):
            if tags[r, c]:
                quads.append(q9(r, c))
                qtags.append(tags[r, c])
    lines = []

    def edge(n0, nm, n1, tag):
        lines.append([n0, n1, nm, tag])

    for r in range(nrow):
        for c in range(ncol):
            if not tags[r, c]:
                continue
            j, i = 2 * r, 2 * c
            if r == 0:
                edge(grid[j, i], grid[j, i + 1], grid[j, i + 2], TAG_BOTTOM)
            if c == 0:
                edge(grid[j, i], grid[j + 1, i], grid[j + 2, i], TAG_LEFT)
            if c == ncol - 1:
                edge(grid[j, i + 2], grid[j + 1, i + 2], grid[j + 2, i + 2], TAG_RIGHT)
            s = strip_of[c]
            if band_of[r] == e_band and s in teeth:
                lt = teeth[s]
                if r == 0 or band_of[r - 1] != e_band:            # contact with the piezo surface
                    edge(grid[j, i], grid[j, i + 1], grid[j, i + 2], lt)
                if r == nrow - 1 or band_of[r + 1] != e_band:     # electrode top
                    edge(grid[j + 2, i], grid[j + 2, i + 1], grid[j + 2, i + 2], lt)
                if s in (1, 5) and (c == 0 or strip_of[c - 1] != s):
                    edge(grid[j, i], grid[j + 1, i], grid[j + 2, i], lt)            # outer flank
                if s in (2, 6) and (c == ncol - 1 or strip_of[c + 1] != s):
                    edge(grid[j, i + 2], grid[j + 1, i + 2], grid[j + 2, i + 2], lt)  # outer flank
    used = np.unique(np.array(quads).ravel())
    renum = np.full(grid.size, -1, dtype=np.int64)
    renum[used] = np.arange(used.size)
    X, Y = np.meshgrid(xn, yn)
    P = np.column_stack([X.ravel()[used], Y.ravel()[used], np.zeros(used.size)])
    POS = _clean13(P)
    Q = renum[np.array(quads)]
    QUADS9 = np.column_stack([Q.astype(float) + 1, np.array(qtags, dtype=float)])
    Ln = np.array(lines, dtype=np.int64)
    LINES3 = np.column_stack([renum[Ln[:, :3]].astype(float) + 1, Ln[:, 3].astype(float)])
    tb, tc = meta['tag_backing'], meta['tag_coating']
    tag_map = {TAG_PIEZO: 0, TAG_ELECTRODE: 1, meta['tag_pml']: (1 + len(tb)) if tb else 0}
    tag_map.update({t: i + 2 for i, t in enumerate(tb + tc)})
    bottom = float(POS[:, 1].min())
    return Q9Cell(POS=POS, QUADS9=QUADS9, LINES3=LINES3, tag_map=tag_map, pml_tag=meta['tag_pml'],
                  pml_top_um=bottom + meta['pml_thickness_um'], pml_bottom_um=bottom, period_um=w,
                  info=dict(rows=[b[3] for b in bands], cols=cols, levels=[b[1] for b in bands] + [bands[-1][2]],
                            cuts=cuts, h_near=meta['h_near'], h_deep=meta['h_deep'],
                            tag_backing=tb, tag_coating=tc, pml_thickness_um=meta['pml_thickness_um']))


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


# ---------------------------------------------------------------------------- Hex27 slab
HEX_TAG_PIEZO, HEX_TAG_ELECTRODE, HEX_TAG_LAYER = 7, 8, 9   # volume tags of sp_hex_meshes/double.py:120-123


def _h27_factor(code, t):
    return t * (t - 1.0) if code == 0 else t * (t + 1.0) if code == 1 else (t + 1.0) * (t - 1.0)


# raw H27 functions (factor codes per axis: 0 t(t-1), 1 t(t+1), 2 (t+1)(t-1)) and the
# sortSF27 permutation (src/sawsim/saw2d/saw3d/elements.py:28-44)
_H27_RAW = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1),
            (2, 0, 0), (1, 2, 0), (2, 1, 0), (0, 2, 0), (0, 0, 2), (1, 0, 2), (1, 1, 2), (0, 1, 2),
            (2, 0, 1), (1, 2, 1), (2, 1, 1), (0, 2, 1), (2, 2, 0), (2, 0, 2), (1, 2, 2), (2, 1, 2),
            (0, 2, 2), (2, 2, 1), (2, 2, 2)]
_H27_PERM = [6, 5, 4, 7, 2, 1, 0, 3, 17, 18, 14, 16, 13, 19, 12, 15, 9, 10, 8, 11, 25, 22, 23, 21, 24, 20, 26]


def h27_local_nodes() -> np.ndarray:
    """(27, 3) natural coordinates in {-1, 0, 1} of the node of each H27 function:
    per axis, t(t-1) vanishes except at -1, t(t+1) except at +1, (t+1)(t-1) except at 0."""
    return np.array([[-1.0 if c == 0 else 1.0 if c == 1 else 0.0 for c in _H27_RAW[r]] for r in _H27_PERM])


@dataclass
class HexCell:
    """A structured Hex27 slab: nodes (um), 0-based connectivity, volume tags and the
    boundary node sets of ``find_saw_boundary_3ds`` (src/sawsim/saw2d/saw3d/boundary.py:32-51)."""

    POS: np.ndarray
    HEXAS27: np.ndarray
    hex_tag: np.ndarray
    sets: dict
    tag_map: dict
    pml_tag: int
    pml_top_um: float
    pml_bottom_um: float
    period_um: float
    aperture_um: float
    info: dict = field(default_factory=dict)


def hex_slab_cell(pitch_um: float, nx: int, ny: int, bands, electrode: Band, aperture_um: float,
                  metal_ratio: float = 0.5) -> HexCell:
    """Two-pitch-wide periodic Hex27 slab (the layout of src/sawsim/sp_hex_meshes/double.py:21-135).

    x in [0, 2p] (nx uniform cells, L/R periodic), y in [0, aperture] (ny cells,
    front/back periodic), z downward from the surface through ``bands`` (last band
    = PML, tagged by its own tag); the + and - electrode blocks of width
    ``metal_ratio * p`` centred at p/2 and 3p/2 stand ``electrode.thickness_um``
    above the surface with ``electrode.rows`` element layers.  Node sets: L (x=0),
    R (x=2p), front (y=0), back (y=aperture), bottom (z=min), zheng / fu = the outer
    surface nodes of the + / - electrode blocks, base included.
    """
    p = float(pitch_um)
    w = 2 * p
    xs = np.array([w * i / nx for i in range(nx + 1)])
    edges = [p * (1 - metal_ratio) / 2, p * (1 + metal_ratio) / 2, p * (3 - metal_ratio) / 2,
             p * (3 + metal_ratio) / 2]
    cols = []
    for a, b in ((edges[0], edges[1]), (edges[2], edges[3])):
        ia, ib = int(np.argmin(np.abs(xs - a))), int(np.argmin(np.abs(xs - b)))
        if abs(xs[ia] - a) > 1e-9 * w or abs(xs[ib] - b) > 1e-9 * w or ib <= ia:
            raise ValueError('electrode edges must fall on cell edges')
        cols.append((ia, ib))
    levels, owner = _band_levels(0.0, bands)                  # bottom -> top, z
    nz = len(owner)
    tl = [electrode.thickness_um * r / electrode.rows for r in range(1, electrode.rows + 1)]
    zlev = np.array(list(levels) + tl)
    xn = np.empty(2 * nx + 1)
    xn[0::2] = xs
    xn[1::2] = 0.5 * (xs[:-1] + xs[1:])
    ys = np.array([aperture_um * j / ny for j in range(ny + 1)])
    yn = np.empty(2 * ny + 1)
    yn[0::2] = ys
    yn[1::2] = 0.5 * (ys[:-1] + ys[1:])
    zn = np.empty(2 * len(zlev) - 1)
    zn[0::2] = zlev
    zn[1::2] = 0.5 * (zlev[:-1] + zlev[1:])

    ids = {}
    pos = []

    def node(i, j, k):
        key = (i, j, k)
        if key not in ids:
            ids[key] = len(pos)
            pos.append((xn[i], yn[j], zn[k]))
        return ids[key]

    loc = h27_local_nodes().astype(int)
    hexas, tags = [], []

    def add(ex, ey, ez, tag):
        hexas.append([node(2 * ex + 1 + lx, 2 * ey + 1 + ly, 2 * ez + 1 + lz) for lx, ly, lz in loc])
        tags.append(tag)

    for ez in range(nz):
        for ey in range(ny):
            for ex in range(nx):
                add(ex, ey, ez, bands[owner[ez]].tag)
    elec = []
    for ia, ib in cols:
        members = set()
        for ez in range(nz, nz + electrode.rows):
            for ey in range(ny):
                for ex in range(ia, ib):
                    add(ex, ey, ez, electrode.tag)
        # outer surface of the block (lattice box [2ia, 2ib] x [0, 2ny] x [2nz, 2nz + 2 rows])
        k0, k1 = 2 * nz, 2 * (nz + electrode.rows)
        for (i, j, k), n in ids.items():
            if 2 * ia <= i <= 2 * ib and k0 <= k <= k1 and (i in (2 * ia, 2 * ib) or j in (0, 2 * ny) or
                                                           k in (k0, k1)):
                members.add(n)
        elec.append(np.array(sorted(members), dtype=np.int64))
    P = _clean13(np.array(pos))
    H = np.array(hexas, dtype=np.int64)
    T = np.array(tags, dtype=np.int64)
    lat = np.array(list(ids.keys()))
    nid = np.array(list(ids.values()))
    order = np.argsort(nid)
    lat = lat[order]

    def where(mask):
        return np.sort(nid[order][mask]).astype(np.int64)

    kmin = 0
    sets = dict(L=where(lat[:, 0] == 0), R=where(lat[:, 0] == 2 * nx), front=where(lat[:, 1] == 0),
                back=where(lat[:, 1] == 2 * ny), bottom=where(lat[:, 2] == kmin), zheng=elec[0], fu=elec[1])
    pml = bands[-1]
    layer_tags = [b.tag for b in bands[1:-1]]
    tag_map = {HEX_TAG_PIEZO: 0, HEX_TAG_ELECTRODE: 1}
    tag_map.update({t: i + 2 for i, t in enumerate(layer_tags)})
    tag_map[pml.tag] = len(layer_tags) + 1 if layer_tags else 0
    bottom = float(P[:, 2].min())
    return HexCell(POS=P, HEXAS27=H, hex_tag=T, sets=sets, tag_map=tag_map, pml_tag=pml.tag,
                   pml_top_um=bottom + pml.thickness_um, pml_bottom_um=bottom, period_um=w,
                   aperture_um=float(aperture_um), info=dict(nx=nx, ny=ny, nz=nz, electrode_cols=cols))


# Element layers of the Hex27 templates (src/sawsim/sp_hex_meshes/{single,double,triple,quad}.py):
# every band gets max(1, ceil(coef * thickness / base * ref / mesh_um)) layers; rows per
# template (piezo, backings..., PML), then the reference size ``ref`` those coefficients assume
_HEX_TEMPLATE_LAYERS = {
    'single': ([(30, 6.51)], (10, 2.17), 0.217),
    'double': ([(3, 0.6), (30, 6.51)], (10, 2.17), 0.217),
    'triple': ([(3, 0.6), (3, 0.5), (30, 6.51)], (11, 2.17), 0.217),
    'quad': ([(3, 0.6), (3, 0.5), (5, 1.0), (30, 6.0)], (10, 2.0), 0.2),
}


def sp_2p5d_template_cell(kind: str, pitch_um: float = 1.085, electrode_um: float = 0.17,
                          substrate_um: float = 0.6, layers_um=(6.51,), metal_ratio: float = 0.5,
                          mesh_um: float = 0.217, aperture_um: float = 0.217, nx: int = 16) -> HexCell:
    """The reference's 2.5D Hex27 templates (``sp_2p5d_{kind}_layer``, kind single /
    double / triple / quad; ``src/sawsim/sp_hex_meshes/*.py``) rebuilt without Gmsh.

    Down (z): the piezo substrate, the backing layers and a 2p PML, each with the
    element layers of the template's own rule (``_HEX_TEMPLATE_LAYERS``); the
    electrodes stand ``electrode_um`` high with their layers of the same rule.
    Across the aperture (y): one element, as the templates' transfinite y edges
    give.  Along x the templates leave the division to Gmsh's mesh size
    (``mesh_um``); ``nx`` uniform columns stand in for it: at the templates'
    defaults (strips of 1.25 and 2.5 x mesh_um) nx = 16 reproduces the reference's
    published curves within its own regression tolerance.  Tags: 7 piezo, 8
    electrode, 9.. backings, the PML after them with the last backing's material
    (the piezo's for the single layer).
    """
    rows, pml_rule, ref = _HEX_TEMPLATE_LAYERS[kind]
    hs = [float(substrate_um)] + [float(t) for t in layers_um]
    if len(hs) != len(rows):
        raise ValueError(f'sp_2p5d_{kind}_layer takes {len(rows) - 1} backing layers')

    def layers(coef, h, base):
        return max(1, math.ceil(coef * h / base * ref / mesh_um - 1e-12))

    p = float(pitch_um)
    bands = [Band(HEX_TAG_PIEZO, hs[0], layers(*rows[0][:1], hs[0], rows[0][1]))]
    for i, h in enumerate(hs[1:]):
        bands.append(Band(HEX_TAG_LAYER + i, h, layers(rows[i + 1][0], h, rows[i + 1][1])))
    bands.append(Band(HEX_TAG_LAYER + len(hs) - 1, 2 * p, layers(pml_rule[0], 2 * p, pml_rule[1])))
    electrode = Band(HEX_TAG_ELECTRODE, float(electrode_um), max(1, math.ceil(electrode_um / 0.17 * ref / mesh_um - 1e-12)))
    return hex_slab_cell(p, nx, 1, bands, electrode, aperture_um, metal_ratio=metal_ratio)


def hex_double_layer_slab(nx: int = 8, ny: int = 4, nz: int = 48, pitch_um: float = 1.085) -> HexCell:
    """Double-layer Hex27 slab: 3m film 0.6p / SiO2 1.4p / SiO2 PML 2p (z), aperture
    0.5p, Al electrodes 0.08p (one layer) on top.  ``nz`` element layers split
    1/6 film, 1/3 SiO2, 1/2 PML (8/16/24 at 48).  Material order: 0 piezo, 1 Al, 2 SiO2."""
    p = pitch_um
    r_film = nz // 6
    r_ox = nz // 3
    r_pml = nz - r_film - r_ox
    return hex_slab_cell(p, nx, ny, [Band(HEX_TAG_PIEZO, 0.6 * p, r_film), Band(HEX_TAG_LAYER, 1.4 * p, r_ox),
                                     Band(10, 2 * p, r_pml)], Band(HEX_TAG_ELECTRODE, 0.08 * p, 1), 0.5 * p)


def hex_four_layer_slab(nx: int = 12, ny: int = 6, nz: int = 80, pitch_um: float = 1.085) -> HexCell:
    """Four-layer Hex27 slab: 3m film 0.5p / SiO2 0.25p / poly-Si 0.5p / Si 1.75p / Si PML 1p
    (z), aperture 0.5p, Al electrodes 0.08p (one layer) of width p/3 (metal ratio 1/3, so
    that their edges fall on the p/6 cells of nx = 12).  ``nz`` layers split
    1/8, 1/16, 1/8, 7/16, 1/4 (10/5/10/35/20 at 80).  Material order: 0 piezo, 1 Al,
    2 SiO2, 3 poly-Si, 4 Si."""
    p = pitch_um
    r = [nz // 8, nz // 16, nz // 8]
    r_pml = nz // 4
    r_si = nz - sum(r) - r_pml
    return hex_slab_cell(p, nx, ny, [Band(HEX_TAG_PIEZO, 0.5 * p, r[0]), Band(HEX_TAG_LAYER, 0.25 * p, r[1]),
                                     Band(11, 0.5 * p, r[2]), Band(12, 1.75 * p, r_si), Band(13, p, r_pml)],
                         Band(HEX_TAG_ELECTRODE, 0.08 * p, 1), 0.5 * p, metal_ratio=1.0 / 3.0)
