"""Oracle: vectorised Q9 assembly of the piezoelectric K and M (test infrastructure).

Restates ``src/sawsim/saw2d/piezo_fem.py`` of the reference:

* Gauss rule and Q9 shapes: ``_gauss_3x3`` :48-53, ``_q9_shapes`` :56-103;
* 9-component gradient form of C / e: ``_C9`` :109-116, ``_e9`` :119-124,
  strain selectors ``_STRAIN_SEL`` :31-35;
* PML stretch tensors ``_T9`` :127-142, ``_Teps`` :145-155, per-element stretch
  at the centre node ``element_alpha`` :222-242;
* element Gram matrices ``_element_geometry`` :248-280;
* block scatter with the ``SCALE`` column scaling and COO->CSR: ``assemble``
  :283-367; ME0 lift-and-slice ``assemble_ME0`` :373-405.

DOF layout ``[ux | uy | uz | phi]`` (component-major, node-minor).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

SCALE = 6.173191780858575e-11               # piezo_fem.py:26

# strain row / derivative pairs for each displacement component (piezo_fem.py:31-35)
STRAIN_SEL = ((( 0, 0), (5, 1)),            # u_x: dux/dx -> row 0, dux/dy -> row 5
              (( 1, 1), (8, 0)),            # u_y: duy/dy -> row 1, duy/dx -> row 8
              (( 6, 1), (7, 0)))            # u_z: duz/dy -> row 6, duz/dx -> row 7


@dataclass
class Model:
    """Mesh container (piezo_fem.py:161-186): coordinates in metres, 0-based Q9."""

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
        sel = lines[lines[:, 3] == tag][:, :3].astype(int) - 1
        return np.unique(sel)


def build_model(msh) -> Model:
    return Model(pos_m=np.asarray(msh['POS'])[:, :2] * 1e-6,
                 quads=np.asarray(msh['QUADS9'])[:, :9].astype(int) - 1,
                 elem_tag=np.asarray(msh['QUADS9'])[:, 9].astype(int))


@dataclass
class PMLRegion:
    """One PML sub-region (piezo_fem.py:192-208)."""

    tag: int
    kind: str
    dmax: float = 1e11
    n: int = 3
    xa: float = 0.0
    xp: float = 0.0
    ya: float = 0.0
    yp: float = 0.0


def material_index(model: Model, tag_map: dict) -> np.ndarray:
    idx = np.full(model.ne, -1, dtype=int)
    for tag, mi in tag_map.items():
        idx[model.elem_tag == tag] = mi
    if (idx < 0).any():
        raise ValueError('element tags missing from the material map')
    return idx


def gauss_3x3():
    g = np.array([-0.774596669241483, 0.0, 0.774596669241483])
    w = np.array([5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0])
    # x varies fastest (piezo_fem.py:51-52)
    pts = np.array([(g[i], g[j]) for j in range(3) for i in range(3)])
    wts = np.array([w[i] * w[j] for j in range(3) for i in range(3)])
    return pts, wts


def q9_shapes(xi, eta):
    """Q9 shape functions (nq, 9) and reference derivatives (nq, 9, 2)."""
    x = np.asarray(xi, float)
    y = np.asarray(eta, float)
    N = 0.25 * np.stack([
        x * y * (x - 1) * (y - 1), x * y * (x + 1) * (y - 1),
        x * y * (x + 1) * (y + 1), x * y * (x - 1) * (y + 1),
        -2 * y * (x * x - 1) * (y - 1), -2 * x * (x + 1) * (y * y - 1),
        -2 * y * (x * x - 1) * (y + 1), -2 * x * (x - 1) * (y * y - 1),
        4 * (x * x - 1) * (y * y - 1)], axis=-1)
    dx = 0.25 * np.stack([
        y * (2 * x - 1) * (y - 1), y * (2 * x + 1) * (y - 1),
        y * (2 * x + 1) * (y + 1), y * (2 * x - 1) * (y + 1),
        -4 * x * y * (y - 1), -2 * (2 * x + 1) * (y + 1) * (y - 1),
        -4 * x * y * (y + 1), -2 * (2 * x - 1) * (y + 1) * (y - 1),
        8 * x * (y * y - 1)], axis=-1)
    dy = 0.25 * np.stack([
        x * (x - 1) * (2 * y - 1), x * (x + 1) * (2 * y - 1),
        x * (x + 1) * (2 * y + 1), x * (x - 1) * (2 * y + 1),
        -2 * (x + 1) * (x - 1) * (2 * y - 1), -4 * x * y * (x + 1),
        -2 * (x + 1) * (x - 1) * (2 * y + 1), -4 * x * y * (x - 1),
        8 * y * (x * x - 1)], axis=-1)
    return N, np.stack([dx, dy], axis=-1)


def c9(C):
    """6x6 -> 9x9 gradient-form stiffness (piezo_fem.py:109-116)."""
    out = np.zeros((9, 9), dtype=np.result_type(C, float))
    out[:6, :6] = C
    out[:6, 6:] = C[:, 3:6]
    out[6:, :6] = C[3:6, :]
    out[6:, 6:] = C[3:6, 3:6]
    return out


def e9(e):
    """3x6 -> 3x9 gradient-form piezo tensor (piezo_fem.py:119-124)."""
    out = np.zeros((3, 9), dtype=np.result_type(e, float))
    out[:, :6] = e
    out[:, 6:] = e[:, 3:6]
    return out


def stretch_T9(a1, a2, a3):
    """(9, 9, ne) PML multiplier of the gradient-form stiffness (piezo_fem.py:127-142)."""
    A, D, F = a2 * a3 / a1, a1 * a3 / a2, a1 * a2 / a3
    code = dict(A=A, b=a3, c=a2, D=D, e=a1, F=F)
    rows = ['AbcccbbAA', 'bDeeeDDbb', 'ceFFFeecc']
    rows = rows + [rows[2], rows[2], rows[1], rows[1], rows[0], rows[0]]
    T = np.empty((9, 9, np.shape(a1)[0]), dtype=complex)
    for r, word in enumerate(rows):
        for c, ch in enumerate(word):
            T[r, c] = code[ch]
    return T


def stretch_eps(a1, a2, a3):
    """(3, 3, ne) PML multiplier of the permittivity (piezo_fem.py:145-155)."""
    T = np.empty((3, 3, np.shape(a1)[0]), dtype=complex)
    T[0, 0], T[0, 1], T[0, 2] = a2 * a3 / a1, a3, a2
    T[1, 0], T[1, 1], T[1, 2] = a3, a1 * a3 / a2, a1
    T[2, 0], T[2, 1], T[2, 2] = a2, a1, a1 * a2 / a3
    return T


def element_alpha(model: Model, pml_regions, omega: float):
    """Per-element complex stretches (a1, a2, a3) at the centre node (piezo_fem.py:222-242)."""
    ne = model.ne
    a1 = np.ones(ne, dtype=complex)
    a2 = np.ones(ne, dtype=complex)
    a3 = np.ones(ne, dtype=complex)
    xc = model.pos_m[model.quads[:, 8], 0]
    yc = model.pos_m[model.quads[:, 8], 1]
    for reg in pml_regions:
        sel = model.elem_tag == reg.tag
        if 'x' in reg.kind:
            r = np.clip((xc - reg.xp) ** 2 / (reg.xa - reg.xp) ** 2, 0.0, 1.0)
            a1[sel] = 1.0 + (reg.dmax * (1.0 - r) ** reg.n)[sel] / (1j * omega)
        if 'y' in reg.kind:
            r = np.clip((yc - reg.yp) ** 2 / (reg.ya - reg.yp) ** 2, 0.0, 1.0)
            a2[sel] = 1.0 + (reg.dmax * (1.0 - r) ** reg.n)[sel] / (1j * omega)
    return a1, a2, a3


def element_grams(model: Model):
    """Gradient Grams G[(d1, d2)] (ne, 9, 9) and mass Gram GM (ne, 9, 9) (piezo_fem.py:248-280)."""
    pts, wts = gauss_3x3()
    Nq, dNr = q9_shapes(pts[:, 0], pts[:, 1])
    xy = model.pos_m[model.quads]                            # (ne, 9, 2)
    J = np.einsum('eai,qaj->eqij', xy, dNr)
    det = J[..., 0, 0] * J[..., 1, 1] - J[..., 0, 1] * J[..., 1, 0]
    inv = np.empty_like(J)
    inv[..., 0, 0], inv[..., 1, 1] = J[..., 1, 1], J[..., 0, 0]
    inv[..., 0, 1], inv[..., 1, 0] = -J[..., 0, 1], -J[..., 1, 0]
    inv /= det[..., None, None]
    dN = np.einsum('qaj,eqjk->eqak', dNr, inv)               # (ne, nq, 9, 2)
    dV = wts[None, :] * det
    G = {(d1, d2): np.einsum('eq,eqa,eqb->eab', dV, dN[..., d1], dN[..., d2])
         for d1 in (0, 1) for d2 in (0, 1)}
    GM = np.einsum('eq,qa,qb->eab', dV, Nq, Nq)
    return G, GM


def element_tensors(model, materials, mat_idx, pml_regions, omega_top):
    """Per-element stretched tensors C_eff (9,9,ne), E_eff (3,9,ne), P_eff (3,3,ne), rho_eff (ne,)."""
    a1, a2, a3 = element_alpha(model, pml_regions, omega_top)
    T9 = stretch_T9(a1, a2, a3)
    Teps = stretch_eps(a1, a2, a3)
    mat_idx = np.asarray(mat_idx, dtype=int)
    C9 = np.stack([c9(m.C) for m in materials])
    E9 = np.stack([e9(m.e) for m in materials])
    P = np.stack([np.asarray(m.eps) for m in materials])
    R = np.array([m.rho for m in materials])
    C_eff = T9 * np.moveaxis(C9[mat_idx], 0, -1)
    E_eff = T9[:3] * np.moveaxis(E9[mat_idx], 0, -1)
    P_eff = Teps * np.moveaxis(P[mat_idx], 0, -1)
    rho_eff = R[mat_idx] * a1 * a2 * a3
    return C_eff, E_eff, P_eff, rho_eff


def element_blocks(model, materials, mat_idx, pml_regions, omega_top):
    """Element matrices before scaling: Kuu[a][b], Kuf[a], Kff (each (ne, 9, 9)), Mel (ne, 9, 9).

    Accumulation order of piezo_fem.py:328-350.
    """
    G, GM = element_grams(model)
    C_eff, E_eff, P_eff, rho_eff = element_tensors(model, materials, mat_idx, pml_regions, omega_top)
    ne = model.ne
    Kuu = [[None] * 3 for _ in range(3)]
    for a in range(3):
        for b in range(3):
            blk = np.zeros((ne, 9, 9), dtype=complex)
            for rv, dv in STRAIN_SEL[a]:
                for ru, du in STRAIN_SEL[b]:
                    blk += C_eff[rv, ru][:, None, None] * G[(dv, du)]
            Kuu[a][b] = blk
    Kuf = []
    for a in range(3):
        blk = np.zeros((ne, 9, 9), dtype=complex)
        for rv, dv in STRAIN_SEL[a]:
            for k in (0, 1):
                blk += E_eff[k, rv][:, None, None] * G[(dv, k)]
        Kuf.append(blk)
    Kff = np.zeros((ne, 9, 9), dtype=complex)
    for j in (0, 1):
        for k in (0, 1):
            Kff += P_eff[j, k][:, None, None] * G[(j, k)]
    Mel = rho_eff[:, None, None] * GM
    return Kuu, Kuf, Kff, Mel


def assemble(model, materials, mat_idx, pml_regions, omega_top):
    """Global (K, M), 4N x 4N complex CSR (piezo_fem.py:283-367)."""
    N, ne = model.N, model.ne
    Kuu, Kuf, Kff, Mel = element_blocks(model, materials, mat_idx, pml_regions, omega_top)
    ri = np.broadcast_to(model.quads[:, :, None], (ne, 9, 9))
    ci = np.broadcast_to(model.quads[:, None, :], (ne, 9, 9))
    R, Cc, V = [], [], []

    def put(blk, roff, coff, fac):
        R.append((ri + roff).ravel())
        Cc.append((ci + coff).ravel())
        V.append((blk * fac).ravel())

    for a in range(3):
        for b in range(3):
            put(Kuu[a][b], a * N, b * N, SCALE)
    for a in range(3):
        put(Kuf[a], a * N, 3 * N, 1.0)
        put(Kuf[a].transpose(0, 2, 1), 3 * N, a * N, SCALE)
    put(Kff, 3 * N, 3 * N, -1.0)
    K = sp.coo_matrix((np.concatenate(V), (np.concatenate(R), np.concatenate(Cc))),
                      shape=(4 * N, 4 * N), dtype=complex).tocsr()
    mblk = Mel * SCALE
    M = sp.coo_matrix((np.concatenate([mblk.ravel()] * 3),
                       (np.concatenate([(ri + a * N).ravel() for a in range(3)]),
                        np.concatenate([(ci + a * N).ravel() for a in range(3)]))),
                      shape=(4 * N, 4 * N), dtype=complex).tocsr()
    return K, M


def _lift(m):
    """Zero-filled full tensors from projected xy ones (piezo_fem.py:389-401)."""
    from types import SimpleNamespace
    s, el = [0, 1, 5], [0, 1]
    C = np.zeros((6, 6), dtype=np.result_type(m.C, float))
    e = np.zeros((3, 6), dtype=np.result_type(m.e, float))
    eps = np.zeros((3, 3), dtype=np.result_type(m.eps, float))
    C[np.ix_(s, s)] = m.C
    e[np.ix_(el, s)] = m.e
    eps[np.ix_(el, el)] = m.eps
    return SimpleNamespace(rho=m.rho, C=C, e=e, eps=eps)


def assemble_me0(model, materials_projected, mat_idx, pml_regions, omega_top):
    """Plane-strain (K, M), 3N x 3N: lift projected tensors, assemble at 4N, keep
    [ux, uy, phi] (piezo_fem.py:373-405)."""
    lifted = [_lift(m) for m in materials_projected]
    K, M = assemble(model, lifted, mat_idx, pml_regions, omega_top)
    n = model.N
    keep = np.r_[0:2 * n, 3 * n:4 * n]
    return K[keep][:, keep].tocsr(), M[keep][:, keep].tocsr()
