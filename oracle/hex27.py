"""Oracle: Hex27 assembly, periodic boundary sets and the 3D frequency solve (test infrastructure).

Restates the reference's 2.5D slab path (src/sawsim/saw2d/saw3d/):

* H27 basis and 27-point Gauss rule with the truncated literals:
  ``elements.py:22-44`` (table, sortSF27 permutation), ``:63-105``;
* Jacobian, |det| weights: ``assembly.py:31-70``;
* strain-displacement selection with the reference's quirk (the yz strain keeps
  only duy/dz): ``assembly.py:81-101``; potential gradient ``:104-123``;
* Voigt PML multipliers at the centre node (node 26), no clamp:
  ``assembly.py:127-213``;
* K = [[S K_uu, K_uphi], [S conj(K_uphi)^T, -K_phiphi]], M = S rho N N on the u
  components, S = KM_SCALE: ``assembly.py:230-327``; u interleaved 3n + c,
  phi at 3N + n;
* boundary sets and the periodic DOF lists: ``boundary.py:32-148``;
* two-stage fold (front/back, then left/right), prescribed DOFs, the
  per-frequency solve and Q = sum over the + electrode rows of the unfolded K
  times disp: ``bc_solve.py:25-175``; the finite-device variant (front/back, then
  the floating electrodes' equipotential fold): ``bc_solve.py:214-335``.

Element matrices are formed per element from gradient Grams (the reference forms
global B^T D B products); the two agree to rounding.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

KM_SCALE = 6.723363908816403e-11                                # assembly.py:24
_G, _W5, _W8 = 0.774596669241483, 0.555555555555556, 0.888888888888889   # elements.py:22-24
_RAW = [(1 / 8, 0, 0, 0), (1 / 8, 1, 0, 0), (1 / 8, 1, 1, 0), (1 / 8, 0, 1, 0), (1 / 8, 0, 0, 1),
        (1 / 8, 1, 0, 1), (1 / 8, 1, 1, 1), (1 / 8, 0, 1, 1), (-1 / 4, 2, 0, 0), (-1 / 4, 1, 2, 0),
        (-1 / 4, 2, 1, 0), (-1 / 4, 0, 2, 0), (-1 / 4, 0, 0, 2), (-1 / 4, 1, 0, 2), (-1 / 4, 1, 1, 2),
        (-1 / 4, 0, 1, 2), (-1 / 4, 2, 0, 1), (-1 / 4, 1, 2, 1), (-1 / 4, 2, 1, 1), (-1 / 4, 0, 2, 1),
        (1 / 2, 2, 2, 0), (1 / 2, 2, 0, 2), (1 / 2, 1, 2, 2), (1 / 2, 2, 1, 2), (1 / 2, 0, 2, 2),
        (1 / 2, 2, 2, 1), (-1.0, 2, 2, 2)]
_PERM = [6, 5, 4, 7, 2, 1, 0, 3, 17, 18, 14, 16, 13, 19, 12, 15, 9, 10, 8, 11, 25, 22, 23, 21, 24, 20, 26]
# component c -> (Voigt strain row, derivative direction) of the reference B matrix
_SEL = {0: [(0, 0), (5, 1), (4, 2)], 1: [(5, 0), (1, 1), (3, 2)], 2: [(4, 0), (2, 2)]}


def _f(code, t):
    return t * (t - 1.0) if code == 0 else t * (t + 1.0) if code == 1 else (t + 1.0) * (t - 1.0)


def _df(code, t):
    return 2.0 * t - 1.0 if code == 0 else 2.0 * t + 1.0 if code == 1 else 2.0 * t


def basis():
    """(N[q, a], dN[r, q, a], wf[q]) of the 27-point rule, sortSF27 order."""
    g, w = [-_G, 0.0, _G], [_W5, _W8, _W5]
    xi = np.array([(g[k1], g[k2], g[k3]) for k3 in range(3) for k2 in range(3) for k1 in range(3)])
    wf = np.array([w[k1] * w[k2] * w[k3] for k3 in range(3) for k2 in range(3) for k1 in range(3)])
    N = np.zeros((27, 27))
    dN = np.zeros((3, 27, 27))
    for a, r in enumerate(_PERM):
        c, f1, f2, f3 = _RAW[r]
        x1, x2, x3 = xi[:, 0], xi[:, 1], xi[:, 2]
        N[:, a] = c * _f(f1, x1) * _f(f2, x2) * _f(f3, x3)
        dN[0, :, a] = c * _df(f1, x1) * _f(f2, x2) * _f(f3, x3)
        dN[1, :, a] = c * _f(f1, x1) * _df(f2, x2) * _f(f3, x3)
        dN[2, :, a] = c * _f(f1, x1) * _f(f2, x2) * _df(f3, x3)
    return N, dN, wf


def _stretch(pml, centre_xyz, omega):
    """Per-element (a1, a2, a3) of a PML dict (assembly.py:127-143)."""
    n = centre_xyz.shape[0]
    a = [np.ones(n, complex) for _ in range(3)]
    region = pml['region']
    if region in {1, 5, 6, 7, 8, 9, 10, 11} or region in (2, 4):
        d = pml['dmax'] * (1.0 - (centre_xyz[:, 0] - pml['xp']) ** 2 / (pml['xa'] - pml['xp']) ** 2) ** pml['n']
        a[0] = 1.0 + d / (1j * omega)
    if region == 3 or region in (2, 4):
        d = pml['dmax'] * (1.0 - (centre_xyz[:, 2] - pml['zp']) ** 2 / (pml['za'] - pml['zp']) ** 2) ** pml['n']
        a[2] = 1.0 + d / (1j * omega)
    return a


def _multipliers(a1, a2, a3):
    """Voigt stretch multipliers for C (6x6), e (3x6), eps (3x3) (assembly.py:146-179)."""
    r1, r2, r3 = a2 * a3 / a1, a1 * a3 / a2, a1 * a2 / a3
    row0, row1, row2 = [r1, a3, a2, a3, r1, r1], [a3, r2, a1, r2, a3, a3], [a2, a1, r3, a1, a2, a2]
    c = np.stack([np.stack(r, -1) for r in (row0, row1, row2, row2, row2, row1)], -2)
    e = np.stack([np.stack(r, -1) for r in ([r1, a3, a2, a2, a2, a3], [a3, r2, a1, a1, a1, r2],
                                             [a2, a1, r3, r3, r3, a1])], -2)
    p = np.stack([np.stack(r, -1) for r in ([r1, a3, a2], [a3, r2, a1], [a2, a1, r3])], -2)
    return c, e, p


def form_stiffness_mass_3d(elem, coord, material_list, pml_list, omega):
    """(mass, stiffness) like assembly.form_stiffness_mass_3d (assembly.py:230-308).

    material_list: dicts rho, C, e, eps, indx; pml_list: dicts region, indx and,
    when indx is non-empty, za, zp, xa, xp, dmax, n, rho, C, e, eps.
    """
    elem = np.asarray(elem, dtype=np.int64)
    ne, nn = elem.shape[0], coord.shape[0]
    Nq, dN, wf = basis()
    X = coord[elem]                                                    # (ne, 27, 3)
    J = np.einsum('rqa,eac->eqrc', dN, X)
    det = (J[..., 0, 0] * (J[..., 1, 1] * J[..., 2, 2] - J[..., 2, 1] * J[..., 1, 2])
           - J[..., 0, 1] * (J[..., 1, 0] * J[..., 2, 2] - J[..., 1, 2] * J[..., 2, 0])
           + J[..., 0, 2] * (J[..., 1, 0] * J[..., 2, 1] - J[..., 1, 1] * J[..., 2, 0]))
    Ji = np.linalg.inv(J)
    dNx = np.einsum('eqir,rqa->eqai', Ji, dN)                        # (ne, 27q, 27a, 3)
    w = np.abs(det) * wf[None, :]
    G = np.einsum('eq,eqai,eqbj->eabij', w, dNx, dNx, optimize=True)
    GM = np.einsum('eq,qa,qb->eab', w, Nq, Nq)

    C = np.zeros((ne, 6, 6), complex)
    E = np.zeros((ne, 3, 6), complex)
    P = np.zeros((ne, 3, 3), complex)
    rho = np.zeros(ne, complex)
    for m in material_list:
        ids = np.asarray(m['indx'], dtype=np.int64)
        C[ids], E[ids], P[ids], rho[ids] = m['C'], m['e'], m['eps'], m['rho']
    for pml in pml_list:
        ids = np.asarray(pml.get('indx', []), dtype=np.int64)
        if ids.size == 0:
            continue
        a1, a2, a3 = _stretch(pml, coord[elem[ids, 26]], omega)
        mc, me, mp = _multipliers(a1, a2, a3)
        C[ids] = pml['C'][None] * mc
        E[ids] = pml['e'][None] * me
        P[ids] = pml['eps'][None] * mp
        rho[ids] = pml['rho'] * a1 * a2 * a3

    S = np.zeros((3, 6, 3))                                            # selector [c, strain, dir]
    for c, lst in _SEL.items():
        for s, i in lst:
            S[c, s, i] = 1.0
    Kuu = np.einsum('csi,est,dtj,eabij->eacbd', S, C, S, G, optimize=True)           # (ne, a, c, b, d)
    Kuf = np.einsum('csi,ejs,eabij->eacb', S, E, G, optimize=True)                   # (ne, a, c, b)
    Kff = np.einsum('eij,eabij->eab', P, G)
    Me = rho[:, None, None] * GM

    ud = 3 * elem[:, :, None] + np.arange(3)[None, None, :]           # (ne, 27, 3)
    fd = 3 * nn + elem                                                # (ne, 27)
    rows, cols, vals = [], [], []

    def put(r, c, v):
        rows.append(np.broadcast_to(r, v.shape).ravel())
        cols.append(np.broadcast_to(c, v.shape).ravel())
        vals.append(v.ravel())

    put(ud[:, :, :, None, None], ud[:, None, None, :, :], Kuu * KM_SCALE)
    put(ud[:, :, :, None], fd[:, None, None, :], Kuf)
    put(fd[:, None, None, :], ud[:, :, :, None], np.conj(Kuf) * KM_SCALE)   # K_phiu[b, (a,c)] = S conj(K_uphi[(a,c), b])
    put(fd[:, :, None], fd[:, None, :], -Kff)
    K = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(4 * nn, 4 * nn)).tocsr()
    mr, mc_, mv = [], [], []
    for c in range(3):
        mr.append(np.broadcast_to(ud[:, :, None, c], Me.shape).ravel())
        mc_.append(np.broadcast_to(ud[:, None, :, c], Me.shape).ravel())
        mv.append((Me * KM_SCALE).ravel())
    M = sp.coo_matrix((np.concatenate(mv), (np.concatenate(mr), np.concatenate(mc_))),
                      shape=(4 * nn, 4 * nn)).tocsr()
    return M, K


# ------------------------------------------------------------------ boundary (boundary.py:32-148)
def _sort_lr(left, right, xyz):
    cor = np.round(xyz * 1e9, 1)
    return left[np.lexsort((cor[left, 2], cor[left, 1]))], right[np.lexsort((cor[right, 2], cor[right, 1]))]


def _sort_fb(front, back, xyz):
    cor = np.round(xyz * 1e9, 1)
    return front[np.lexsort((cor[front, 2], cor[front, 0]))], back[np.lexsort((cor[back, 2], cor[back, 0]))]


def _mach(nodes):
    nodes = np.asarray(nodes, dtype=np.int64)
    return np.concatenate([3 * nodes, 3 * nodes + 1, 3 * nodes + 2])


def boundary_idx_vect_3ds(sets, xyz, gdofu):
    """Periodic / prescribed DOF lists (boundary.py:84-148)."""
    I, D = np.intersect1d, np.setdiff1d
    g2, L, R, front, back, zheng, fu = (np.asarray(sets[k], dtype=np.int64) for k in
                                        ('bottom', 'L', 'R', 'front', 'back', 'zheng', 'fu'))
    fz, bz, ff, bf = I(front, zheng), I(back, zheng), I(front, fu), I(back, fu)
    front = D(front, np.concatenate([fz, ff]))
    back = D(back, np.concatenate([bz, bf]))
    g2F, g2b, g2L, g2R = I(g2, front), I(g2, back), I(g2, L), I(g2, R)
    g2Lb, g2Rb = I(g2, I(L, back)), I(g2, I(R, back))
    g2Le, g2Re = D(g2L, g2Lb), D(g2R, g2Rb)
    front, back, L, R = D(front, g2F), D(back, g2b), D(L, g2L), D(R, g2R)
    L, R = D(L, I(L, back)), D(R, I(R, back))
    L, R = _sort_lr(L, R, xyz)
    front, back = _sort_fb(front, back, xyz)
    g2F, g2b = _sort_fb(g2F, g2b, xyz)
    g2Le, g2Re = _sort_lr(g2Le, g2Re, xyz)
    fz, bz = _sort_fb(fz, bz, xyz)
    ff, bf = _sort_fb(ff, bf, xyz)
    m = dict(period_F=np.concatenate([_mach(front), _mach(fz), _mach(ff)]),
             period_B=np.concatenate([_mach(back), _mach(bz), _mach(bf)]),
             period_L=_mach(L), period_R=_mach(R), fix=_mach(g2))
    e = dict(period_F=np.concatenate([front, g2F]) + gdofu, period_B=np.concatenate([back, g2b]) + gdofu,
             period_L=np.concatenate([L, g2Le]) + gdofu, period_R=np.concatenate([R, g2Re]) + gdofu,
             zheng=zheng + gdofu, fu=fu + gdofu)
    return m, e


def _fold(slaves, masters, gdof):
    is_slave = np.zeros(gdof, bool)
    is_slave[slaves] = True
    free = np.where(~is_slave)[0]
    return sp.coo_matrix((np.ones(free.size + slaves.size), (np.concatenate([free, slaves]),
                                                              np.concatenate([free, masters]))),
                         shape=(gdof, gdof)).tocsr()


class FrequencySolver3D:
    """bc_solve.FrequencySolver3D (bc_solve.py:108-175) with the SuperLU route."""

    def __init__(self, K, M, boundary):
        m, e = boundary
        self.K = K.tocsr()
        self.gdof = K.shape[0]
        t_fb = _fold(np.concatenate([m['period_B'], e['period_B']]), np.concatenate([m['period_F'], e['period_F']]),
                     self.gdof)
        t_lr = _fold(np.concatenate([m['period_R'], e['period_R']]), np.concatenate([m['period_L'], e['period_L']]),
                     self.gdof)
        self.T = (t_fb @ t_lr).tocsr()
        kf = (t_lr.T @ (t_fb.T @ self.K @ t_fb) @ t_lr).tocsr()
        mf = (t_lr.T @ (t_fb.T @ M.tocsr() @ t_fb) @ t_lr).tocsr()
        prescribed = np.unique(np.concatenate([m['fix'], m['period_B'], m['period_R'], e['period_R'],
                                               e['period_B'], e['zheng'], e['fu']]))
        self.active = np.setdiff1d(np.arange(self.gdof), prescribed)
        self.n_active = self.active.size
        self.zheng, self.fu, self.m, self.e = e['zheng'], e['fu'], m, e
        self.k_aa = kf[self.active][:, self.active].tocsr()
        self.m_aa = mf[self.active][:, self.active].tocsr()
        self.k_az = kf[self.active][:, self.zheng]
        self.m_az = mf[self.active][:, self.zheng]
        self.kz_rows = self.K[self.zheng, :].tocsr()

    def system(self, omega, V=1.0):
        a_aa = (self.k_aa - omega ** 2 * self.m_aa).tocsr()
        rhs = -V * np.asarray((self.k_az - omega ** 2 * self.m_az).sum(axis=1)).ravel()
        return a_aa, rhs

    def solve(self, omega, V=1.0):
        A, rhs = self.system(omega, V)
        u = spla.splu(A.tocsc()).solve(rhs)
        disp = np.zeros(self.gdof, complex)
        disp[self.active] = u
        m, e = self.m, self.e
        disp[m['period_R']] = disp[m['period_L']]
        disp[m['period_B']] = disp[m['period_F']]
        disp[e['period_R']] = disp[e['period_L']]
        disp[e['period_B']] = disp[e['period_F']]
        disp[self.zheng] = V
        disp[self.fu] = 0.0
        Q = (self.kz_rows @ disp).sum()
        return disp, Q, abs(1j * omega * Q / V)

    def sweep(self, freqs, V=1.0):
        return np.array([self.solve(2 * np.pi * f, V)[1] for f in np.asarray(freqs, float)])


class FrequencySolver3DFP(FrequencySolver3D):
    """bc_solve.FrequencySolver3D_FP (bc_solve.py:214-335): the finite-device variant.
    Front/back fold, then the equipotential fold of the floating electrodes XFL / XFR
    (each node's phi onto the set's first node); no left/right periodicity.
    ``boundary`` = (machine, electric) dicts with electric['XFL'], ['XFR']."""

    def __init__(self, K, M, boundary):
        m, e = boundary
        self.K = K.tocsr()
        self.gdof = K.shape[0]
        t_fb = _fold(np.concatenate([m['period_B'], e['period_B']]), np.concatenate([m['period_F'], e['period_F']]),
                     self.gdof)
        t_fl = float_fold(e, self.gdof)
        kf = (t_fl.T @ (t_fb.T @ self.K @ t_fb) @ t_fl).tocsr()
        mf = (t_fl.T @ (t_fb.T @ M.tocsr() @ t_fb) @ t_fl).tocsr()
        xfl, xfr = e['XFL'], e['XFR']
        prescribed = np.unique(np.concatenate([m['fix'], m['period_B'], e['period_B'], xfl[1:], xfr[1:],
                                               e['zheng'], e['fu']]))
        self.active = np.setdiff1d(np.arange(self.gdof), prescribed)
        self.n_active = self.active.size
        self.zheng, self.fu, self.m, self.e = e['zheng'], e['fu'], m, e
        self.k_aa = kf[self.active][:, self.active].tocsr()
        self.m_aa = mf[self.active][:, self.active].tocsr()
        self.k_az = kf[self.active][:, self.zheng]
        self.m_az = mf[self.active][:, self.zheng]
        self.kz_rows = self.K[self.zheng, :].tocsr()

    def solve(self, omega, V=1.0):
        A, rhs = self.system(omega, V)
        u = spla.splu(A.tocsc()).solve(rhs)
        disp = np.zeros(self.gdof, complex)
        disp[self.active] = u
        m, e = self.m, self.e
        disp[m['period_B']] = disp[m['period_F']]            # bc_solve.py:242-253
        disp[e['period_B']] = disp[e['period_F']]
        for xs in (e['XFL'], e['XFR']):
            if xs.size > 1:
                disp[xs[1:]] = disp[xs[0]]
        disp[self.zheng] = V
        disp[self.fu] = 0.0
        Q = (self.kz_rows @ disp).sum()
        return disp, Q, abs(1j * omega * Q / V)


def float_fold(e, gdof):
    """The equipotential fold operator of bc_solve.py:219-231 (XFL / XFR slaves onto
    their first node)."""
    s, mst = [], []
    for xs in (e['XFL'], e['XFR']):
        if xs.size > 1:
            s.append(xs[1:])
            mst.append(np.full(xs.size - 1, xs[0]))
    slaves = np.concatenate(s) if s else np.zeros(0, np.int64)
    masters = np.concatenate(mst) if mst else np.zeros(0, np.int64)
    return _fold(slaves, masters, gdof)
