"""Oracle: Bloch boundary sets, master-slave fold and the per-frequency solve.

Restates ``src/sawsim/saw2d/sweep.py`` of the reference (test infrastructure):

* ``bc_periodic`` :41-72 — L/R pairs sorted by y, bottom corners dropped from the
  displacement pairs, bottom u fixed, + / - electrode phi DOFs;
* ``merge_transform`` :97-144 — union-find master/slave, 0/1 ``T``;
* ``FrequencySolver`` :275-364 — ``Km = T^T K T``, active set, ``Km_s``, ``Mm_s``,
  ``kts = K^T s``, condensed ``Km_aa``/``Mm_aa``; per frequency the complex solve
  and ``Q = kts . disp``; ``set_damping`` :316-323.

The reference solves each point either with MKL PARDISO or, when pypardiso is
absent, with ``scipy.sparse.linalg.spsolve`` (SuperLU) on the real-block form
``[[Ar, -Ai], [Ai, Ar]]`` (:346-353).  ``route='realblock'`` reproduces that
fallback exactly; ``route='complex'`` factors the complex matrix with SuperLU,
which gives the same solution about 3x faster.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def bc_periodic(model, lines, tag_bottom=21, tag_left=19, tag_right=20,
                tag_zheng=17, tag_fu=18, ndisp=3):
    """(fix, zheng, fu, merge_groups) for the SP cell (sweep.py:41-72)."""
    N = model.N
    bottom = model.nodes_with_tag(tag_bottom, lines)
    left = model.nodes_with_tag(tag_left, lines)
    right = model.nodes_with_tag(tag_right, lines)
    zheng = model.nodes_with_tag(tag_zheng, lines)
    fu = model.nodes_with_tag(tag_fu, lines)
    cL = np.intersect1d(bottom, left)
    cR = np.intersect1d(bottom, right)
    L = np.setdiff1d(left, cL)
    R = np.setdiff1d(right, cR)
    L = L[np.argsort(model.pos_m[L, 1])]
    R = R[np.argsort(model.pos_m[R, 1])]
    if L.size != R.size:
        raise RuntimeError('left/right periodic node counts differ')
    masters = np.concatenate([L + a * N for a in range(ndisp)] + [L + ndisp * N, cL + ndisp * N])
    slaves = np.concatenate([R + a * N for a in range(ndisp)] + [R + ndisp * N, cR + ndisp * N])
    groups = [np.array([m, s]) for m, s in zip(masters, slaves)]
    fix = np.concatenate([bottom + a * N for a in range(ndisp)])
    return fix, zheng + ndisp * N, fu + ndisp * N, groups


def merge_transform(gdof, groups):
    """0/1 fold ``T`` with ``A_merged = T^T A T`` by union-find (sweep.py:97-144).

    The first DOF of each group is its master; the root of an equivalence class is
    the master listed first.
    """
    parent = {}
    pairs = []
    for g in groups:
        g = [int(x) for x in np.asarray(g).ravel()]
        if not g:
            continue
        for x in g:
            parent.setdefault(x, x)
        pairs.extend((s, g[0]) for s in g[1:])

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for s, m in pairs:
        rs, rm = find(s), find(m)
        if rs != rm:
            parent[rs] = rm
    slaves, masters = [], []
    is_slave = np.zeros(gdof, dtype=bool)
    for x in parent:
        r = find(x)
        if r != x:
            slaves.append(x)
            masters.append(r)
            is_slave[x] = True
    slaves = np.array(slaves, dtype=int)
    masters = np.array(masters, dtype=int)
    keep = np.flatnonzero(~is_slave)
    T = sp.coo_matrix((np.ones(keep.size + slaves.size),
                       (np.concatenate([keep, slaves]), np.concatenate([keep, masters]))),
                      shape=(gdof, gdof)).tocsr()
    return T, slaves, masters


class FrequencySolver:
    """Oracle engine with the reference's constructor and ``solve`` (sweep.py:283-364)."""

    def __init__(self, K, M, fix, zheng, fu, groups):
        self.K = K.tocsr()
        gdof = K.shape[0]
        self.gdof = gdof
        self.zheng = np.asarray(zheng, dtype=int)
        self.fu = np.asarray(fu, dtype=int)
        T, self.slaves, self.masters = merge_transform(gdof, groups)
        Km = (T.T @ self.K @ T).tocsr()
        Mm = (T.T @ M.tocsr() @ T).tocsr()
        prescribed = np.unique(np.concatenate([np.asarray(fix, dtype=int), self.slaves,
                                               self.zheng, self.fu]))
        self.active = np.setdiff1d(np.arange(gdof), prescribed)
        self.n_active = self.active.size
        s = np.zeros(gdof)
        s[self.zheng] = 1.0
        self.Km_s = np.asarray(Km @ s).ravel()
        self.Mm_s = np.asarray(Mm @ s).ravel()
        self.kts = np.asarray(self.K.T @ s).ravel()
        self.Km_aa = Km[self.active][:, self.active].tocsr()
        self.Mm_aa = Mm[self.active][:, self.active].tocsr()
        self._T = T
        self.beta = 0.0

    def set_damping(self, D, beta):
        """Rayleigh stiffness damping A = K + i w beta D - w^2 M (sweep.py:316-323)."""
        Dm = (self._T.T @ D.tocsr() @ self._T).tocsr()
        s = np.zeros(self.gdof)
        s[self.zheng] = 1.0
        self.Dm_s = np.asarray(Dm @ s).ravel()
        self.Dm_aa = Dm[self.active][:, self.active].tocsr()
        self.beta = float(beta)

    def system(self, omega, V=1.0):
        """(A_aa, rhs) at angular frequency ``omega`` (sweep.py:337-347)."""
        w2 = omega ** 2
        Ks, Ka = self.Km_s, self.Km_aa
        if self.beta:
            Ks = Ks + 1j * omega * self.beta * self.Dm_s
            Ka = Ka + 1j * omega * self.beta * self.Dm_aa
        rhs = -(Ks - w2 * self.Mm_s)[self.active] * V
        return (Ka - w2 * self.Mm_aa).tocsr(), rhs

    def charge(self, x, V=1.0):
        """Full DOF vector and Q = kts . disp from the active solution (sweep.py:356-363)."""
        disp = np.zeros(self.gdof, dtype=complex)
        disp[self.active] = x
        disp[self.slaves] = disp[self.masters]
        disp[self.zheng] = V
        disp[self.fu] = 0.0
        return disp, self.kts @ disp

    def solve(self, omega, V=1.0, route='complex'):
        A, rhs = self.system(omega, V)
        n = self.n_active
        if route == 'realblock':
            A2 = sp.bmat([[A.real, -A.imag], [A.imag, A.real]], format='csr')
            A2.sort_indices()
            z = spla.spsolve(A2.tocsc(), np.concatenate([rhs.real, rhs.imag]))
            x = z[:n] + 1j * z[n:]
        else:
            x = spla.splu(A.tocsc()).solve(rhs)
        disp, Q = self.charge(x, V)
        return disp, Q, abs(1j * omega * Q / V)

    def sweep(self, freqs, V=1.0, route='complex'):
        Q = np.array([self.solve(2 * np.pi * f, V, route)[1] for f in np.asarray(freqs, float)])
        return Q


def admittance_2d(freqs, Q, V=1.0):
    """Passive-sign 2D admittance Y = -i w Q / V (solver.py:128)."""
    return -1j * 2 * np.pi * np.asarray(freqs) * np.asarray(Q) / V
