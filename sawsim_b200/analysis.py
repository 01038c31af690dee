"""Host-only analysis of a cell (``ss_analyze_host``): the condensation, the
nested-dissection ordering and the front tree that a GPU engine would use, with
no CUDA device.  ``analyze_q9`` / ``analyze_hex27`` take the inputs of the
engine constructors (mesh and boundary sets; no materials) and return the
sizes, the work and memory per frequency point, and the front tree."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .engine import _bc_arrays


@dataclass
class Analysis:
    n_active: int
    flops_per_point: float          # factorisation flops of one frequency point
    nnz_lu: float
    max_front: int
    max_pivots: int
    front_bytes_per_point: dict     # complex128 / complex64 fronts of one point
    condensed_nnz: int
    levels: int
    active: np.ndarray              # global DOF of each active DOF, ascending
    order: np.ndarray               # elimination position of each active DOF
    k: np.ndarray                   # pivots per front (fronts in postorder)
    m: np.ndarray                   # rows per front
    parent: np.ndarray              # parent front, -1 at a root
    level: np.ndarray               # tree level (leaves 0)
    rows_ptr: np.ndarray
    rows: np.ndarray                # front rows in elimination positions (pivots first)


def _bc_args(bc, two_stage):
    fix, zheng, fu, gptr, gd = _bc_arrays(bc)
    return [fix.size, L.ptr(fix, C.c_int64), zheng.size, L.ptr(zheng, C.c_int64), fu.size, L.ptr(fu, C.c_int64),
            gptr.size - 1, L.ptr(gptr, C.c_int64), L.ptr(gd, C.c_int64), int(two_stage)], (fix, zheng, fu, gptr, gd)


def _run(kind, pos, conn, gdof, bc, two_stage):
    pos, conn = L.f64(pos), L.i64(conn)
    bca, keep = _bc_args(bc, two_stage)
    args = [kind, pos.shape[0], L.ptr(pos, C.c_double), conn.shape[0], L.ptr(conn, C.c_int64), int(gdof)] + bca
    return _call(L.load().ss_analyze_host, args)


def _call(fn, args):
    sizes = np.zeros(4, dtype=np.int64)
    stats = np.zeros(6)
    rc = fn(*args, L.ptr(sizes, C.c_int64), L.ptr(stats, C.c_double), *([None] * 8))
    if rc != L.SS_OK:
        raise L.SawsimError(rc, 'host analysis failed')
    n, nf, nr, _ = (int(x) for x in sizes)
    active, order = np.zeros(n, np.int64), np.zeros(n, np.int64)
    k, m, parent, level = (np.zeros(nf, np.int32) for _ in range(4))
    rows_ptr, rows = np.zeros(nf + 1, np.int64), np.zeros(nr, np.int64)
    rc = fn(*args, L.ptr(sizes, C.c_int64), L.ptr(stats, C.c_double), L.ptr(active, C.c_int64),
            L.ptr(order, C.c_int64), L.ptr(k, C.c_int32), L.ptr(m, C.c_int32), L.ptr(parent, C.c_int32),
            L.ptr(level, C.c_int32), L.ptr(rows_ptr, C.c_int64), L.ptr(rows, C.c_int64))
    if rc != L.SS_OK:
        raise L.SawsimError(rc, 'host analysis failed')
    return Analysis(n_active=n, flops_per_point=float(stats[0]), nnz_lu=float(stats[1]), max_front=int(stats[2]),
                    max_pivots=int(stats[3]),
                    front_bytes_per_point=dict(complex128=16 * stats[4], complex64=8 * stats[4]),
                    condensed_nnz=int(stats[5]), levels=int(sizes[3]), active=active, order=order, k=k, m=m,
                    parent=parent, level=level, rows_ptr=rows_ptr, rows=rows)


def analyze_q9(pos_m, quads, bc, mode_extension=1) -> Analysis:
    """Analysis of a Q9 cell: ``pos_m`` (N, 2) node coordinates, ``quads`` (ne, 9)
    0-based connectivity, ``bc`` the ``(fix, zheng, fu, merge_groups)`` tuple of
    ``sweep.bc_periodic`` (as ``FrequencySolver.from_q9`` takes them)."""
    pos = np.asarray(pos_m)[:, :2]
    nc = 4 if mode_extension else 3
    kind = L.SS_Q9_ME1 if mode_extension else L.SS_Q9_ME0
    return _run(kind, pos, quads, nc * pos.shape[0], bc, 0)


def analyze_hex27(pos_m, hexas, bc) -> Analysis:
    """Analysis of a Hex27 slab with ``bc = (fix, zheng, fu, groups, two_stage)``
    (as ``FrequencySolver.from_hex27`` takes them)."""
    fix, zheng, fu, groups, two_stage = bc
    pos = np.asarray(pos_m)
    return _run(L.SS_HEX27, pos, hexas, 4 * pos.shape[0], (fix, zheng, fu, groups), two_stage)


def analyze_csr(pattern, bc, two_stage=0, dof_node=None, node_xyz=None) -> Analysis:
    """Analysis from an assembled pattern (``ss_analyze_host_csr``): ``pattern`` a
    scipy sparse matrix whose structure is the union of K's and M's (for example
    ``abs(K) + abs(M)``, which no cancellation can thin out), ``bc`` the
    ``(fix, zheng, fu, groups)`` of the reference engine's constructor
    (``FrequencySolver.from_matrices`` takes the same); ``dof_node`` and
    ``node_xyz`` (nodes x 2 or 3) give the geometric ordering of the mesh path,
    else the graph nested dissection."""
    A = pattern.tocsr(copy=True)
    A.sort_indices()
    A.sum_duplicates()
    indptr, indices = L.i64(A.indptr), L.i64(A.indices)
    gdof = A.shape[0]
    if node_xyz is not None:
        xyz = L.f64(node_xyz)
        n_nodes, dim = xyz.shape
        xp = L.ptr(xyz, C.c_double)
    else:
        n_nodes, dim, xp = (int(np.max(dof_node)) + 1 if dof_node is not None else 0), 0, None
    dn = L.i64(dof_node) if dof_node is not None else None
    bca, keep = _bc_args(bc, two_stage)
    args = [gdof, L.ptr(indptr, C.c_int64), L.ptr(indices, C.c_int64), n_nodes, dim,
            None if dn is None else L.ptr(dn, C.c_int64), xp] + bca
    return _call(L.load().ss_analyze_host_csr, args)


def level_work(a: Analysis, itemsize: int = 16) -> list:
    """Work and traffic of one frequency point's factorisation, level by level
    (leaves first): fronts, pivots, the Schur-update flops (8 k (m-k)^2 per front,
    complex multiply-adds x 8) and bytes (the update block read and written once,
    the two panels read once), the rest of the factorisation's flops (the panel
    LU, L21 and U12: 8 (k^3/3 + k^2 (m-k) + k (m-k)^2) minus the Schur part), the
    bytes the front assembly moves at the least (each front written once, m x m,
    each child's update block read once) and the factors' bytes (L+U entries, read
    once by each triangular solve)."""
    k = a.k.astype(float)
    u = (a.m - a.k).astype(float)
    schur = 8.0 * k * u * u
    total = 8.0 * (k ** 3 / 3 + k * k * u + k * u * u)
    front_bytes = itemsize * a.m.astype(float) ** 2
    cb_bytes = itemsize * u * u                     # read by the parent's assembly
    lu_bytes = itemsize * (k * k + 2 * k * u)
    schur_bytes = itemsize * (2 * u * u + 2 * k * u)   # F22 read and written, F21 and F12 read
    out = []
    for lev in range(a.levels):
        sel = a.level == lev
        kids = np.isin(a.parent, np.flatnonzero(sel))
        out.append(dict(level=lev, fronts=int(sel.sum()), pivots=int(a.k[sel].sum()),
                        max_front=int(a.m[sel].max()), schur_flops=float(schur[sel].sum()),
                        schur_bytes=float(schur_bytes[sel].sum()),
                        other_flops=float((total - schur)[sel].sum()),
                        assembly_bytes=float(front_bytes[sel].sum() + cb_bytes[kids].sum()),
                        lu_bytes=float(lu_bytes[sel].sum())))
    return out


def _main(argv=None):
    """Per-level work of a cell's factorisation as a markdown table:
    ``python -m sawsim_b200.analysis --case me1_64x256 --points 37``."""
    import argparse
    from . import cases
    p = argparse.ArgumentParser(description=_main.__doc__)
    p.add_argument('--case', default='me1_64x256')
    p.add_argument('--points', type=int, default=1, help='points per factorisation (the chunk)')
    p.add_argument('--itemsize', type=int, default=16, help='16 complex128, 8 complex64')
    args = p.parse_args(argv)
    if args.case.startswith('hex'):
        c = cases.make_hex_case(args.case)
        a = analyze_hex27(c.pos_m, c.hexas, c.bc)
    else:
        c = cases.make_case(args.case)
        a = analyze_q9(c.mesh.pos_m, c.mesh.quads, c.bc, c.mode_extension)
    n = args.points
    print(f'{args.case}: {a.n_active} active DOFs, {a.k.size} fronts, {a.levels} levels; '
          f'{a.flops_per_point / 1e9:.1f} GFLOP and {a.nnz_lu / 1e6:.2f} M L+U entries per point; x {n} points')
    print()
    print('| level | fronts | pivots | widest front | Schur GFLOP | Schur GB | other GFLOP | assembly GB | L+U GB |')
    print('|---:|---:|---:|---:|---:|---:|---:|---:|---:|')
    for r in level_work(a, args.itemsize):
        print(f"| {r['level']} | {r['fronts']} | {r['pivots']} | {r['max_front']} | {n * r['schur_flops'] / 1e9:.1f} | "
              f"{n * r['schur_bytes'] / 1e9:.2f} | {n * r['other_flops'] / 1e9:.1f} | "
              f"{n * r['assembly_bytes'] / 1e9:.2f} | {n * r['lu_bytes'] / 1e9:.2f} |")


if __name__ == '__main__':
    _main()
