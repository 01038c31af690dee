"""Python host layer of the B200 sweep backend.

``FrequencySolver`` mirrors the engine the reference's pipeline builds and
drives (``src/sawsim/saw2d/sweep.py:275-393``): ``solve(omega, V)`` returns
``(disp, Q, |Y|)``, ``sweep(freqs, V)`` the charges, ``n_active`` the size of the
condensed system.  Construction goes either from the inputs of the reference's
assembly (``piezo_fem.assemble``, ``piezo_fem.py:283``) and boundary builder
(``sweep.bc_periodic``, ``sweep.py:41``), so that assembly, condensation and
every frequency's factorisation run on the GPU (``from_q9``, ``from_hex27``), or
from the reference engine's own constructor arguments, the assembled K and M and
the boundary sets (``from_matrices``, ``from_matrices_3d``).  All numerical work
is done by ``libsawsim_b200.so``; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from . import _lib as L
from .materials import pack

PRECISION = {'fp64': L.SS_PREC_FP64, 'mixed': L.SS_PREC_MIXED, 'auto': L.SS_PREC_AUTO}


class Handle:
    """Owns one ``ss_handle``; raises ``SawsimError`` on any non-zero status."""

    def __init__(self, device: int = 0):
        self.lib = L.load()
        self.h = C.c_void_p()
        rc = self.lib.ss_create(C.byref(self.h), int(device))
        if rc != L.SS_OK:
            raise L.SawsimError(rc, 'ss_create failed (no CUDA device?)')

    def __call__(self, name, *args):
        rc = getattr(self.lib, name)(self.h, *args)
        if rc != L.SS_OK:
            raise L.SawsimError(rc, self.lib.ss_last_error(self.h).decode())
        return rc

    def close(self):
        if self.h:
            self.lib.ss_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _pml_arrays(elem_tag, pml_regions, ne):
    """Region arrays for ss_set_pml from reference-style PML regions: Q9
    ``PMLRegion`` (piezo_fem.py:192-242, axes x/y) or the Hex27 bottom region
    (saw3d/assembly.py:127-143, axis z with za the interface, zp the outer face)."""
    regions = list(pml_regions or [])
    region = np.full(ne, -1, dtype=np.int32)
    axis, dmax, npow, inner, outer = [], [], [], [], []
    for r, reg in enumerate(regions):
        region[np.asarray(elem_tag) == reg.tag] = r
        mask = (1 if 'x' in reg.kind else 0) | (2 if 'y' in reg.kind else 0) | (4 if 'z' in reg.kind else 0)
        axis.append(mask)
        dmax.append(reg.dmax)
        npow.append(reg.n)
        inner.append([reg.xa, reg.ya, getattr(reg, 'za', 0.0)])
        outer.append([reg.xp, reg.yp, getattr(reg, 'zp', 0.0)])
    return (len(regions), L.i32(axis), L.f64(dmax), L.i32(npow), L.f64(np.reshape(inner, (-1, 3))),
            L.f64(np.reshape(outer, (-1, 3))), region)


def _bc_arrays(bc):
    fix, zheng, fu, groups = bc
    groups = [np.asarray(g, dtype=np.int64).ravel() for g in groups]
    gptr = np.zeros(len(groups) + 1, dtype=np.int64)
    gptr[1:] = np.cumsum([g.size for g in groups])
    gd = np.concatenate(groups) if groups else np.zeros(0, dtype=np.int64)
    return L.i64(fix), L.i64(zheng), L.i64(fu), L.i64(gptr), L.i64(gd)


def _canonical(A, n):
    """Complex CSR with sorted columns and duplicates summed (explicit zeros kept,
    as the reference's COO -> CSR assembly keeps them)."""
    A = sp.csr_matrix(A, dtype=np.complex128, copy=True)
    if A.shape != (n, n):
        raise ValueError(f'matrix shape {A.shape} != ({n}, {n})')
    A.sum_duplicates()
    return A


def _keys(A):
    rows = np.repeat(np.arange(A.shape[0], dtype=np.int64), np.diff(A.indptr))
    return rows * A.shape[1] + A.indices.astype(np.int64)


def _union_pattern(mats):
    """CSR pattern (indptr, indices) holding every stored entry of ``mats``."""
    n = mats[0].shape[0]
    keys = np.unique(np.concatenate([_keys(A) for A in mats]))
    rows = keys // n
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=indptr[1:])
    return indptr, (keys % n).astype(np.int64), keys


def _on_pattern(A, keys):
    """Values of canonical ``A`` scattered onto the pattern with sorted ``keys``."""
    k = _keys(A)
    pos = np.searchsorted(keys, k)
    if k.size and (pos.max() >= keys.size or not np.array_equal(keys[np.minimum(pos, keys.size - 1)], k)):
        raise ValueError('matrix has entries outside the engine\'s pattern')
    v = np.zeros(keys.size, dtype=np.complex128)
    v[pos] = A.data
    return v


def _fold_pairs(T):
    """(slave, master) pairs of a fold operator (bc_solve.py:25-33: row ``slave``
    holds a single 1 in column ``master``; other rows are identity rows)."""
    T = sp.csr_matrix(T)
    rows = np.repeat(np.arange(T.shape[0], dtype=np.int64), np.diff(T.indptr))
    cols = T.indices.astype(np.int64)
    off = rows != cols
    return rows[off], cols[off]


class FrequencySolver:
    """Sweep engine on one B200 with the reference engine's ``solve``/``sweep`` surface."""

    def __init__(self, handle: Handle, gdof: int, ndisp: int, kind: int, zheng, fu):
        self._h = handle
        self.gdof = int(gdof)
        self.ndisp = ndisp
        self.kind = kind
        self.zheng = np.asarray(zheng, dtype=np.int64)
        self.fu = np.asarray(fu, dtype=np.int64)

    @classmethod
    def from_q9(cls, model, materials, mat_idx, pml_regions, omega_top, bc, mode_extension=1,
                damping_materials=None, beta=0.0, device=0):
        """Assemble on the GPU from the inputs of ``piezo_fem.assemble`` (ME1) or
        ``piezo_fem.assemble_ME0`` (``mode_extension=0``, projected xy tensors) and
        the ``(fix, zheng, fu, merge_groups)`` tuple of ``sweep.bc_periodic``."""
        h = Handle(device)
        ndisp = 3 if mode_extension else 2
        kind = L.SS_Q9_ME1 if mode_extension else L.SS_Q9_ME0
        pos = L.f64(model.pos_m[:, :2])
        quads = L.i64(model.quads)
        emat = L.i32(mat_idx)
        h('ss_set_mesh', kind, pos.shape[0], L.ptr(pos, C.c_double), quads.shape[0], L.ptr(quads, C.c_int64),
          L.ptr(emat, C.c_int32))
        rho, Cm, em, epsm = pack(materials, ndisp)
        h('ss_set_materials', L.SS_MAT_K, len(rho), L.ptr(rho, C.c_double), L.ptr(Cm, C.c_double),
          L.ptr(em, C.c_double), L.ptr(epsm, C.c_double))
        if damping_materials is not None:
            rho, Cm, em, epsm = pack(damping_materials, ndisp)
            h('ss_set_materials', L.SS_MAT_D, len(rho), L.ptr(rho, C.c_double), L.ptr(Cm, C.c_double),
              L.ptr(em, C.c_double), L.ptr(epsm, C.c_double))
        nreg, axis, dmax, npow, inner, outer, region = _pml_arrays(model.elem_tag, pml_regions, quads.shape[0])
        h('ss_set_pml', nreg, L.ptr(axis, C.c_int32), L.ptr(dmax, C.c_double), L.ptr(npow, C.c_int32),
          L.ptr(inner, C.c_double), L.ptr(outer, C.c_double), 1, L.ptr(region, C.c_int32), float(omega_top))
        h('ss_assemble')
        eng = cls(h, (ndisp + 1) * pos.shape[0], ndisp, kind, bc[1], bc[2])
        eng._pml = (nreg, axis, dmax, npow, inner, outer, 1, region)
        eng.omega_top = float(omega_top)
        eng._set_bc(bc, two_stage=0)
        if damping_materials is not None and beta:
            h('ss_set_damping', float(beta))
        return eng

    @classmethod
    def from_hex27(cls, pos_m, hexas, elem_tag, materials, mat_idx, pml_regions, omega_top, bc, device=0):
        """Assemble a Hex27 slab on the GPU from the inputs of
        ``form_stiffness_mass_3d`` (saw3d/assembly.py:230: 0-based H27 connectivity,
        coordinates in metres, full 3D tensors; the PML elements carry the PML
        material; PML regions select elements by ``elem_tag``, no clamp) and
        ``bc = (fix, zheng, fu, groups, two_stage)`` from ``cases.bc_periodic_3d``
        (the two-stage fold of saw3d/bc_solve.py:36-44)."""
        h = Handle(device)
        pos = L.f64(pos_m)
        conn = L.i64(hexas)
        emat = L.i32(mat_idx)
        h('ss_set_mesh', L.SS_HEX27, pos.shape[0], L.ptr(pos, C.c_double), conn.shape[0], L.ptr(conn, C.c_int64),
          L.ptr(emat, C.c_int32))
        rho, Cm, em, epsm = pack(materials, 3)
        h('ss_set_materials', L.SS_MAT_K, len(rho), L.ptr(rho, C.c_double), L.ptr(Cm, C.c_double),
          L.ptr(em, C.c_double), L.ptr(epsm, C.c_double))
        nreg, axis, dmax, npow, inner, outer, region = _pml_arrays(elem_tag, pml_regions, conn.shape[0])
        h('ss_set_pml', nreg, L.ptr(axis, C.c_int32), L.ptr(dmax, C.c_double), L.ptr(npow, C.c_int32),
          L.ptr(inner, C.c_double), L.ptr(outer, C.c_double), 0, L.ptr(region, C.c_int32), float(omega_top))
        h('ss_assemble')
        fix, zheng, fu, groups, two_stage = bc
        eng = cls(h, 4 * pos.shape[0], 3, L.SS_HEX27, zheng, fu)
        eng._pml = (nreg, axis, dmax, npow, inner, outer, 0, region)
        eng.omega_top = float(omega_top)
        eng._set_bc((fix, zheng, fu, groups), two_stage=two_stage)
        return eng

    @classmethod
    def from_matrices(cls, K, M, fix, zheng, fu, merge_groups, dof_node=None, node_xyz=None, device=0):
        """The reference engine's constructor, ``sweep.FrequencySolver(K, M, fix,
        zheng, fu, merge_groups)`` (sweep.py:283-314): assembled global K and M
        (any mesh, e.g. the Gmsh-meshed templates), the fixed DOFs, the electrode
        DOFs and the periodic merge groups.  Fold, condensation, analysis and every
        frequency's factorisation run on the GPU.  Optional ``dof_node`` (node of
        each DOF) and ``node_xyz`` (node coordinates, n_nodes x 2 or 3) give the
        geometric nested dissection of the mesh path; without them the ordering
        is a graph nested dissection of the matrix (more fill)."""
        return cls._from_csr(K, M, (fix, zheng, fu, merge_groups), 0, dof_node, node_xyz, device)

    @classmethod
    def from_matrices_3d(cls, K, M, boundary, t_fb, t_lr, dof_node=None, node_xyz=None, device=0):
        """``FrequencySolver3D(K, M, boundary, t_fb, t_lr)`` (bc_solve.py:108-136):
        the unfolded K and M, the boundary DOF container (an object with the
        ``machine`` / ``electric`` dicts of boundary.py:84-148, or the pair of
        dicts) and the two fold operators of ``build_periodic_operators``
        (front/back first, then left/right)."""
        s_fb, m_fb = _fold_pairs(t_fb)
        s_lr, m_lr = _fold_pairs(t_lr)
        groups = [[m, s] for s, m in zip(s_fb, m_fb)] + [[m, s] for s, m in zip(s_lr, m_lr)]
        mach, elec = (boundary.machine, boundary.electric) if hasattr(boundary, 'machine') else boundary
        bc = (np.asarray(mach['fix'], dtype=np.int64), elec['zheng'], elec['fu'], groups)
        return cls._from_csr(K, M, bc, len(s_fb), dof_node, node_xyz, device)

    @classmethod
    def _from_csr(cls, K, M, bc, two_stage, dof_node, node_xyz, device):
        n = K.shape[0]
        Kc, Mc = _canonical(K, n), _canonical(M, n)
        indptr, indices, keys = _union_pattern([Kc, Mc])
        h = Handle(device)
        dn = None if dof_node is None else L.i64(dof_node)
        xyz = None if node_xyz is None else L.f64(node_xyz)
        if dn is not None and dn.size != n:
            raise ValueError('dof_node needs one node id per DOF')
        n_nodes = 0 if dn is None else int(dn.max()) + 1 if xyz is None else xyz.shape[0]
        dim = 0 if xyz is None else xyz.shape[1]
        h('ss_set_csr', n, L.ptr(indptr, C.c_int64), L.ptr(indices, C.c_int64), n_nodes, dim,
          None if dn is None else L.ptr(dn, C.c_int64), None if xyz is None else L.ptr(xyz, C.c_double))
        for which, A in ((L.SS_MAT_K, Kc), (L.SS_MAT_M, Mc)):
            v = L.cplx(_on_pattern(A, keys))
            h('ss_set_values', which, L.ptr(v, C.c_double))
        eng = cls(h, n, 0, L.SS_MATRIX, bc[1], bc[2])
        eng._keys = keys
        eng._set_bc(bc, two_stage=two_stage)
        return eng

    def update_matrices(self, K=None, M=None):
        """New K and/or M values on the engine's pattern (e.g. reassembled with the
        PML frozen at a new top frequency): the analysis, the factorisation plans and
        their autotuner picks are kept."""
        self._matrix_only('update_matrices')
        for which, A in ((L.SS_MAT_K, K), (L.SS_MAT_M, M)):
            if A is not None:
                v = L.cplx(_on_pattern(_canonical(A, self.gdof), self._keys))
                self._h('ss_set_values', which, L.ptr(v, C.c_double))

    def set_damping(self, D=None, beta: float = 0.0):
        """Rayleigh stiffness damping A = K + i w beta D - w^2 M (sweep.py:316-323).
        Matrix engines take D itself (the damped part of K, on the engine's
        pattern); mesh engines assemble D from their damping materials and take
        ``beta`` only."""
        if D is not None:
            self._matrix_only('set_damping(D)')
            v = L.cplx(_on_pattern(_canonical(D, self.gdof), self._keys))
            self._h('ss_set_values', L.SS_MAT_D, L.ptr(v, C.c_double))
        self._h('ss_set_damping', float(beta))

    def _matrix_only(self, what):
        if self.kind != L.SS_MATRIX:
            raise ValueError(f'{what}: the engine was built from a mesh; it assembles its own matrices')

    def _set_bc(self, bc, two_stage=0):
        fix, zheng, fu, gptr, gd = _bc_arrays(bc)
        self._h('ss_set_bc', self.gdof, fix.size, L.ptr(fix, C.c_int64), zheng.size, L.ptr(zheng, C.c_int64),
                fu.size, L.ptr(fu, C.c_int64), gptr.size - 1, L.ptr(gptr, C.c_int64), L.ptr(gd, C.c_int64),
                int(two_stage))
        self._h('ss_analyze')

    def set_freeze_frequency(self, omega_top: float):
        """Reassemble K and M with the PML stretch frozen at ``omega_top`` (the
        reference assembles at each sweep's top frequency, solver.py:106-107).
        The mesh and the boundary sets are unchanged, so the analysis, the
        factorisation plans and their autotuner picks are kept."""
        if float(omega_top) == self.omega_top:
            return
        nreg, axis, dmax, npow, inner, outer, clip, region = self._pml
        self._h('ss_set_pml', nreg, L.ptr(axis, C.c_int32), L.ptr(dmax, C.c_double), L.ptr(npow, C.c_int32),
                L.ptr(inner, C.c_double), L.ptr(outer, C.c_double), clip, L.ptr(region, C.c_int32),
                float(omega_top))
        self._h('ss_assemble')
        self.omega_top = float(omega_top)

    # ------------------------------------------------------------------ queries
    STAT_KEYS = ['n_active', 'n_fronts', 'max_front', 'factor_flops_per_point', 'nnz_lu', 'analyze_s',
                 'assemble_ms', 'sweep_ms', 'factor_ms', 'solve_ms', 'chunk', 'schur_gemm_ms',
                 'schur_gemm_flops', 'levels', 'perturbed_pivots', 'launches', 'schur_launches',
                 'sweep_device_ms', 'refine_solves', 'precision_used', 'schur_candidate0', 'schur_candidate1',
                 'schur_candidate2', 'panel_gemm_dmma', 'panel_tune_simt_ms', 'panel_tune_dmma_ms', 'small_fronts',
                 'schur_tune_ms', 'auto_probe_ms', 'fp64_resolved', 'krylov_steps_primal', 'krylov_steps_adjoint',
                 'mixed_not_converged', 'fp64_resolve_ms', 'element_kernel_ms', 'scatter_kernel_ms',
                 'schur_candidate3', 'panel_thin_tiles']

    def stats(self) -> dict:
        n = len(self.STAT_KEYS)
        out = np.zeros(n)
        self._h('ss_stats', L.ptr(out, C.c_double), n)
        return dict(zip(self.STAT_KEYS, out.tolist()))

    def gemm_ceiling(self, kernel: int, m: int = 2560, k: int = 512, n_fronts: int = 8, reps: int = 5) -> float:
        """Measured algorithmic TFLOP/s of a Schur-update kernel on dense fronts
        (``ss_measure_gemm_ceiling``; kernel 0 FP64 DMMA, 1 FP64 SIMT, 2 / 3
        complex64 TMA + tcgen05 3xTF32 with 128 / 64-column tiles, 4 complex64
        SIMT FP32, 5 FP64 DMMA with three real products per complex block, 6 the
        same with the C tile staged in shared memory)."""
        out = C.c_double()
        self._h('ss_measure_gemm_ceiling', int(kernel), int(m), int(k), int(n_fronts), int(reps), C.byref(out))
        return out.value

    def set_option(self, name: str, value: float):
        """Solver option by name (``ss_set_option``): krylov_restart, krylov_cycles,
        krylov_tol, pivot_tiny_c128, pivot_tiny_c64, fp64_fallback, auto_probe_steps."""
        self._h('ss_set_option', name.encode(), float(value))

    @property
    def n_active(self) -> int:
        return int(self.stats()['n_active'])

    def export(self, which: int):
        """Device matrix as scipy CSR (global K/M/D, or condensed KC/MC in active order)."""
        n = C.c_int64()
        nnz = C.c_int64()
        self._h('ss_export_csr', which, C.byref(n), C.byref(nnz), None, None, None)
        ip = np.zeros(n.value + 1, dtype=np.int64)
        ix = np.zeros(nnz.value, dtype=np.int64)
        v = np.zeros(2 * nnz.value, dtype=np.float64)
        self._h('ss_export_csr', which, C.byref(n), C.byref(nnz), L.ptr(ip, C.c_int64), L.ptr(ix, C.c_int64),
                L.ptr(v, C.c_double))
        return sp.csr_matrix((v.view(np.complex128), ix, ip), shape=(n.value, n.value))

    # ------------------------------------------------------------------ solves
    def charges(self, omegas, V: float = 1.0, precision: str = 'fp64'):
        """Batched sweep: (Q complex[n_f], status int[n_f], refinement steps int[n_f])."""
        om = L.f64(np.atleast_1d(omegas))
        Q = np.zeros(2 * om.size)
        st = np.zeros(om.size, dtype=np.int32)
        it = np.zeros(om.size, dtype=np.int32)
        self._h('ss_sweep', om.size, L.ptr(om, C.c_double), float(V), PRECISION[precision], L.ptr(Q, C.c_double),
                L.ptr(st, C.c_int), L.ptr(it, C.c_int))
        return Q.view(np.complex128), st, it

    def sweep(self, fre, V: float = 1.0, precision: str = 'fp64'):
        """Charges at frequencies ``fre`` (Hz), all points in batched GPU factorisations.
        Raises ``SawsimError`` when a point fails (a singular or non-finite solve, or
        an unconverged refinement), as the reference's solve raises on a singular
        matrix and its pipeline on a non-finite charge (solver.py:121-122);
        ``charges`` returns the per-point statuses instead."""
        fre = np.asarray(fre, dtype=float)
        Q, st, _ = self.charges(2 * np.pi * fre, V, precision)
        bad = np.flatnonzero(st)
        if bad.size:
            code = int(st[bad[0]])
            raise L.SawsimError(code, f'{bad.size} of {st.size} points failed, the first at '
                                      f'{fre.ravel()[bad[0]] * 1e-9:.9f} GHz')
        return Q

    def solve(self, omega: float, V: float = 1.0):
        """One point: ``(disp, Q, |Y|)`` like ``FrequencySolver.solve`` (sweep.py:335-364)."""
        disp = np.zeros(2 * self.gdof)
        q = np.zeros(2)
        self._h('ss_solve_fields', float(omega), float(V), L.ptr(disp, C.c_double), L.ptr(q, C.c_double))
        Q = complex(q[0], q[1])
        return disp.view(np.complex128), Q, abs(1j * omega * Q / V)

    def solve_adjoint(self, omega: float, precision: str = 'fp64'):
        """lambda (complex, n_active, active-DOF order) with A_aa^T lambda = kq, the
        folded charge row: dQ = -lambda^T dA x for a perturbation dA of the system."""
        n = self.n_active
        lam = np.zeros(2 * n)
        self._h('ss_solve_adjoint', float(omega), PRECISION[precision], L.ptr(lam, C.c_double))
        return lam.view(np.complex128)

    def gradient(self, omegas, seeds, V: float = 1.0, precision: str = 'fp64'):
        """Charges and dQ/dp by the adjoint (``ss_adjoint_gradient``).

        ``seeds``: one dict per parameter with optional keys dpos (n_nodes x 2,
        metres per unit p), dC (n_mat x 6 x 6), de (n_mat x 3 x 6), deps
        (n_mat x 3 x 3) complex, drho (n_mat,), dinner / douter (n_regions x 3).
        Returns ``(Q[n_f], dQ[n_f, n_params], status[n_f])``."""
        om = L.f64(np.atleast_1d(omegas))
        npar = len(seeds)

        def stack(key, shape, cplx):
            if all(sd.get(key) is None for sd in seeds):
                return None
            out = []
            for sd in seeds:
                a = sd.get(key)
                a = np.zeros(shape, complex if cplx else float) if a is None else np.asarray(a)
                if cplx:
                    a = np.stack([np.real(a), np.imag(a)], axis=-1)
                out.append(np.asarray(a, dtype=np.float64).reshape(-1))
            return np.ascontiguousarray(np.concatenate(out))

        n_nodes = self.gdof // (self.ndisp + 1)
        first = next((sd for sd in seeds if sd.get('dC') is not None or sd.get('drho') is not None), None)
        n_mat = 0 if first is None else len(first['dC'] if first.get('dC') is not None else first['drho'])
        nreg_src = next((sd for sd in seeds if sd.get('dinner') is not None or sd.get('douter') is not None), None)
        nreg = 0 if nreg_src is None else np.asarray(
            nreg_src['dinner'] if nreg_src.get('dinner') is not None else nreg_src['douter']).shape[0]
        arrs = [stack('dpos', (n_nodes, 2), False), stack('dC', (n_mat, 6, 6), True), stack('de', (n_mat, 3, 6), True),
                stack('deps', (n_mat, 3, 3), True), stack('drho', (n_mat,), False),
                stack('dinner', (nreg, 3), False), stack('douter', (nreg, 3), False)]
        ptrs = [None if a is None else L.ptr(a, C.c_double) for a in arrs]
        Q = np.zeros(2 * om.size)
        dQ = np.zeros(2 * om.size * npar)
        st = np.zeros(om.size, dtype=np.int32)
        self._h('ss_adjoint_gradient', om.size, L.ptr(om, C.c_double), float(V), PRECISION[precision], npar, *ptrs,
                L.ptr(Q, C.c_double), L.ptr(dQ, C.c_double), L.ptr(st, C.c_int))
        return Q.view(np.complex128), dQ.view(np.complex128).reshape(om.size, npar), st

    def close(self):
        self._h.close()
