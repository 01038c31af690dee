/*
 * sawsim_b200 — B200 frequency-sweep backend for SawSim's piezoelectric FEM.
 *
 * C ABI: opaque handle, plain pointers and sizes, int status returns, no
 * exceptions across the boundary.  Complex arrays are interleaved (re, im)
 * float64.  The caller keeps ownership of host memory; the handle owns all
 * device memory.  A handle is single-threaded and uses one CUDA stream; do not
 * fork a process after ss_create.
 *
 * The reference (Duane245/sawsim 2.1.0) has no C interface: its de-facto plugin
 * boundary is the frequency-solver engine object built by
 *   src/sawsim/solver.py:108   sweep.FrequencySolver(K, M, *bc)
 *   src/sawsim/hex_solver.py:92 FrequencySolver3D(K, M, boundary, t_fb, t_lr)
 * and driven per frequency by src/sawsim/frequency_tasks.py:33-55.  Each entry
 * point below names the reference function whose work it replaces.
 */
#ifndef SAWSIM_B200_H
#define SAWSIM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ss_handle ss_handle;

/* status codes */
#define SS_OK          0
#define SS_EINVAL     -1   /* bad argument or size                              */
#define SS_ECUDA      -2   /* CUDA runtime / driver error                       */
#define SS_ESINGULAR  -3   /* zero pivot after static perturbation              */
#define SS_ENOCONV    -4   /* iterative refinement did not converge             */
#define SS_ETIMEOUT   -5   /* a bounded device wait ran out                     */
#define SS_ENOMEM     -6   /* device allocation failed                          */
#define SS_ESTATE     -7   /* call out of order (e.g. sweep before analyze)      */

/* element families (src/sawsim/saw2d/piezo_fem.py:283, :373; saw3d/assembly.py:230) */
#define SS_Q9_ME0   0      /* plane strain [ux | uy | phi], 3 DOF/node           */
#define SS_Q9_ME1   1      /* [ux | uy | uz | phi], 4 DOF/node                   */
#define SS_HEX27    2      /* u interleaved 3n+c, phi at 3N+n                    */
#define SS_MATRIX   3      /* assembled global matrices from ss_set_csr          */

/* precision modes for ss_sweep */
#define SS_PREC_FP64   0   /* complex128 fronts, FP64 throughout (the drop-in)   */
#define SS_PREC_MIXED  1   /* complex64 fronts, 3xTF32 tensor-core Schur updates
                              (or SIMT FP32 where the autotuner finds it faster),
                              FP64 residual, FP64 flexible GMRES on the primal and
                              the adjoint, dual-weighted charge correction; points
                              that do not converge are re-solved in FP64         */
#define SS_PREC_AUTO   2   /* probe MIXED on the two band ends with 12 Krylov
                              steps; MIXED if both converge, else FP64; the
                              decision is kept for the same two end
                              frequencies until the system changes               */

/* matrix selectors for ss_export_csr */
#define SS_MAT_K    0      /* global stiffness                                   */
#define SS_MAT_M    1      /* global mass                                        */
#define SS_MAT_D    2      /* global damping (Rayleigh beta*D part)              */
#define SS_MAT_KC   3      /* condensed active stiffness, active-DOF order       */
#define SS_MAT_MC   4      /* condensed active mass, active-DOF order            */

/* Create / destroy.  `device` is the CUDA ordinal. */
int ss_create(ss_handle **out, int device);
void ss_destroy(ss_handle *h);
/* Last error message of this handle (never NULL). */
const char *ss_last_error(const ss_handle *h);

/*
 * Mesh input of the GPU assembly (replaces the inputs of piezo_fem.assemble,
 * src/sawsim/saw2d/piezo_fem.py:283, and form_stiffness_mass_3d,
 * src/sawsim/saw2d/saw3d/assembly.py:230).
 *   pos_m   : n_nodes x 2 (Q9) or x 3 (Hex27) coordinates in metres
 *   conn    : n_elem x 9 (Q9) or x 27 (Hex27) 0-based node ids
 *   elem_mat: n_elem material indices
 */
int ss_set_mesh(ss_handle *h, int element_kind, int64_t n_nodes, const double *pos_m,
                int64_t n_elem, const int64_t *conn, const int32_t *elem_mat);

/*
 * Materials in device axes (already rotated).  Complex interleaved:
 * C: n_mat x 6 x 6 x 2, e: n_mat x 3 x 6 x 2, eps: n_mat x 3 x 3 x 2; rho real.
 * For SS_Q9_ME0 pass the zero-lifted full tensors, as piezo_fem.py:389-401 does.
 * `which` = SS_MAT_K for the stiffness/mass materials, SS_MAT_D for the Rayleigh
 * damping materials (solver.py:109-115).
 */
int ss_set_materials(ss_handle *h, int which, int n_mat, const double *rho,
                     const double *C, const double *e, const double *eps);

/*
 * PML regions (piezo_fem.py:192-242 for Q9, saw3d/assembly.py:127-143 for Hex27).
 * Region r stretches axis a (bit a of axis_mask[r]) by
 *   alpha = 1 + dmax*(1 - ((c - outer)/(inner - outer))^2)^npow / (i omega_top)
 * with c the element's centre-node coordinate; `clip` clamps the ratio to [0,1]
 * (the Q9 form clamps, the Hex27 form does not).  elem_region[e] = -1 for none.
 * inner/outer: n_regions x 3.
 */
int ss_set_pml(ss_handle *h, int n_regions, const int32_t *axis_mask, const double *dmax,
               const int32_t *npow, const double *inner, const double *outer, int clip,
               const int32_t *elem_region, double omega_top);

/*
 * Boundary sets (sweep.py:41-72 / saw3d/boundary.py:84-148).
 * merge groups as CSR: group g = group_dofs[group_ptr[g] .. group_ptr[g+1]),
 * first entry the master (sweep.py:97-144).  For the Hex27 two-stage fold pass
 * the front/back groups first and then the left/right groups with
 * `two_stage` = number of groups in the first stage (bc_solve.py:25-44); 0 for
 * the single union-find fold.
 */
int ss_set_bc(ss_handle *h, int64_t gdof, int64_t n_fix, const int64_t *fix,
              int64_t n_zheng, const int64_t *zheng, int64_t n_fu, const int64_t *fu,
              int64_t n_groups, const int64_t *group_ptr, const int64_t *group_dofs,
              int64_t two_stage);

/* GPU assembly of K and M (and D when damping materials were set).  On an
 * analysed handle whose mesh and boundary sets are unchanged (new materials,
 * PML or freeze frequency only) the analysis, the factorisation plans and their
 * autotuner picks are kept and only the condensed values are gathered again;
 * the reference rebuilds its engine for every sweep (agent.py:406-477 runs 2-9
 * of them per locate). */
int ss_assemble(ss_handle *h);

/*
 * Assembled-matrix input, the alternative to ss_set_mesh + ss_assemble: the
 * arguments of the reference engine's constructor,
 *   src/sawsim/saw2d/sweep.py:283  FrequencySolver(K, M, fix, zheng, fu, merge_groups)
 *   src/sawsim/saw2d/saw3d/bc_solve.py:108  FrequencySolver3D(K, M, boundary, t_fb, t_lr)
 * as a global pattern here, values by ss_set_values and the boundary sets by
 * ss_set_bc.  The pattern is CSR over gdof rows with strictly ascending columns in
 * each row; K, M (and D) share it (pass the union of their patterns).
 *   dof_node : gdof node ids in [0, n_nodes), or NULL.  The DOFs of one node are
 *              eliminated together; without it, DOFs whose condensed rows have
 *              the same columns are grouped.
 *   node_xyz : n_nodes x dim coordinates (dim 2 or 3), or NULL; needs dof_node.
 *              With them the fill-reducing ordering is the geometric nested
 *              dissection of the mesh path (the same ordering as ss_set_mesh on
 *              the same mesh); without them a graph nested dissection (level-set
 *              separators from a pseudo-peripheral node), which needs no geometry
 *              but leaves more fill.
 * Resets the mesh, the values and any analysis.
 */
int ss_set_csr(ss_handle *h, int64_t gdof, const int64_t *indptr, const int64_t *indices,
               int64_t n_nodes, int dim, const int64_t *dof_node, const double *node_xyz);

/*
 * Values on the ss_set_csr pattern, complex interleaved (2 x nnz doubles):
 * which = SS_MAT_K, SS_MAT_M or SS_MAT_D (the Rayleigh-damped part of K,
 * sweep.py:316-323; ss_set_damping sets beta).  On an analysed handle only the
 * condensed values are gathered again: the analysis, the factorisation plans and
 * their autotuner picks are kept (a new PML freeze frequency, new damping).
 */
int ss_set_values(ss_handle *h, int which, const double *vals);

/*
 * Copy a matrix to host.  Call with vals == NULL to get sizes in *nnz.
 * indptr: n+1, indices: nnz, vals: 2*nnz.  For SS_MAT_KC/MC the order is the
 * reference's active-DOF order (sweep.py:308-309) on the structural pattern.
 */
int ss_export_csr(ss_handle *h, int which, int64_t *n, int64_t *nnz, int64_t *indptr,
                  int64_t *indices, double *vals);

/* Condensation maps, fill-reducing ordering and symbolic factorisation (host). */
int ss_analyze(ss_handle *h);

/* Rayleigh stiffness damping A = K + i w beta D - w^2 M (sweep.py:316-323). */
int ss_set_damping(ss_handle *h, double beta);

/*
 * Sweep n_f angular frequencies at drive voltage V (FrequencySolver.solve,
 * sweep.py:335-364, for every point; charge_stream, frequency_tasks.py:33).
 * Q: n_f x 2 reaction charges (the reference's Q = kts . disp).
 * status: n_f per-point status (0 ok); iters: n_f refinement steps (may be NULL).
 */
int ss_sweep(ss_handle *h, int n_f, const double *omega, double V, int precision,
             double *Q, int *status, int *iters);

/* Full DOF vector at one frequency (fields.npz, solver.py:131-140): gdof x 2,
 * and the charge of the same solve in Q (2 doubles; may be NULL), as
 * FrequencySolver.solve returns both (sweep.py:335-364). */
int ss_solve_fields(ss_handle *h, double omega, double V, double *disp, double *Q);

/*
 * Adjoint of the charge at one frequency: lambda (n_active x 2, the reference's
 * active-DOF order) solves A_aa^T lambda = kq, where A_aa = Km_aa - w^2 Mm_aa
 * (+ i w beta Dm_aa) and kq is the charge row kts = K^T s folded onto the
 * active DOFs (sweep.py:301-305, :356-362), so that dQ = -lambda^T dA x for a
 * perturbation dA of the condensed system.  The reference has no adjoint; this
 * is the transposed solve with the same factors that its PARDISO/SuperLU call
 * (sweep.py:346-353) would need.  Returns the solve status (SS_ENOCONV when the
 * mixed-precision refinement did not reach its tolerance).
 */
int ss_solve_adjoint(ss_handle *h, double omega, int precision, double *lambda);

/*
 * Charges and their derivatives with respect to n_params parameters, by the
 * adjoint: dQ/dp = sum_e (s - mu)_e^T dK_e/dp d_e + w^2 mu_e^T dM_e/dp d_e with d
 * the full DOF vector, mu the folded adjoint (ss_solve_adjoint) and s the +
 * electrode indicator; dK_e/dp, dM_e/dp are recomputed per element by
 * forward-mode differentiation of the element routine.  The reference has no
 * derivative; its charge is Q = kts . disp (sweep.py:303-305, :356-363) and the
 * element routine is piezo_fem.py:248-367.  A parameter is described by its
 * seeds (parameter-major, any pointer may be NULL = zero):
 *   dpos   n_params x n_nodes x dim     node velocities dX/dp (metres per unit p;
 *                                       dim 2 for Q9, 3 for Hex27)
 *   dC     n_params x n_mat x 6 x 6 x 2 d(material C)/dp, complex interleaved
 *   de     n_params x n_mat x 3 x 6 x 2
 *   deps   n_params x n_mat x 3 x 3 x 2
 *   drho   n_params x n_mat
 *   dinner, douter  n_params x n_regions x 3   d(PML bounds)/dp
 * Outputs: Q (n_f x 2) and dQ (n_f x n_params x 2).  Q9 and Hex27 meshes
 * (saw3d/assembly.py:230-327 for the Hex27 element routine); no Rayleigh
 * damping.  status: n_f per-point status as ss_sweep (may be NULL).
 */
int ss_adjoint_gradient(ss_handle *h, int n_f, const double *omega, double V, int precision, int n_params,
                        const double *dpos, const double *dC, const double *de, const double *deps,
                        const double *drho, const double *dinner, const double *douter, double *Q, double *dQ,
                        int *status);

/*
 * Counters of the last calls: out[0..n) filled with
 *  0 n_active, 1 n_fronts, 2 max_front, 3 factor_flops_per_point (complex fronts,
 *  8 real flops per complex multiply-add), 4 nnz(L+U), 5 analyze_s, 6 assemble_ms,
 *  7 sweep_ms, 8 factor_ms, 9 solve_ms, 10 chunk, 11 schur_gemm_ms,
 *  12 schur_gemm_flops, 13 levels, 14 perturbed pivots, 15 kernel launches,
 *  16 Schur GEMM launches, 17 device time of the last ss_sweep (ms, CUDA events),
 *  18 refinement / Krylov steps of the last ss_sweep (sum over points),
 *  19 precision the last ss_sweep ran in (SS_PREC_FP64 or SS_PREC_MIXED),
 *  20-22 levels whose Schur update uses the autotuner's candidate 0, 1, 2
 *  (FP64 sweep: SIMT 128x64, FP64 tensor-core DMMA 64x64 with three real
 *  products per complex block, the same with four; mixed
 *  sweep: packed operands + TMA + tcgen05 3xTF32 with 128 / 64 complex columns
 *  per tile, SIMT FP32 128x64),
 *  23 panel-step GEMM tiles (128x32 / 32x128): 0 SIMT, 1 DMMA, 2 DMMA with
 *  three real products per complex block, 3 the same with C staged, 4 SIMT
 *  with C staged (complex64), 24-25 autotuner time of all
 *  panel-step GEMMs with SIMT / the faster DMMA tiles (ms),
 *  26 fronts factored whole in shared memory, 27 autotuner time of all
 *  Schur candidates (ms, sum over candidates and levels),
 *  28 device time of the last SS_PREC_AUTO probe (ms), 29 points of the last
 *  mixed sweep re-solved in FP64 (option fp64_fallback), 30 / 31 Krylov steps of
 *  the primal / adjoint solves of the last sweep (sums over points), 32 points
 *  whose mixed refinement did not converge (before any FP64 re-solve), 33 device
 *  time of the FP64 re-solves (ms, included in 17), 34 / 35 device time of the
 *  element kernel / of the scatter into the CSR pattern of the last
 *  ss_assemble (ms, CUDA events), 36 levels whose FP64 Schur update uses
 *  candidate 3 (DMMA 64x64, three real products, C tile staged in shared
 *  memory while the K loop runs), 37 panel-step GEMM tiles per point run as
 *  thin SIMT 128x8 / 8x128 tiles (tasks at most 8 columns wide or 8 rows high,
 *  beside the DMMA tiles; 0 when the autotuner kept them in DMMA tiles).
 *  Slots past 37 read 0.
 */
int ss_stats(const ss_handle *h, double *out, int n);

/*
 * Solver options, by name (the reference's PARDISO / SuperLU calls,
 * sweep.py:346-353, take none; these tune the replacement's refinement):
 *   krylov_restart    FGMRES restart length of the mixed sweep (default 30)
 *   krylov_cycles     FGMRES restarts (default 1)
 *   krylov_tol        relative residual target of the primal and adjoint
 *                     Krylov solves (default 1e-8; with the dual-weighted
 *                     charge correction the charge error is about the product
 *                     of the two residuals' effects)
 *   pivot_tiny_c128   static pivot perturbation of complex128 fronts: a pivot
 *                     of modulus below it is replaced by it (default 1e-13; the
 *                     system is equilibrated to unit row and column maxima)
 *   pivot_tiny_c64    the same for complex64 fronts (default 1e-6)
 *   fp64_fallback     1: points of a mixed sweep whose refinement does not
 *                     converge are re-solved in FP64 in the same call (default)
 *   auto_probe_steps  Krylov steps of SS_PREC_AUTO's probe (default 12)
 * Options persist in the handle; changing one drops a kept SS_PREC_AUTO
 * decision.  SS_EINVAL for an unknown name or a value out of range.
 */
int ss_set_option(ss_handle *h, const char *name, double value);

/*
 * Roofline denominator of the Schur update (no counterpart in the reference):
 * the median algorithmic rate in TFLOP/s (8 real flops per complex
 * multiply-add) of one Schur-update kernel of this library on n_fronts dense
 * synthetic fronts of m rows with k pivots (update block (m-k)^2, K = k), one
 * launch covering all fronts, timed by CUDA events over `reps` launches after a
 * warm-up.  kernel: 0 FP64 DMMA 64x64 tiles, 1 FP64 SIMT 128x64, 2 complex64
 * TMA + tcgen05 3xTF32 with 128-column tiles, 3 the same with 64-column tiles
 * (operands packed once before the timed launches), 4 complex64 SIMT FP32
 * 128x64, 5 FP64 DMMA 64x64 with three real products per complex block, 6 the
 * same with the C tile staged in shared memory while the K loop runs.
 * Allocates and frees its fronts (at most 64 GB).
 */
int ss_measure_gemm_ceiling(ss_handle *h, int kernel, int m, int k, int n_fronts, int reps,
                            double *tflops);

/*
 * Host-only analysis of a mesh system: the global pattern, the Bloch fold and
 * condensation, the nested-dissection ordering and the multifrontal front tree
 * that ss_analyze builds, computed on the host with no CUDA device and no handle
 * (no counterpart in the reference, whose SuperLU / PARDISO calls analyse inside
 * every per-frequency solve, src/sawsim/saw2d/sweep.py:346-353).  It shows the
 * fronts, fill, flops and front memory of a cell before it runs on a GPU.
 *
 * Inputs as for ss_set_mesh (without materials) and ss_set_bc.  Outputs:
 * sizes[4] = {active DOFs n, fronts F, total front rows R, tree levels};
 * stats[6] = {factorisation flops per point, nnz(L+U), widest front, most
 * pivots of a front, complex front elements per point (m x padded ld, summed),
 * condensed nonzeros}.  Arrays that are not NULL are filled: active[n] (global
 * DOF of each active DOF, ascending), order[n] (elimination position of each
 * active DOF), k[F], m[F] (pivots, rows), parent[F] (-1 at a root), level[F],
 * rows_ptr[F+1] and rows[R] (each front's rows in elimination positions: its
 * pivots, then its update rows ascending).  Call once with NULL arrays for the
 * sizes, then with arrays of those sizes.  Errors: SS_EINVAL for bad inputs or
 * an analysis that fails (there is no handle, so no error text).
 */
int ss_analyze_host(int element_kind, int64_t n_nodes, const double *pos_m, int64_t n_elem,
                    const int64_t *conn, int64_t gdof, int64_t n_fix, const int64_t *fix, int64_t n_zheng,
                    const int64_t *zheng, int64_t n_fu, const int64_t *fu, int64_t n_groups,
                    const int64_t *group_ptr, const int64_t *group_dofs, int64_t two_stage, int64_t *sizes,
                    double *stats, int64_t *active, int64_t *order, int32_t *k, int32_t *m, int32_t *parent,
                    int32_t *level, int64_t *rows_ptr, int64_t *rows);

/*
 * The same host-only analysis from an assembled pattern, as ss_set_csr takes it
 * (the reference engine's FrequencySolver(K, M, ...), sweep.py:283-314): the
 * union pattern of K and M (gdof rows, columns strictly ascending), and
 * optionally the node of every DOF and the node coordinates (dim 2 or 3), which
 * give the geometric ordering of the mesh path; without them the ordering is the
 * graph nested dissection of ss_analyze.  Boundary sets and outputs as for
 * ss_analyze_host.
 */
int ss_analyze_host_csr(int64_t gdof, const int64_t *indptr, const int64_t *indices, int64_t n_nodes, int dim,
                        const int64_t *dof_node, const double *node_xyz, int64_t n_fix, const int64_t *fix,
                        int64_t n_zheng, const int64_t *zheng, int64_t n_fu, const int64_t *fu, int64_t n_groups,
                        const int64_t *group_ptr, const int64_t *group_dofs, int64_t two_stage, int64_t *sizes,
                        double *stats, int64_t *active, int64_t *order, int32_t *k, int32_t *m, int32_t *parent,
                        int32_t *level, int64_t *rows_ptr, int64_t *rows);

/*
 * Q9 assembly that allocates nothing (no counterpart in the reference).  It is
 * for callers of this library that may not allocate device memory: a host
 * framework that hands out all device memory from its own pool (a caching
 * allocator, a serving runtime with a fixed memory budget) and forbids
 * allocations behind its back.  Such a caller still owns every input and
 * output buffer; only the scratch is fixed.
 *
 * Every pointer is a device pointer the caller owns: the mesh and materials as
 * for ss_set_mesh / ss_set_materials (materials already zero-lifted for
 * ndisp == 2), the PML as for ss_set_pml (n_regions == 0: no PML; the Q9 form
 * clamps the ratio), and the global pattern: indptr (ndisp+1)*n_nodes+1 row
 * pointers of the component-major K layout and the node adjacency nadj_ptr /
 * nadj (sorted neighbours, self included).  K and M (nnz complex values each)
 * are zeroed and then filled.
 *
 * Scratch: element matrices go through one fixed file-scope device array of
 * 512 elements (11.3 MB), which every GPU that loads the library holds until
 * the process exits; larger meshes are processed in 512-element batches.  All
 * calls share that array and it keeps the last call's contents, so calls that
 * overlap on the GPU (other streams, other host threads) race.  Shared slots are
 * summed with atomic adds, so results equal ss_assemble's to rounding, not bit
 * for bit.  The first call on a device, with that device current, resolves the
 * array's device address and keeps it for the life of the process: make that
 * first call before any stream capture, and do not call this entry point on a
 * device after cudaDeviceReset of that device.
 *
 * The call synchronises `stream` (a cudaStream_t, NULL for the legacy default
 * stream) to read back its pattern check, and returns SS_EINVAL when the
 * pattern does not contain an element's node pair (the skipped entries are
 * then missing from K and M).
 */
int ss_assemble_q9_noalloc(int ndisp, int64_t n_nodes, const double *pos, int64_t n_elem,
                           const int64_t *conn, const int32_t *elem_mat, const double *rho,
                           const double *C, const double *e, const double *eps, int n_regions,
                           const int32_t *elem_region, const int32_t *pml_axis,
                           const double *pml_dmax, const int32_t *pml_npow,
                           const double *pml_inner, const double *pml_outer, double omega_top,
                           const int64_t *indptr, const int64_t *nadj_ptr, const int64_t *nadj,
                           int64_t nnz, double *K, double *M, void *stream);

#ifdef __cplusplus
}
#endif
#endif
