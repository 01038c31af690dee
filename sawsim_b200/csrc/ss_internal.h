// Internal declarations shared by the host runtime (ss_api.cpp, symbolic.cpp)
// and the device code (*.cu).
#pragma once
#include <cstdint>
#include <functional>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/sawsim_b200.h"

namespace ss {

template <class T>
struct cplx;   // dev_complex.cuh
struct cplx_d {   // host view of a device cplx<double>
  double re, im;
};

// ---------------------------------------------------------------- device buffer
struct DBuf {
  void *p = nullptr;
  size_t bytes = 0;
  ~DBuf() { release(); }
  void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
  template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

// FGMRES workspace (basis, preconditioned basis, Hessenberg data); held by the
// handle so that repeated mixed sweeps reuse it
struct KrylovWork {
  DBuf V, Z, w, h, hn, y, kf, sc;
  size_t bytes() const { return V.bytes + Z.bytes + w.bytes + h.bytes + hn.bytes + y.bytes + kf.bytes + sc.bytes; }
  void release() { V.release(); Z.release(); w.release(); h.release(); hn.release(); y.release(); kf.release(); sc.release(); }
};

// frequencies per thread in the sparse products (residual, Krylov SpMV): the
// matrix row is read once per block of this many frequencies
constexpr int kSpmvFreqs = 8;
inline unsigned spmv_blocks(int nb) { return (unsigned)((nb + kSpmvFreqs - 1) / kSpmvFreqs); }

// Allocate (or grow) a device buffer; returns cudaError_t.
cudaError_t dalloc(DBuf &b, size_t bytes);
template <class T>
cudaError_t dupload(DBuf &b, const std::vector<T> &v) {
  cudaError_t e = dalloc(b, v.size() * sizeof(T) + 16);
  if (e != cudaSuccess) return e;
  return v.empty() ? cudaSuccess : cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// ---------------------------------------------------------------- symbolic data
struct Symbolic {
  int64_t n = 0;                    // active DOFs (condensed system size)
  std::vector<int64_t> new_of_act;  // active index -> elimination order index
  std::vector<int64_t> act_of_new;  // inverse
  // fronts in postorder (children first)
  int nfront = 0;
  std::vector<int> k, m, ld, parent, level;
  std::vector<int64_t> p0;          // first pivot (new index)
  std::vector<int64_t> rows_ptr;    // rows of front s: rows[rows_ptr[s] .. +m[s])
  std::vector<int64_t> rows;        // new indices, pivots first then update rows ascending
  std::vector<int64_t> child_ptr;   // children of s
  std::vector<int> child;
  std::vector<int64_t> off;         // element offset of front s in one frequency's arena
  int64_t arena = 0;                // elements per frequency (sum m*ld)
  std::vector<int64_t> relpos_ptr;  // per front: CB row -> parent position (m-k entries)
  std::vector<int> relpos;
  std::vector<int64_t> arrow_ptr;   // per front: condensed entries owned by this front
  std::vector<int32_t> arrow_pos;   // row*ld + col inside the front
  std::vector<int64_t> arrow_slot;  // index into the condensed CSR values
  int nlevel = 0;
  std::vector<int64_t> level_ptr;   // fronts of level l: level_fronts[level_ptr[l]..]
  std::vector<int> level_fronts;
  double flops = 0, nnz_lu = 0;
  int max_m = 0, max_k = 0;
};

struct Handle {
  int device = 0;
  int num_sms = 148;                     // streaming multiprocessors of the device
  cudaStream_t stream = nullptr;
  std::string err;
  // mesh
  int kind = -1, npe = 0, dim = 2, nc = 0;  // nc: DOF components per node
  int64_t N = 0, ne = 0, gdof = 0;
  std::vector<double> pos;
  std::vector<int64_t> conn;
  std::vector<int32_t> emat;
  std::vector<int64_t> dof_node;         // SS_MATRIX: node of each global DOF (empty: none given)
  // materials (per which: 0 K/M, 1 D)
  int nmat[2] = {0, 0};
  std::vector<double> rho[2], C[2], e[2], eps[2];
  // pml
  int npml = 0, pml_clip = 1;
  std::vector<int32_t> pml_axis, pml_npow, elem_region;
  std::vector<double> pml_dmax, pml_inner, pml_outer;
  double omega_top = 0;
  // boundary
  std::vector<int64_t> fix, zheng, fu, gptr, gdofs;
  int64_t two_stage = 0;
  bool have_bc = false;
  // global pattern (host) and values (device)
  std::vector<int64_t> nadj_ptr, nadj;   // node graph
  std::vector<int64_t> indptr, indices;  // global K pattern
  int64_t nnz = 0;
  bool have_K = false, have_M = false, have_D = false;
  DBuf dK, dM, dD;                       // complex128 values on the K pattern
  // condensation (new-order CSR)
  std::vector<int64_t> rep;              // gdof -> representative (master) dof
  std::vector<int64_t> active;           // active gdofs ascending
  std::vector<int64_t> act_of_gdof;      // gdof -> active index or -1
  std::vector<int64_t> a_ptr, a_idx;     // condensed pattern, active order
  std::vector<int64_t> ag_ptr, ag_src;   // its gather lists (global slots, ascending)
  std::vector<int64_t> vg_ptr, vg_src;   // gathers of ks|ms|kq (3*n_act+1), active order
  std::vector<int64_t> qz_src;           // global slots summed into Qz
  std::vector<int64_t> sv_of_act;        // active dof -> supervariable (node)
  int64_t nsv = 0;
  std::vector<double> sv_xyz;            // supervariable coordinates (nsv x 3)
  std::vector<int64_t> c_ptr, c_idx;     // condensed pattern in NEW order
  std::vector<int64_t> c_perm;           // new-order entry -> active-order entry
  int64_t c_nnz = 0;
  DBuf dc_ptr, dc_idx, dKc, dMc, dDc;    // device condensed CSR
  DBuf dg_ptr, dg_src;                   // gather lists: condensed slot <- global slots
  DBuf dks, dms, dds, dkq;               // rhs/charge vectors (new order)
  DBuf dv_ptr, dv_src;                   // gather lists of ks | kq (and ms, ds)
  DBuf dq_ptr, dq_src;                   // gather list of Qz
  std::vector<int64_t> v_ptr;            // host copy (sizes)
  double Qz_dummy = 0;
  DBuf dQz;                              // complex: sum over zheng rows/cols of K
  DBuf drow_scale, dcol_scale;           // equilibration (new order)
  double beta = 0;
  bool analyzed = false;
  Symbolic sym;
  // device copies of symbolic data
  DBuf d_k, d_m, d_ld, d_off, d_rows_ptr, d_rows, d_child_ptr, d_child, d_relpos_ptr,
      d_relpos, d_arrow_ptr, d_arrow_pos, d_arrow_slot, d_level_fronts, d_p0;
  // numeric work
  DBuf arena, piv, dperm_new, work;
  DBuf wk[16];                           // sweep work buffers, kept across calls
  DBuf dct_ptr, dct_idx, dct_src;        // transposed condensed pattern (new order) and value slots
  size_t arena_chunk = 0;
  void *plan[2] = {nullptr, nullptr};   // factorisation plans per precision
  KrylovWork kw;                         // FGMRES workspace of the mixed sweeps
  // SS_PREC_AUTO's decision for the last probed band (its two end frequencies);
  // dropped with the plans whenever the system changes
  double auto_w0 = 0, auto_w1 = 0;
  int auto_prec = -1;
  DBuf dKs, dMs, dDs;                    // equilibrated condensed values
  DBuf tc_stage;                         // packed tensor-core Schur operands (mixed sweeps)
  DBuf dmask;                            // per chunk frequency: still iterating in a Krylov loop
  double scale_w = -1;                   // frequency the scaling was computed at
  // solver options (ss_set_option); kept until changed
  struct Options {
    int krylov_m = 30;                   // FGMRES restart length of the mixed sweep
    int krylov_cycles = 1;               // FGMRES restarts
    double krylov_tol = 1e-8;            // relative residual target (primal and adjoint)
    double tiny_c128 = 1e-13;            // static pivot perturbation, complex128 fronts
    double tiny_c64 = 1e-6;              // static pivot perturbation, complex64 fronts
    int fp64_fallback = 1;               // re-solve unconverged mixed points in FP64
    int auto_probe_m = 12;               // Krylov steps of SS_PREC_AUTO's probe
  } opt;
  // stats
  static constexpr int kStats = 38;
  double st[kStats] = {0};
};

// ---------------------------------------------------------------- kernels
// assemble.cu
int launch_assemble(Handle &h, int which);  // which 0: K+M, 1: D
// numeric.cu
int launch_condense(Handle &h);
int gather_values(Handle &h);   // condensed values again after a value-only reassembly
// Optional work of a sweep beyond the charges: per_chunk(c0, nb, x, mu) is called
// for every chunk of frequencies with the scaled primal solutions x' and adjoint
// solutions mu' (A'^T mu' = cs * kq) of that chunk on the device (nb x n each).
struct SweepExtra {
  std::function<int(int, int, const cplx<double> *, const cplx<double> *)> per_chunk;
};
int run_sweep(Handle &h, int n_f, const double *omega, double V, int precision,
              double *Q, int *status, int *iters, double *disp_out, const SweepExtra *ex = nullptr);
// Median algorithmic TFLOP/s of one Schur-update kernel on dense synthetic fronts
int measure_ceiling(Handle &h, int kernel, int m, int k, int nb, int reps, double *tflops);
// adjoint.cu: Q (n_f x 2) and dQ (n_f x n_params x 2) with the seeds of ss_adjoint_gradient
int run_adjoint_gradient(Handle &h, int n_f, const double *omega, double V, int precision, int n_params,
                         const double *dpos, const double *dC, const double *de, const double *deps,
                         const double *drho, const double *dinner, const double *douter, double *Q, double *dQ,
                         int *status);
// hex27.cu: tangent element matrices of a parameter (Seed: dual.cuh)
struct Seed;
struct PmlDev;
cudaError_t launch_hex27_tangent(cudaStream_t st, int64_t ne, const double *pos, const int64_t *conn,
                                 const int32_t *emat, const double *rho, const double *C, const double *e,
                                 const double *eps, const PmlDev &pml, const Seed &sd, cplx<double> *dKel,
                                 cplx<double> *dMel);
// symbolic.cpp
int build_global_pattern(Handle &h);
int build_condensation(Handle &h);
int build_symbolic(Handle &h);

int fail(Handle &h, int code, const std::string &msg);
int cuda_fail(Handle &h, cudaError_t e, const char *where);

}  // namespace ss

struct ss_handle {
  ss::Handle h;
};
