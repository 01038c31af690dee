// C ABI of the sweep backend (declared in include/sawsim_b200.h).
#include "ss_internal.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>

namespace ss {

int fail(Handle &h, int code, const std::string &msg) {
  h.err = msg;
  return code;
}
int cuda_fail(Handle &h, cudaError_t e, const char *where) {
  h.err = std::string(where) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? SS_ENOMEM : SS_ECUDA;
}
int build_new_order(Handle &h);
void free_plans(Handle &h);

}  // namespace ss

using namespace ss;

#define H_CHECK(hp)                       \
  if (!(hp)) return SS_EINVAL;            \
  Handle &h = (hp)->h;                    \
  cudaSetDevice(h.device)

static const char *kNoHandle = "null handle";

static bool all_finite(const double *p, int64_t n) {
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

extern "C" int ss_create(ss_handle **out, int device) {
  if (!out) return SS_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return SS_ECUDA;
  ss_handle *p = new (std::nothrow) ss_handle();
  if (!p) return SS_ENOMEM;
  p->h.device = device;
  cudaSetDevice(device);
  cudaDeviceGetAttribute(&p->h.num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&p->h.stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete p;
    return SS_ECUDA;
  }
  *out = p;
  return SS_OK;
}

extern "C" void ss_destroy(ss_handle *hp) {
  if (!hp) return;
  cudaSetDevice(hp->h.device);
  cudaStreamSynchronize(hp->h.stream);
  free_plans(hp->h);
  cudaStreamDestroy(hp->h.stream);
  delete hp;
}

extern "C" const char *ss_last_error(const ss_handle *hp) { return hp ? hp->h.err.c_str() : kNoHandle; }

static void reset_derived(Handle &h) {
  h.analyzed = false;
  h.scale_w = -1;
  free_plans(h);
}

extern "C" int ss_set_mesh(ss_handle *hp, int kind, int64_t n_nodes, const double *pos, int64_t n_elem,
                           const int64_t *conn, const int32_t *emat) {
  H_CHECK(hp);
  if (kind < SS_Q9_ME0 || kind > SS_HEX27) return fail(h, SS_EINVAL, "unknown element kind (SS_MATRIX: ss_set_csr)");
  if (n_nodes <= 0 || n_elem <= 0 || !pos || !conn || !emat) return fail(h, SS_EINVAL, "empty mesh or null array");
  if (!all_finite(pos, n_nodes * (kind == SS_HEX27 ? 3 : 2))) return fail(h, SS_EINVAL, "non-finite coordinate");
  h.kind = kind;
  h.npe = kind == SS_HEX27 ? 27 : 9;
  h.dim = kind == SS_HEX27 ? 3 : 2;
  h.nc = kind == SS_Q9_ME0 ? 3 : 4;
  h.N = n_nodes;
  h.ne = n_elem;
  h.pos.assign(pos, pos + n_nodes * h.dim);
  h.dof_node.clear();
  h.conn.assign(conn, conn + n_elem * h.npe);
  h.emat.assign(emat, emat + n_elem);
  for (int64_t v : h.conn)
    if (v < 0 || v >= n_nodes) return fail(h, SS_EINVAL, "connectivity index out of range");
  for (int32_t v : h.emat)
    if (v < 0) return fail(h, SS_EINVAL, "negative material index");
  h.indptr.clear();
  h.have_K = h.have_M = h.have_D = false;
  reset_derived(h);
  return build_global_pattern(h);
}

extern "C" int ss_set_materials(ss_handle *hp, int which, int n_mat, const double *rho, const double *C,
                                const double *e, const double *eps) {
  H_CHECK(hp);
  if (which != SS_MAT_K && which != SS_MAT_D) return fail(h, SS_EINVAL, "materials: which must be K or D");
  if (n_mat <= 0 || !rho || !C || !e || !eps) return fail(h, SS_EINVAL, "materials: empty or null");
  if (!all_finite(rho, n_mat) || !all_finite(C, n_mat * 72) || !all_finite(e, n_mat * 36) ||
      !all_finite(eps, n_mat * 18))
    return fail(h, SS_EINVAL, "materials: non-finite value");
  const int w = which == SS_MAT_D;
  h.nmat[w] = n_mat;
  h.rho[w].assign(rho, rho + n_mat);
  h.C[w].assign(C, C + n_mat * 72);
  h.e[w].assign(e, e + n_mat * 36);
  h.eps[w].assign(eps, eps + n_mat * 18);
  return SS_OK;
}

extern "C" int ss_set_pml(ss_handle *hp, int n_regions, const int32_t *axis, const double *dmax, const int32_t *npow,
                          const double *inner, const double *outer, int clip, const int32_t *elem_region,
                          double omega_top) {
  H_CHECK(hp);
  if (!(omega_top > 0) || !std::isfinite(omega_top)) return fail(h, SS_EINVAL, "omega_top must be positive and finite");
  if (n_regions < 0 || (n_regions > 0 && (!axis || !dmax || !npow || !inner || !outer || !elem_region)))
    return fail(h, SS_EINVAL, "pml: null array");
  if (n_regions > 0 && (!all_finite(dmax, n_regions) || !all_finite(inner, 3 * n_regions) ||
                        !all_finite(outer, 3 * n_regions)))
    return fail(h, SS_EINVAL, "pml: non-finite value");
  h.omega_top = omega_top;
  h.npml = n_regions;
  h.pml_clip = clip;
  h.pml_axis.assign(axis, axis + n_regions);
  h.pml_npow.assign(npow, npow + n_regions);
  h.pml_dmax.assign(dmax, dmax + n_regions);
  h.pml_inner.assign(inner, inner + 3 * n_regions);
  h.pml_outer.assign(outer, outer + 3 * n_regions);
  if (n_regions > 0) {
    if (h.ne <= 0) return fail(h, SS_ESTATE, "set the mesh before the PML");
    h.elem_region.assign(elem_region, elem_region + h.ne);
    for (int32_t r : h.elem_region)
      if (r >= n_regions) return fail(h, SS_EINVAL, "pml region index out of range");
  }
  return SS_OK;
}

extern "C" int ss_set_bc(ss_handle *hp, int64_t gdof, int64_t n_fix, const int64_t *fix, int64_t n_zheng,
                         const int64_t *zheng, int64_t n_fu, const int64_t *fu, int64_t n_groups,
                         const int64_t *group_ptr, const int64_t *group_dofs, int64_t two_stage) {
  H_CHECK(hp);
  if (gdof <= 0) return fail(h, SS_EINVAL, "gdof must be positive");
  if (h.gdof && gdof != h.gdof) return fail(h, SS_EINVAL, "gdof does not match the mesh");
  auto in = [&](const int64_t *p, int64_t cnt) {
    for (int64_t i = 0; i < cnt; ++i)
      if (p[i] < 0 || p[i] >= gdof) return false;
    return true;
  };
  if ((n_fix && !fix) || (n_zheng && !zheng) || (n_fu && !fu) || (n_groups && (!group_ptr || !group_dofs)))
    return fail(h, SS_EINVAL, "bc: null array");
  if (!in(fix, n_fix) || !in(zheng, n_zheng) || !in(fu, n_fu)) return fail(h, SS_EINVAL, "bc: dof out of range");
  if (n_zheng == 0) return fail(h, SS_EINVAL, "bc: no driven electrode DOFs");
  if (two_stage < 0 || two_stage > n_groups) return fail(h, SS_EINVAL, "bc: bad two_stage");
  h.fix.assign(fix, fix + n_fix);
  h.zheng.assign(zheng, zheng + n_zheng);
  h.fu.assign(fu, fu + n_fu);
  h.gptr.assign(group_ptr, group_ptr + n_groups + 1);
  if (n_groups == 0) h.gptr.assign(1, 0);
  h.gdofs.assign(group_dofs, group_dofs + h.gptr.back());
  if (!in(h.gdofs.data(), (int64_t)h.gdofs.size())) return fail(h, SS_EINVAL, "bc: group dof out of range");
  h.two_stage = two_stage;
  h.have_bc = true;
  if (!h.gdof) h.gdof = gdof;
  reset_derived(h);
  return SS_OK;
}

extern "C" int ss_assemble(ss_handle *hp) {
  H_CHECK(hp);
  if (h.kind < 0 || h.kind == SS_MATRIX) return fail(h, SS_ESTATE, "assemble: no mesh (matrix input takes ss_set_values)");
  if (h.nmat[0] <= 0) return fail(h, SS_ESTATE, "assemble: no materials");
  int mx = *std::max_element(h.emat.begin(), h.emat.end());
  if (mx >= h.nmat[0]) return fail(h, SS_EINVAL, "element material index >= number of materials");
  if (h.omega_top <= 0 && h.npml > 0) return fail(h, SS_ESTATE, "assemble: set the PML first");
  auto t0 = std::chrono::steady_clock::now();
  // a reassembly of an analysed system with the same mesh and boundary sets (new
  // materials, PML or freeze frequency) keeps the analysis, the factorisation
  // plans, their autotuner picks and launch graphs: only the values change
  const bool keep = h.analyzed;
  const bool had_D = h.have_D;
  if (h.nmat[1] > 0 && mx >= h.nmat[1]) return fail(h, SS_EINVAL, "damping materials fewer than element materials");
  int rc = launch_assemble(h, 0);
  if (rc) return rc;
  if (h.nmat[1] > 0) {
    rc = launch_assemble(h, 1);
    if (rc) return rc;
  }
  h.st[6] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (keep) {
    if (h.have_D != had_D) free_plans(h);   // the launch graphs bake the damping matrix in
    rc = gather_values(h);
    if (rc) {
      reset_derived(h);
      return rc;
    }
    h.scale_w = -1;      // equilibrate again at the next sweep
    h.auto_prec = -1;    // a kept SS_PREC_AUTO decision was for the old values
  } else {
    reset_derived(h);
  }
  return SS_OK;
}

extern "C" int ss_set_csr(ss_handle *hp, int64_t gdof, const int64_t *indptr, const int64_t *indices,
                          int64_t n_nodes, int dim, const int64_t *dof_node, const double *node_xyz) {
  H_CHECK(hp);
  if (gdof <= 0 || !indptr || !indices) return fail(h, SS_EINVAL, "csr: empty pattern or null array");
  if (indptr[0] != 0) return fail(h, SS_EINVAL, "csr: indptr[0] must be 0");
  for (int64_t r = 0; r < gdof; ++r) {
    if (indptr[r + 1] < indptr[r]) return fail(h, SS_EINVAL, "csr: indptr not ascending");
    for (int64_t s = indptr[r]; s < indptr[r + 1]; ++s) {
      if (indices[s] < 0 || indices[s] >= gdof) return fail(h, SS_EINVAL, "csr: column out of range");
      if (s > indptr[r] && indices[s] <= indices[s - 1])
        return fail(h, SS_EINVAL, "csr: columns of a row not strictly ascending");
    }
  }
  if (node_xyz && !dof_node) return fail(h, SS_EINVAL, "csr: node coordinates need dof_node");
  if (dof_node) {
    if (n_nodes <= 0) return fail(h, SS_EINVAL, "csr: n_nodes must be positive with dof_node");
    for (int64_t d = 0; d < gdof; ++d)
      if (dof_node[d] < 0 || dof_node[d] >= n_nodes) return fail(h, SS_EINVAL, "csr: dof_node out of range");
  }
  if (node_xyz && (dim < 2 || dim > 3)) return fail(h, SS_EINVAL, "csr: dim must be 2 or 3");
  if (node_xyz && !all_finite(node_xyz, n_nodes * dim)) return fail(h, SS_EINVAL, "csr: non-finite coordinate");
  reset_derived(h);
  h.kind = SS_MATRIX;
  h.npe = 0;
  h.nc = 0;
  h.ne = 0;
  h.conn.clear();
  h.emat.clear();
  h.elem_region.clear();
  h.npml = 0;
  h.nmat[0] = h.nmat[1] = 0;
  h.nadj_ptr.clear();
  h.nadj.clear();
  h.N = dof_node ? n_nodes : 0;
  h.dim = node_xyz ? dim : 0;
  h.pos.assign(node_xyz ? node_xyz : nullptr, node_xyz ? node_xyz + n_nodes * dim : nullptr);
  h.dof_node.assign(dof_node ? dof_node : nullptr, dof_node ? dof_node + gdof : nullptr);
  h.gdof = gdof;
  h.indptr.assign(indptr, indptr + gdof + 1);
  h.nnz = h.indptr[gdof];
  h.indices.assign(indices, indices + h.nnz);
  h.have_K = h.have_M = h.have_D = false;
  h.have_bc = false;
  h.beta = 0;
  return SS_OK;
}

extern "C" int ss_set_values(ss_handle *hp, int which, const double *vals) {
  H_CHECK(hp);
  if (h.kind != SS_MATRIX) return fail(h, SS_ESTATE, "set_values: no ss_set_csr pattern");
  if (which != SS_MAT_K && which != SS_MAT_M && which != SS_MAT_D)
    return fail(h, SS_EINVAL, "set_values: which must be K, M or D");
  if (!vals) return fail(h, SS_EINVAL, "set_values: null array");
  if (!all_finite(vals, 2 * h.nnz)) return fail(h, SS_EINVAL, "set_values: non-finite value");
  DBuf &dst = which == SS_MAT_K ? h.dK : which == SS_MAT_M ? h.dM : h.dD;
  cudaError_t e = dalloc(dst, (size_t)h.nnz * 16 + 16);
  if (e != cudaSuccess) return cuda_fail(h, e, "set_values alloc");
  e = cudaMemcpyAsync(dst.p, vals, (size_t)h.nnz * 16, cudaMemcpyHostToDevice, h.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h.stream);
  if (e != cudaSuccess) return cuda_fail(h, e, "set_values copy");
  const bool had_D = h.have_D;
  (which == SS_MAT_K ? h.have_K : which == SS_MAT_M ? h.have_M : h.have_D) = true;
  if (h.analyzed) {
    // same pattern and boundary sets: keep the analysis and the plans, gather the
    // condensed values again (as a value-only reassembly does)
    if (h.have_D != had_D) free_plans(h);
    int rc = gather_values(h);
    if (rc) {
      reset_derived(h);
      return rc;
    }
    h.scale_w = -1;
    h.auto_prec = -1;
  }
  return SS_OK;
}

extern "C" int ss_export_csr(ss_handle *hp, int which, int64_t *n_out, int64_t *nnz_out, int64_t *indptr,
                             int64_t *indices, double *vals) {
  H_CHECK(hp);
  if (!n_out || !nnz_out) return fail(h, SS_EINVAL, "export: null size pointers");
  if (which == SS_MAT_K || which == SS_MAT_M || which == SS_MAT_D) {
    const DBuf &src = which == SS_MAT_K ? h.dK : which == SS_MAT_M ? h.dM : h.dD;
    const bool ok = which == SS_MAT_K ? h.have_K : which == SS_MAT_M ? h.have_M : h.have_D;
    if (!ok) return fail(h, SS_ESTATE, "export: matrix not assembled");
    // M lives on the K pattern; the reference M has only same-component u blocks
    const int ndisp = h.kind == SS_Q9_ME0 ? 2 : 3;
    auto comp = [&](int64_t d) -> int {
      if (h.kind == SS_HEX27) return d < 3 * h.N ? (int)(d % 3) : 3;
      return (int)(d / h.N);
    };
    std::vector<char> keep;
    int64_t nnz = h.nnz;
    if (which == SS_MAT_M && h.kind != SS_MATRIX) {
      keep.assign(h.nnz, 0);
      nnz = 0;
      for (int64_t r = 0; r < h.gdof; ++r)
        for (int64_t s = h.indptr[r]; s < h.indptr[r + 1]; ++s) {
          const int a = comp(r), b = comp(h.indices[s]);
          keep[s] = (a == b && a < ndisp);
          nnz += keep[s];
        }
    }
    *n_out = h.gdof;
    *nnz_out = nnz;
    if (!vals) return SS_OK;
    std::vector<double> v(2 * h.nnz);
    cudaError_t e = cudaMemcpy(v.data(), src.p, h.nnz * 16, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(h, e, "export copy");
    int64_t q = 0;
    indptr[0] = 0;
    for (int64_t r = 0; r < h.gdof; ++r) {
      for (int64_t s = h.indptr[r]; s < h.indptr[r + 1]; ++s) {
        if (!keep.empty() && !keep[s]) continue;
        indices[q] = h.indices[s];
        vals[2 * q] = v[2 * s];
        vals[2 * q + 1] = v[2 * s + 1];
        ++q;
      }
      indptr[r + 1] = q;
    }
    return SS_OK;
  }
  if (which == SS_MAT_KC || which == SS_MAT_MC) {
    if (!h.analyzed) return fail(h, SS_ESTATE, "export: analyze first");
    const int64_t n = (int64_t)h.active.size();
    *n_out = n;
    *nnz_out = (int64_t)h.a_idx.size();
    if (!vals) return SS_OK;
    std::vector<double> v(2 * h.c_nnz);
    cudaError_t e = cudaMemcpy(v.data(), (which == SS_MAT_KC ? h.dKc : h.dMc).p, h.c_nnz * 16, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(h, e, "export copy");
    std::copy(h.a_ptr.begin(), h.a_ptr.end(), indptr);
    std::copy(h.a_idx.begin(), h.a_idx.end(), indices);
    for (int64_t t = 0; t < h.c_nnz; ++t) {
      vals[2 * h.c_perm[t]] = v[2 * t];
      vals[2 * h.c_perm[t] + 1] = v[2 * t + 1];
    }
    return SS_OK;
  }
  return fail(h, SS_EINVAL, "export: unknown matrix");
}

extern "C" int ss_analyze(ss_handle *hp) {
  H_CHECK(hp);
  if (!h.have_K || !h.have_M) return fail(h, SS_ESTATE, "analyze: assemble (or set) K and M first");
  if (!h.have_bc) return fail(h, SS_ESTATE, "analyze: boundary sets missing");
  auto t0 = std::chrono::steady_clock::now();
  reset_derived(h);
  int rc = build_condensation(h);
  if (!rc) rc = build_symbolic(h);
  if (!rc) rc = build_new_order(h);
  if (!rc) rc = launch_condense(h);
  if (rc) return rc;
  h.analyzed = true;
  const Symbolic &S = h.sym;
  h.st[0] = (double)S.n;
  h.st[1] = S.nfront;
  h.st[2] = S.max_m;
  h.st[3] = S.flops;
  h.st[4] = S.nnz_lu;
  h.st[5] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  h.st[13] = S.nlevel;
  return SS_OK;
}

extern "C" int ss_set_damping(ss_handle *hp, double beta) {
  H_CHECK(hp);
  if (!std::isfinite(beta) || beta < 0.0) return fail(h, SS_EINVAL, "damping: beta must be finite and >= 0");
  if (beta != 0.0 && !h.have_D) return fail(h, SS_ESTATE, "damping: assemble D first (damping materials, or ss_set_values)");
  h.beta = beta;
  h.scale_w = -1;
  free_plans(h);   // the captured launch graphs bake beta and the damping matrix in
  return SS_OK;
}

extern "C" int ss_sweep(ss_handle *hp, int n_f, const double *omega, double V, int precision, double *Q, int *status,
                        int *iters) {
  H_CHECK(hp);
  if (!h.analyzed) return fail(h, SS_ESTATE, "sweep: analyze first");
  if (n_f < 0 || (n_f > 0 && (!omega || !Q))) return fail(h, SS_EINVAL, "sweep: bad frequency arrays");
  if (precision != SS_PREC_FP64 && precision != SS_PREC_MIXED && precision != SS_PREC_AUTO)
    return fail(h, SS_EINVAL, "sweep: bad precision");
  if (V == 0.0 || !std::isfinite(V)) return fail(h, SS_EINVAL, "sweep: V must be nonzero and finite");
  for (int i = 0; i < n_f; ++i)
    if (!(omega[i] > 0.0) || !std::isfinite(omega[i])) return fail(h, SS_EINVAL, "sweep: omega must be positive and finite");
  if (n_f == 0) return SS_OK;
  return run_sweep(h, n_f, omega, V, precision, Q, status, iters, nullptr);
}

extern "C" int ss_solve_fields(ss_handle *hp, double omega, double V, double *disp, double *Q) {
  H_CHECK(hp);
  if (!h.analyzed) return fail(h, SS_ESTATE, "fields: analyze first");
  if (!disp || !(omega > 0.0) || V == 0.0) return fail(h, SS_EINVAL, "fields: bad arguments");
  double q[2];
  int st = 0, it = 0;
  const int rc = run_sweep(h, 1, &omega, V, SS_PREC_FP64, q, &st, &it, disp);
  if (rc == SS_OK && Q) Q[0] = q[0], Q[1] = q[1];
  return rc;
}

extern "C" int ss_stats(const ss_handle *hp, double *out, int n) {
  if (!hp || !out || n < 0) return SS_EINVAL;
  for (int i = 0; i < n && i < Handle::kStats; ++i) out[i] = hp->h.st[i];
  for (int i = Handle::kStats; i < n; ++i) out[i] = 0.0;
  return SS_OK;
}

extern "C" int ss_set_option(ss_handle *hp, const char *name, double value) {
  H_CHECK(hp);
  if (!name) return fail(h, SS_EINVAL, "option: null name");
  const std::string k(name);
  Handle::Options &o = h.opt;
  auto whole = [&](double lo, double hi) { return value == std::floor(value) && value >= lo && value <= hi; };
  if (k == "krylov_restart") {
    if (!whole(1, 200)) return fail(h, SS_EINVAL, "option krylov_restart: integer in [1, 200]");
    o.krylov_m = (int)value;
  } else if (k == "krylov_cycles") {
    if (!whole(1, 100)) return fail(h, SS_EINVAL, "option krylov_cycles: integer in [1, 100]");
    o.krylov_cycles = (int)value;
  } else if (k == "krylov_tol") {
    if (!(value > 0.0 && value < 1.0)) return fail(h, SS_EINVAL, "option krylov_tol: in (0, 1)");
    o.krylov_tol = value;
  } else if (k == "pivot_tiny_c128" || k == "pivot_tiny_c64") {
    if (!(value >= 0.0 && value < 1.0)) return fail(h, SS_EINVAL, "option pivot_tiny: in [0, 1)");
    (k == "pivot_tiny_c128" ? o.tiny_c128 : o.tiny_c64) = value;
    free_plans(h);   // the captured factorisation graphs bake the threshold in
  } else if (k == "fp64_fallback") {
    if (!whole(0, 1)) return fail(h, SS_EINVAL, "option fp64_fallback: 0 or 1");
    o.fp64_fallback = (int)value;
  } else if (k == "auto_probe_steps") {
    if (!whole(1, 200)) return fail(h, SS_EINVAL, "option auto_probe_steps: integer in [1, 200]");
    o.auto_probe_m = (int)value;
  } else {
    return fail(h, SS_EINVAL, "option: unknown name '" + k + "'");
  }
  h.auto_prec = -1;   // a kept SS_PREC_AUTO decision was taken under the old options
  return SS_OK;
}

extern "C" int ss_solve_adjoint(ss_handle *hp, double omega, int precision, double *lambda) {
  H_CHECK(hp);
  if (!h.analyzed) return fail(h, SS_ESTATE, "adjoint: analyze first");
  if (!lambda || !(omega > 0.0)) return fail(h, SS_EINVAL, "adjoint: bad arguments");
  if (precision != SS_PREC_FP64 && precision != SS_PREC_MIXED) return fail(h, SS_EINVAL, "adjoint: bad precision");
  const int64_t n = h.sym.n;
  std::vector<cplx_d> mu(n);
  std::vector<double> rs(n);
  SweepExtra ex;
  ex.per_chunk = [&](int, int, const cplx<double> *, const cplx<double> *dmu) -> int {
    cudaError_t e = cudaMemcpyAsync(mu.data(), dmu, n * sizeof(cplx_d), cudaMemcpyDeviceToHost, h.stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(rs.data(), h.drow_scale.p, n * sizeof(double), cudaMemcpyDeviceToHost, h.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h.stream);
    return e == cudaSuccess ? SS_OK : cuda_fail(h, e, "adjoint copy");
  };
  double Q[2];
  int st = 0, it = 0;
  int rc = run_sweep(h, 1, &omega, 1.0, precision, Q, &st, &it, nullptr, &ex);
  if (rc) return rc;
  // lambda = Dr mu' in the reference's active-DOF order
  for (int64_t P = 0; P < n; ++P) {
    const int64_t R = h.sym.new_of_act[P];
    lambda[2 * P] = mu[R].re * rs[R];
    lambda[2 * P + 1] = mu[R].im * rs[R];
  }
  return st;
}

extern "C" int ss_adjoint_gradient(ss_handle *hp, int n_f, const double *omega, double V, int precision,
                                   int n_params, const double *dpos, const double *dC, const double *de,
                                   const double *deps, const double *drho, const double *dinner,
                                   const double *douter, double *Q, double *dQ, int *status) {
  H_CHECK(hp);
  if (!h.analyzed) return fail(h, SS_ESTATE, "gradient: analyze first");
  if (h.kind == SS_MATRIX) return fail(h, SS_ESTATE, "gradient: the element derivatives need a mesh (ss_set_mesh)");
  if (n_f <= 0 || !omega || !Q || !dQ || n_params <= 0) return fail(h, SS_EINVAL, "gradient: bad arguments");
  if (precision != SS_PREC_FP64 && precision != SS_PREC_MIXED && precision != SS_PREC_AUTO)
    return fail(h, SS_EINVAL, "gradient: bad precision");
  if (V == 0.0) return fail(h, SS_EINVAL, "gradient: V must be nonzero");
  for (int i = 0; i < n_f; ++i)
    if (!(omega[i] > 0.0)) return fail(h, SS_EINVAL, "gradient: omega must be positive");
  return run_adjoint_gradient(h, n_f, omega, V, precision, n_params, dpos, dC, de, deps, drho, dinner, douter, Q,
                              dQ, status);
}

extern "C" int ss_measure_gemm_ceiling(ss_handle *hp, int kernel, int m, int k, int n_fronts, int reps,
                                       double *tflops) {
  H_CHECK(hp);
  if (!tflops || kernel < 0 || kernel > 6 || k <= 0 || m <= k || n_fronts <= 0 || reps <= 0 || reps > 1000)
    return fail(h, SS_EINVAL, "ceiling: bad arguments");
  if ((double)n_fronts * m * m * 16.0 > 64e9) return fail(h, SS_EINVAL, "ceiling: more than 64 GB of fronts");
  return measure_ceiling(h, kernel, m, k, n_fronts, reps, tflops);
}
