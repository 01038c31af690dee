// Host-only analysis of a system: the global pattern, the Bloch fold and the
// condensation to the active DOFs, the nested-dissection ordering and the
// multifrontal front tree, computed by the same host code that ss_analyze runs
// (symbolic.cpp) on a local handle that never touches a CUDA device.  Callers
// use it to see front sizes, fill, flops and the per-point front memory of a
// cell before they run it on a GPU; the tests use it to check the analysis on a
// machine without one.  Two inputs, as for the handle: a mesh (ss_set_mesh) or
// an assembled pattern with optional node map and coordinates (ss_set_csr).
#include "ss_internal.h"

#include <algorithm>
#include <cmath>

namespace ss {
int build_new_order(Handle &h);
}  // namespace ss

using namespace ss;

namespace {

// Boundary sets (checked as ss_set_bc checks them), the analysis, and the outputs
// of ss_analyze_host / ss_analyze_host_csr.
int analyze_and_report(Handle &h, int64_t n_fix, const int64_t *fix, int64_t n_zheng, const int64_t *zheng,
                       int64_t n_fu, const int64_t *fu, int64_t n_groups, const int64_t *group_ptr,
                       const int64_t *group_dofs, int64_t two_stage, int64_t *sizes, double *stats, int64_t *active,
                       int64_t *order, int32_t *k, int32_t *m, int32_t *parent, int32_t *level, int64_t *rows_ptr,
                       int64_t *rows) {
  const int64_t gdof = h.gdof;
  if ((n_fix && !fix) || (n_zheng && !zheng) || (n_fu && !fu) || (n_groups && (!group_ptr || !group_dofs)))
    return SS_EINVAL;
  if (n_fix < 0 || n_zheng <= 0 || n_fu < 0 || n_groups < 0 || two_stage < 0 || two_stage > n_groups)
    return SS_EINVAL;
  auto in = [&](const int64_t *p, int64_t cnt) {
    for (int64_t i = 0; i < cnt; ++i)
      if (p[i] < 0 || p[i] >= gdof) return false;
    return true;
  };
  if (!in(fix, n_fix) || !in(zheng, n_zheng) || !in(fu, n_fu)) return SS_EINVAL;
  h.fix.assign(fix, fix + n_fix);
  h.zheng.assign(zheng, zheng + n_zheng);
  h.fu.assign(fu, fu + n_fu);
  if (n_groups == 0) {
    h.gptr.assign(1, 0);
  } else {
    h.gptr.assign(group_ptr, group_ptr + n_groups + 1);
    if (h.gptr[0] != 0) return SS_EINVAL;
    for (int64_t g = 0; g < n_groups; ++g)
      if (h.gptr[g + 1] < h.gptr[g]) return SS_EINVAL;
  }
  h.gdofs.assign(group_dofs, group_dofs + h.gptr.back());
  if (!in(h.gdofs.data(), (int64_t)h.gdofs.size())) return SS_EINVAL;
  h.two_stage = two_stage;
  h.have_bc = true;
  int rc = build_condensation(h);
  if (!rc) rc = build_symbolic(h);
  if (!rc) rc = build_new_order(h);
  if (rc) return rc;
  const Symbolic &S = h.sym;
  sizes[0] = S.n;
  sizes[1] = S.nfront;
  sizes[2] = S.rows_ptr[S.nfront];
  sizes[3] = S.nlevel;
  stats[0] = S.flops;
  stats[1] = S.nnz_lu;
  stats[2] = S.max_m;
  stats[3] = S.max_k;
  stats[4] = (double)S.arena;
  stats[5] = (double)h.c_nnz;
  if (active) std::copy(h.active.begin(), h.active.end(), active);
  if (order) std::copy(S.new_of_act.begin(), S.new_of_act.end(), order);
  if (k) std::copy(S.k.begin(), S.k.end(), k);
  if (m) std::copy(S.m.begin(), S.m.end(), m);
  if (parent) std::copy(S.parent.begin(), S.parent.end(), parent);
  if (level) std::copy(S.level.begin(), S.level.end(), level);
  if (rows_ptr) std::copy(S.rows_ptr.begin(), S.rows_ptr.end(), rows_ptr);
  if (rows) std::copy(S.rows.begin(), S.rows.end(), rows);
  return SS_OK;
}

}  // namespace

extern "C" int ss_analyze_host(int element_kind, int64_t n_nodes, const double *pos, int64_t n_elem,
                               const int64_t *conn, int64_t gdof, int64_t n_fix, const int64_t *fix,
                               int64_t n_zheng, const int64_t *zheng, int64_t n_fu, const int64_t *fu,
                               int64_t n_groups, const int64_t *group_ptr, const int64_t *group_dofs,
                               int64_t two_stage, int64_t *sizes, double *stats, int64_t *active, int64_t *order,
                               int32_t *k, int32_t *m, int32_t *parent, int32_t *level, int64_t *rows_ptr,
                               int64_t *rows) {
  if (element_kind < SS_Q9_ME0 || element_kind > SS_HEX27) return SS_EINVAL;
  if (n_nodes <= 0 || n_elem <= 0 || !pos || !conn || !sizes || !stats) return SS_EINVAL;
  Handle h;   // host fields only: no device, no stream, no device buffers
  h.device = -1;
  h.kind = element_kind;
  h.npe = element_kind == SS_HEX27 ? 27 : 9;
  h.dim = element_kind == SS_HEX27 ? 3 : 2;
  h.nc = element_kind == SS_Q9_ME0 ? 3 : 4;
  h.N = n_nodes;
  h.ne = n_elem;
  for (int64_t i = 0; i < n_nodes * h.dim; ++i)
    if (!std::isfinite(pos[i])) return SS_EINVAL;
  for (int64_t i = 0; i < n_elem * h.npe; ++i)
    if (conn[i] < 0 || conn[i] >= n_nodes) return SS_EINVAL;
  h.pos.assign(pos, pos + n_nodes * h.dim);
  h.conn.assign(conn, conn + n_elem * h.npe);
  const int rc = build_global_pattern(h);
  if (rc) return rc;
  if (gdof != h.gdof) return SS_EINVAL;
  return analyze_and_report(h, n_fix, fix, n_zheng, zheng, n_fu, fu, n_groups, group_ptr, group_dofs, two_stage,
                            sizes, stats, active, order, k, m, parent, level, rows_ptr, rows);
}

extern "C" int ss_analyze_host_csr(int64_t gdof, const int64_t *indptr, const int64_t *indices, int64_t n_nodes,
                                   int dim, const int64_t *dof_node, const double *node_xyz, int64_t n_fix,
                                   const int64_t *fix, int64_t n_zheng, const int64_t *zheng, int64_t n_fu,
                                   const int64_t *fu, int64_t n_groups, const int64_t *group_ptr,
                                   const int64_t *group_dofs, int64_t two_stage, int64_t *sizes, double *stats,
                                   int64_t *active, int64_t *order, int32_t *k, int32_t *m, int32_t *parent,
                                   int32_t *level, int64_t *rows_ptr, int64_t *rows) {
  // the pattern and node data, checked as ss_set_csr checks them
  if (gdof <= 0 || !indptr || !indices || !sizes || !stats || indptr[0] != 0) return SS_EINVAL;
  for (int64_t r = 0; r < gdof; ++r) {
    if (indptr[r + 1] < indptr[r]) return SS_EINVAL;
    for (int64_t s = indptr[r]; s < indptr[r + 1]; ++s)
      if (indices[s] < 0 || indices[s] >= gdof || (s > indptr[r] && indices[s] <= indices[s - 1])) return SS_EINVAL;
  }
  if (node_xyz && !dof_node) return SS_EINVAL;
  if (dof_node) {
    if (n_nodes <= 0) return SS_EINVAL;
    for (int64_t d = 0; d < gdof; ++d)
      if (dof_node[d] < 0 || dof_node[d] >= n_nodes) return SS_EINVAL;
  }
  if (node_xyz && (dim < 2 || dim > 3)) return SS_EINVAL;
  if (node_xyz)
    for (int64_t i = 0; i < n_nodes * dim; ++i)
      if (!std::isfinite(node_xyz[i])) return SS_EINVAL;
  Handle h;   // host fields only
  h.device = -1;
  h.kind = SS_MATRIX;
  h.N = dof_node ? n_nodes : 0;
  h.dim = node_xyz ? dim : 0;
  if (node_xyz) h.pos.assign(node_xyz, node_xyz + n_nodes * dim);
  if (dof_node) h.dof_node.assign(dof_node, dof_node + gdof);
  h.gdof = gdof;
  h.indptr.assign(indptr, indptr + gdof + 1);
  h.nnz = h.indptr[gdof];
  h.indices.assign(indices, indices + h.nnz);
  return analyze_and_report(h, n_fix, fix, n_zheng, zheng, n_fu, fu, n_groups, group_ptr, group_dofs, two_stage,
                            sizes, stats, active, order, k, m, parent, level, rows_ptr, rows);
}
