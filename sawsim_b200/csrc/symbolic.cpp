// Host setup: global sparsity pattern, Bloch condensation maps, fill-reducing
// nested dissection and the multifrontal symbolic factorisation.
//
// Pattern and fold semantics follow the reference:
//  * global K/M pattern: every element scatters all nc x nc component blocks of
//    all its node pairs and COO->CSR keeps explicit zeros
//    (src/sawsim/saw2d/piezo_fem.py:318-365);
//  * fold: union-find master/slave with the first-listed master as the class root
//    (src/sawsim/saw2d/sweep.py:97-144), or the two-stage front/back then
//    left/right fold of src/sawsim/saw2d/saw3d/bc_solve.py:25-44;
//  * active DOFs = all minus (fix, slaves, + electrode, - electrode), ascending
//    (sweep.py:296-299, bc_solve.py:47-53, :131-132).
#include "ss_internal.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>

namespace ss {

static inline int64_t dof_of(const Handle &h, int64_t node, int c) {
  if (h.kind == SS_HEX27) return c < 3 ? 3 * node + c : 3 * h.N + node;
  return (int64_t)c * h.N + node;
}
static inline int64_t node_of_dof(const Handle &h, int64_t d) {
  if (h.kind == SS_MATRIX) return h.dof_node[d];
  if (h.kind == SS_HEX27) return d < 3 * h.N ? d / 3 : d - 3 * h.N;
  return d % h.N;
}

int build_global_pattern(Handle &h) {
  const int64_t N = h.N;
  // node adjacency: all node pairs sharing an element (self included)
  std::vector<std::vector<int64_t>> adj(N);
  for (int64_t e = 0; e < h.ne; ++e) {
    const int64_t *c = &h.conn[e * h.npe];
    for (int a = 0; a < h.npe; ++a)
      for (int b = 0; b < h.npe; ++b) adj[c[a]].push_back(c[b]);
  }
  h.nadj_ptr.assign(N + 1, 0);
  for (int64_t i = 0; i < N; ++i) {
    auto &v = adj[i];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    h.nadj_ptr[i + 1] = h.nadj_ptr[i] + (int64_t)v.size();
  }
  h.nadj.resize(h.nadj_ptr[N]);
  for (int64_t i = 0; i < N; ++i) std::copy(adj[i].begin(), adj[i].end(), h.nadj.begin() + h.nadj_ptr[i]);
  adj.clear();
  adj.shrink_to_fit();

  const int nc = h.nc;
  h.gdof = (int64_t)nc * N;
  h.indptr.assign(h.gdof + 1, 0);
  for (int64_t i = 0; i < N; ++i)
    for (int a = 0; a < nc; ++a) h.indptr[dof_of(h, i, a) + 1] = (int64_t)nc * (h.nadj_ptr[i + 1] - h.nadj_ptr[i]);
  for (int64_t r = 0; r < h.gdof; ++r) h.indptr[r + 1] += h.indptr[r];
  h.nnz = h.indptr[h.gdof];
  h.indices.resize(h.nnz);
  for (int64_t i = 0; i < N; ++i) {
    const int64_t d = h.nadj_ptr[i + 1] - h.nadj_ptr[i];
    const int64_t *nb = &h.nadj[h.nadj_ptr[i]];
    for (int a = 0; a < nc; ++a) {
      int64_t *out = &h.indices[h.indptr[dof_of(h, i, a)]];
      if (h.kind == SS_HEX27) {
        for (int64_t r = 0; r < d; ++r)
          for (int b = 0; b < 3; ++b) out[3 * r + b] = 3 * nb[r] + b;
        for (int64_t r = 0; r < d; ++r) out[3 * d + r] = 3 * N + nb[r];
      } else {
        for (int b = 0; b < nc; ++b)
          for (int64_t r = 0; r < d; ++r) out[b * d + r] = (int64_t)b * N + nb[r];
      }
    }
  }
  return SS_OK;
}

// slot of global entry (row dof of node i comp a, col dof of node j comp b) with
// j the r-th neighbour of i
int64_t global_slot(const Handle &h, int64_t i, int a, int64_t r, int b) {
  const int64_t d = h.nadj_ptr[i + 1] - h.nadj_ptr[i];
  const int64_t base = h.indptr[dof_of(h, i, a)];
  if (h.kind == SS_HEX27) return base + (b < 3 ? 3 * r + b : 3 * d + r);
  return base + (int64_t)b * d + r;
}

// ---------------------------------------------------------------- fold maps
static void fold_union_find(const Handle &h, int64_t g0, int64_t g1, std::vector<int64_t> &parent) {
  // parent[] preset to identity; union s -> root of master (sweep.py:114-126)
  auto find = [&](int64_t x) {
    while (parent[x] != x) {
      parent[x] = parent[parent[x]];
      x = parent[x];
    }
    return x;
  };
  for (int64_t g = g0; g < g1; ++g) {
    const int64_t b = h.gptr[g], e = h.gptr[g + 1];
    if (e <= b) continue;
    const int64_t m = h.gdofs[b];
    for (int64_t t = b + 1; t < e; ++t) {
      int64_t rs = find(h.gdofs[t]), rm = find(m);
      if (rs != rm) parent[rs] = rm;
    }
  }
  for (int64_t x = 0; x < (int64_t)parent.size(); ++x) parent[x] = find(x);
}

static void fold_single_stage(const Handle &h, int64_t g0, int64_t g1, std::vector<int64_t> &rep) {
  // slave takes its paired master's value, no transitive closure (bc_solve.py:25-33)
  for (int64_t g = g0; g < g1; ++g) {
    const int64_t b = h.gptr[g], e = h.gptr[g + 1];
    for (int64_t t = b + 1; t < e; ++t) rep[h.gdofs[t]] = h.gdofs[b];
  }
}

int build_fold(Handle &h, std::vector<char> &is_slave) {
  const int64_t G = h.gdof;
  const int64_t ng = (int64_t)h.gptr.size() - 1;
  h.rep.resize(G);
  std::iota(h.rep.begin(), h.rep.end(), 0);
  is_slave.assign(G, 0);
  if (h.two_stage > 0) {
    std::vector<int64_t> fb(G), lr(G);
    std::iota(fb.begin(), fb.end(), 0);
    std::iota(lr.begin(), lr.end(), 0);
    fold_single_stage(h, 0, h.two_stage, fb);
    fold_single_stage(h, h.two_stage, ng, lr);
    for (int64_t i = 0; i < G; ++i) {
      h.rep[i] = lr[fb[i]];
      is_slave[i] = (fb[i] != i) || (lr[i] != i);
    }
  } else {
    fold_union_find(h, 0, ng, h.rep);
    for (int64_t i = 0; i < G; ++i) is_slave[i] = h.rep[i] != i;
  }
  return SS_OK;
}

}  // namespace ss

namespace ss {

// Condensed active system on the structural pattern: entry (P, Q) gathers every
// global slot (i, j) with rep(i) = active[P], rep(j) = active[Q], i.e. the
// entries of (T^T K T)[active][:, active] (sweep.py:293, :308).  Also the
// gathers of Km_s (= Mm_s, Dm_s lists) and of the charge vector kts folded onto
// the active DOFs (sweep.py:301-305, :356-362).
int build_condensation(Handle &h) {
  std::vector<char> is_slave;
  build_fold(h, is_slave);
  const int64_t G = h.gdof;
  std::vector<char> presc(G, 0), inz(G, 0), inf(G, 0);
  for (int64_t d : h.fix) presc[d] = 1;
  for (int64_t d : h.zheng) presc[d] = 1, inz[d] = 1;
  for (int64_t d : h.fu) presc[d] = 1, inf[d] = 1;
  for (int64_t d = 0; d < G; ++d)
    if (is_slave[d]) presc[d] = 1;
  h.active.clear();
  h.act_of_gdof.assign(G, -1);
  for (int64_t d = 0; d < G; ++d)
    if (!presc[d]) {
      h.act_of_gdof[d] = (int64_t)h.active.size();
      h.active.push_back(d);
    }
  const int64_t n = (int64_t)h.active.size();
  if (n == 0) return fail(h, SS_EINVAL, "no active DOFs after boundary conditions");

  // active index of each DOF's representative, -1 when prescribed
  std::vector<int64_t> ar(G);
  for (int64_t d = 0; d < G; ++d) ar[d] = h.act_of_gdof[h.rep[d]];

  // bucket the (Q, slot) contributions by condensed row P
  std::vector<int64_t> cnt(n + 1, 0);
  for (int64_t i = 0; i < G; ++i) {
    const int64_t P = ar[i];
    if (P < 0) continue;
    for (int64_t s = h.indptr[i]; s < h.indptr[i + 1]; ++s)
      if (ar[h.indices[s]] >= 0) ++cnt[P + 1];
  }
  for (int64_t P = 0; P < n; ++P) cnt[P + 1] += cnt[P];
  std::vector<std::pair<int64_t, int64_t>> qs(cnt[n]);
  std::vector<int64_t> fillp(cnt.begin(), cnt.end() - 1);
  for (int64_t i = 0; i < G; ++i) {
    const int64_t P = ar[i];
    if (P < 0) continue;
    for (int64_t s = h.indptr[i]; s < h.indptr[i + 1]; ++s) {
      const int64_t Q = ar[h.indices[s]];
      if (Q >= 0) qs[fillp[P]++] = {Q, s};
    }
  }
  h.a_ptr.assign(n + 1, 0);
  h.a_idx.clear();
  h.ag_ptr.assign(1, 0);
  h.ag_src.resize(qs.size());
  int64_t w = 0;
  for (int64_t P = 0; P < n; ++P) {
    std::sort(qs.begin() + cnt[P], qs.begin() + cnt[P + 1]);
    for (int64_t t = cnt[P]; t < cnt[P + 1]; ++t) {
      if (t == cnt[P] || qs[t].first != qs[t - 1].first) {
        h.a_idx.push_back(qs[t].first);
        h.ag_ptr.push_back(w);
      }
      h.ag_src[w++] = qs[t].second;
      h.ag_ptr.back() = w;
    }
    h.a_ptr[P + 1] = (int64_t)h.a_idx.size();
  }
  // ag_ptr currently holds end offsets per entry; shift into begin/end form
  {
    std::vector<int64_t> p(h.a_idx.size() + 1, 0);
    for (size_t t = 0; t < h.a_idx.size(); ++t) p[t + 1] = h.ag_ptr[t + 1];
    h.ag_ptr.swap(p);
  }
  qs.clear();
  qs.shrink_to_fit();

  // vector gathers: ks[P] over rows rep(i)=P, cols rep(j) in zheng; kq[P] over
  // rows i in zheng, cols j not in zheng/fu with rep(j) = P; Qz over zheng x zheng
  std::vector<std::vector<int64_t>> ks(n), kq(n);
  h.qz_src.clear();
  for (int64_t i = 0; i < G; ++i) {
    const int64_t P = ar[i];
    for (int64_t s = h.indptr[i]; s < h.indptr[i + 1]; ++s) {
      const int64_t j = h.indices[s];
      if (P >= 0 && inz[h.rep[j]]) ks[P].push_back(s);
      if (inz[i]) {
        if (inz[j]) h.qz_src.push_back(s);
        else if (!inf[j] && ar[j] >= 0) kq[ar[j]].push_back(s);
      }
    }
  }
  h.vg_ptr.assign(2 * n + 1, 0);
  h.vg_src.clear();
  for (int64_t P = 0; P < n; ++P) {
    h.vg_src.insert(h.vg_src.end(), ks[P].begin(), ks[P].end());
    h.vg_ptr[P + 1] = (int64_t)h.vg_src.size();
  }
  for (int64_t P = 0; P < n; ++P) {
    std::sort(kq[P].begin(), kq[P].end());
    h.vg_src.insert(h.vg_src.end(), kq[P].begin(), kq[P].end());
    h.vg_ptr[n + P + 1] = (int64_t)h.vg_src.size();
  }
  // supervariables: active DOFs of one mesh node
  h.sv_of_act.resize(n);
  h.sv_xyz.clear();
  h.nsv = 0;
  if (h.kind == SS_MATRIX && h.dof_node.empty()) {
    // no node map: active DOFs whose condensed rows hold the same columns
    // (indistinguishable in the elimination) form one supervariable
    std::vector<uint64_t> hv(n);
    for (int64_t P = 0; P < n; ++P) {
      uint64_t x = 1469598103934665603ull ^ (uint64_t)(h.a_ptr[P + 1] - h.a_ptr[P]);
      for (int64_t t = h.a_ptr[P]; t < h.a_ptr[P + 1]; ++t) x = (x ^ (uint64_t)h.a_idx[t]) * 1099511628211ull;
      hv[P] = x;
    }
    std::vector<int64_t> by(n);
    std::iota(by.begin(), by.end(), 0);
    std::sort(by.begin(), by.end(), [&](int64_t a, int64_t b) { return hv[a] != hv[b] ? hv[a] < hv[b] : a < b; });
    auto same = [&](int64_t a, int64_t b) {
      return hv[a] == hv[b] && h.a_ptr[a + 1] - h.a_ptr[a] == h.a_ptr[b + 1] - h.a_ptr[b] &&
             std::equal(h.a_idx.begin() + h.a_ptr[a], h.a_idx.begin() + h.a_ptr[a + 1], h.a_idx.begin() + h.a_ptr[b]);
    };
    // group leader = the smallest P of its group; ids in ascending leader order
    std::vector<int64_t> lead(n);
    for (int64_t i = 0; i < n;) {
      int64_t j = i;
      while (j < n && hv[by[j]] == hv[by[i]]) ++j;
      // within one hash bucket, match each DOF against the bucket's earlier leaders
      std::vector<int64_t> leaders;
      for (int64_t t = i; t < j; ++t) {
        const int64_t P = by[t];
        int64_t L = -1;
        for (int64_t q : leaders)
          if (same(q, P)) { L = q; break; }
        if (L < 0) leaders.push_back(L = P);
        lead[P] = L;
      }
      i = j;
    }
    std::vector<int64_t> sv_of_lead(n, -1);
    for (int64_t P = 0; P < n; ++P) {
      const int64_t L = lead[P];
      if (sv_of_lead[L] < 0) sv_of_lead[L] = h.nsv++;
      h.sv_of_act[P] = sv_of_lead[L];
    }
    return SS_OK;
  }
  std::vector<int64_t> sv_of_node(h.N, -1);
  for (int64_t P = 0; P < n; ++P) {
    const int64_t nd = node_of_dof(h, h.active[P]);
    if (sv_of_node[nd] < 0) {
      sv_of_node[nd] = h.nsv++;
      if (!h.pos.empty())
        for (int c = 0; c < 3; ++c) h.sv_xyz.push_back(c < h.dim ? h.pos[nd * h.dim + c] : 0.0);
    }
    h.sv_of_act[P] = sv_of_node[nd];
  }
  return SS_OK;
}

}  // namespace ss

namespace ss {

// ------------------------------------------------------------------------------
// Geometric nested dissection on the supervariable (mesh node) graph of the
// condensed system.  A subset is split by a coordinate cut; the vertex
// separator is the boundary of the cut on its smaller side.  Candidate cuts
// around the median on every axis are scored by |S| / balance, so a Bloch
// cylinder is cut into rings before it is cut lengthwise.  The separator tree is
// the assembly tree: leaves are whole subdomains, interior fronts separators.
// Without coordinates (assembled-matrix input) the cut is a breadth-first level
// set from a pseudo-peripheral supervariable (George and Liu's level structure),
// chosen among the levels that leave at least a quarter of the set on each side
// by the same |S| / balance score and trimmed to its vertices that touch the next
// level.
// ------------------------------------------------------------------------------
struct ND {
  const std::vector<int64_t> &ap, &aj;   // supervariable adjacency
  const std::vector<double> &xyz;
  int dim;
  int leaf;
  std::vector<int64_t> stamp, side;
  int64_t tick = 0;
  std::vector<int64_t> vis, lvl;         // breadth-first search marks and levels
  int64_t vtick = 0;
  std::vector<std::vector<int64_t>> piv;  // pivots (supervariables) per front
  std::vector<std::vector<int>> kids;

  ND(const std::vector<int64_t> &p, const std::vector<int64_t> &j, const std::vector<double> &x, int d, int lf,
     int64_t n)
      : ap(p), aj(j), xyz(x), dim(d), leaf(lf), stamp(n, -1), side(n, 0), vis(n, -1), lvl(n, 0) {}

  // breadth-first levels of the set stamped t from root: level l is
  // order[lptr[l] .. lptr[l+1]); returns the number of levels
  int64_t bfs(int64_t root, int64_t t, std::vector<int64_t> &order, std::vector<int64_t> &lptr) {
    const int64_t mark = ++vtick;
    order.clear();
    lptr.assign(1, 0);
    order.push_back(root);
    vis[root] = mark;
    lvl[root] = 0;
    int64_t cur = 0;
    for (size_t head = 0; head < order.size(); ++head) {
      const int64_t v = order[head];
      if (lvl[v] != cur) {
        lptr.push_back((int64_t)head);
        cur = lvl[v];
      }
      for (int64_t q = ap[v]; q < ap[v + 1]; ++q) {
        const int64_t w = aj[q];
        if (stamp[w] == t && vis[w] != mark) {
          vis[w] = mark;
          lvl[w] = lvl[v] + 1;
          order.push_back(w);
        }
      }
    }
    lptr.push_back((int64_t)order.size());
    return (int64_t)lptr.size() - 1;
  }

  // level-set separator of a connected set stamped t (no coordinates)
  std::vector<int64_t> graph_separator(const std::vector<int64_t> &nodes, int64_t t) {
    const int64_t nn = (int64_t)nodes.size();
    auto deg = [&](int64_t v) { return ap[v + 1] - ap[v]; };
    int64_t r = nodes[0];
    for (int64_t v : nodes)
      if (deg(v) < deg(r)) r = v;
    std::vector<int64_t> order, lptr;
    int64_t nl = bfs(r, t, order, lptr);
    for (int it = 0; it < 8; ++it) {   // pseudo-peripheral root
      int64_t c = order[lptr[nl - 1]];
      for (int64_t i = lptr[nl - 1]; i < lptr[nl]; ++i)
        if (deg(order[i]) < deg(c)) c = order[i];
      std::vector<int64_t> o2, l2;
      const int64_t n2 = bfs(c, t, o2, l2);
      if (n2 <= nl) break;
      order.swap(o2);
      lptr.swap(l2);
      nl = n2;
      r = c;
    }
    if (nl < 3) return nodes;
    nl = bfs(r, t, order, lptr);   // the levels (and marks) of the kept root
    const int64_t mark = vtick;
    // per level: its vertices with a neighbour in the next level
    std::vector<int64_t> touch(nl, 0);
    std::vector<char> keep(order.size(), 0);
    for (int64_t l = 0; l + 1 < nl; ++l)
      for (int64_t i = lptr[l]; i < lptr[l + 1]; ++i) {
        const int64_t v = order[i];
        for (int64_t q = ap[v]; q < ap[v + 1]; ++q) {
          const int64_t w = aj[q];
          if (stamp[w] == t && vis[w] == mark && lvl[w] == l + 1) {
            keep[i] = 1;
            ++touch[l];
            break;
          }
        }
      }
    double best = 1e300;
    int64_t bl = -1;
    for (int64_t l = 1; l + 1 < nl; ++l) {
      const int64_t before = lptr[l + 1] - touch[l], after = nn - lptr[l + 1];
      if (touch[l] == 0 || before <= 0 || after <= 0) continue;
      const double bal = (double)std::min(before, after) / (double)nn;
      if (bal < 0.25) continue;
      const double score = (double)touch[l] / bal;
      if (score < best) best = score, bl = l;
    }
    if (bl < 0) {   // no balanced level: the one holding the median vertex
      bl = std::min<int64_t>(std::max<int64_t>(lvl[order[nn / 2]], 1), nl - 2);
      if (touch[bl] == 0) return nodes;
    }
    std::vector<int64_t> S;
    for (int64_t i = lptr[bl]; i < lptr[bl + 1]; ++i)
      if (keep[i]) S.push_back(order[i]);
    std::sort(S.begin(), S.end());
    return S;
  }

  void components(const std::vector<int64_t> &nodes, std::vector<std::vector<int64_t>> &out) {
    const int64_t t = ++tick;
    for (int64_t v : nodes) stamp[v] = t;
    const int64_t seen = ++tick;
    std::vector<int64_t> st;
    for (int64_t v0 : nodes) {
      if (stamp[v0] != t) continue;
      out.emplace_back();
      auto &cc = out.back();
      stamp[v0] = seen;
      st.push_back(v0);
      while (!st.empty()) {
        int64_t v = st.back();
        st.pop_back();
        cc.push_back(v);
        for (int64_t q = ap[v]; q < ap[v + 1]; ++q) {
          int64_t w = aj[q];
          if (stamp[w] == t) {
            stamp[w] = seen;
            st.push_back(w);
          }
        }
      }
      std::sort(cc.begin(), cc.end());
    }
  }

  // best separator of a connected set
  std::vector<int64_t> separator(const std::vector<int64_t> &nodes) {
    const int64_t nn = (int64_t)nodes.size();
    const int64_t t = ++tick;
    for (int64_t v : nodes) stamp[v] = t;
    if (xyz.empty()) return graph_separator(nodes, t);
    double best = 1e300;
    std::vector<int64_t> bestS;
    std::vector<int64_t> key(nn);
    for (int ax = 0; ax < dim; ++ax) {
      for (int64_t i = 0; i < nn; ++i) key[i] = (int64_t)std::llround(xyz[nodes[i] * 3 + ax] * 1e12);
      std::vector<int64_t> u(key);
      std::sort(u.begin(), u.end());
      const int64_t med = u[nn / 2];
      u.erase(std::unique(u.begin(), u.end()), u.end());
      if (u.size() < 3) continue;
      int64_t k0 = std::lower_bound(u.begin(), u.end(), med) - u.begin();
      for (int64_t kk = std::max<int64_t>(1, k0 - 3); kk <= std::min<int64_t>((int64_t)u.size() - 1, k0 + 3); ++kk) {
        const int64_t cut = u[kk];
        int64_t na = 0;
        for (int64_t i = 0; i < nn; ++i) {
          side[nodes[i]] = key[i] < cut ? 0 : 1;
          na += key[i] < cut;
        }
        const int64_t nb = nn - na;
        if (na == 0 || nb == 0) continue;
        std::vector<int64_t> SA, SB;
        for (int64_t v : nodes) {
          bool touches = false;
          for (int64_t q = ap[v]; q < ap[v + 1] && !touches; ++q) {
            int64_t w = aj[q];
            touches = stamp[w] == t && side[w] != side[v];
          }
          if (touches) (side[v] == 0 ? SA : SB).push_back(v);
        }
        std::vector<int64_t> &S = SA.size() <= SB.size() ? SA : SB;
        const double bal = (double)std::min(na, nb) / (double)nn;
        const double score = (double)S.size() / std::max(bal, 0.2);
        if (score < best) {
          best = score;
          bestS = S;
        }
      }
    }
    if (bestS.empty()) bestS = nodes;  // cannot be cut: one dense front
    return bestS;
  }

  int add_front(std::vector<int64_t> p, std::vector<int> c) {
    piv.push_back(std::move(p));
    kids.push_back(std::move(c));
    return (int)piv.size() - 1;
  }

  void run(const std::vector<int64_t> &nodes, std::vector<int> &roots) {
    std::vector<std::vector<int64_t>> comps;
    components(nodes, comps);
    for (auto &cc : comps) {
      if ((int64_t)cc.size() <= leaf) {
        roots.push_back(add_front(cc, {}));
        continue;
      }
      std::vector<int64_t> S = separator(cc);
      if (S.size() == cc.size()) {
        roots.push_back(add_front(cc, {}));
        continue;
      }
      const int64_t t = ++tick;
      for (int64_t v : S) stamp[v] = t;
      std::vector<int64_t> rest;
      for (int64_t v : cc)
        if (stamp[v] != t) rest.push_back(v);
      std::vector<int> ch;
      run(rest, ch);
      roots.push_back(add_front(S, ch));
    }
  }
};

}  // namespace ss

namespace ss {

int build_symbolic(Handle &h) {
  Symbolic &S = h.sym;
  S = Symbolic();
  const int64_t n = (int64_t)h.active.size();
  const int64_t nsv = h.nsv;
  S.n = n;
  // supervariable -> active dofs, and supervariable graph
  std::vector<int64_t> svp(nsv + 1, 0), svd(n);
  for (int64_t P = 0; P < n; ++P) ++svp[h.sv_of_act[P] + 1];
  for (int64_t v = 0; v < nsv; ++v) svp[v + 1] += svp[v];
  {
    std::vector<int64_t> f(svp.begin(), svp.end() - 1);
    for (int64_t P = 0; P < n; ++P) svd[f[h.sv_of_act[P]]++] = P;
  }
  std::vector<std::vector<int64_t>> sadj(nsv);
  for (int64_t P = 0; P < n; ++P)
    for (int64_t t = h.a_ptr[P]; t < h.a_ptr[P + 1]; ++t) {
      int64_t a = h.sv_of_act[P], b = h.sv_of_act[h.a_idx[t]];
      if (a != b) sadj[a].push_back(b), sadj[b].push_back(a);
    }
  std::vector<int64_t> ap(nsv + 1, 0), aj;
  for (int64_t v = 0; v < nsv; ++v) {
    auto &x = sadj[v];
    std::sort(x.begin(), x.end());
    x.erase(std::unique(x.begin(), x.end()), x.end());
    ap[v + 1] = ap[v] + (int64_t)x.size();
  }
  aj.resize(ap[nsv]);
  for (int64_t v = 0; v < nsv; ++v) std::copy(sadj[v].begin(), sadj[v].end(), aj.begin() + ap[v]);
  sadj.clear();

  // leaf subdomain size: 12 supervariables in 2D, 8 in 3D (without coordinates,
  // 3D is told apart by the mean supervariable degree: ~20 for Q9, ~60 for Hex27)
  int leaf = h.dim == 3 ? 8 : 12;
  if (h.dim == 0 && nsv > 0 && (double)ap[nsv] / (double)nsv > 40.0) leaf = 8;
  if (const char *e = getenv("SS_ND_LEAF")) leaf = std::max(1, atoi(e));
  ND nd(ap, aj, h.sv_xyz, h.dim, leaf, nsv);
  std::vector<int64_t> all(nsv);
  std::iota(all.begin(), all.end(), 0);
  std::vector<int> roots;
  nd.run(all, roots);
  const int nf = (int)nd.piv.size();
  S.nfront = nf;

  // elimination order: fronts in creation (post)order, pivots in sv order
  std::vector<int64_t> sv_order(nsv, -1), front_of_sv(nsv, -1);
  S.new_of_act.assign(n, -1);
  S.act_of_new.assign(n, -1);
  S.p0.assign(nf, 0);
  S.k.assign(nf, 0);
  int64_t nxt = 0, so = 0;
  for (int f = 0; f < nf; ++f) {
    S.p0[f] = nxt;
    for (int64_t v : nd.piv[f]) {
      sv_order[v] = so++;
      front_of_sv[v] = f;
      for (int64_t t = svp[v]; t < svp[v + 1]; ++t) {
        S.new_of_act[svd[t]] = nxt;
        S.act_of_new[nxt] = svd[t];
        ++nxt;
      }
    }
    S.k[f] = (int)(nxt - S.p0[f]);
  }
  S.parent.assign(nf, -1);
  S.child_ptr.assign(nf + 1, 0);
  for (int f = 0; f < nf; ++f) {
    for (int c : nd.kids[f]) S.parent[c] = f;
    S.child_ptr[f + 1] = S.child_ptr[f] + (int64_t)nd.kids[f].size();
  }
  for (int f = 0; f < nf; ++f) S.child.insert(S.child.end(), nd.kids[f].begin(), nd.kids[f].end());

  // update sets at supervariable level, sorted by elimination order
  std::vector<std::vector<int64_t>> U(nf);
  std::vector<int64_t> mark(nsv, -1);
  for (int f = 0; f < nf; ++f) {
    int64_t last = -1;
    for (int64_t v : nd.piv[f]) last = std::max(last, sv_order[v]);
    std::vector<int64_t> u;
    for (int64_t v : nd.piv[f])
      for (int64_t q = ap[v]; q < ap[v + 1]; ++q) {
        int64_t w = aj[q];
        if (sv_order[w] > last && mark[w] != f) mark[w] = f, u.push_back(w);
      }
    for (int64_t c = S.child_ptr[f]; c < S.child_ptr[f + 1]; ++c)
      for (int64_t w : U[S.child[c]])
        if (sv_order[w] > last && mark[w] != f) mark[w] = f, u.push_back(w);
    std::sort(u.begin(), u.end(), [&](int64_t a, int64_t b) { return sv_order[a] < sv_order[b]; });
    U[f].swap(u);
  }
  // dof-level rows
  S.m.assign(nf, 0);
  S.ld.assign(nf, 0);
  S.rows_ptr.assign(nf + 1, 0);
  S.off.assign(nf, 0);
  int64_t off = 0;
  for (int f = 0; f < nf; ++f) {
    int64_t mm = S.k[f];
    for (int64_t w : U[f]) mm += svp[w + 1] - svp[w];
    S.m[f] = (int)mm;
    S.ld[f] = (int)((mm + 3) / 4 * 4);
    S.rows_ptr[f + 1] = S.rows_ptr[f] + mm;
    S.off[f] = off;
    off += ((int64_t)mm * S.ld[f] + 31) / 32 * 32;
    S.max_m = std::max(S.max_m, (int)mm);
    S.max_k = std::max(S.max_k, S.k[f]);
    const double k = S.k[f], r = (double)mm - k;
    S.flops += 8.0 * (k * k * k / 3.0 + k * k * r + k * r * r);
    S.nnz_lu += k * k + 2.0 * k * r;
  }
  S.arena = off;
  S.rows.resize(S.rows_ptr[nf]);
  for (int f = 0; f < nf; ++f) {
    int64_t *r = &S.rows[S.rows_ptr[f]];
    int64_t q = 0;
    for (int i = 0; i < S.k[f]; ++i) r[q++] = S.p0[f] + i;
    for (int64_t w : U[f])
      for (int64_t t = svp[w]; t < svp[w + 1]; ++t) r[q++] = S.new_of_act[svd[t]];
    std::sort(r + S.k[f], r + q);
  }
  // extend-add maps: child CB row -> parent position
  S.relpos_ptr.assign(nf + 1, 0);
  for (int f = 0; f < nf; ++f) S.relpos_ptr[f + 1] = S.relpos_ptr[f] + (S.m[f] - S.k[f]);
  S.relpos.assign(S.relpos_ptr[nf], -1);
  for (int f = 0; f < nf; ++f) {
    const int p = S.parent[f];
    if (p < 0) {
      if (S.m[f] != S.k[f]) return fail(h, SS_EINVAL, "root front with update rows");
      continue;
    }
    const int64_t *pr = &S.rows[S.rows_ptr[p]];
    for (int i = S.k[f]; i < S.m[f]; ++i) {
      const int64_t r = S.rows[S.rows_ptr[f] + i];
      int pos;
      if (r >= S.p0[p] && r < S.p0[p] + S.k[p]) pos = (int)(r - S.p0[p]);
      else {
        const int64_t *it = std::lower_bound(pr + S.k[p], pr + S.m[p], r);
        if (it == pr + S.m[p] || *it != r) return fail(h, SS_EINVAL, "extend-add row missing in parent");
        pos = (int)(it - pr);
      }
      S.relpos[S.relpos_ptr[f] + i - S.k[f]] = pos;
    }
  }
  // levels by height
  S.level.assign(nf, 0);
  for (int f = 0; f < nf; ++f)
    for (int64_t c = S.child_ptr[f]; c < S.child_ptr[f + 1]; ++c)
      S.level[f] = std::max(S.level[f], S.level[S.child[c]] + 1);
  S.nlevel = nf ? 1 + *std::max_element(S.level.begin(), S.level.end()) : 0;
  S.level_ptr.assign(S.nlevel + 1, 0);
  for (int f = 0; f < nf; ++f) ++S.level_ptr[S.level[f] + 1];
  for (int l = 0; l < S.nlevel; ++l) S.level_ptr[l + 1] += S.level_ptr[l];
  S.level_fronts.resize(nf);
  {
    std::vector<int64_t> fl(S.level_ptr.begin(), S.level_ptr.end() - 1);
    for (int f = 0; f < nf; ++f) S.level_fronts[fl[S.level[f]]++] = f;
  }
  return SS_OK;
}

}  // namespace ss

namespace ss {

// Condensed CSR and gathers in elimination order, plus the arrowhead lists that
// place each condensed entry into the front that owns min(row, col).
int build_new_order(Handle &h) {
  Symbolic &S = h.sym;
  const int64_t n = S.n;
  h.c_ptr.assign(n + 1, 0);
  h.c_idx.clear();
  h.c_perm.clear();
  h.c_idx.reserve(h.a_idx.size());
  h.c_perm.reserve(h.a_idx.size());
  std::vector<std::pair<int64_t, int64_t>> row;
  for (int64_t R = 0; R < n; ++R) {
    const int64_t P = S.act_of_new[R];
    row.clear();
    for (int64_t t = h.a_ptr[P]; t < h.a_ptr[P + 1]; ++t) row.push_back({S.new_of_act[h.a_idx[t]], t});
    std::sort(row.begin(), row.end());
    for (auto &x : row) h.c_idx.push_back(x.first), h.c_perm.push_back(x.second);
    h.c_ptr[R + 1] = (int64_t)h.c_idx.size();
  }
  h.c_nnz = (int64_t)h.c_idx.size();
  // front of each pivot
  std::vector<int> fo(n, -1);
  for (int f = 0; f < S.nfront; ++f)
    for (int i = 0; i < S.k[f]; ++i) fo[S.p0[f] + i] = f;
  auto pos_in = [&](int f, int64_t r) -> int64_t {
    if (r >= S.p0[f] && r < S.p0[f] + S.k[f]) return r - S.p0[f];
    const int64_t *b = &S.rows[S.rows_ptr[f]];
    const int64_t *it = std::lower_bound(b + S.k[f], b + S.m[f], r);
    if (it == b + S.m[f] || *it != r) return -1;
    return it - b;
  };
  std::vector<int64_t> cnt(S.nfront + 1, 0);
  std::vector<int> own(h.c_nnz);
  for (int64_t R = 0; R < n; ++R)
    for (int64_t t = h.c_ptr[R]; t < h.c_ptr[R + 1]; ++t) {
      own[t] = fo[std::min(R, h.c_idx[t])];
      ++cnt[own[t] + 1];
    }
  for (int f = 0; f < S.nfront; ++f) cnt[f + 1] += cnt[f];
  S.arrow_ptr = cnt;
  S.arrow_pos.assign(h.c_nnz, 0);
  S.arrow_slot.assign(h.c_nnz, 0);
  std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
  for (int64_t R = 0; R < n; ++R)
    for (int64_t t = h.c_ptr[R]; t < h.c_ptr[R + 1]; ++t) {
      const int f = own[t];
      const int64_t pr = pos_in(f, R), pc = pos_in(f, h.c_idx[t]);
      if (pr < 0 || pc < 0) return fail(h, SS_EINVAL, "condensed entry outside its front");
      const int64_t q = fill[f]++;
      S.arrow_pos[q] = (int32_t)(pr * S.ld[f] + pc);
      S.arrow_slot[q] = t;
    }
  return SS_OK;
}

}  // namespace ss
