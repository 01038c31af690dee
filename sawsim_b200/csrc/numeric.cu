// Numeric phase of the sweep: Bloch condensation on the device, equilibration,
// batched multifrontal LU of A(w) = Kc - w^2 Mc (+ i w beta Dc) over a chunk of
// frequencies that share one symbolic analysis, triangular solves, FP64
// iterative refinement and the electrode charge Q.
//
// Reference semantics (src/sawsim/saw2d/sweep.py:335-364): per frequency
//   rhs = -(Km_s - w^2 Mm_s (+ i w beta Dm_s))[active] V,  A = Km_aa - w^2 Mm_aa,
//   disp[active] = A^-1 rhs, slaves <- masters, zheng <- V, fu <- 0, Q = kts . disp.
// Here Q = kq . x + V * Qz with kq the charge row folded onto the active DOFs.
#include "ss_internal.h"
#include "dev_complex.cuh"
#include "krylov.cuh"
#include "tc_gemm.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>

namespace ss {

// ------------------------------------------------------------------ gathers
// out[t] = sum of src[list[ptr[t] .. ptr[t+1])] in list order (fixed order)
__global__ void gather_sum_kernel(int64_t n, const int64_t *__restrict__ ptr, const int64_t *__restrict__ list,
                                  const cd *__restrict__ src, cd *__restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  cd acc{0.0, 0.0};
  for (int64_t q = ptr[t]; q < ptr[t + 1]; ++q) acc = acc + src[list[q]];
  out[t] = acc;
}

// ------------------------------------------------------------------ equilibration
// Ruiz scaling of |Kc| + w2 |Mc| (+ wb |Dc|): rows then columns to unit max norm.
__global__ void row_absmax_kernel(int64_t n, const int64_t *__restrict__ rp, const int64_t *__restrict__ ci,
                                  const cd *__restrict__ K, const cd *__restrict__ M, const cd *__restrict__ D,
                                  double w2, double wb, const double *__restrict__ rs,
                                  const double *__restrict__ cs, double *__restrict__ rmax,
                                  unsigned long long *__restrict__ cmax) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double m = 0.0;
  for (int64_t t = rp[r]; t < rp[r + 1]; ++t) {
    const int64_t c = ci[t];
    double a = sqrt(cabs2(K[t])) + w2 * sqrt(cabs2(M[t]));
    if (D) a += wb * sqrt(cabs2(D[t]));
    a *= rs[r] * cs[c];
    m = fmax(m, a);
    if (cmax) atomicMax(&cmax[c], (unsigned long long)__double_as_longlong(a));
  }
  rmax[r] = m;
}

__global__ void scale_update_kernel(int64_t n, double *__restrict__ s, const double *__restrict__ mx,
                                    const unsigned long long *__restrict__ cmx) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const double m = cmx ? __longlong_as_double((long long)cmx[r]) : mx[r];
  if (m > 0.0) s[r] /= sqrt(m);
}

// scaled copy: A'[t] = rs[r] * A[t] * cs[c]
__global__ void scale_csr_kernel(int64_t n, const int64_t *__restrict__ rp, const int64_t *__restrict__ ci,
                                 const double *__restrict__ rs, const double *__restrict__ cs,
                                 const cd *__restrict__ in, cd *__restrict__ out) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  for (int64_t t = rp[r]; t < rp[r + 1]; ++t) out[t] = in[t] * (rs[r] * cs[ci[t]]);
}

// ------------------------------------------------------------------ vectors
// scaled right-hand sides for a chunk: b[f][R] = -V rs[R] (ks - w^2 ms + i w beta ds)[R]
__global__ void rhs_kernel(int64_t n, int nb, const double *__restrict__ omega, double V, double beta,
                           const cd *__restrict__ ks, const cd *__restrict__ ms, const cd *__restrict__ ds,
                           const double *__restrict__ rs, cd *__restrict__ b) {
  const int64_t R = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (R >= n || f >= nb) return;
  const double w = omega[f];
  cd v = ks[R] - ms[R] * (w * w);
  if (ds) v = v + cmul(cd{0.0, w * beta}, ds[R]);
  b[(int64_t)f * n + R] = v * (-V * rs[R]);
}

// Q[f] = sum_R kq[R] cs[R] x[f][R] + V Qz, one block per frequency, fixed-order tree
__global__ void charge_kernel(int64_t n, const cd *__restrict__ kq, const double *__restrict__ cs,
                              const cd *__restrict__ x, const cd *__restrict__ Qz, double V, cd *__restrict__ Q) {
  __shared__ cd red[256];
  const int f = blockIdx.x;
  cd acc{0.0, 0.0};
  for (int64_t R = threadIdx.x; R < n; R += blockDim.x)
    acc = acc + cmul(kq[R] * cs[R], x[(int64_t)f * n + R]);
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) Q[f] = red[0] + Qz[0] * V;
}

// r[f] = b[f] - A'(w_f) x[f]   (scaled system, FP64); a thread owns a row for a
// block of kSpmvFreqs frequencies (the row's matrix data read once per block; each
// frequency's sum in the order of a one-frequency product).
// (vp: value slot of each pattern entry, for the transposed operator; nullptr = own slot)
__global__ void residual_kernel(int64_t n, int nb, const int64_t *__restrict__ rp, const int64_t *__restrict__ ci,
                                const int64_t *__restrict__ vp, const cd *__restrict__ K, const cd *__restrict__ M,
                                const cd *__restrict__ D, const double *__restrict__ omega, double beta,
                                const cd *__restrict__ b, const cd *__restrict__ x, cd *__restrict__ r) {
  const int64_t R = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int f0 = blockIdx.y * kSpmvFreqs;
  if (R >= n || f0 >= nb) return;
  const int nf = min(kSpmvFreqs, nb - f0);
  double w2[kSpmvFreqs], wb[kSpmvFreqs];
  cd acc[kSpmvFreqs];
#pragma unroll
  for (int q = 0; q < kSpmvFreqs; ++q) {
    const double w = q < nf ? omega[f0 + q] : 0.0;
    w2[q] = w * w;
    wb[q] = w * beta;
    acc[q] = q < nf ? b[(int64_t)(f0 + q) * n + R] : cd{0.0, 0.0};
  }
  const cd *xb = x + (int64_t)f0 * n;
  for (int64_t t = rp[R]; t < rp[R + 1]; ++t) {
    const int64_t s = vp ? vp[t] : t;
    const int64_t j = ci[t];
    const cd Ks = K[s], Ms = M[s];
    const cd Ds = D ? D[s] : cd{0.0, 0.0};
#pragma unroll
    for (int q = 0; q < kSpmvFreqs; ++q)
      if (q < nf) {
        cd a = Ks - Ms * w2[q];
        if (D) a = a + cmul(cd{0.0, wb[q]}, Ds);
        acc[q] = acc[q] - cmul(a, xb[(int64_t)q * n + j]);
      }
  }
#pragma unroll
  for (int q = 0; q < kSpmvFreqs; ++q)
    if (q < nf) r[(int64_t)(f0 + q) * n + R] = acc[q];
}

}  // namespace ss

namespace ss {

// Everything a front kernel needs; device pointers.
template <class T>
struct FrontArgs {
  const int *fronts;                 // front ids of this launch
  const int *k, *m, *ld;
  const int64_t *off, *p0;
  const int64_t *rows_ptr, *rows;    // front row lists (new indices)
  const int64_t *child_ptr;
  const int *child;
  const int64_t *relpos_ptr;
  const int *relpos;
  const int64_t *arrow_ptr;
  const int32_t *arrow_pos;
  const int64_t *arrow_slot;
  const cd *Kc, *Mc, *Dc;            // scaled condensed values (new order)
  double beta;
  const double *omega;               // chunk frequencies
  cplx<T> *arena;                    // fronts of frequency f at arena + f * stride
  int64_t stride;
  int *piv;                          // piv[f * n + p0 + j] = local pivot row
  int64_t n;
  T tiny;                            // static pivot perturbation threshold
  int *nperturb;
  const int *active;                 // solves: frequencies still iterating (nullptr = all)
};

template <class T>
__device__ inline cplx<T> to_t(cd v) { return cplx<T>{(T)v.x, (T)v.y}; }

// entry of A'(w) at a condensed slot
__device__ inline cd a_entry(const cd *K, const cd *M, const cd *D, int64_t s, double w, double beta) {
  cd v = K[s] - M[s] * (w * w);
  if (D) v = v + cmul(cd{0.0, w * beta}, D[s]);
  return v;
}

// block-wide argmax of |col| over rows [lo, hi) of a column (stride ldc); ties -> lowest row
template <class T, class Get>
__device__ int block_argmax(int lo, int hi, Get get, T *sv, int *si) {
  T best = (T)-1;
  int bi = lo;
  for (int r = lo + threadIdx.x; r < hi; r += blockDim.x) {
    const T v = cabs1(get(r));
    if (v > best) best = v, bi = r;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const T ov = __shfl_down_sync(0xffffffffu, best, o);
    const int oi = __shfl_down_sync(0xffffffffu, bi, o);
    if (ov > best || (ov == best && oi < bi)) best = ov, bi = oi;
  }
  const int wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if ((threadIdx.x & 31) == 0) sv[wid] = best, si[wid] = bi;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < nw; ++q)
      if (sv[q] > sv[0] || (sv[q] == sv[0] && si[q] < si[0])) sv[0] = sv[q], si[0] = si[q];
  }
  __syncthreads();
  const int r = si[0];
  __syncthreads();
  return r;
}

// Fronts small enough for shared memory: one CTA per (front, frequency) assembles
// the front (arrowhead entries of A'(w) + extend-add of the children's update
// blocks), eliminates its k pivots with row pivoting restricted to the k
// fully-summed rows, and writes factors and update block to the arena.  Every
// row-wise loop is one warp per row with the lanes along the columns (no
// per-element index division; conflict-free shared accesses).
constexpr int kSmallThreads = 512;
template <class T>
__global__ void __launch_bounds__(kSmallThreads) front_small_kernel(FrontArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T> *F = reinterpret_cast<cplx<T> *>(smem_raw);
  __shared__ T s_v[kSmallThreads / 32];
  __shared__ int s_i[kSmallThreads / 32];
  __shared__ T s_cv[2][kSmallThreads / 32];      // per-warp pivot candidates, by pivot parity
  __shared__ int s_ci[2][kSmallThreads / 32];
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  const double w = a.omega[fq];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  cplx<T> *arena = a.arena + (int64_t)fq * a.stride;
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) F[t] = cplx<T>{0, 0};
  __syncthreads();
  for (int64_t q = a.arrow_ptr[f] + threadIdx.x; q < a.arrow_ptr[f + 1]; q += blockDim.x) {
    const int pos = a.arrow_pos[q];
    F[(pos / ld) * m + pos % ld] = to_t<T>(a_entry(a.Kc, a.Mc, a.Dc, a.arrow_slot[q], w, a.beta));
  }
  __syncthreads();
  for (int64_t cc = a.child_ptr[f]; cc < a.child_ptr[f + 1]; ++cc) {
    const int ch = a.child[cc];
    const int kc = a.k[ch], nn = a.m[ch] - kc, ldc = a.ld[ch];
    const cplx<T> *CB = arena + a.off[ch] + (int64_t)kc * ldc + kc;
    const int *rel = a.relpos + a.relpos_ptr[ch];
    for (int i = wid; i < nn; i += nw) {
      cplx<T> *d = F + rel[i] * m;
      const cplx<T> *src = CB + (int64_t)i * ldc;
      for (int j = lane; j < nn; j += 32) d[rel[j]] = d[rel[j]] + src[j];
    }
    __syncthreads();
  }
  // One barrier per pivot: while a warp updates its rows for pivot j, lane 0
  // (which owns column j + 1) keeps the largest |F[r][j+1]| over its rows r < k;
  // after the barrier every thread reduces the warps' candidates to the same next
  // pivot row (largest modulus, lowest row on ties), as a block-wide argmax would.
  int *piv = a.piv + (int64_t)fq * a.n + a.p0[f];
  int p = k > 0 ? block_argmax<T>(0, k, [&](int r) { return F[r * m]; }, s_v, s_i) : 0;
  bool pert_prev = false;
  cplx<T> pv_prev{0, 0};
  for (int j = 0; j < k; ++j) {
    if (p != j) {   // p is the same in every thread
      for (int c = threadIdx.x; c < m; c += blockDim.x) {
        const cplx<T> t = F[j * m + c];
        F[j * m + c] = F[p * m + c];
        F[p * m + c] = t;
      }
      __syncthreads();   // the swapped pivot row is read below
    }
    cplx<T> pv = F[j * m + j];
    const bool pert = cabs1(pv) < a.tiny;
    if (pert) pv = cplx<T>{a.tiny, (T)0};
    if (threadIdx.x == 0) {
      piv[j] = p;
      if (pert) atomicAdd(a.nperturb + fq, 1);
    }
    const cplx<T> inv = cdiv(cplx<T>{1, 0}, pv);
    // rows below the pivot: multiplier, then the rank-1 update of the row.  The
    // pivot row's columns are held in registers (CU per lane covers m - 1 columns
    // at the widest small front), and each row's loads are all issued before its
    // stores, so that a warp keeps them in flight together.
    constexpr int CU = sizeof(T) == 8 ? 4 : 5;
    const cplx<T> *prow = F + j * m;
    cplx<T> pr[CU];
#pragma unroll
    for (int u = 0; u < CU; ++u) {
      const int c = j + 1 + lane + 32 * u;
      pr[u] = c < m ? prow[c] : cplx<T>{0, 0};
    }
    T best = (T)-1;
    int bi = j + 1;
    for (int r = j + 1 + wid; r < m; r += nw) {
      cplx<T> *row = F + r * m;
      const cplx<T> l = cmul(row[j], inv);
      cplx<T> rv[CU];
#pragma unroll
      for (int u = 0; u < CU; ++u) {
        const int c = j + 1 + lane + 32 * u;
        if (c < m) rv[u] = row[c];
      }
#pragma unroll
      for (int u = 0; u < CU; ++u) {
        const int c = j + 1 + lane + 32 * u;
        if (c < m) {
          rv[u] = cfms(rv[u], l, pr[u]);
          row[c] = rv[u];
        }
      }
      __syncwarp();
      if (lane == 0) {
        row[j] = l;
        if (r < k && j + 1 < k) {
          const T v = cabs1(rv[0]);   // the updated F[r][j + 1]: lane 0's first column
          if (v > best) best = v, bi = r;
        }
      }
    }
    if (lane == 0) {
      s_cv[j & 1][wid] = best;
      s_ci[j & 1][wid] = bi;
    }
    // the previous pivot's perturbed diagonal is read by no one any more
    if (pert_prev && threadIdx.x == 0) F[(j - 1) * m + j - 1] = pv_prev;
    pert_prev = pert;
    pv_prev = pv;
    __syncthreads();
    if (j + 1 < k) {
      // largest modulus, lowest row on ties: a total order, so the shuffle tree
      // gives the same row in every warp (and as a serial scan would)
      T bv = lane < nw ? s_cv[j & 1][lane] : (T)-1;
      int bq = lane < nw ? s_ci[j & 1][lane] : j + 1;
      for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bq, o);
        if (ov > bv || (ov == bv && oi < bq)) bv = ov, bq = oi;
      }
      p = bq;
    }
  }
  if (pert_prev && threadIdx.x == 0) F[(k - 1) * m + k - 1] = pv_prev;
  __syncthreads();
  cplx<T> *G = arena + a.off[f];
  for (int r = wid; r < m; r += nw)
    for (int c = lane; c < m; c += 32) G[(int64_t)r * ld + c] = F[r * m + c];
}

}  // namespace ss

namespace ss {

constexpr int kPanel = 32;      // panel width of the blocked partial LU

// rows per CTA of the large-front assembly: about SS_ASM_ELEMS elements per CTA
// (default 16k), at least 32 rows, a whole front when it is that small (narrow
// fronts would otherwise make hundreds of thousands of near-empty CTAs)
static inline int asm_rows(int maxm) {
  int elems = 16384;
  if (const char *e = getenv("SS_ASM_ELEMS")) elems = std::max(1024, atoi(e));
  return std::max(32, std::min(maxm, elems / std::max(1, maxm)));
}

// Whole-element accesses of arena entries: one 16-byte (complex128) or 8-byte
// (complex64) load or store; the arena is cudaMalloc'd and every front offset is
// a whole number of elements, so each entry is aligned to its size.  ld_once
// marks data read once (a child's update block) as evict-first, so that it does
// not push the parent rows being summed out of L2.
template <class T> struct VecOf;
template <> struct VecOf<double> { using V = double2; };
template <> struct VecOf<float> { using V = float2; };
template <class T>
__device__ __forceinline__ cplx<T> ld_el(const cplx<T> *p) {
  const auto v = *reinterpret_cast<const typename VecOf<T>::V *>(p);
  return {v.x, v.y};
}
template <class T>
__device__ __forceinline__ cplx<T> ld_once(const cplx<T> *p) {
  const auto v = __ldcs(reinterpret_cast<const typename VecOf<T>::V *>(p));
  return {v.x, v.y};
}
template <class T>
__device__ __forceinline__ void st_el(cplx<T> *p, cplx<T> v) {
  typename VecOf<T>::V w;
  w.x = v.x;
  w.y = v.y;
  *reinterpret_cast<typename VecOf<T>::V *>(p) = w;
}
// Which assembly kernel: 0 the row-chunk one, 1 the row-owned one in global
// memory, 2 the row-owned one with each row staged in shared memory.  Defaults:
// the row-owned one for complex64 fronts, the row-chunk one for complex128
// (measured: 94.7 vs 92.1 points/s on the Hex27 slab's mixed sweep, 72.4 vs 74.6 on
// the ME1 cell's FP64 sweep); SS_ASM_BY_ROWS=0|1|2 overrides.
template <class T>
static inline int asm_variant() {
  if (const char *e = getenv("SS_ASM_BY_ROWS")) return std::max(0, std::min(2, atoi(e)));
  return sizeof(T) == 4 ? 1 : 0;
}
constexpr int kAsmSmemMax = 227 * 1024;   // shared memory of one CTA of the staged kernel

// Large fronts, assembly in global memory: CTA (frequency, front, row chunk)
// zeroes its rows, drops in the arrowhead entries of those rows, then adds the
// children's update rows that map into them (children in order: deterministic).
// Frequencies are the fastest grid index, so the CTAs of one front's chunk run
// together and read its arrowhead entries (shared by all frequencies) from L2.
template <class T>
__global__ void __launch_bounds__(256) front_assemble_large_kernel(FrontArgs<T> a, int rows) {
  const int f = a.fronts[blockIdx.y], fq = blockIdx.x;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  const int r0 = blockIdx.z * rows;
  if (r0 >= m) return;
  const int r1 = min(m, r0 + rows);
  const double w = a.omega[fq];
  cplx<T> *arena = a.arena + (int64_t)fq * a.stride;
  cplx<T> *F = arena + a.off[f];
  for (int t = threadIdx.x; t < (r1 - r0) * m; t += blockDim.x) {
    const int r = r0 + t / m, c = t % m;
    st_el(F + (int64_t)r * ld + c, cplx<T>{0, 0});
  }
  __syncthreads();
  {
    // arrow entries are sorted by row position
    int64_t lo = a.arrow_ptr[f], hi = a.arrow_ptr[f + 1];
    int64_t b = lo, e = hi;
    while (b < e) {
      int64_t mid = (b + e) / 2;
      if (a.arrow_pos[mid] / ld < r0) b = mid + 1; else e = mid;
    }
    const int64_t q0 = b;
    e = hi;
    while (b < e) {
      int64_t mid = (b + e) / 2;
      if (a.arrow_pos[mid] / ld < r1) b = mid + 1; else e = mid;
    }
    for (int64_t q = q0 + threadIdx.x; q < b; q += blockDim.x)
      F[a.arrow_pos[q]] = to_t<T>(a_entry(a.Kc, a.Mc, a.Dc, a.arrow_slot[q], w, a.beta));
  }
  __syncthreads();
  for (int64_t cc = a.child_ptr[f]; cc < a.child_ptr[f + 1]; ++cc) {
    const int ch = a.child[cc];
    const int kc = a.k[ch], nn = a.m[ch] - kc, ldc = a.ld[ch];
    const int *rel = a.relpos + a.relpos_ptr[ch];
    int b = 0, e = nn;
    while (b < e) { int mid = (b + e) / 2; if (rel[mid] < r0) b = mid + 1; else e = mid; }
    const int i0 = b;
    e = nn;
    while (b < e) { int mid = (b + e) / 2; if (rel[mid] < r1) b = mid + 1; else e = mid; }
    const int i1 = b;
    const cplx<T> *CB = arena + a.off[ch] + (int64_t)kc * ldc + kc;
    // four elements per thread and pass, every load issued before any store (the
    // targets of one child are distinct), so that each thread keeps several
    // memory requests in flight
    constexpr int U = 4;
    const int tot = (i1 - i0) * nn;
    for (int t0 = threadIdx.x; t0 < tot; t0 += U * blockDim.x) {
      cplx<T> *dp[U];
      cplx<T> cv[U], dv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int t = t0 + u * blockDim.x;
        dp[u] = nullptr;
        if (t < tot) {
          const int i = i0 + t / nn, j = t % nn;
          dp[u] = F + (int64_t)rel[i] * ld + rel[j];
          cv[u] = ld_once(CB + (int64_t)i * ldc + j);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (dp[u]) dv[u] = ld_el(dp[u]);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (dp[u]) st_el(dp[u], dv[u] + cv[u]);
    }
    __syncthreads();
  }
}

// The same assembly organised by parent row: a warp owns one row at a time and
// takes it through zero, arrowhead entries and every child's update row that maps
// into it (children in order, found by binary search in the child's sorted row
// map), with only warp-level ordering between the steps.  Each element sees the
// same operations in the same order as in front_assemble_large_kernel, and a
// row's zeroes are still in cache when its children's adds arrive.
constexpr int kAsmRowsPerCta = 32;
template <class T>
__global__ void __launch_bounds__(256) front_assemble_rows_kernel(FrontArgs<T> a) {
  const int f = a.fronts[blockIdx.y], fq = blockIdx.x;
  const int m = a.m[f], ld = a.ld[f];
  const int r0 = blockIdx.z * kAsmRowsPerCta;
  if (r0 >= m) return;
  const int r1 = min(m, r0 + kAsmRowsPerCta);
  const double w = a.omega[fq];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  cplx<T> *arena = a.arena + (int64_t)fq * a.stride;
  cplx<T> *F = arena + a.off[f];
  const int64_t alo = a.arrow_ptr[f], ahi = a.arrow_ptr[f + 1];
  for (int r = r0 + wid; r < r1; r += nw) {
    cplx<T> *row = F + (int64_t)r * ld;
    for (int c = lane; c < m; c += 32) row[c] = cplx<T>{0, 0};
    __syncwarp();
    {
      // arrow entries are sorted by position: those of row r are one range
      int64_t b = alo, e = ahi;
      while (b < e) {
        const int64_t mid = (b + e) / 2;
        if (a.arrow_pos[mid] < r * ld) b = mid + 1; else e = mid;
      }
      for (int64_t q = b + lane; q < ahi && a.arrow_pos[q] < (r + 1) * ld; q += 32)
        F[a.arrow_pos[q]] = to_t<T>(a_entry(a.Kc, a.Mc, a.Dc, a.arrow_slot[q], w, a.beta));
    }
    __syncwarp();
    for (int64_t cc = a.child_ptr[f]; cc < a.child_ptr[f + 1]; ++cc) {
      const int ch = a.child[cc];
      const int kc = a.k[ch], nn = a.m[ch] - kc, ldc = a.ld[ch];
      const int *rel = a.relpos + a.relpos_ptr[ch];
      int b = 0, e = nn;
      while (b < e) {
        const int mid = (b + e) / 2;
        if (rel[mid] < r) b = mid + 1; else e = mid;
      }
      if (b == nn || rel[b] != r) continue;
      const cplx<T> *src = arena + a.off[ch] + (int64_t)(kc + b) * ldc + kc;
      constexpr int U = 4;
      for (int j0 = lane; j0 < nn; j0 += 32 * U) {
        int cj[U];
        cplx<T> cv[U], dv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int j = j0 + 32 * u;
          cj[u] = j < nn ? rel[j] : -1;
          if (cj[u] >= 0) cv[u] = ld_once(src + j);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (cj[u] >= 0) dv[u] = ld_el(row + cj[u]);
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (cj[u] >= 0) st_el(row + cj[u], dv[u] + cv[u]);
      }
      __syncwarp();
    }
  }
}

// The row-owned assembly with each warp's row staged in shared memory (rows of
// `sld` elements): the zero, the arrowhead entries and the children's update rows
// are summed there in the same order as in the two kernels above (so all three
// give identical fronts), and the finished row is written to the arena once: the
// arena sees each front written once and each child block read once, with no
// read-modify-write of global memory.  Each warp owns rows r0 + wid, + nw, ...
template <class T>
__global__ void __launch_bounds__(256) front_assemble_rows_smem_kernel(FrontArgs<T> a, int rows_per_cta, int sld) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int f = a.fronts[blockIdx.y], fq = blockIdx.x;
  const int m = a.m[f], ld = a.ld[f];
  const int r0 = blockIdx.z * rows_per_cta;
  if (r0 >= m) return;
  const int r1 = min(m, r0 + rows_per_cta);
  const double w = a.omega[fq];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  cplx<T> *srow = reinterpret_cast<cplx<T> *>(smem_raw) + (int64_t)wid * sld;
  cplx<T> *arena = a.arena + (int64_t)fq * a.stride;
  cplx<T> *F = arena + a.off[f];
  const int64_t alo = a.arrow_ptr[f], ahi = a.arrow_ptr[f + 1];
  for (int r = r0 + wid; r < r1; r += nw) {
    for (int c = lane; c < m; c += 32) srow[c] = cplx<T>{0, 0};
    __syncwarp();
    {
      int64_t b = alo, e = ahi;
      while (b < e) {
        const int64_t mid = (b + e) / 2;
        if (a.arrow_pos[mid] < r * ld) b = mid + 1; else e = mid;
      }
      for (int64_t q = b + lane; q < ahi && a.arrow_pos[q] < (r + 1) * ld; q += 32)
        srow[a.arrow_pos[q] - r * ld] = to_t<T>(a_entry(a.Kc, a.Mc, a.Dc, a.arrow_slot[q], w, a.beta));
    }
    __syncwarp();
    for (int64_t cc = a.child_ptr[f]; cc < a.child_ptr[f + 1]; ++cc) {
      const int ch = a.child[cc];
      const int kc = a.k[ch], nn = a.m[ch] - kc, ldc = a.ld[ch];
      const int *rel = a.relpos + a.relpos_ptr[ch];
      int b = 0, e = nn;
      while (b < e) {
        const int mid = (b + e) / 2;
        if (rel[mid] < r) b = mid + 1; else e = mid;
      }
      if (b == nn || rel[b] != r) continue;
      const cplx<T> *src = arena + a.off[ch] + (int64_t)(kc + b) * ldc + kc;
      constexpr int U = 4;
      for (int j0 = lane; j0 < nn; j0 += 32 * U) {
        int cj[U];
        cplx<T> cv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int j = j0 + 32 * u;
          cj[u] = j < nn ? rel[j] : -1;
          if (cj[u] >= 0) cv[u] = ld_once(src + j);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (cj[u] >= 0) srow[cj[u]] = srow[cj[u]] + cv[u];
      }
      __syncwarp();
    }
    cplx<T> *row = F + (int64_t)r * ld;
    for (int c = lane; c < m; c += 32) st_el(row + c, srow[c]);
    __syncwarp();
  }
}

// Rows [k, m) of the panel columns: L21[:, j0:j1] = F21[:, j0:j1] U_jj^-1 (each
// row independent, one thread per row; U_jj and its diagonal reciprocals staged in
// shared memory).  The 32 columns go in two halves of 16 held in registers: the
// second half first takes the first half's finished values back from the row in
// the order t = 0, 1, ..., so every entry sees the operations of a single
// 32-column substitution in the same order.  `row` is the row in global memory or
// in a staged tile.
template <class T>
__device__ __forceinline__ void l21_row(cplx<T> *row, int w, const cplx<T> (*U)[kPanel], const cplx<T> *Uinv) {
  constexpr int H = kPanel / 2;
  for (int h0 = 0; h0 < w; h0 += H) {
    const int hw = min(H, w - h0);
    cplx<T> x[H];
#pragma unroll
    for (int c = 0; c < H; ++c)
      if (c < hw) x[c] = row[h0 + c];
    // the finished columns left of this half
    for (int t = 0; t < h0; ++t) {
      const cplx<T> xt = row[t];
#pragma unroll
      for (int c = 0; c < H; ++c)
        if (c < hw) x[c] = cfms(x[c], xt, U[t][h0 + c]);
    }
#pragma unroll
    for (int c = 0; c < H; ++c) {
      if (c >= hw) break;
      cplx<T> v = x[c];
#pragma unroll
      for (int t = 0; t < c; ++t) v = cfms(v, x[t], U[h0 + t][h0 + c]);
      x[c] = cmul(v, Uinv[h0 + c]);
    }
#pragma unroll
    for (int c = 0; c < H; ++c)
      if (c < hw) row[h0 + c] = x[c];
  }
}

// RPW > 0 (staged): each warp stages RPW rows of the panel columns in shared memory
// with coalesced loads (lane = column), solves them with lanes 0..RPW-1 = rows,
// and writes them back coalesced.  RPW = 0: each thread works on its row in global
// memory (a warp's loads then touch 32 rows at once).  The arithmetic is the same.
// Defaults (measured): 32 staged rows per warp for complex64 (Hex27 slab mixed sweep
// 139.6 points/s, 137.3 with 16, 132.0 direct); 16 for complex128, whose 32-row tiles
// take 135 KB per 256-thread CTA (ME1 FP64 sweep 80.2 points/s, 79.1 with 32, 79.4
// direct); SS_L21_STAGED=0|16|32 overrides.
template <class T, int RPW>
__global__ void __launch_bounds__(256) front_l21_kernel(FrontArgs<T> a, int j0) {
  constexpr int TS = kPanel + 1;            // staged tile row stride (conflict-free)
  __shared__ cplx<T> U[kPanel][kPanel];
  __shared__ cplx<T> Uinv[kPanel];          // reciprocals of the diagonal, once per CTA
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  if (j0 >= k) return;
  const int j1 = min(k, j0 + kPanel), w = j1 - j0;
  const cplx<T> *Fc = a.arena + (int64_t)fq * a.stride + a.off[f];
  for (int t = threadIdx.x; t < w * w; t += blockDim.x) U[t / w][t % w] = Fc[(int64_t)(j0 + t / w) * ld + j0 + t % w];
  __syncthreads();
  if (threadIdx.x < w) Uinv[threadIdx.x] = cdiv(cplx<T>{1, 0}, U[threadIdx.x][threadIdx.x]);
  __syncthreads();
  cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  if constexpr (RPW == 0) {
    const int r = k + blockIdx.z * blockDim.x + threadIdx.x;
    if (r < m) l21_row<T>(F + (int64_t)r * ld + j0, w, U, Uinv);
  } else {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int rw = k + blockIdx.z * (blockDim.x / 32) * RPW + wid * RPW;
    if (rw >= m) return;
    const int nr = min(RPW, m - rw);
    cplx<T> *tile = reinterpret_cast<cplx<T> *>(smem_raw) + wid * RPW * TS;
    cplx<T> *gp = F + (int64_t)rw * ld + j0;
    if (lane < w) {
#pragma unroll 8
      for (int i = 0; i < nr; ++i) tile[i * TS + lane] = ld_el(gp + (int64_t)i * ld + lane);
    }
    __syncwarp();
    if (lane < nr) l21_row<T>(tile + lane * TS, w, U, Uinv);
    __syncwarp();
    if (lane < w) {
#pragma unroll 8
      for (int i = 0; i < nr; ++i) st_el(gp + (int64_t)i * ld + lane, tile[i * TS + lane]);
    }
  }
}
template <class T>
static inline int l21_rpw() {
  if (const char *e = getenv("SS_L21_STAGED")) {
    const int v = atoi(e);
    return v >= 32 ? 32 : v >= 16 ? 16 : 0;
  }
  return sizeof(T) == 4 ? 32 : 16;
}
// dynamic shared memory of the staged front_l21_kernel (RPW rows per warp)
template <class T>
static inline size_t l21_smem(int threads, int rpw) {
  return (size_t)(threads / 32) * rpw * (kPanel + 1) * sizeof(cplx<T>);
}

// Unblocked LU of panel columns [j0, j1) over the fully-summed rows [j0, k).
template <class T>
__global__ void __launch_bounds__(256) front_panel_kernel(FrontArgs<T> a, int j0) {
  __shared__ T s_v[8];
  __shared__ int s_i[8];
  __shared__ cplx<T> s_pivot;
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  if (j0 >= k) return;
  const int j1 = min(k, j0 + kPanel);
  cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  int *piv = a.piv + (int64_t)fq * a.n + a.p0[f];
  for (int j = j0; j < j1; ++j) {
    const int p = block_argmax<T>(j, k, [&](int r) { return F[(int64_t)r * ld + j]; }, s_v, s_i);
    if (p != j)
      for (int c = j0 + threadIdx.x; c < j1; c += blockDim.x) {
        const cplx<T> t = F[(int64_t)j * ld + c];
        F[(int64_t)j * ld + c] = F[(int64_t)p * ld + c];
        F[(int64_t)p * ld + c] = t;
      }
    __syncthreads();
    if (threadIdx.x == 0) {
      piv[j] = p;
      cplx<T> pv = F[(int64_t)j * ld + j];
      if (cabs1(pv) < a.tiny) {
        pv = cplx<T>{a.tiny, (T)0};
        F[(int64_t)j * ld + j] = pv;
        atomicAdd(a.nperturb + fq, 1);
      }
      s_pivot = pv;
    }
    __syncthreads();
    const cplx<T> inv = cdiv(cplx<T>{1, 0}, s_pivot);
    for (int r = j + 1 + threadIdx.x; r < k; r += blockDim.x)
      F[(int64_t)r * ld + j] = cmul(F[(int64_t)r * ld + j], inv);
    __syncthreads();
    const int nc = j1 - j - 1;
    if (nc > 0) {
      const int nr = k - j - 1;
      for (int t = threadIdx.x; t < nr * nc; t += blockDim.x) {
        const int r = j + 1 + t / nc, c = j + 1 + t % nc;
        F[(int64_t)r * ld + c] = cfms(F[(int64_t)r * ld + c], F[(int64_t)r * ld + j], F[(int64_t)j * ld + c]);
      }
    }
    __syncthreads();
  }
}

// The same panel LU with the panel block -- rows [j0, k) x columns [j0, j1) -- held
// in shared memory (row stride kPanel + 1 complex: row and column walks are both
// conflict-free); one warp per row for the multipliers and the rank-1 update.
// Operation for operation the arithmetic of front_panel_kernel.  The next column's
// pivot search rides on the update: lane 0 of each warp (which updates column
// j + 1) keeps the largest |F[r][j+1]| of its rows, and after the barrier a warp
// shuffle picks the largest over the warps, lowest row on ties, as a block-wide
// argmax over the updated column would.
constexpr int kPanelThreads = 512;
constexpr int kPanelSmemMax = 224 * 1024;
template <class T>
__global__ void __launch_bounds__(kPanelThreads) front_panel_smem_kernel(FrontArgs<T> a, int j0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T> *P = reinterpret_cast<cplx<T> *>(smem_raw);
  constexpr int PS = kPanel + 1;
  __shared__ T s_v[kPanelThreads / 32];
  __shared__ int s_i[kPanelThreads / 32];
  __shared__ cplx<T> s_pivot;
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], ld = a.ld[f];
  if (j0 >= k) return;
  const int w = min(k, j0 + kPanel) - j0, R = k - j0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f] + (int64_t)j0 * ld + j0;
  int *piv = a.piv + (int64_t)fq * a.n + a.p0[f] + j0;
  __shared__ T s_cv[2][kPanelThreads / 32];      // per-warp pivot candidates, by column parity
  __shared__ int s_ci[2][kPanelThreads / 32];
  for (int r = wid; r < R; r += nw)
    if (lane < w) P[r * PS + lane] = F[(int64_t)r * ld + lane];
  __syncthreads();
  int p = block_argmax<T>(0, R, [&](int r) { return P[r * PS]; }, s_v, s_i);
  for (int j = 0; j < w; ++j) {
    if (p != j) {   // p is the same in every thread
      if (threadIdx.x < w) {
        const cplx<T> t = P[j * PS + threadIdx.x];
        P[j * PS + threadIdx.x] = P[p * PS + threadIdx.x];
        P[p * PS + threadIdx.x] = t;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      piv[j] = j0 + p;
      cplx<T> pv = P[j * PS + j];
      if (cabs1(pv) < a.tiny) {
        pv = cplx<T>{a.tiny, (T)0};
        P[j * PS + j] = pv;
        atomicAdd(a.nperturb + fq, 1);
      }
      s_pivot = pv;
    }
    __syncthreads();
    const cplx<T> inv = cdiv(cplx<T>{1, 0}, s_pivot);
    const int c = j + 1 + lane;
    const cplx<T> pc = c < w ? P[j * PS + c] : cplx<T>{0, 0};
    T best = (T)-1;
    int bi = j + 1;
    for (int r = j + 1 + wid; r < R; r += nw) {
      cplx<T> *row = P + r * PS;
      const cplx<T> l = cmul(row[j], inv);
      cplx<T> v{0, 0};
      if (c < w) {
        v = cfms(row[c], l, pc);
        row[c] = v;
      }
      __syncwarp();
      if (lane == 0) {
        row[j] = l;
        const T av = cabs1(v);   // the updated F[r][j + 1] (c = j + 1 for lane 0)
        if (j + 1 < w && av > best) best = av, bi = r;
      }
    }
    if (lane == 0) {
      s_cv[j & 1][wid] = best;
      s_ci[j & 1][wid] = bi;
    }
    __syncthreads();
    if (j + 1 < w) {
      T bv = lane < nw ? s_cv[j & 1][lane] : (T)-1;
      int bq = lane < nw ? s_ci[j & 1][lane] : j + 1;
      for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bq, o);
        if (ov > bv || (ov == bv && oi < bq)) bv = ov, bq = oi;
      }
      p = bq;
    }
  }
  for (int r = wid; r < R; r += nw)
    if (lane < w) F[(int64_t)r * ld + lane] = P[r * PS + lane];
}

// The panel's row swaps applied to every column outside it (one thread per
// column; the panel's pivots read once into shared memory).
template <class T>
__global__ void __launch_bounds__(256) front_swap_kernel(FrontArgs<T> a, int j0) {
  __shared__ int sp[kPanel];
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  if (j0 >= k) return;
  const int j1 = min(k, j0 + kPanel), w = j1 - j0;
  cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  if (threadIdx.x < w) sp[threadIdx.x] = a.piv[(int64_t)fq * a.n + a.p0[f] + j0 + threadIdx.x];
  __syncthreads();
  const int idx = blockIdx.z * blockDim.x + threadIdx.x;
  if (idx >= m - w) return;
  const int c = idx < j0 ? idx : idx + w;
  for (int j = j0; j < j1; ++j) {
    const int p = sp[j - j0];
    if (p != j) {
      const cplx<T> t = F[(int64_t)j * ld + c];
      F[(int64_t)j * ld + c] = F[(int64_t)p * ld + c];
      F[(int64_t)p * ld + c] = t;
    }
  }
}

// The unit-lower diagonal block solved into the row block U[j0:j1, j1:m) (one
// thread per column, L_jj staged in shared memory).  The 32 rows go in two halves
// of 16 held in registers: the second half first takes the first half's finished
// values back from the arena (still in L1) in the order t = 0, 1, ..., so every
// entry sees the same operations in the same order as a single 32-row pass.
template <class T>
__global__ void __launch_bounds__(256) front_u12_trsm_kernel(FrontArgs<T> a, int j0) {
  constexpr int H = kPanel / 2;
  __shared__ cplx<T> L[kPanel][kPanel];
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  if (j0 >= k) return;
  const int j1 = min(k, j0 + kPanel), w = j1 - j0;
  cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  const int idx = blockIdx.z * blockDim.x + threadIdx.x;
  for (int t = threadIdx.x; t < w * w; t += blockDim.x) L[t / w][t % w] = F[(int64_t)(j0 + t / w) * ld + j0 + t % w];
  __syncthreads();
  const int c = j1 + idx;
  if (c >= m) return;
  cplx<T> *col = F + (int64_t)j0 * ld + c;
  for (int h0 = 0; h0 < w; h0 += H) {
    const int hw = min(H, w - h0);
    cplx<T> v[H];
#pragma unroll
    for (int i = 0; i < H; ++i)
      if (i < hw) v[i] = col[(int64_t)(h0 + i) * ld];
    // the finished rows above this half
    for (int t = 0; t < h0; ++t) {
      const cplx<T> xt = col[(int64_t)t * ld];
#pragma unroll
      for (int i = 0; i < H; ++i)
        if (i < hw) v[i] = cfms(v[i], L[h0 + i][t], xt);
    }
#pragma unroll
    for (int i = 1; i < H; ++i) {
      if (i >= hw) break;
      cplx<T> x = v[i];
#pragma unroll
      for (int t = 0; t < i; ++t) x = cfms(x, L[h0 + i][h0 + t], v[t]);
      v[i] = x;
    }
#pragma unroll
    for (int i = 0; i < H; ++i)
      if (i < hw) col[(int64_t)(h0 + i) * ld] = v[i];
  }
}

constexpr int kGemmBK = 8;
// tile shapes: square (Schur update), skinny (panel column update), short (U row update)
// tile shapes: square (Schur update; two candidates the autotuner picks from per
// level), skinny (panel column update), short (U row update)
// thin column / row tiles: panel-step tasks at most 8 columns wide (panel columns)
// or 8 rows high (U rows), e.g. a 4-pivot tail panel after a full 32-wide one
enum GemmShape { kSquare = 0, kSkinny = 1, kShort = 2, kSquare64 = 3, kThinCol = 4, kThinRow = 5 };
template <int S> struct Tile;
template <> struct Tile<kSquare> { static constexpr int BM = 128, BN = 64, TM = 8, TN = 4; };
template <> struct Tile<kSkinny> { static constexpr int BM = 256, BN = 32, TM = 8, TN = 4; };
template <> struct Tile<kShort> { static constexpr int BM = 32, BN = 256, TM = 4, TN = 8; };
template <> struct Tile<kSquare64> { static constexpr int BM = 64, BN = 64, TM = 4, TN = 4; };
template <> struct Tile<kThinCol> { static constexpr int BM = 128, BN = 8, TM = 2, TN = 2; };
template <> struct Tile<kThinRow> { static constexpr int BM = 8, BN = 128, TM = 2, TN = 2; };
static inline int tile_bm(int s) {
  return s == kSquare ? 128 : s == kSkinny ? 256 : s == kShort ? 32 : s == kThinCol ? 128 : s == kThinRow ? 8 : 64;
}
static inline int tile_bn(int s) {
  return s == kSquare ? 64 : s == kSkinny ? 32 : s == kShort ? 256 : s == kThinCol ? 8 : s == kThinRow ? 128 : 64;
}

// One BMxBN complex tile of C -= A B per CTA, TMxTN outputs per thread; K in
// chunks of 8 with the next chunk prefetched into registers.  CST: the C tile is
// copied into shared memory by cp.async when the CTA starts (row stride BN + 1),
// so that its latency overlaps the K loop (dynamic shared memory gemm_cst_bytes).
template <class T, int S>
constexpr int gemm_cst_bytes() { return Tile<S>::BM * (Tile<S>::BN + 1) * (int)sizeof(cplx<T>); }
// (the thin tiles: four CTAs per SM, so that more tiles hide their load latency)
template <class T, int S, bool CST = false>
__global__ void __launch_bounds__(256, (S == kThinCol || S == kThinRow) ? 4 : sizeof(T) == 4 ? 2 : 1)
    front_gemm_kernel(FrontArgs<T> a, const GemmTask *__restrict__ tasks) {
  constexpr int BM = Tile<S>::BM, BN = Tile<S>::BN, TM = Tile<S>::TM, TN = Tile<S>::TN, BK = kGemmBK;
  constexpr int TX = BN / TN, TY = BM / TM, CS = BN + 1;
  static_assert(TX * TY == 256, "256 threads");
  // staged A / B elements per thread; the thin tiles' narrow side has fewer than
  // 256 elements per K chunk, so only the first BM*BK (BN*BK) threads load it
  constexpr int NA = (BM * BK + 255) / 256, NBt = (BN * BK + 255) / 256;
  constexpr bool A_ALL = BM * BK % 256 == 0, B_ALL = BN * BK % 256 == 0;
  // A rows padded by 4: the transposing stores (8 k values x 4 rows per warp) hit
  // 32 distinct slots
  __shared__ cplx<T> As[BK][BM + 4];
  __shared__ cplx<T> Bs[BK][BN];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const GemmTask tk = tasks[blockIdx.x];
  const int fq = blockIdx.y;
  const int ld = a.ld[tk.f];
  cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[tk.f];
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  cplx<T> *Cs = reinterpret_cast<cplx<T> *>(smem_raw);
  if constexpr (CST) {
    constexpr uint32_t EB = sizeof(cplx<T>);
    for (int idx = threadIdx.x; idx < BM * BN; idx += 256) {
      const int r = idx / BN, c = idx % BN;
      const int gr = tk.r0 + r, gc = tk.c0 + c;
      const bool ok = gr < tk.rhi && gc < tk.chi;
      const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&Cs[r * CS + c]);
      const void *src = ok ? (const void *)(F + (int64_t)gr * ld + gc) : (const void *)F;
      if constexpr (EB == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(ok ? 16u : 0u) : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(ok ? 8u : 0u) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  cplx<T> acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = cplx<T>{0, 0};
  cplx<T> pa[NA], pb[NBt];
  auto fetch = [&](int kb) {
#pragma unroll
    for (int q = 0; q < NA; ++q) {
      const int idx = threadIdx.x + 256 * q, rr = idx / BK, kk = idx % BK;
      const int r = tk.r0 + rr, c = kb + kk;
      pa[q] = ((A_ALL || idx < BM * BK) && r < tk.rhi && c < tk.kk1) ? F[(int64_t)r * ld + c] : cplx<T>{0, 0};
    }
#pragma unroll
    for (int q = 0; q < NBt; ++q) {
      const int idx = threadIdx.x + 256 * q, kk = idx / BN, cc = idx % BN;
      const int r = kb + kk, c = tk.c0 + cc;
      pb[q] = ((B_ALL || idx < BN * BK) && c < tk.chi && r < tk.kk1) ? F[(int64_t)r * ld + c] : cplx<T>{0, 0};
    }
  };
  fetch(tk.kk0);
  for (int kb = tk.kk0; kb < tk.kk1; kb += BK) {
#pragma unroll
    for (int q = 0; q < NA; ++q) {
      const int idx = threadIdx.x + 256 * q;
      if (A_ALL || idx < BM * BK) As[idx % BK][idx / BK] = pa[q];
    }
#pragma unroll
    for (int q = 0; q < NBt; ++q) {
      const int idx = threadIdx.x + 256 * q;
      if (B_ALL || idx < BN * BK) Bs[idx / BN][idx % BN] = pb[q];
    }
    __syncthreads();
    if (kb + BK < tk.kk1) fetch(kb + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      cplx<T> av[TM], bv[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) av[i] = As[kk][ty + TY * i];
#pragma unroll
      for (int j = 0; j < TN; ++j) bv[j] = Bs[kk][tx + TX * j];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) {
          acc[i][j].x = fma(av[i].x, bv[j].x, fma(-av[i].y, bv[j].y, acc[i][j].x));
          acc[i][j].y = fma(av[i].x, bv[j].y, fma(av[i].y, bv[j].x, acc[i][j].y));
        }
    }
    __syncthreads();
  }
  if constexpr (CST) {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
  }
  // epilogue: per output row, all TN loads of C first, then the stores
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int r = tk.r0 + ty + TY * i;
    const bool rok = r < tk.rhi;
    cplx<T> *Fr = F + (int64_t)(rok ? r : tk.r0) * ld;
    cplx<T> cv[TN];
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int c = tk.c0 + tx + TX * j;
      if constexpr (CST)
        cv[j] = Cs[(ty + TY * i) * CS + tx + TX * j];
      else
        cv[j] = (rok && c < tk.chi) ? Fr[c] : cplx<T>{0, 0};
    }
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int c = tk.c0 + tx + TX * j;
      if (rok && c < tk.chi) Fr[c] = cv[j] - acc[i][j];
    }
  }
}

// FP64 complex tile C -= A B on the FP64 tensor cores (DMMA, mma.sync m8n8k4 f64):
// 4 warps in a WM x WN grid, each a 32x32 complex warp tile (4x4 blocks of 8x8), so
// (32 WM) x (32 WN) complex outputs per 128-thread CTA (64x64 Schur tiles, 128x32
// panel-column tiles, 32x128 U-row tiles); K in chunks of 8 complex staged by
// cp.async (double-buffered).  Each
// 8x8x4 complex block is four real MMAs: Dr += Ar Br - Ai Bi, Di += Ar Bi + Ai Br.
// Fragments (PTX m8n8k4 .f64): A[g][t], B[t][g], C[g][2t + i] with g = lane / 4,
// t = lane % 4.
constexpr int kDmmaBK = 8;
// shared layouts (complex): A rows of 8 with the halves of odd rows swapped
// (column k stored at k ^ 4), B rows padded by 2 (32 bytes off a 128-byte line):
// each 8-lane phase of a 16-byte fragment load then hits eight distinct 16-byte
// slots (conflict-free)
constexpr int kDmmaAS = kDmmaBK;
__device__ __forceinline__ int dmma_acol(int r, int k) { return k ^ ((r & 1) << 2); }

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}
__device__ __forceinline__ void cp_async16_cd(uint32_t dst, const void *src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

template <int WM, int WN>
__global__ void __launch_bounds__(128, 3) front_dmma_kernel(FrontArgs<double> a, const GemmTask *__restrict__ tasks) {
  constexpr int kDmmaBM = 32 * WM, kDmmaBN = 32 * WN, kDmmaBS = kDmmaBN + 2;
  static_assert(WM * WN == 4, "four warps");
  __shared__ __align__(16) cd As[2][kDmmaBM * kDmmaAS];
  __shared__ __align__(16) cd Bs[2][kDmmaBK * kDmmaBS];
  const GemmTask tk = tasks[blockIdx.x];
  const int fq = blockIdx.y;
  const int ld = a.ld[tk.f];
  cd *F = a.arena + (int64_t)fq * a.stride + a.off[tk.f];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wm = wid / WN, wn = wid % WN;       // warp tile origin (32 x 32 complex)
  const int g = lane >> 2, t = lane & 3;
  double dr[4][4][2], di[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) dr[i][j][0] = dr[i][j][1] = di[i][j][0] = di[i][j][1] = 0.0;
  auto issue = [&](int buf, int kb) {
#pragma unroll
    for (int q = 0; q < kDmmaBM * kDmmaBK / 128; ++q) {
      const int idx = threadIdx.x + 128 * q;
      const int r = idx / kDmmaBK, k = idx % kDmmaBK;   // A: BM rows x 8
      const int gr = tk.r0 + r, gk = kb + k;
      const bool ok = gr < tk.rhi && gk < tk.kk1;
      cp_async16_cd((uint32_t)__cvta_generic_to_shared(&As[buf][r * kDmmaAS + dmma_acol(r, k)]),
                    ok ? F + (int64_t)gr * ld + gk : F, ok ? 16u : 0u);
    }
#pragma unroll
    for (int q = 0; q < kDmmaBK * kDmmaBN / 128; ++q) {
      const int idx = threadIdx.x + 128 * q;
      const int k = idx / kDmmaBN, c = idx % kDmmaBN;   // B: 8 rows x BN
      const int gk = kb + k, gc = tk.c0 + c;
      const bool ok = gk < tk.kk1 && gc < tk.chi;
      cp_async16_cd((uint32_t)__cvta_generic_to_shared(&Bs[buf][k * kDmmaBS + c]),
                    ok ? F + (int64_t)gk * ld + gc : F, ok ? 16u : 0u);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  const int nk = (tk.kk1 - tk.kk0 + kDmmaBK - 1) / kDmmaBK;
  issue(0, tk.kk0);
  for (int kc = 0; kc < nk; ++kc) {
    const int buf = kc & 1;
    if (kc + 1 < nk) {
      issue(buf ^ 1, tk.kk0 + (kc + 1) * kDmmaBK);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kDmmaBK; kk += 4) {
      cd av[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int ar = wm * 32 + i * 8 + g;
        av[i] = As[buf][ar * kDmmaAS + dmma_acol(ar, kk + t)];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const cd bv = Bs[buf][(kk + t) * kDmmaBS + wn * 32 + j * 8 + g];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          dmma(dr[i][j][0], dr[i][j][1], av[i].x, bv.x);
          dmma(dr[i][j][0], dr[i][j][1], -av[i].y, bv.y);
          dmma(di[i][j][0], di[i][j][1], av[i].x, bv.y);
          dmma(di[i][j][0], di[i][j][1], av[i].y, bv.x);
        }
      }
    }
    __syncthreads();
  }
  // epilogue: per fragment row, all eight C loads first, then the stores (one
  // memory round trip per row instead of one per element)
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = tk.r0 + wm * 32 + i * 8 + g;
    const bool rok = r < tk.rhi;
    cd *Fr = F + (int64_t)(rok ? r : tk.r0) * ld;
    cd cv[4][2];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = tk.c0 + wn * 32 + j * 8 + 2 * t + e;
        cv[j][e] = (rok && c < tk.chi) ? Fr[c] : cd{0.0, 0.0};
      }
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = tk.c0 + wn * 32 + j * 8 + 2 * t + e;
        if (rok && c < tk.chi) Fr[c] = cv[j][e] - cd{dr[i][j][e], di[i][j][e]};
      }
  }
}

// The same 64x64 Schur tile with Gauss's three-multiplication complex product:
// P1 = Ar Br, P2 = Ai Bi, P3 = (Ar + Ai)(Br + Bi), then Re = P1 - P2 and
// Im = P3 - P1 - P2, so each 8x8x4 complex block is three real DMMAs instead of
// four (the FP64 tensor pipe is the bound of this update).  The algorithmic flop
// count is unchanged (8 per complex multiply-add).  Normwise the product is as
// stable as the four-product form; the imaginary part's error is bounded by
// u (|Ar| + |Ai|)(|Br| + |Bi|) per term instead of u (|Ar||Bi| + |Ai||Br|).
// Three accumulator sets (96 doubles per thread): two CTAs per SM.  WM x WN warps
// of 32x32 complex, as front_dmma_kernel (2x2 Schur tiles, 4x1 / 1x4 panel steps).
// CST: the C tile is copied into shared memory by cp.async when the CTA starts (row
// stride BN + 1: conflict-free fragment reads), so its DRAM latency overlaps the K
// loop instead of following it; for the updates with short K (12-36 pivots on the
// lower levels of a nested dissection), where the tile's read-modify-write of C is
// most of its time.  Dynamic shared memory: dmma_cst_bytes<WM, WN>().
template <int WM, int WN>
constexpr int dmma_cst_bytes() { return 32 * WM * (32 * WN + 1) * (int)sizeof(cd); }
template <int WM, int WN, bool CST = false>
__global__ void __launch_bounds__(128, 2) front_dmma3_kernel(FrontArgs<double> a, const GemmTask *__restrict__ tasks) {
  constexpr int kDmmaBM = 32 * WM, kDmmaBN = 32 * WN, kDmmaBS = kDmmaBN + 2, kCS = kDmmaBN + 1;
  static_assert(WM * WN == 4, "four warps");
  __shared__ __align__(16) cd As[2][kDmmaBM * kDmmaAS];
  __shared__ __align__(16) cd Bs[2][kDmmaBK * kDmmaBS];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const GemmTask tk = tasks[blockIdx.x];
  const int fq = blockIdx.y;
  const int ld = a.ld[tk.f];
  cd *F = a.arena + (int64_t)fq * a.stride + a.off[tk.f];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wm = wid / WN, wn = wid % WN;       // warp tile origin (32 x 32 complex)
  const int g = lane >> 2, t = lane & 3;
  cd *Cs = reinterpret_cast<cd *>(smem_raw);
  if constexpr (CST) {
    // the C tile (zeros outside the front's block), one cp.async group of its own
    // committed before the first operand chunk's
    for (int idx = threadIdx.x; idx < kDmmaBM * kDmmaBN; idx += 128) {
      const int r = idx / kDmmaBN, c = idx % kDmmaBN;
      const int gr = tk.r0 + r, gc = tk.c0 + c;
      const bool ok = gr < tk.rhi && gc < tk.chi;
      cp_async16_cd((uint32_t)__cvta_generic_to_shared(&Cs[r * kCS + c]), ok ? F + (int64_t)gr * ld + gc : F,
                    ok ? 16u : 0u);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  double p1[4][4][2], p2[4][4][2], p3[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) p1[i][j][e] = p2[i][j][e] = p3[i][j][e] = 0.0;
  auto issue = [&](int buf, int kb) {
#pragma unroll
    for (int q = 0; q < kDmmaBM * kDmmaBK / 128; ++q) {
      const int idx = threadIdx.x + 128 * q;
      const int r = idx / kDmmaBK, k = idx % kDmmaBK;
      const int gr = tk.r0 + r, gk = kb + k;
      const bool ok = gr < tk.rhi && gk < tk.kk1;
      cp_async16_cd((uint32_t)__cvta_generic_to_shared(&As[buf][r * kDmmaAS + dmma_acol(r, k)]),
                    ok ? F + (int64_t)gr * ld + gk : F, ok ? 16u : 0u);
    }
#pragma unroll
    for (int q = 0; q < kDmmaBK * kDmmaBN / 128; ++q) {
      const int idx = threadIdx.x + 128 * q;
      const int k = idx / kDmmaBN, c = idx % kDmmaBN;
      const int gk = kb + k, gc = tk.c0 + c;
      const bool ok = gk < tk.kk1 && gc < tk.chi;
      cp_async16_cd((uint32_t)__cvta_generic_to_shared(&Bs[buf][k * kDmmaBS + c]),
                    ok ? F + (int64_t)gk * ld + gc : F, ok ? 16u : 0u);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  const int nk = (tk.kk1 - tk.kk0 + kDmmaBK - 1) / kDmmaBK;
  issue(0, tk.kk0);
  for (int kc = 0; kc < nk; ++kc) {
    const int buf = kc & 1;
    if (kc + 1 < nk) {
      issue(buf ^ 1, tk.kk0 + (kc + 1) * kDmmaBK);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kDmmaBK; kk += 4) {
      cd av[4];
      double as[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int ar = wm * 32 + i * 8 + g;
        av[i] = As[buf][ar * kDmmaAS + dmma_acol(ar, kk + t)];
        as[i] = av[i].x + av[i].y;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const cd bv = Bs[buf][(kk + t) * kDmmaBS + wn * 32 + j * 8 + g];
        const double bs = bv.x + bv.y;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          dmma(p1[i][j][0], p1[i][j][1], av[i].x, bv.x);
          dmma(p2[i][j][0], p2[i][j][1], av[i].y, bv.y);
          dmma(p3[i][j][0], p3[i][j][1], as[i], bs);
        }
      }
    }
    __syncthreads();
  }
  if constexpr (CST) {
    if (nk == 0) {   // no operand chunk waited for the C tile
      asm volatile("cp.async.wait_group 0;" ::: "memory");
      __syncthreads();
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int rl = wm * 32 + i * 8 + g, r = tk.r0 + rl;
    const bool rok = r < tk.rhi;
    cd *Fr = F + (int64_t)(rok ? r : tk.r0) * ld;
    cd cv[4][2];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int cl = wn * 32 + j * 8 + 2 * t + e, c = tk.c0 + cl;
        if constexpr (CST)
          cv[j][e] = Cs[rl * kCS + cl];
        else
          cv[j][e] = (rok && c < tk.chi) ? Fr[c] : cd{0.0, 0.0};
      }
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = tk.c0 + wn * 32 + j * 8 + 2 * t + e;
        const double re = p1[i][j][e] - p2[i][j][e];
        const double im = p3[i][j][e] - p1[i][j][e] - p2[i][j][e];
        if (rok && c < tk.chi) Fr[c] = cv[j][e] - cd{re, im};
      }
  }
}

}  // namespace ss

namespace ss {

// Triangular solves stage each 32x32 diagonal block in shared memory (row stride
// 33: row and column walks conflict-free) with one coalesced pass of all threads,
// so that warp 0's sequential block solve reads shared memory instead of making a
// chain of dependent global loads.
constexpr int kDiagS = 33;
constexpr int kDiagElems = 32 * kDiagS;
template <class T>
__device__ __forceinline__ void stage_diag(cplx<T> *D, const cplx<T> *F, int ld, int jb, int bw) {
  for (int t = threadIdx.x; t < bw * 32; t += blockDim.x) {
    const int i = t >> 5, j = t & 31;
    if (j < bw) D[i * kDiagS + j] = F[(int64_t)(jb + i) * ld + jb + j];
  }
}

// Forward substitution for one level: CTA per (front, frequency).  v = b[pivots] +
// children's update vectors; apply the front's row swaps; solve L11; the update
// rows receive v[k:m] - L21 y for the parent.  y overwrites x[pivots].
template <class T>
__global__ void __launch_bounds__(256) front_fwd_kernel(FrontArgs<T> a, const cd *__restrict__ b,
                                                        cd *__restrict__ x, cplx<T> *__restrict__ wv,
                                                        int64_t wstride) {
  if (a.active && !a.active[blockIdx.y]) return;   // converged in the Krylov loop
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T> *D = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *v = D + kDiagElems;
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  const cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  const int64_t p0 = a.p0[f];
  for (int i = threadIdx.x; i < m; i += blockDim.x)
    v[i] = i < k ? to_t<T>(b[(int64_t)fq * a.n + p0 + i]) : cplx<T>{0, 0};
  int *sp = reinterpret_cast<int *>(v + m);   // this front's pivots, loaded in parallel
  for (int j = threadIdx.x; j < k; j += blockDim.x) sp[j] = a.piv[(int64_t)fq * a.n + p0 + j];
  __syncthreads();
  cplx<T> *w = wv + (int64_t)fq * wstride;
  for (int64_t cc = a.child_ptr[f]; cc < a.child_ptr[f + 1]; ++cc) {
    const int ch = a.child[cc];
    const int nn = a.m[ch] - a.k[ch];
    const int *rel = a.relpos + a.relpos_ptr[ch];
    const cplx<T> *wc = w + a.relpos_ptr[ch];
    for (int i = threadIdx.x; i < nn; i += blockDim.x) v[rel[i]] = v[rel[i]] + wc[i];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int j = 0; j < k; ++j) {
      const int p = sp[j];
      if (p != j) {
        const cplx<T> t = v[j];
        v[j] = v[p];
        v[p] = t;
      }
    }
  }
  __syncthreads();
  // blocked unit-lower solve: warp 0 solves each 32x32 diagonal block with
  // shuffles, then one thread per row below it subtracts the block (each thread's
  // entries are one contiguous run of its row, all of them in flight at once)
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int jb = 0; jb < k; jb += 32) {
    const int je = min(k, jb + 32), bw = je - jb;
    stage_diag(D, F, ld, jb, bw);
    __syncthreads();
    if (wid == 0) {
      cplx<T> x = lane < bw ? v[jb + lane] : cplx<T>{0, 0};
      for (int t = 0; t < bw - 1; ++t) {
        cplx<T> xt;
        xt.x = __shfl_sync(0xffffffffu, x.x, t);
        xt.y = __shfl_sync(0xffffffffu, x.y, t);
        if (lane > t && lane < bw) x = cfms(x, D[lane * kDiagS + t], xt);
      }
      if (lane < bw) v[jb + lane] = x;
    }
    __syncthreads();
    for (int r = je + threadIdx.x; r < k; r += blockDim.x) {
      const cplx<T> *Lr = F + (int64_t)r * ld + jb;
      cplx<T> acc = v[r];
#pragma unroll 8
      for (int t = 0; t < bw; ++t) acc = cfms(acc, Lr[t], v[jb + t]);
      v[r] = acc;
    }
    __syncthreads();
  }
  // update rows keep the children's sums; front_fwd_l21_kernel subtracts L21 y
  for (int r = k + threadIdx.x; r < m; r += blockDim.x) w[a.relpos_ptr[f] + r - k] = v[r];
  for (int i = threadIdx.x; i < k; i += blockDim.x) x[(int64_t)fq * a.n + p0 + i] = cd{(double)v[i].x, (double)v[i].y};
}

constexpr int kSolveRows = 64;   // rows per CTA of the solve GEMV kernels

// Update rows of the forward solve: w[r - k] -= L21[r, :] y, CTA per
// (front, frequency, 64-row chunk), one warp per row with coalesced dots.
template <class T>
__global__ void __launch_bounds__(256) front_fwd_l21_kernel(FrontArgs<T> a, const cd *__restrict__ x,
                                                            cplx<T> *__restrict__ wv, int64_t wstride) {
  if (a.active && !a.active[blockIdx.y]) return;   // converged in the Krylov loop
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T> *y = reinterpret_cast<cplx<T> *>(smem_raw);
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  const int r0 = k + blockIdx.z * kSolveRows;
  if (r0 >= m) return;
  const int r1 = min(m, r0 + kSolveRows);
  const cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  const int64_t p0 = a.p0[f];
  for (int i = threadIdx.x; i < k; i += blockDim.x) y[i] = to_t<T>(x[(int64_t)fq * a.n + p0 + i]);
  __syncthreads();
  cplx<T> *w = wv + (int64_t)fq * wstride + a.relpos_ptr[f] - k;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int r = r0 + wid; r < r1; r += nw) {
    cplx<T> acc{0, 0};
    for (int t = lane; t < k; t += 32) acc = acc + cmul(F[(int64_t)r * ld + t], y[t]);
    for (int o = 16; o > 0; o >>= 1) {
      acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
      acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
    }
    if (lane == 0) w[r] = w[r] - acc;
  }
}

// First phase of the backward solve: x[pivots] -= U12 x_U, CTA per (front,
// frequency, 64 pivot rows); x_U gathered from the ancestors' solution.
template <class T>
__global__ void __launch_bounds__(256) front_bwd_u12_kernel(FrontArgs<T> a, cd *__restrict__ x) {
  if (a.active && !a.active[blockIdx.y]) return;   // converged in the Krylov loop
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T> *xu = reinterpret_cast<cplx<T> *>(smem_raw);
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  const int q0 = blockIdx.z * kSolveRows;
  if (q0 >= k || m == k) return;
  const int q1 = min(k, q0 + kSolveRows);
  const cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  cd *xf = x + (int64_t)fq * a.n;
  const int64_t *rows = a.rows + a.rows_ptr[f];
  for (int i = threadIdx.x; i < m - k; i += blockDim.x) xu[i] = to_t<T>(xf[rows[k + i]]);
  __syncthreads();
  const int64_t p0 = a.p0[f];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int r = q0 + wid; r < q1; r += nw) {
    cplx<T> acc{0, 0};
    for (int c = lane; c < m - k; c += 32) acc = acc + cmul(F[(int64_t)r * ld + k + c], xu[c]);
    for (int o = 16; o > 0; o >>= 1) {
      acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
      acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
    }
    if (lane == 0) {
      const cd cur = xf[p0 + r];
      xf[p0 + r] = cd{cur.x - (double)acc.x, cur.y - (double)acc.y};
    }
  }
}

// Backward substitution for one level (levels run root first): z = y - U12 x_U,
// then U11 back substitution; x[pivots] <- z.
template <class T>
__global__ void __launch_bounds__(256) front_bwd_kernel(FrontArgs<T> a, cd *__restrict__ x) {
  if (a.active && !a.active[blockIdx.y]) return;   // converged in the Krylov loop
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T> *D = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *z = D + kDiagElems;
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], ld = a.ld[f];
  const cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  const int64_t p0 = a.p0[f];
  cd *xf = x + (int64_t)fq * a.n;
  for (int i = threadIdx.x; i < k; i += blockDim.x) z[i] = to_t<T>(xf[p0 + i]);   // y - U12 x_U
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // blocked upper solve from the bottom: warp 0 solves each diagonal block,
  // then one thread per row above it subtracts the block (contiguous runs of the
  // rows, all of a thread's loads in flight at once)
  for (int je = k; je > 0; je -= 32) {
    const int jb = max(0, je - 32), bw = je - jb;
    stage_diag(D, F, ld, jb, bw);
    __syncthreads();
    if (wid == 0) {
      cplx<T> x = lane < bw ? z[jb + lane] : cplx<T>{0, 0};
      // each lane's diagonal reciprocal up front: the chain below multiplies
      const cplx<T> rd = lane < bw ? cdiv(cplx<T>{1, 0}, D[lane * kDiagS + lane]) : cplx<T>{0, 0};
      for (int t = bw - 1; t >= 0; --t) {
        if (lane == t) x = cmul(x, rd);
        cplx<T> xt;
        xt.x = __shfl_sync(0xffffffffu, x.x, t);
        xt.y = __shfl_sync(0xffffffffu, x.y, t);
        if (lane < t) x = cfms(x, D[lane * kDiagS + t], xt);
      }
      if (lane < bw) z[jb + lane] = x;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < jb; r += blockDim.x) {
      const cplx<T> *Ur = F + (int64_t)r * ld + jb;
      cplx<T> acc = z[r];
#pragma unroll 8
      for (int t = 0; t < bw; ++t) acc = cfms(acc, Ur[t], z[jb + t]);
      z[r] = acc;
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < k; i += blockDim.x) xf[p0 + i] = cd{(double)z[i].x, (double)z[i].y};
}

// ------------------------------------------------------------------ transposed solves
// A'^T mu = c with P A' = L U (P: the row swaps inside each front, in pivot
// order):  U^T w = c (levels bottom-up), L^T z = w (levels top-down), mu = P^T z.
// The adjoint of the charge functional and the dual-weighted charge correction
// of the mixed-precision sweep use these.

// U^T solve for one level: v = c[pivots] + the children's update vectors;
// U11^T w = v[0:k] (lower triangular, non-unit); the update rows keep the
// children's sums and front_tfwd_u12_kernel subtracts U12^T w.  w -> x[pivots].
template <class T>
__global__ void __launch_bounds__(256) front_tfwd_kernel(FrontArgs<T> a, const cd *__restrict__ c,
                                                         cd *__restrict__ x, cplx<T> *__restrict__ wv,
                                                         int64_t wstride) {
  if (a.active && !a.active[blockIdx.y]) return;   // converged in the Krylov loop
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T> *D = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *v = D + kDiagElems;
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  const cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  const int64_t p0 = a.p0[f];
  for (int i = threadIdx.x; i < m; i += blockDim.x)
    v[i] = i < k ? to_t<T>(c[(int64_t)fq * a.n + p0 + i]) : cplx<T>{0, 0};
  __syncthreads();
  cplx<T> *w = wv + (int64_t)fq * wstride;
  for (int64_t cc = a.child_ptr[f]; cc < a.child_ptr[f + 1]; ++cc) {
    const int ch = a.child[cc];
    const int nn = a.m[ch] - a.k[ch];
    const int *rel = a.relpos + a.relpos_ptr[ch];
    const cplx<T> *wc = w + a.relpos_ptr[ch];
    for (int i = threadIdx.x; i < nn; i += blockDim.x) v[rel[i]] = v[rel[i]] + wc[i];
    __syncthreads();
  }
  // entry (i, t) of U11^T is F[t * ld + i]; warp 0 solves each 32-wide diagonal
  // block, then one thread per row below it subtracts the block (coalesced in r)
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int jb = 0; jb < k; jb += 32) {
    const int je = min(k, jb + 32), bw = je - jb;
    stage_diag(D, F, ld, jb, bw);
    __syncthreads();
    if (wid == 0) {
      cplx<T> xv = lane < bw ? v[jb + lane] : cplx<T>{0, 0};
      const cplx<T> rd = lane < bw ? cdiv(cplx<T>{1, 0}, D[lane * kDiagS + lane]) : cplx<T>{0, 0};
      for (int t = 0; t < bw; ++t) {
        if (lane == t) xv = cmul(xv, rd);
        cplx<T> xt;
        xt.x = __shfl_sync(0xffffffffu, xv.x, t);
        xt.y = __shfl_sync(0xffffffffu, xv.y, t);
        if (lane > t && lane < bw) xv = cfms(xv, D[t * kDiagS + lane], xt);
      }
      if (lane < bw) v[jb + lane] = xv;
    }
    __syncthreads();
    for (int r = je + threadIdx.x; r < k; r += blockDim.x) {
      cplx<T> acc = v[r];
      for (int t = 0; t < bw; ++t) acc = cfms(acc, F[(int64_t)(jb + t) * ld + r], v[jb + t]);
      v[r] = acc;
    }
    __syncthreads();
  }
  for (int r = k + threadIdx.x; r < m; r += blockDim.x) w[a.relpos_ptr[f] + r - k] = v[r];
  for (int i = threadIdx.x; i < k; i += blockDim.x) x[(int64_t)fq * a.n + p0 + i] = cd{(double)v[i].x, (double)v[i].y};
}

// Update rows of the U^T solve: w[r - k] -= sum_i U12[i, r] x_i; CTA per (front,
// frequency, 256 update rows), one thread per row (coalesced column reads).
// Update rows of the U^T solve: w[r - k] -= (U12^T w_piv)[r].  CTA per (front,
// frequency, 32 update rows), lane = row (32 consecutive entries of a U12 row per
// load); the 8 warps split the pivots and their partial sums are added in warp
// order (fixed-order, deterministic).
constexpr int kTColWarps = 8;
template <class T>
__global__ void __launch_bounds__(32 * kTColWarps) front_tfwd_u12_kernel(FrontArgs<T> a, const cd *__restrict__ x,
                                                                         cplx<T> *__restrict__ wv, int64_t wstride) {
  if (a.active && !a.active[blockIdx.y]) return;   // converged in the Krylov loop
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T> *y = reinterpret_cast<cplx<T> *>(smem_raw);
  __shared__ cplx<T> red[kTColWarps][32];
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  const int rb = k + blockIdx.z * 32;
  if (rb >= m) return;
  const cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  const int64_t p0 = a.p0[f];
  for (int i = threadIdx.x; i < k; i += blockDim.x) y[i] = to_t<T>(x[(int64_t)fq * a.n + p0 + i]);
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int r = rb + lane;
  cplx<T> acc{0, 0};
  if (r < m) {
#pragma unroll 4
    for (int i = wid; i < k; i += kTColWarps) acc = acc + cmul(F[(int64_t)i * ld + r], y[i]);
  }
  red[wid][lane] = acc;
  __syncthreads();
  if (wid == 0 && r < m) {
    cplx<T> s = red[0][lane];
    for (int q = 1; q < kTColWarps; ++q) s = s + red[q][lane];
    cplx<T> *w = wv + (int64_t)fq * wstride + a.relpos_ptr[f] - k;
    w[r] = w[r] - s;
  }
}

// First phase of the L^T solve (levels top-down): x[pivots] -= L21^T x_U, with
// x_U the ancestors' solution at this front's update rows; CTA per (front,
// frequency, 256 pivots), one thread per pivot (coalesced row reads).
template <class T>
__global__ void __launch_bounds__(32 * kTColWarps) front_tbwd_l21_kernel(FrontArgs<T> a, cd *__restrict__ x) {
  if (a.active && !a.active[blockIdx.y]) return;   // converged in the Krylov loop
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T> *xu = reinterpret_cast<cplx<T> *>(smem_raw);
  __shared__ cplx<T> red[kTColWarps][32];
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], m = a.m[f], ld = a.ld[f];
  const int ib = blockIdx.z * 32;
  if (ib >= k || m == k) return;
  const cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  cd *xf = x + (int64_t)fq * a.n;
  const int64_t *rows = a.rows + a.rows_ptr[f];
  for (int i = threadIdx.x; i < m - k; i += blockDim.x) xu[i] = to_t<T>(xf[rows[k + i]]);
  __syncthreads();
  // lane = pivot column (32 consecutive entries of an L21 row per load); the 8
  // warps split the update rows, partial sums added in warp order
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int i = ib + lane;
  cplx<T> acc{0, 0};
  if (i < k) {
#pragma unroll 4
    for (int r = wid; r < m - k; r += kTColWarps) acc = acc + cmul(F[(int64_t)(k + r) * ld + i], xu[r]);
  }
  red[wid][lane] = acc;
  __syncthreads();
  if (wid == 0 && i < k) {
    cplx<T> s = red[0][lane];
    for (int q = 1; q < kTColWarps; ++q) s = s + red[q][lane];
    const int64_t p = a.p0[f] + i;
    xf[p] = cd{xf[p].x - (double)s.x, xf[p].y - (double)s.y};
  }
}

// L11^T z = x[pivots] (upper triangular, unit diagonal; entry (i, t) is
// F[t * ld + i]) from the last pivot up, then this front's row swaps undone in
// reverse pivot order; the result -> x[pivots].  The forward solve applies a
// front's swaps before its L11 solve, so the transposed sequence undoes them
// right after the L11^T solve, before any descendant reads these entries.
template <class T>
__global__ void __launch_bounds__(256) front_tbwd_kernel(FrontArgs<T> a, cd *__restrict__ x) {
  if (a.active && !a.active[blockIdx.y]) return;   // converged in the Krylov loop
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T> *D = reinterpret_cast<cplx<T> *>(smem_raw);
  cplx<T> *z = D + kDiagElems;
  const int f = a.fronts[blockIdx.x], fq = blockIdx.y;
  const int k = a.k[f], ld = a.ld[f];
  const cplx<T> *F = a.arena + (int64_t)fq * a.stride + a.off[f];
  const int64_t p0 = a.p0[f];
  cd *xf = x + (int64_t)fq * a.n;
  for (int i = threadIdx.x; i < k; i += blockDim.x) z[i] = to_t<T>(xf[p0 + i]);
  int *sp = reinterpret_cast<int *>(z + k);   // this front's pivots, loaded in parallel
  for (int j = threadIdx.x; j < k; j += blockDim.x) sp[j] = a.piv[(int64_t)fq * a.n + p0 + j];
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int je = k; je > 0; je -= 32) {
    const int jb = max(0, je - 32), bw = je - jb;
    stage_diag(D, F, ld, jb, bw);
    __syncthreads();
    if (wid == 0) {
      cplx<T> xv = lane < bw ? z[jb + lane] : cplx<T>{0, 0};
      for (int t = bw - 1; t > 0; --t) {
        cplx<T> xt;
        xt.x = __shfl_sync(0xffffffffu, xv.x, t);
        xt.y = __shfl_sync(0xffffffffu, xv.y, t);
        if (lane < t) xv = cfms(xv, D[t * kDiagS + lane], xt);
      }
      if (lane < bw) z[jb + lane] = xv;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < jb; r += blockDim.x) {
      cplx<T> acc = z[r];
      for (int t = 0; t < bw; ++t) acc = cfms(acc, F[(int64_t)(jb + t) * ld + r], z[jb + t]);
      z[r] = acc;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int j = k - 1; j >= 0; --j) {
      const int p = sp[j];
      if (p != j) {
        const cplx<T> t = z[j];
        z[j] = z[p];
        z[p] = t;
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < k; i += blockDim.x) xf[p0 + i] = cd{(double)z[i].x, (double)z[i].y};
}

// out[f] = sum_R u[f][R] * v[f][R] (bilinear, no conjugate), fixed-order tree
__global__ void dotu_kernel(int64_t n, const cd *__restrict__ u, const cd *__restrict__ v, cd *__restrict__ out) {
  __shared__ cd red[256];
  const int f = blockIdx.x;
  cd acc{0.0, 0.0};
  for (int64_t R = threadIdx.x; R < n; R += blockDim.x) acc = acc + cmul(u[(int64_t)f * n + R], v[(int64_t)f * n + R]);
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[f] = red[0];
}

// c[f][R] = kq[R] * cs[R] for every frequency of the chunk (the charge row in the
// scaled variables: Q = c^T x' + V Qz)
__global__ void charge_row_kernel(int64_t n, int nb, const cd *__restrict__ kq, const double *__restrict__ cs,
                                  cd *__restrict__ c) {
  const int64_t R = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (R >= n || f >= nb) return;
  c[(int64_t)f * n + R] = kq[R] * cs[R];
}

// x += dx and per-frequency max |dx|, max |x| (for the refinement stopping test)
__global__ void axpy_norm_kernel(int64_t n, cd *__restrict__ x, const cd *__restrict__ dx,
                                 double *__restrict__ nrm) {
  __shared__ double s_dx[256], s_x[256];
  const int f = blockIdx.x;
  double mdx = 0.0, mx = 0.0;
  for (int64_t R = threadIdx.x; R < n; R += blockDim.x) {
    const int64_t t = (int64_t)f * n + R;
    const cd v = x[t] + dx[t];
    x[t] = v;
    mdx = fmax(mdx, sqrt(cabs2(dx[t])));
    mx = fmax(mx, sqrt(cabs2(v)));
  }
  s_dx[threadIdx.x] = mdx;
  s_x[threadIdx.x] = mx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      s_dx[threadIdx.x] = fmax(s_dx[threadIdx.x], s_dx[threadIdx.x + s]);
      s_x[threadIdx.x] = fmax(s_x[threadIdx.x], s_x[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    nrm[2 * f] = s_dx[0];
    nrm[2 * f + 1] = s_x[0];
  }
}

}  // namespace ss

namespace ss {

#define SS_CK(x)                                                   \
  do {                                                             \
    cudaError_t e_ = (x);                                          \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, #x);            \
  } while (0)

// Per-level launch plan of the factorisation, built once after the analysis.
struct Plan {
  std::vector<int> small_ptr, large_ptr;   // per level offsets into fronts_small / fronts_large
  std::vector<int> fronts_small, fronts_large;
  std::vector<int> small_maxm;             // per level max m among small fronts
  std::vector<int> nsteps;                 // per level panel steps of the large fronts
  std::vector<int> maxm_large;             // per level
  std::vector<int> maxk_large;             // per level max k among large fronts
  std::vector<int64_t> step_ptr;           // per (level, step): tasks of that step (flattened)
  std::vector<int64_t> level_step0;        // first (level, step) index of level l
  std::vector<int64_t> schur_ptr;          // per level: Schur tasks
  std::vector<GemmTask> tasks;
  DBuf d_small, d_large, d_tasks;
  int small_m = 0;                         // threshold used
  double schur_flops = 0;
  std::vector<int> lvl_maxk, lvl_maxu;     // per level max k and max m-k (solve grids)
  // CUDA graphs of the per-chunk launch sequences, replayed for every chunk with
  // the same batch size and buffers (key: nb and the device pointers they bake in)
  struct Graph {
    int kind;                              // 0 factorisation, 1 solve, 2 transposed solve
    int nb;
    const void *key[8];
    cudaGraphExec_t exec = nullptr;
    int launches = 0, schur_launches = 0;
  };
  std::vector<Graph> graphs;
  std::vector<cudaEvent_t> ev;             // Schur GEMM timing, one pair per level (owned here so
                                           // that captured event-record nodes stay valid)
  // Schur-tile autotuner (FP64): candidates 0 SIMT 128x64, 1 SIMT 64x64, 2 DMMA
  // 64x64 (the 64x64 candidates share the second task list); per-level pick,
  // decided once per plan by timing every candidate on every level before the
  // first factorisation, so that every sweep of the plan runs the same tiles
  std::vector<int64_t> schur_ptr_b;
  std::vector<int64_t> step_ptr_d;         // panel-step tasks in DMMA tiles (same indexing as step_ptr)
  int panel_dmma = 0;                      // panel-step GEMMs: 0 SIMT, 1 DMMA, 2 DMMA with three
                                           // real products per complex block, 3 the same with the
                                           // C tile staged (tuned once per plan)
  float panel_ms[4] = {0, 0, 0, 0};        // tuner's panel-GEMM times: SIMT, DMMA, DMMA 3M, DMMA 3M C staged
  // FP64 panel-step GEMMs with thin tiles for the narrow tasks: the same (level,
  // step) slots as step_ptr_d, each split into its wide tasks in DMMA tiles
  // (step_ptr_tw) and its narrow ones (at most 8 columns or rows) in SIMT 128x8 /
  // 8x128 tiles (step_ptr_tn); used with the DMMA candidates when panel_thin
  std::vector<int64_t> step_ptr_tw, step_ptr_tn;
  bool panel_thin = false;
  int64_t thin_tasks = 0;                  // narrow-task tiles of one factorisation (per frequency)
  float panel_thin_ms = 0;                 // tuner's time of the picked DMMA candidate with thin tiles
  bool panel_cst = false;                  // complex64 SIMT panel-step tiles stage C (tuned once per plan)
  std::vector<char> pick;                  // per level candidate
  std::vector<float> tune_ms;              // [candidate][level] measured times
  bool tuned = true;
  // complex64 TMA Schur candidates: per level the packed fronts, the pack items
  // (packed front, K chunk) and the output tiles of 128 and 64 complex columns
  std::vector<int64_t> pk_ptr, pi_ptr, tt_ptr[2];
  std::vector<tc::PackFront> pk;
  std::vector<int2> pitems;
  std::vector<tc::TmaTask> tt[2];
  int64_t stage_rows = 0;                  // packed rows of the widest level, per frequency
  bool tma_ok = false;                     // staging buffer and tensor map ready for this sweep
  DBuf d_pk, d_pitems, d_tt[2];
  CUtensorMap tmap{};                      // 2D map over the staging buffer (128-byte rows)
  ~Plan() {
    for (auto &g : graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto &e : ev) cudaEventDestroy(e);
  }
};

static void add_tiles(std::vector<GemmTask> &v, int bm, int bn, int f, int r0, int r1, int c0, int c1, int k0,
                      int k1) {
  for (int r = r0; r < r1; r += bm)
    for (int c = c0; c < c1; c += bn) v.push_back(GemmTask{f, r, c, r1, c1, k0, k1});
}
static void add_tiles(std::vector<GemmTask> &v, int shape, int f, int r0, int r1, int c0, int c1, int k0, int k1) {
  add_tiles(v, tile_bm(shape), tile_bn(shape), f, r0, r1, c0, c1, k0, k1);
}

// Panel-step GEMMs of one front at panel j0 (left-looking, blocked in two levels).
// The pivots are taken in blocks of kOuter columns [b0, b1): when a block starts,
// its columns (rows [b0, m)) get every earlier pivot at once (K = [0, b0)), so the
// L columns left of the block are read once per block instead of once per panel;
// the block's later panels then need only the pivots [b0, j0).  The U rows of a
// panel are updated after its row swaps: their columns inside the block by the
// pivots [b0, j0) (the block update already applied [0, b0)), the columns right of
// the block by all pivots [0, j0).  (Row swaps stay inside [j0, k), and every row in
// [b0, m) received the same block update, so the swaps keep the updates consistent.)
constexpr int kOuter = 128;
static void add_panel_col_tiles(std::vector<GemmTask> &v, int bm, int bn, int f, int k, int m, int j0) {
  const int b0 = j0 / kOuter * kOuter, b1 = std::min(k, b0 + kOuter);
  if (j0 == b0) {
    if (j0 > 0) add_tiles(v, bm, bn, f, j0, m, j0, b1, 0, j0);
  } else {
    add_tiles(v, bm, bn, f, j0, m, j0, std::min(k, j0 + kPanel), b0, j0);
  }
}
static void add_panel_row_tiles(std::vector<GemmTask> &v, int bm, int bn, int f, int k, int m, int j0) {
  const int b0 = j0 / kOuter * kOuter, b1 = std::min(k, b0 + kOuter), j1 = std::min(k, j0 + kPanel);
  if (j0 > b0 && j1 < b1) add_tiles(v, bm, bn, f, j0, j1, j1, b1, b0, j0);
  if (j0 > 0 && std::max(j1, b1) < m) add_tiles(v, bm, bn, f, j0, j1, std::max(j1, b1), m, 0, j0);
}
// Narrow panel-step regions: the columns add_panel_col_tiles updates at panel j0
// (the block's columns when j0 starts a block, else the panel's), and the rows
// [j0, j1) of add_panel_row_tiles, at most kThinMax wide / high
constexpr int kThinMax = 8;
static bool panel_col_narrow(int k, int j0) {
  const int b0 = j0 / kOuter * kOuter, b1 = std::min(k, b0 + kOuter);
  return (j0 == b0 ? b1 : std::min(k, j0 + kPanel)) - j0 <= kThinMax;
}
static bool panel_row_narrow(int k, int j0) { return std::min(k, j0 + kPanel) - j0 <= kThinMax; }

Plan *build_plan(Handle &h, int small_m, bool tensor_schur) {
  Symbolic &S = h.sym;
  Plan *P = new Plan();
  P->small_m = small_m;
  P->small_ptr.assign(1, 0);
  P->large_ptr.assign(1, 0);
  P->schur_ptr.assign(1, 0);
  P->step_ptr.assign(1, 0);
  for (int l = 0; l < S.nlevel; ++l) {
    int lk = 0, lu = 0;
    for (int64_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
      const int f = S.level_fronts[q];
      lk = std::max(lk, S.k[f]);
      lu = std::max(lu, S.m[f] - S.k[f]);
    }
    P->lvl_maxk.push_back(lk);
    P->lvl_maxu.push_back(lu);
    int mm = 0, ml = 0, kmax = 0;
    std::vector<int> large;
    for (int64_t q = S.level_ptr[l]; q < S.level_ptr[l + 1]; ++q) {
      const int f = S.level_fronts[q];
      if (S.m[f] <= small_m) {
        P->fronts_small.push_back(f);
        mm = std::max(mm, S.m[f]);
      } else {
        large.push_back(f);
        ml = std::max(ml, S.m[f]);
        kmax = std::max(kmax, S.k[f]);
      }
    }
    P->fronts_large.insert(P->fronts_large.end(), large.begin(), large.end());
    P->small_ptr.push_back((int)P->fronts_small.size());
    P->large_ptr.push_back((int)P->fronts_large.size());
    P->small_maxm.push_back(mm);
    P->maxm_large.push_back(ml);
    P->maxk_large.push_back(kmax);
    const int ns = (kmax + kPanel - 1) / kPanel;
    P->nsteps.push_back(ns);
    P->level_step0.push_back((int64_t)P->step_ptr.size() - 1);
    // left-looking (Crout) steps: before panel j0 its columns get all earlier
    // pivots (skinny GEMM, K = j0), after it the U row block does (short GEMM)
    for (int s = 0; s < ns; ++s) {
      const int j0 = s * kPanel;
      for (int f : large)
        if (j0 < S.k[f]) add_panel_col_tiles(P->tasks, tile_bm(kSkinny), tile_bn(kSkinny), f, S.k[f], S.m[f], j0);
      P->step_ptr.push_back((int64_t)P->tasks.size());
      for (int f : large)
        if (j0 < S.k[f]) add_panel_row_tiles(P->tasks, tile_bm(kShort), tile_bn(kShort), f, S.k[f], S.m[f], j0);
      P->step_ptr.push_back((int64_t)P->tasks.size());
    }
    P->schur_ptr.push_back((int64_t)P->tasks.size());
  }
  // Schur tasks appended after all step tasks (own index range per level)
  std::vector<int64_t> sp(1, (int64_t)P->tasks.size());
  for (int l = 0; l < S.nlevel; ++l) {
    for (int q = P->large_ptr[l]; q < P->large_ptr[l + 1]; ++q) {
      const int f = P->fronts_large[q], k = S.k[f], m = S.m[f];
      if (m > k) add_tiles(P->tasks, kSquare, f, k, m, k, m, 0, k);
      P->schur_flops += 8.0 * k * (double)(m - k) * (m - k);
    }
    sp.push_back((int64_t)P->tasks.size());
  }
  P->schur_ptr = sp;
  P->pick.assign(S.nlevel, 0);
  P->tuned = false;
  if (tensor_schur) {
    // packed operands of every front with an update block, level by level (the
    // staging buffer is reused per level), and the TMA kernels' tiles
    P->pk_ptr.assign(1, 0);
    P->pi_ptr.assign(1, 0);
    P->tt_ptr[0].assign(1, 0);
    P->tt_ptr[1].assign(1, 0);
    for (int l = 0; l < S.nlevel; ++l) {
      int64_t base = 0;
      // levels whose fronts are mostly padding in 128-row tiles stay on the SIMT
      // candidate (no packed operands, no staging rows)
      double work = 0, padded = 0;
      for (int q = P->large_ptr[l]; q < P->large_ptr[l + 1]; ++q) {
        const int f = P->fronts_large[q], k = S.k[f], u = S.m[f] - k;
        if (u <= 0 || k <= 0) continue;
        const double au = (u + tc::PADC - 1) / tc::PADC * tc::PADC, kp = (k + tc::KCH - 1) / tc::KCH * tc::KCH;
        work += (double)u * u * k;
        padded += au * au * kp;
      }
      const bool eligible = work > 0 && padded <= 2.5 * work;
      for (int q = P->large_ptr[l]; q < P->large_ptr[l + 1] && eligible; ++q) {
        const int f = P->fronts_large[q], k = S.k[f], m = S.m[f], u = m - k;
        if (u <= 0 || k <= 0) continue;
        const int kc = (k + tc::KCH - 1) / tc::KCH, au = (u + tc::PADC - 1) / tc::PADC * tc::PADC;
        const int pf = (int)P->pk.size();
        P->pk.push_back(tc::PackFront{base, f, kc, au, au});
        for (int c = 0; c < kc; ++c) P->pitems.push_back(make_int2(pf, c));
        for (int v = 0; v < 2; ++v) {
          const int bnc = v == 0 ? 128 : 64;
          for (int r0 = k; r0 < m; r0 += tc::BM)
            for (int c0 = k; c0 < m; c0 += bnc)
              P->tt[v].push_back(tc::TmaTask{base, f, r0, c0, m, m, kc, au, au, r0 - k, 2 * (c0 - k)});
        }
        base += tc::pack_rows(kc, au, au);
      }
      P->stage_rows = std::max(P->stage_rows, base);
      P->pk_ptr.push_back((int64_t)P->pk.size());
      P->pi_ptr.push_back((int64_t)P->pitems.size());
      P->tt_ptr[0].push_back((int64_t)P->tt[0].size());
      P->tt_ptr[1].push_back((int64_t)P->tt[1].size());
    }
  }
  if (!tensor_schur) {
    std::vector<int64_t> sb(1, (int64_t)P->tasks.size());
    for (int l = 0; l < S.nlevel; ++l) {
      for (int q = P->large_ptr[l]; q < P->large_ptr[l + 1]; ++q) {
        const int f = P->fronts_large[q], k = S.k[f], m = S.m[f];
        if (m > k) add_tiles(P->tasks, kSquare64, f, k, m, k, m, 0, k);
      }
      sb.push_back((int64_t)P->tasks.size());
    }
    P->schur_ptr_b = sb;
    // panel-step GEMMs in DMMA tiles: 128x32 for the panel columns, 32x128 for the
    // U rows, in the (level, step) order of step_ptr
    P->step_ptr_d.assign(1, (int64_t)P->tasks.size());
    for (int l = 0; l < S.nlevel; ++l) {
      for (int st = 0; st < P->nsteps[l]; ++st) {
        const int j0 = st * kPanel;
        for (int q = P->large_ptr[l]; q < P->large_ptr[l + 1]; ++q) {
          const int f = P->fronts_large[q];
          if (j0 < S.k[f]) add_panel_col_tiles(P->tasks, 128, 32, f, S.k[f], S.m[f], j0);
        }
        P->step_ptr_d.push_back((int64_t)P->tasks.size());
        for (int q = P->large_ptr[l]; q < P->large_ptr[l + 1]; ++q) {
          const int f = P->fronts_large[q];
          if (j0 < S.k[f]) add_panel_row_tiles(P->tasks, 32, 128, f, S.k[f], S.m[f], j0);
        }
        P->step_ptr_d.push_back((int64_t)P->tasks.size());
      }
    }
    // the same slots split into wide tasks (DMMA tiles) and narrow ones (thin tiles)
    P->step_ptr_tw.assign(1, (int64_t)P->tasks.size());
    for (int l = 0; l < S.nlevel; ++l)
      for (int st = 0; st < P->nsteps[l]; ++st) {
        const int j0 = st * kPanel;
        for (int q = P->large_ptr[l]; q < P->large_ptr[l + 1]; ++q) {
          const int f = P->fronts_large[q];
          if (j0 < S.k[f] && !panel_col_narrow(S.k[f], j0)) add_panel_col_tiles(P->tasks, 128, 32, f, S.k[f], S.m[f], j0);
        }
        P->step_ptr_tw.push_back((int64_t)P->tasks.size());
        for (int q = P->large_ptr[l]; q < P->large_ptr[l + 1]; ++q) {
          const int f = P->fronts_large[q];
          if (j0 < S.k[f] && !panel_row_narrow(S.k[f], j0)) add_panel_row_tiles(P->tasks, 32, 128, f, S.k[f], S.m[f], j0);
        }
        P->step_ptr_tw.push_back((int64_t)P->tasks.size());
      }
    P->step_ptr_tn.assign(1, (int64_t)P->tasks.size());
    for (int l = 0; l < S.nlevel; ++l)
      for (int st = 0; st < P->nsteps[l]; ++st) {
        const int j0 = st * kPanel;
        for (int q = P->large_ptr[l]; q < P->large_ptr[l + 1]; ++q) {
          const int f = P->fronts_large[q];
          if (j0 < S.k[f] && panel_col_narrow(S.k[f], j0))
            add_panel_col_tiles(P->tasks, tile_bm(kThinCol), tile_bn(kThinCol), f, S.k[f], S.m[f], j0);
        }
        P->step_ptr_tn.push_back((int64_t)P->tasks.size());
        for (int q = P->large_ptr[l]; q < P->large_ptr[l + 1]; ++q) {
          const int f = P->fronts_large[q];
          if (j0 < S.k[f] && panel_row_narrow(S.k[f], j0))
            add_panel_row_tiles(P->tasks, tile_bm(kThinRow), tile_bn(kThinRow), f, S.k[f], S.m[f], j0);
        }
        P->step_ptr_tn.push_back((int64_t)P->tasks.size());
      }
    P->thin_tasks = P->step_ptr_tn.back() - P->step_ptr_tn.front();
    P->tuned = false;
  }
  return P;
}

// Condensed values from the global K, M (and D) through the fixed-order gather
// lists: the condensed matrices (new order), ks | kq, ms (and ds), Qz.  Run after
// the analysis and again after a value-only reassembly (same mesh and pattern).
int gather_values(Handle &h) {
  const int64_t n = h.sym.n;
  const size_t cb = (size_t)h.c_nnz * sizeof(cd);
  SS_CK(dalloc(h.dKc, cb));
  SS_CK(dalloc(h.dMc, cb));
  SS_CK(dalloc(h.dks, 2 * n * sizeof(cd)));   // ks | kq
  SS_CK(dalloc(h.dms, n * sizeof(cd)));
  SS_CK(dalloc(h.dQz, sizeof(cd)));
  const unsigned gb = (unsigned)((h.c_nnz + 255) / 256), vb = (unsigned)((n + 255) / 256);
  const int64_t *gp = h.dg_ptr.as<int64_t>(), *gs = h.dg_src.as<int64_t>();
  const int64_t *vp = h.dv_ptr.as<int64_t>(), *vs = h.dv_src.as<int64_t>();
  gather_sum_kernel<<<gb, 256, 0, h.stream>>>(h.c_nnz, gp, gs, h.dK.as<cd>(), h.dKc.as<cd>());
  gather_sum_kernel<<<gb, 256, 0, h.stream>>>(h.c_nnz, gp, gs, h.dM.as<cd>(), h.dMc.as<cd>());
  gather_sum_kernel<<<(unsigned)((2 * n + 255) / 256), 256, 0, h.stream>>>(2 * n, vp, vs, h.dK.as<cd>(), h.dks.as<cd>());
  gather_sum_kernel<<<vb, 256, 0, h.stream>>>(n, vp, vs, h.dM.as<cd>(), h.dms.as<cd>());
  gather_sum_kernel<<<1, 256, 0, h.stream>>>(1, h.dq_ptr.as<int64_t>(), h.dq_src.as<int64_t>(), h.dK.as<cd>(),
                                             h.dQz.as<cd>());
  if (h.have_D) {
    SS_CK(dalloc(h.dDc, cb));
    SS_CK(dalloc(h.dds, n * sizeof(cd)));
    gather_sum_kernel<<<gb, 256, 0, h.stream>>>(h.c_nnz, gp, gs, h.dD.as<cd>(), h.dDc.as<cd>());
    gather_sum_kernel<<<vb, 256, 0, h.stream>>>(n, vp, vs, h.dD.as<cd>(), h.dds.as<cd>());
  }
  SS_CK(cudaGetLastError());
  SS_CK(cudaStreamSynchronize(h.stream));
  return SS_OK;
}

int launch_condense(Handle &h) {
  Symbolic &S = h.sym;
  const int64_t n = S.n;
  // gathers in the new entry order
  std::vector<int64_t> gp(h.c_nnz + 1, 0), gs;
  gs.reserve(h.ag_src.size());
  for (int64_t t = 0; t < h.c_nnz; ++t) {
    const int64_t o = h.c_perm[t];
    gs.insert(gs.end(), h.ag_src.begin() + h.ag_ptr[o], h.ag_src.begin() + h.ag_ptr[o + 1]);
    gp[t + 1] = (int64_t)gs.size();
  }
  std::vector<int64_t> vp(2 * n + 1, 0), vs;
  for (int w = 0; w < 2; ++w)
    for (int64_t R = 0; R < n; ++R) {
      const int64_t P = S.act_of_new[R] + w * n;
      vs.insert(vs.end(), h.vg_src.begin() + h.vg_ptr[P], h.vg_src.begin() + h.vg_ptr[P + 1]);
      vp[w * n + R + 1] = (int64_t)vs.size();
    }
  std::vector<int64_t> qp = {0, (int64_t)h.qz_src.size()};
  SS_CK(dupload(h.dc_ptr, h.c_ptr));
  SS_CK(dupload(h.dc_idx, h.c_idx));
  SS_CK(dupload(h.dg_ptr, gp));
  SS_CK(dupload(h.dg_src, gs));
  SS_CK(dupload(h.dv_ptr, vp));
  SS_CK(dupload(h.dv_src, vs));
  SS_CK(dupload(h.dq_ptr, qp));
  SS_CK(dupload(h.dq_src, h.qz_src));
  {
    const int rc = gather_values(h);
    if (rc) return rc;
  }
  // symbolic arrays
  SS_CK(dupload(h.d_k, S.k));
  SS_CK(dupload(h.d_m, S.m));
  SS_CK(dupload(h.d_ld, S.ld));
  SS_CK(dupload(h.d_off, S.off));
  SS_CK(dupload(h.d_p0, S.p0));
  SS_CK(dupload(h.d_rows_ptr, S.rows_ptr));
  SS_CK(dupload(h.d_rows, S.rows));
  SS_CK(dupload(h.d_child_ptr, S.child_ptr));
  SS_CK(dupload(h.d_child, S.child));
  SS_CK(dupload(h.d_relpos_ptr, S.relpos_ptr));
  SS_CK(dupload(h.d_relpos, S.relpos));
  SS_CK(dupload(h.d_arrow_ptr, S.arrow_ptr));
  SS_CK(dupload(h.d_arrow_pos, S.arrow_pos));
  SS_CK(dupload(h.d_arrow_slot, S.arrow_slot));
  SS_CK(dupload(h.d_level_fronts, S.level_fronts));
  return SS_OK;
}

}  // namespace ss

namespace ss {

// Krylov settings of one sweep (the handle's options): FGMRES restart length,
// restarts and the relative residual target of the primal and adjoint solves.
// With the dual-weighted charge correction the charge error is about the product
// of the two residuals' effects.
struct SweepOpts {
  int krylov_m = 30;
  int restarts = 1;
  double tol = 1e-8;
};

// Fronts with m up to this are factored whole in shared memory (one CTA each);
// wider ones take the level-batched panel path.  The ceiling is what one CTA's
// shared memory holds (112^2 x 16 bytes, 160^2 x 8 bytes); SS_SMALL_FRONT_M
// overrides the default (a tuning knob).  On the 262k-DOF ME1 cell the batched
// path is as fast as the one-CTA kernel up to m = 96 and faster beyond it, in both
// precisions (measured: the complex64 factorisation takes 1446 ms for 201 points
// at 96, 1521 ms at 128, where the cell's 4256 leaves of m = 97 fall into the
// one-CTA kernel).
template <class T>
static int small_limit() {
  const int cap = sizeof(T) == 8 ? 112 : 160;
  int v = 96;
  if (const char *e = getenv("SS_SMALL_FRONT_M")) v = atoi(e);
  return std::max(0, std::min(cap, v));
}

// 2D tensor map over a staging buffer of `rows` rows of 32 fp32 (128 bytes):
// boxes of 32 x 128 with the 128-byte swizzle the MMA operand descriptors use.
// The encoder is the driver's cuTensorMapEncodeTiled, reached through the
// runtime's entry-point query (no link against the driver library).
static int encode_stage_map(Handle &h, CUtensorMap &map, void *base, int64_t rows) {
  using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                              const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Encode fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      return fail(h, SS_ECUDA, "tensor map: cuTensorMapEncodeTiled not available");
    fn = reinterpret_cast<Encode>(p);
  }
  const cuuint64_t dim[2] = {32, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)tc::ROWB};
  const cuuint32_t box[2] = {32, 128};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dim, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(h, SS_ECUDA, "tensor map: cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return SS_OK;
}

// equilibration at angular frequency w (Ruiz, 3 sweeps)
static int equilibrate(Handle &h, double w) {
  const int64_t n = h.sym.n;
  const unsigned nb = (unsigned)((n + 255) / 256);
  SS_CK(dalloc(h.drow_scale, n * sizeof(double)));
  SS_CK(dalloc(h.dcol_scale, n * sizeof(double)));
  DBuf rmax, cmax;
  SS_CK(dalloc(rmax, n * sizeof(double)));
  SS_CK(dalloc(cmax, n * sizeof(unsigned long long)));
  std::vector<double> ones(n, 1.0);
  SS_CK(cudaMemcpy(h.drow_scale.p, ones.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  SS_CK(cudaMemcpy(h.dcol_scale.p, ones.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  const cd *D = h.have_D && h.beta ? h.dDc.as<cd>() : nullptr;
  for (int it = 0; it < 3; ++it) {
    row_absmax_kernel<<<nb, 256, 0, h.stream>>>(n, h.dc_ptr.as<int64_t>(), h.dc_idx.as<int64_t>(), h.dKc.as<cd>(),
                                                h.dMc.as<cd>(), D, w * w, w * h.beta, h.drow_scale.as<double>(),
                                                h.dcol_scale.as<double>(), rmax.as<double>(), nullptr);
    scale_update_kernel<<<nb, 256, 0, h.stream>>>(n, h.drow_scale.as<double>(), rmax.as<double>(), nullptr);
    SS_CK(cudaMemsetAsync(cmax.p, 0, n * sizeof(unsigned long long), h.stream));
    row_absmax_kernel<<<nb, 256, 0, h.stream>>>(n, h.dc_ptr.as<int64_t>(), h.dc_idx.as<int64_t>(), h.dKc.as<cd>(),
                                                h.dMc.as<cd>(), D, w * w, w * h.beta, h.drow_scale.as<double>(),
                                                h.dcol_scale.as<double>(), rmax.as<double>(),
                                                cmax.as<unsigned long long>());
    scale_update_kernel<<<nb, 256, 0, h.stream>>>(n, h.dcol_scale.as<double>(), nullptr,
                                                  cmax.as<unsigned long long>());
  }
  const size_t cb = (size_t)h.c_nnz * sizeof(cd);
  SS_CK(dalloc(h.dKs, cb));
  SS_CK(dalloc(h.dMs, cb));
  scale_csr_kernel<<<nb, 256, 0, h.stream>>>(n, h.dc_ptr.as<int64_t>(), h.dc_idx.as<int64_t>(),
                                             h.drow_scale.as<double>(), h.dcol_scale.as<double>(), h.dKc.as<cd>(),
                                             h.dKs.as<cd>());
  scale_csr_kernel<<<nb, 256, 0, h.stream>>>(n, h.dc_ptr.as<int64_t>(), h.dc_idx.as<int64_t>(),
                                             h.drow_scale.as<double>(), h.dcol_scale.as<double>(), h.dMc.as<cd>(),
                                             h.dMs.as<cd>());
  if (h.have_D) {
    SS_CK(dalloc(h.dDs, cb));
    scale_csr_kernel<<<nb, 256, 0, h.stream>>>(n, h.dc_ptr.as<int64_t>(), h.dc_idx.as<int64_t>(),
                                               h.drow_scale.as<double>(), h.dcol_scale.as<double>(),
                                               h.dDc.as<cd>(), h.dDs.as<cd>());
  }
  SS_CK(cudaGetLastError());
  h.scale_w = w;
  return SS_OK;
}

template <class T>
struct Sweeper {
  static constexpr size_t kDiagBytes = (size_t)kDiagElems * sizeof(cplx<T>);
  Handle &h;
  Plan &P;
  size_t pivb = 0;   // shared bytes for one front's pivot list (solve kernels)
  // CTA width of a level's solve kernels: no wider than its widest front
  int solve_threads(int l) const {
    const int w = P.lvl_maxk[l] + P.lvl_maxu[l];
    return w <= 64 ? 64 : w <= 128 ? 128 : 256;
  }
  FrontArgs<T> a{};
  int64_t wstride = 0;
  int launches = 0, schur_launches = 0;
  int *tc_err = nullptr;                     // device flag: a tensor-core tile timed out
  std::vector<cudaEvent_t> &ev;              // Schur GEMM timing (the plan's events)
  int nev = 0;
  double schur_ms = 0;
  cplx<T> *stage_wv = nullptr;               // solve workspace baked into the solve graphs
  cd *stage_b = nullptr, *stage_x = nullptr; // solve input / output staging for the graphs
  explicit Sweeper(Handle &hh, Plan &pp) : h(hh), P(pp), ev(pp.ev) {
    pivb = ((size_t)std::max(1, h.sym.max_k) * sizeof(int) + 15) / 16 * 16;
    if (ev.empty()) {
      ev.resize(2 * std::max(1, h.sym.nlevel));
      // recorded once outside any capture: the graphs' event-record nodes then
      // re-record them at every replay and their elapsed times can be read
      for (auto &e : ev) {
        cudaEventCreate(&e);
        cudaEventRecord(e, h.stream);
      }
    }
  }

  // Run `body` (a launch sequence on h.stream) through a cached CUDA graph keyed by
  // (kind, nb, key pointers): captured on first use, replayed afterwards.
  template <class Body>
  int graphed(int kind, int nb, std::initializer_list<const void *> key, Body body) {
    const void *k[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    int i = 0;
    for (const void *p : key) k[i++] = p;
    for (auto &g : P.graphs) {
      if (g.kind != kind || g.nb != nb) continue;
      bool same = true;
      for (int j = 0; j < 8; ++j) same = same && g.key[j] == k[j];
      if (!same) continue;
      SS_CK(cudaGraphLaunch(g.exec, h.stream));
      launches += g.launches;
      schur_launches += g.schur_launches;
      return SS_OK;
    }
    const int l0 = launches, s0 = schur_launches;
    cudaGraph_t graph = nullptr;
    SS_CK(cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal));
    const int rc = body();
    const cudaError_t ce = cudaStreamEndCapture(h.stream, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    SS_CK(ce);
    Plan::Graph g;
    g.kind = kind;
    g.nb = nb;
    for (int j = 0; j < 8; ++j) g.key[j] = k[j];
    const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    SS_CK(ie);
    g.launches = launches - l0;
    g.schur_launches = schur_launches - s0;
    P.graphs.push_back(g);
    SS_CK(cudaGraphLaunch(g.exec, h.stream));
    return SS_OK;
  }
  // factorisation of a chunk as one graph replay
  int factor_graphed(int nb) {
    {
      const int rc = tune(nb);
      if (rc) return rc;
    }
    // every level's launch chain is one graph replay; the Schur update between
    // levels is a direct, event-timed launch (timed kernel time of the dominant GEMM)
    nev = 0;
    for (int l = 0; l < h.sym.nlevel; ++l) {
      int rc = graphed(100 + l, nb, {a.arena, a.piv, a.omega, a.Kc, a.Mc, a.Dc, a.nperturb, tc_err},
                       [&] { return factor_level(l, nb); });
      if (rc) return rc;
      rc = schur_level(l, nb);
      if (rc) return rc;
    }
    return SS_OK;
  }
  // x <- A'^-1 b (kind 1) or A'^-T b (kind 2) through a graph over fixed staging buffers
  int solve_graphed(int kind, int nb, const cd *b, cd *x) {
    const int64_t n = h.sym.n;
    SS_CK(cudaMemcpyAsync(stage_b, b, (size_t)nb * n * sizeof(cd), cudaMemcpyDeviceToDevice, h.stream));
    int rc = graphed(kind, nb, {a.arena, a.piv, stage_b, stage_x, stage_wv, a.Kc, a.active},
                     [&] { return kind == 1 ? solve(nb, stage_b, stage_x, stage_wv) : solve_t(nb, stage_b, stage_x, stage_wv); });
    if (rc) return rc;
    SS_CK(cudaMemcpyAsync(x, stage_x, (size_t)nb * n * sizeof(cd), cudaMemcpyDeviceToDevice, h.stream));
    return SS_OK;
  }
  // after the stream reached the end of factor(): add up the Schur GEMM time
  void collect(int) {
    for (int i = 0; i < nev; ++i) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
      schur_ms += ms;
    }
    nev = 0;
  }

  // panel-step GEMM of (level, step) slot q: which 0 = panel columns (skinny),
  // 1 = U rows (short); SIMT tiles, or DMMA tiles when the tuner chose them
  int panel_gemm(const FrontArgs<T> &b, int64_t q, int which, int nb) {
    const GemmTask *tasks = P.d_tasks.template as<GemmTask>();
    if constexpr (sizeof(T) == 8) {
      if (P.panel_dmma) {
        const bool thin = P.panel_thin;
        int nl = 0;
        if (thin) {   // the narrow tasks of the slot in thin SIMT tiles
          const int64_t n0 = P.step_ptr_tn[q + which], n1 = P.step_ptr_tn[q + which + 1];
          if (n1 > n0) {
            ++nl;
            const dim3 g((unsigned)(n1 - n0), nb);
            if (which == 0)
              front_gemm_kernel<T, kThinCol><<<g, 256, 0, h.stream>>>(b, tasks + n0);
            else
              front_gemm_kernel<T, kThinRow><<<g, 256, 0, h.stream>>>(b, tasks + n0);
          }
        }
        const std::vector<int64_t> &sp = thin ? P.step_ptr_tw : P.step_ptr_d;
        const int64_t t0 = sp[q + which], t1 = sp[q + which + 1];
        if (t1 == t0) return nl;
        const dim3 grid((unsigned)(t1 - t0), nb);
        if (P.panel_dmma == 3) {
          if (which == 0)
            front_dmma3_kernel<4, 1, true><<<grid, 128, dmma_cst_bytes<4, 1>(), h.stream>>>(b, tasks + t0);
          else
            front_dmma3_kernel<1, 4, true><<<grid, 128, dmma_cst_bytes<1, 4>(), h.stream>>>(b, tasks + t0);
        } else if (P.panel_dmma == 2) {
          if (which == 0)
            front_dmma3_kernel<4, 1><<<grid, 128, 0, h.stream>>>(b, tasks + t0);
          else
            front_dmma3_kernel<1, 4><<<grid, 128, 0, h.stream>>>(b, tasks + t0);
        } else {
          if (which == 0)
            front_dmma_kernel<4, 1><<<grid, 128, 0, h.stream>>>(b, tasks + t0);
          else
            front_dmma_kernel<1, 4><<<grid, 128, 0, h.stream>>>(b, tasks + t0);
        }
        return nl + 1;
      }
    }
    const int64_t t0 = P.step_ptr[q + which], t1 = P.step_ptr[q + which + 1];
    if (t1 == t0) return 0;
    const dim3 grid((unsigned)(t1 - t0), nb);
    if (P.panel_cst) {
      if (which == 0)
        front_gemm_kernel<T, kSkinny, true><<<grid, 256, gemm_cst_bytes<T, kSkinny>(), h.stream>>>(b, tasks + t0);
      else
        front_gemm_kernel<T, kShort, true><<<grid, 256, gemm_cst_bytes<T, kShort>(), h.stream>>>(b, tasks + t0);
    } else {
      if (which == 0)
        front_gemm_kernel<T, kSkinny><<<grid, 256, 0, h.stream>>>(b, tasks + t0);
      else
        front_gemm_kernel<T, kShort><<<grid, 256, 0, h.stream>>>(b, tasks + t0);
    }
    return 1;
  }

  // FP64 Schur update of level l with candidate tile c (0 SIMT 128x64, 1 DMMA
  // 64x64 with three real products per complex block, 2 DMMA 64x64 with four)
  void schur_launch(const FrontArgs<T> &b, int l, int c, int nb) {
    const GemmTask *tasks = P.d_tasks.template as<GemmTask>();
    if constexpr (sizeof(T) == 4) {
      // complex64: candidates 0 / 1 pack the level's operands and run the TMA +
      // tcgen05 kernel with 128 / 64 complex columns per tile; 2 SIMT FP32 128x64
      const int64_t t0 = P.schur_ptr[l], t1 = P.schur_ptr[l + 1];
      const int v = c;   // tile variant
      // SIMT tiles: the third candidate, and the fallback where a level has no
      // packed operands (mostly padding) or the staging buffer is not available
      if (c == 2 || !P.tma_ok || P.tt_ptr[v > 1 ? 0 : v][l + 1] == P.tt_ptr[v > 1 ? 0 : v][l]) {
        if (t1 > t0)
          front_gemm_kernel<T, kSquare><<<dim3((unsigned)(t1 - t0), nb), 256, 0, h.stream>>>(b, tasks + t0);
        return;
      }
      const int64_t i0 = P.pi_ptr[l], i1 = P.pi_ptr[l + 1], q0 = P.tt_ptr[v][l], q1 = P.tt_ptr[v][l + 1];
      cf *ar = reinterpret_cast<cf *>(b.arena);
      tc::pack_kernel<<<dim3((unsigned)(i1 - i0), nb), tc::PACK_THREADS, 0, h.stream>>>(
          ar, b.stride, b.off, b.ld, b.k, b.m, P.d_pk.template as<tc::PackFront>(), P.d_pitems.template as<int2>() + i0,
          h.tc_stage.template as<float>(), P.stage_rows);
      const int64_t items = (q1 - q0) * nb;
      const unsigned grid = (unsigned)std::min<int64_t>(items, h.num_sms);
      const tc::TmaTask *tt = P.d_tt[v].template as<tc::TmaTask>() + q0;
      if (v == 0)
        tc::tma_gemm_kernel<128, 2><<<grid, tc::TmaCfg<128, 2>::THREADS, tc::TmaCfg<128, 2>::SMEM, h.stream>>>(
            P.tmap, ar, b.stride, b.off, b.ld, tt, (int)(q1 - q0), nb, P.stage_rows, tc_err);
      else
        tc::tma_gemm_kernel<64, 3><<<grid, tc::TmaCfg<64, 3>::THREADS, tc::TmaCfg<64, 3>::SMEM, h.stream>>>(
            P.tmap, ar, b.stride, b.off, b.ld, tt, (int)(q1 - q0), nb, P.stage_rows, tc_err);
      return;
    }
    if (c == 0) {
      const int64_t t0 = P.schur_ptr[l], t1 = P.schur_ptr[l + 1];
      front_gemm_kernel<T, kSquare><<<dim3((unsigned)(t1 - t0), nb), 256, 0, h.stream>>>(b, tasks + t0);
      return;
    }
    const int64_t t0 = P.schur_ptr_b[l], t1 = P.schur_ptr_b[l + 1];
    if constexpr (sizeof(T) == 8) {
      if (c == 1)
        front_dmma3_kernel<2, 2><<<dim3((unsigned)(t1 - t0), nb), 128, 0, h.stream>>>(b, tasks + t0);
      else if (c == 3)
        front_dmma3_kernel<2, 2, true><<<dim3((unsigned)(t1 - t0), nb), 128, dmma_cst_bytes<2, 2>(), h.stream>>>(
            b, tasks + t0);
      else
        front_dmma_kernel<2, 2><<<dim3((unsigned)(t1 - t0), nb), 128, 0, h.stream>>>(b, tasks + t0);
    }
  }

  // Autotuner: time every candidate on every level with Schur work, on the chunk's
  // arena before its first factorisation (GEMM time does not depend on the
  // values), and keep the fastest per level.  SS_SCHUR_TILE=0|1|2 (FP64) and
  // SS_SCHUR_TILE_C64=0|1|2 (complex64) force one.
  int tune(int nb) {
    if (P.tuned) return SS_OK;
    const Symbolic &S = h.sym;
    const char *force = getenv(sizeof(T) == 8 ? "SS_SCHUR_TILE" : "SS_SCHUR_TILE_C64");
    // FP64: SIMT 128x64, DMMA three products, DMMA four products, DMMA three
    // products with C staged; complex64: TMA 128 / 64 columns, SIMT
    constexpr int NC = sizeof(T) == 8 ? 4 : 3;
    P.tune_ms.assign((size_t)NC * S.nlevel, 0.f);
    if (!force) {
      std::vector<cudaEvent_t> e(2 * NC * S.nlevel);
      for (auto &x : e) SS_CK(cudaEventCreate(&x));
      for (int c = 0; c < NC; ++c)
        for (int l = 0; l < S.nlevel; ++l) {
          if (P.schur_ptr[l + 1] == P.schur_ptr[l]) continue;
          FrontArgs<T> b = a;
          cudaEventRecord(e[2 * (c * S.nlevel + l)], h.stream);
          schur_launch(b, l, c, nb);
          cudaEventRecord(e[2 * (c * S.nlevel + l) + 1], h.stream);
        }
      SS_CK(cudaGetLastError());
      SS_CK(cudaStreamSynchronize(h.stream));
      for (int c = 0; c < NC; ++c)
        for (int l = 0; l < S.nlevel; ++l) {
          if (P.schur_ptr[l + 1] == P.schur_ptr[l]) continue;
          cudaEventElapsedTime(&P.tune_ms[c * S.nlevel + l], e[2 * (c * S.nlevel + l)], e[2 * (c * S.nlevel + l) + 1]);
        }
      for (auto &x : e) cudaEventDestroy(x);
      if constexpr (sizeof(T) == 8) {
      // panel-step GEMMs (FP64): all of them once with SIMT tiles, once with DMMA
      // tiles, once with DMMA tiles of three real products per complex block, once
      // with those tiles staging C in shared memory
      constexpr int NP = 4;
      cudaEvent_t pe[2 * NP];
      for (auto &x : pe) SS_CK(cudaEventCreate(&x));
      float pt[NP] = {0, 0, 0, 0};
      P.panel_thin = false;
      for (int c = 0; c < NP; ++c) {
        P.panel_dmma = c;
        cudaEventRecord(pe[2 * c], h.stream);
        for (int l = 0; l < S.nlevel; ++l) {
          FrontArgs<T> b = a;
          b.fronts = P.d_large.as<int>() + P.large_ptr[l];
          for (int st = 0; st < P.nsteps[l]; ++st) {
            const int64_t q = P.level_step0[l] + 2 * st;
            panel_gemm(b, q, 0, nb);
            panel_gemm(b, q, 1, nb);
          }
        }
        cudaEventRecord(pe[2 * c + 1], h.stream);
      }
      SS_CK(cudaGetLastError());
      SS_CK(cudaStreamSynchronize(h.stream));
      for (int c = 0; c < NP; ++c) cudaEventElapsedTime(&pt[c], pe[2 * c], pe[2 * c + 1]);
      P.panel_dmma = 0;
      for (int c = 1; c < NP; ++c)
        if (pt[c] < pt[P.panel_dmma]) P.panel_dmma = c;
      for (int c = 0; c < NP; ++c) P.panel_ms[c] = pt[c];
      // the picked DMMA tiles once more with the narrow tasks in thin SIMT tiles;
      // kept if faster
      P.panel_thin = false;
      if (P.panel_dmma > 0 && P.thin_tasks > 0) {
        P.panel_thin = true;
        cudaEventRecord(pe[0], h.stream);
        for (int l = 0; l < S.nlevel; ++l) {
          FrontArgs<T> b = a;
          b.fronts = P.d_large.as<int>() + P.large_ptr[l];
          for (int st = 0; st < P.nsteps[l]; ++st) {
            const int64_t q = P.level_step0[l] + 2 * st;
            panel_gemm(b, q, 0, nb);
            panel_gemm(b, q, 1, nb);
          }
        }
        cudaEventRecord(pe[1], h.stream);
        SS_CK(cudaGetLastError());
        SS_CK(cudaStreamSynchronize(h.stream));
        cudaEventElapsedTime(&P.panel_thin_ms, pe[0], pe[1]);
        P.panel_thin = P.panel_thin_ms < pt[P.panel_dmma];
      }
      for (auto &x : pe) cudaEventDestroy(x);
      } else {
      // panel-step GEMMs (complex64, SIMT tiles): once reading C after the K loop,
      // once with C staged in shared memory while it runs
      cudaEvent_t pe[4];
      for (auto &x : pe) SS_CK(cudaEventCreate(&x));
      float pt[2] = {0, 0};
      for (int c = 0; c < 2; ++c) {
        P.panel_cst = c == 1;
        cudaEventRecord(pe[2 * c], h.stream);
        for (int l = 0; l < S.nlevel; ++l) {
          FrontArgs<T> b = a;
          b.fronts = P.d_large.as<int>() + P.large_ptr[l];
          for (int st = 0; st < P.nsteps[l]; ++st) {
            const int64_t q = P.level_step0[l] + 2 * st;
            panel_gemm(b, q, 0, nb);
            panel_gemm(b, q, 1, nb);
          }
        }
        cudaEventRecord(pe[2 * c + 1], h.stream);
      }
      SS_CK(cudaGetLastError());
      SS_CK(cudaStreamSynchronize(h.stream));
      for (int c = 0; c < 2; ++c) cudaEventElapsedTime(&pt[c], pe[2 * c], pe[2 * c + 1]);
      for (auto &x : pe) cudaEventDestroy(x);
      P.panel_cst = pt[1] < pt[0];
      P.panel_ms[0] = pt[0];
      P.panel_ms[3] = pt[1];
      }
    } else {
      // a forced DMMA Schur tile puts the panel-step GEMMs on the same kind of tile
      P.panel_dmma = sizeof(T) != 8 ? 0 : atoi(force) == 2 ? 1 : atoi(force) == 1 ? 2 : atoi(force) == 3 ? 3 : 0;
      P.panel_thin = false;
    }
    if constexpr (sizeof(T) == 8) {
      // measurement / test override of the thin tiles (they go with the DMMA tiles)
      if (const char *e = getenv("SS_PANEL_THIN")) P.panel_thin = atoi(e) != 0 && P.panel_dmma > 0 && P.thin_tasks > 0;
    }
    if constexpr (sizeof(T) == 4) {
      if (const char *e = getenv("SS_PANEL_CST")) P.panel_cst = atoi(e) != 0;   // measurement override
    }
    for (int l = 0; l < S.nlevel; ++l) {
      int best = 0;
      // complex64 levels without packed operands run the SIMT tiles whatever the
      // candidate: they count as the SIMT candidate
      const bool no_tma = sizeof(T) == 4 && (!P.tma_ok || P.tt_ptr[0][l + 1] == P.tt_ptr[0][l]);
      if (no_tma) {
        best = 2;
      } else if (force) {
        best = std::max(0, std::min(NC - 1, atoi(force)));
      } else {
        for (int c = 1; c < NC; ++c)
          if (P.tune_ms[c * S.nlevel + l] < P.tune_ms[best * S.nlevel + l]) best = c;
      }
      P.pick[l] = (char)best;
    }
    P.tuned = true;
    return SS_OK;
  }

  // level l of the factorisation up to (not including) its Schur update: small
  // fronts, large-front assembly and the panel steps
  int factor_level(int l, int nb) {
    {
      const int ns = P.small_ptr[l + 1] - P.small_ptr[l];
      if (ns) {
        FrontArgs<T> b = a;
        b.fronts = P.d_small.as<int>() + P.small_ptr[l];
        const int mm = P.small_maxm[l];
        front_small_kernel<T><<<dim3(ns, nb), kSmallThreads, (size_t)mm * mm * sizeof(cplx<T>), h.stream>>>(b);
        ++launches;
      }
      const int nl = P.large_ptr[l + 1] - P.large_ptr[l];
      if (!nl) return SS_OK;
      FrontArgs<T> b = a;
      b.fronts = P.d_large.as<int>() + P.large_ptr[l];
      const int ml = P.maxm_large[l];
      // grid (frequency, front, row chunk); gridDim.y is at most 65535, so a
      // level with more large fronts is launched in slices of fronts
      for (int s0 = 0; s0 < nl; s0 += 65535) {
        const int ns1 = std::min(nl - s0, 65535);
        FrontArgs<T> bs = b;
        bs.fronts = b.fronts + s0;
        const int av = asm_variant<T>();
        // staged kernel: as many warps (<= 8) as rows of the level's widest front
        // fit in one CTA's shared memory, four rows per warp
        const int snw = std::min(8, kAsmSmemMax / (ml * (int)sizeof(cplx<T>)));
        if (av == 2 && snw >= 1) {
          const int rpc = 4 * snw;
          front_assemble_rows_smem_kernel<T><<<dim3(nb, ns1, (ml + rpc - 1) / rpc), 32 * snw,
                                               (size_t)snw * ml * sizeof(cplx<T>), h.stream>>>(bs, rpc, ml);
        } else if (av >= 1) {
          front_assemble_rows_kernel<T><<<dim3(nb, ns1, (ml + kAsmRowsPerCta - 1) / kAsmRowsPerCta), 256, 0,
                                          h.stream>>>(bs);
        } else {
          const int ar = asm_rows(ml);
          front_assemble_large_kernel<T><<<dim3(nb, ns1, (ml + ar - 1) / ar), 256, 0, h.stream>>>(bs, ar);
        }
        ++launches;
      }
      const GemmTask *tasks = P.d_tasks.as<GemmTask>();
      // row/column-parallel panel kernels: CTAs no wider than the level's fronts
      // (narrow fronts then run more CTAs per SM instead of idle threads)
      const int bs = ml <= 64 ? 64 : ml <= 128 ? 128 : 256;
      const unsigned zc = (unsigned)((ml + bs - 1) / bs);
      for (int s = 0; s < P.nsteps[l]; ++s) {
        const int j0 = s * kPanel;
        const int64_t q = P.level_step0[l] + 2 * s;
        const int64_t g0 = P.step_ptr[q], g1 = P.step_ptr[q + 1], g2 = P.step_ptr[q + 2];
        if (g1 > g0) {   // panel columns <- earlier pivots
          launches += panel_gemm(b, q, 0, nb);
        }
        const size_t psm = (size_t)std::max(0, P.maxk_large[l] - j0) * (kPanel + 1) * sizeof(cplx<T>);
        const int prow = P.maxk_large[l] - j0;   // panel rows of the widest front
        const int pth = prow <= 64 ? 128 : prow <= 160 ? 256 : kPanelThreads;
        if (psm <= (size_t)kPanelSmemMax)
          front_panel_smem_kernel<T><<<dim3(nl, nb), pth, psm, h.stream>>>(b, j0);
        else
          front_panel_kernel<T><<<dim3(nl, nb), 256, 0, h.stream>>>(b, j0);
        const int rpw = l21_rpw<T>();
        if (rpw > 0) {
          // rows per CTA: (bs / 32) warps x rpw rows
          const unsigned zl = (unsigned)((ml + (bs / 32) * rpw - 1) / ((bs / 32) * rpw));
          if (rpw == 32)
            front_l21_kernel<T, 32><<<dim3(nl, nb, zl), bs, l21_smem<T>(bs, 32), h.stream>>>(b, j0);
          else
            front_l21_kernel<T, 16><<<dim3(nl, nb, zl), bs, l21_smem<T>(bs, 16), h.stream>>>(b, j0);
        } else {
          front_l21_kernel<T, 0><<<dim3(nl, nb, zc), bs, 0, h.stream>>>(b, j0);
        }
        front_swap_kernel<T><<<dim3(nl, nb, zc), bs, 0, h.stream>>>(b, j0);
        if (g2 > g1) {   // U row block <- earlier pivots
          launches += panel_gemm(b, q, 1, nb);
        }
        front_u12_trsm_kernel<T><<<dim3(nl, nb, zc), bs, 0, h.stream>>>(b, j0);
        launches += 4;
      }
    }
    SS_CK(cudaGetLastError());
    return SS_OK;
  }

  // Schur update of level l's large fronts, launched directly and timed by a pair
  // of events on the launch stream
  int schur_level(int l, int nb) {
    const int64_t t0 = P.schur_ptr[l], t1 = P.schur_ptr[l + 1];
    if (t1 == t0) return SS_OK;
    FrontArgs<T> b = a;
    b.fronts = P.d_large.as<int>() + P.large_ptr[l];
    const GemmTask *tasks = P.d_tasks.as<GemmTask>();
    cudaEventRecord(ev[2 * nev], h.stream);
    schur_launch(b, l, P.pick[l], nb);
    cudaEventRecord(ev[2 * nev + 1], h.stream);
    ++nev;
    ++launches;
    ++schur_launches;
    SS_CK(cudaGetLastError());
    return SS_OK;
  }

  // x <- A'^-1 b for nb frequencies (x may alias nothing; wv workspace)
  int solve(int nb, const cd *b, cd *x, cplx<T> *wv) {
    const Symbolic &S = h.sym;
    const size_t sm = (size_t)S.max_m * sizeof(cplx<T>);
    const size_t smk = (size_t)std::max(1, S.max_k) * sizeof(cplx<T>);
    for (int l = 0; l < S.nlevel; ++l) {
      FrontArgs<T> c = a;
      c.fronts = h.d_level_fronts.as<int>() + S.level_ptr[l];
      const int nf = (int)(S.level_ptr[l + 1] - S.level_ptr[l]);
      const int bs = solve_threads(l);
      front_fwd_kernel<T><<<dim3(nf, nb), bs, sm + kDiagBytes + pivb, h.stream>>>(c, b, x, wv, wstride);
      ++launches;
      if (P.lvl_maxu[l] > 0) {
        const unsigned z = (unsigned)((P.lvl_maxu[l] + kSolveRows - 1) / kSolveRows);
        front_fwd_l21_kernel<T><<<dim3(nf, nb, z), bs, smk, h.stream>>>(c, x, wv, wstride);
        ++launches;
      }
    }
    for (int l = S.nlevel - 1; l >= 0; --l) {
      FrontArgs<T> c = a;
      c.fronts = h.d_level_fronts.as<int>() + S.level_ptr[l];
      const int nf = (int)(S.level_ptr[l + 1] - S.level_ptr[l]);
      const int bs = solve_threads(l);
      if (P.lvl_maxu[l] > 0) {
        const unsigned z = (unsigned)((P.lvl_maxk[l] + kSolveRows - 1) / kSolveRows);
        front_bwd_u12_kernel<T><<<dim3(nf, nb, z), bs, (size_t)P.lvl_maxu[l] * sizeof(cplx<T>), h.stream>>>(c, x);
        ++launches;
      }
      front_bwd_kernel<T><<<dim3(nf, nb), bs, smk + kDiagBytes, h.stream>>>(c, x);
      ++launches;
    }
    SS_CK(cudaGetLastError());
    return SS_OK;
  }
  // mu <- A'^-T c for nb frequencies (same factors; wv workspace)
  int solve_t(int nb, const cd *cvec, cd *mu, cplx<T> *wv) {
    const Symbolic &S = h.sym;
    const size_t sm = (size_t)S.max_m * sizeof(cplx<T>);
    const size_t smk = (size_t)std::max(1, S.max_k) * sizeof(cplx<T>);
    for (int l = 0; l < S.nlevel; ++l) {
      FrontArgs<T> c = a;
      c.fronts = h.d_level_fronts.as<int>() + S.level_ptr[l];
      const int nf = (int)(S.level_ptr[l + 1] - S.level_ptr[l]);
      front_tfwd_kernel<T><<<dim3(nf, nb), solve_threads(l), sm + kDiagBytes, h.stream>>>(c, cvec, mu, wv, wstride);
      ++launches;
      if (P.lvl_maxu[l] > 0) {
        const unsigned z = (unsigned)((P.lvl_maxu[l] + 31) / 32);
        front_tfwd_u12_kernel<T><<<dim3(nf, nb, z), 32 * kTColWarps, smk, h.stream>>>(c, mu, wv, wstride);
        ++launches;
      }
    }
    for (int l = S.nlevel - 1; l >= 0; --l) {
      FrontArgs<T> c = a;
      c.fronts = h.d_level_fronts.as<int>() + S.level_ptr[l];
      const int nf = (int)(S.level_ptr[l + 1] - S.level_ptr[l]);
      if (P.lvl_maxu[l] > 0) {
        const unsigned z = (unsigned)((P.lvl_maxk[l] + 31) / 32);
        front_tbwd_l21_kernel<T><<<dim3(nf, nb, z), 32 * kTColWarps, (size_t)P.lvl_maxu[l] * sizeof(cplx<T>),
                                   h.stream>>>(c, mu);
        ++launches;
      }
      front_tbwd_kernel<T><<<dim3(nf, nb), solve_threads(l), smk + kDiagBytes + pivb, h.stream>>>(c, mu);
      ++launches;
    }
    SS_CK(cudaGetLastError());
    return SS_OK;
  }
};

// Transposed condensed pattern in the new order (built once): row C of A'^T
// lists the rows R with an entry (R, C), ascending, and the slot of (R, C).
static int build_transpose(Handle &h) {
  if (h.dct_ptr.p) return SS_OK;
  const int64_t n = h.sym.n;
  std::vector<int64_t> tp(n + 1, 0), ti(h.c_nnz), ts(h.c_nnz);
  for (int64_t t = 0; t < h.c_nnz; ++t) ++tp[h.c_idx[t] + 1];
  for (int64_t c = 0; c < n; ++c) tp[c + 1] += tp[c];
  std::vector<int64_t> fill(tp.begin(), tp.end() - 1);
  for (int64_t R = 0; R < n; ++R)
    for (int64_t t = h.c_ptr[R]; t < h.c_ptr[R + 1]; ++t) {
      const int64_t q = fill[h.c_idx[t]]++;
      ti[q] = R;
      ts[q] = t;
    }
  SS_CK(dupload(h.dct_ptr, tp));
  SS_CK(dupload(h.dct_idx, ti));
  SS_CK(dupload(h.dct_src, ts));
  return SS_OK;
}

}  // namespace ss

namespace ss {

template <class T>
static int sweep_impl(Handle &h, int n_f, const double *omega, double V, double *Qout, int *status,
                      int *iters, double *disp, const SweepExtra *ex, const SweepOpts &opt) {
  Symbolic &S = h.sym;
  const int64_t n = S.n;
  const int pi = sizeof(T) == 8 ? 0 : 1;
  if (!h.plan[pi]) {
    Plan *P = build_plan(h, small_limit<T>(), sizeof(T) == 4);
    h.plan[pi] = P;
    SS_CK(dupload(P->d_small, P->fronts_small));
    SS_CK(dupload(P->d_large, P->fronts_large));
    SS_CK(dupload(P->d_tasks, P->tasks));
    SS_CK(cudaFuncSetAttribute(front_small_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               small_limit<T>() * small_limit<T>() * (int)sizeof(cplx<T>)));
    SS_CK(cudaFuncSetAttribute(front_panel_smem_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kPanelSmemMax));
    SS_CK(cudaFuncSetAttribute(front_assemble_rows_smem_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kAsmSmemMax));
    SS_CK(cudaFuncSetAttribute(front_gemm_kernel<T, kSkinny, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               gemm_cst_bytes<T, kSkinny>()));
    SS_CK(cudaFuncSetAttribute(front_gemm_kernel<T, kShort, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               gemm_cst_bytes<T, kShort>()));
    if constexpr (sizeof(T) == 8) {
      SS_CK(cudaFuncSetAttribute(front_dmma3_kernel<2, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 dmma_cst_bytes<2, 2>()));
      SS_CK(cudaFuncSetAttribute(front_dmma3_kernel<4, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 dmma_cst_bytes<4, 1>()));
      SS_CK(cudaFuncSetAttribute(front_dmma3_kernel<1, 4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 dmma_cst_bytes<1, 4>()));
    }
    SS_CK(cudaFuncSetAttribute(front_l21_kernel<T, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)l21_smem<T>(256, 32)));
    SS_CK(cudaFuncSetAttribute(front_l21_kernel<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)l21_smem<T>(256, 16)));
    SS_CK(cudaFuncSetAttribute(tc::tma_gemm_kernel<128, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               tc::TmaCfg<128, 2>::SMEM));
    SS_CK(cudaFuncSetAttribute(tc::tma_gemm_kernel<64, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               tc::TmaCfg<64, 3>::SMEM));
    if (sizeof(T) == 4) {
      SS_CK(dupload(P->d_pk, P->pk));
      SS_CK(dupload(P->d_pitems, P->pitems));
      SS_CK(dupload(P->d_tt[0], P->tt[0]));
      SS_CK(dupload(P->d_tt[1], P->tt[1]));
    }
    // solve kernels stage a whole front vector in shared memory
    // (the four triangular kernels also hold one staged 32x32 diagonal block)
    const int vec = (int)std::min<int64_t>(227 * 1024, (int64_t)S.max_m * (int64_t)sizeof(cplx<T>));
    const int vecd = (int)std::min<int64_t>(227 * 1024, vec + (int64_t)kDiagElems * sizeof(cplx<T>) +
                                                           ((int64_t)std::max(1, S.max_k) * 4 + 15) / 16 * 16);
    if (vecd > 48 * 1024) {
      SS_CK(cudaFuncSetAttribute(front_fwd_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, vecd));
      SS_CK(cudaFuncSetAttribute(front_tfwd_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, vecd));
      SS_CK(cudaFuncSetAttribute(front_bwd_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, vecd));
      SS_CK(cudaFuncSetAttribute(front_tbwd_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, vecd));
    }
    if (vec > 48 * 1024) {
      SS_CK(cudaFuncSetAttribute(front_fwd_l21_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, vec));
      // (these two also hold an 8 x 32 static reduction tile)
      SS_CK(cudaFuncSetAttribute(front_tfwd_u12_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 std::min(vec, 223 * 1024)));
      SS_CK(cudaFuncSetAttribute(front_bwd_u12_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, vec));
      SS_CK(cudaFuncSetAttribute(front_tbwd_l21_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 std::min(vec, 223 * 1024)));
    }
  }
  Plan &P = *static_cast<Plan *>(h.plan[pi]);
  double wmax = 0;
  for (int i = 0; i < n_f; ++i) wmax = std::max(wmax, std::fabs(omega[i]));
  if (h.scale_w != wmax) {
    int rc = equilibrate(h, wmax);
    if (rc) return rc;
  }
  const int64_t W = S.relpos_ptr[S.nfront];
  const int krylov_m = opt.krylov_m;
  const int krylov_restarts = opt.restarts;
  const double tol_p = opt.tol, tol_a = opt.tol;
  const double krylov = sizeof(T) == 4 ? (2.0 * krylov_m + 2) * n * sizeof(cd) : 0.0;
  // the mixed sweep always solves the adjoint too (dual-weighted charge correction)
  const bool correct = sizeof(T) == 4;
  const bool need_adjoint = correct || (ex && ex->per_chunk);
  const double per = (double)S.arena * sizeof(cplx<T>) + n * 4.0 + W * (double)sizeof(cplx<T>) + n * 64.0 + krylov +
                     (need_adjoint ? 32.0 * n : 0.0) + 32.0 * n + 256 +
                     (sizeof(T) == 4 ? (double)P.stage_rows * tc::ROWB : 0.0);
  // the Krylov workspace persists in the handle; a sweep without Krylov steps
  // gives its memory back to the fronts
  KrylovWork &kw = h.kw;
  if (!(sizeof(T) == 4 || getenv("SS_FP64_KRYLOV") != nullptr)) kw.release();
  if (sizeof(T) == 8) h.tc_stage.release();   // packed tensor-core operands: mixed sweeps only
  size_t fr = 0, tot = 0;
  SS_CK(cudaMemGetInfo(&fr, &tot));
  fr += kw.bytes();
  // device work buffers persist in the handle: repeated sweeps reuse them
  DBuf &arena = h.wk[0], &piv = h.wk[1], &wv = h.wk[2], &b = h.wk[3], &x = h.wk[4], &r = h.wk[5], &dx = h.wk[6],
       &dom = h.wk[7], &npert = h.wk[8], &nrm = h.wk[9], &dQ = h.wk[10], &mu = h.wk[11], &cvec = h.wk[12];
  // the chunk size counts only memory not already held by these buffers
  for (int i = 0; i < 16; ++i) fr += h.wk[i].bytes;
  fr += h.tc_stage.bytes;
  int B = (int)std::max(1.0, std::min((double)n_f, std::min(256.0, (0.85 * (double)fr - 512e6) / per)));
  // The chunk size counted every buffer above as free, so each one is brought to
  // exactly this sweep's size: larger ones (an earlier sweep's chunk or precision)
  // are released before anything grows, so old and new never coexist.
  {
    const size_t vecb = (size_t)B * n * sizeof(cd);
    const size_t need[16] = {(size_t)B * S.arena * sizeof(cplx<T>), (size_t)B * n * sizeof(int),
                             (size_t)B * std::max<int64_t>(W, 1) * sizeof(cplx<T>), vecb, vecb, vecb, vecb,
                             B * sizeof(double), B * sizeof(int), 2 * B * sizeof(double), 2 * B * sizeof(cd),
                             need_adjoint ? vecb : 0, need_adjoint ? vecb : 0, sizeof(int), vecb, vecb};
    for (int i = 0; i < 16; ++i)
      if (h.wk[i].bytes != need[i]) h.wk[i].release();
    const size_t stage = sizeof(T) == 4 ? (size_t)B * P.stage_rows * tc::ROWB : 0;
    if (h.tc_stage.bytes != stage) h.tc_stage.release();
    if (krylov > 0 && kw.V.bytes != vecb * (size_t)(krylov_m + 1)) kw.release();
  }
  SS_CK(dalloc(arena, (size_t)B * S.arena * sizeof(cplx<T>)));
  if (sizeof(T) == 4) {
    // staging buffer of the packed Schur operands (one level at a time) and the
    // 2D tensor map over it: rows of 32 fp32, boxes of 128 rows, 128-byte swizzle
    P.tma_ok = false;
    const int64_t rows = (int64_t)B * P.stage_rows;
    if (P.stage_rows > 0 && rows < ((int64_t)1 << 31)) {
      SS_CK(dalloc(h.tc_stage, (size_t)rows * tc::ROWB));
      const int rc = encode_stage_map(h, P.tmap, h.tc_stage.p, rows);
      if (rc) return rc;
      P.tma_ok = true;
    }
  }
  SS_CK(dalloc(piv, (size_t)B * n * sizeof(int)));
  SS_CK(dalloc(wv, (size_t)B * std::max<int64_t>(W, 1) * sizeof(cplx<T>)));
  SS_CK(dalloc(b, (size_t)B * n * sizeof(cd)));
  SS_CK(dalloc(x, (size_t)B * n * sizeof(cd)));
  SS_CK(dalloc(r, (size_t)B * n * sizeof(cd)));
  SS_CK(dalloc(dx, (size_t)B * n * sizeof(cd)));
  SS_CK(dalloc(dom, B * sizeof(double)));
  SS_CK(dalloc(npert, B * sizeof(int)));
  SS_CK(dalloc(nrm, 2 * B * sizeof(double)));
  SS_CK(dalloc(dQ, 2 * B * sizeof(cd)));
  if (need_adjoint) {
    SS_CK(dalloc(mu, (size_t)B * n * sizeof(cd)));
    SS_CK(dalloc(cvec, (size_t)B * n * sizeof(cd)));
    int rc = build_transpose(h);
    if (rc) return rc;
  }
  DBuf &stb = h.wk[14], &stx = h.wk[15];
  SS_CK(dalloc(stb, (size_t)B * n * sizeof(cd)));
  SS_CK(dalloc(stx, (size_t)B * n * sizeof(cd)));
  {
    // frequencies still iterating in the Krylov loops (read by the solve kernels)
    SS_CK(dalloc(h.dmask, (size_t)B * sizeof(int)));
    std::vector<int> ones(B, 1);
    SS_CK(cudaMemcpy(h.dmask.p, ones.data(), (size_t)B * sizeof(int), cudaMemcpyHostToDevice));
  }
  DBuf &tcerr = h.wk[13];
  SS_CK(dalloc(tcerr, sizeof(int)));
  SS_CK(cudaMemsetAsync(tcerr.p, 0, sizeof(int), h.stream));
  Sweeper<T> sw(h, P);
  sw.tc_err = tcerr.as<int>();
  sw.stage_b = stb.as<cd>();
  sw.stage_x = stx.as<cd>();
  sw.stage_wv = wv.as<cplx<T>>();
  FrontArgs<T> &a = sw.a;
  a.k = h.d_k.as<int>();
  a.m = h.d_m.as<int>();
  a.ld = h.d_ld.as<int>();
  a.off = h.d_off.as<int64_t>();
  a.p0 = h.d_p0.as<int64_t>();
  a.rows_ptr = h.d_rows_ptr.as<int64_t>();
  a.rows = h.d_rows.as<int64_t>();
  a.child_ptr = h.d_child_ptr.as<int64_t>();
  a.child = h.d_child.as<int>();
  a.relpos_ptr = h.d_relpos_ptr.as<int64_t>();
  a.relpos = h.d_relpos.as<int>();
  a.arrow_ptr = h.d_arrow_ptr.as<int64_t>();
  a.arrow_pos = h.d_arrow_pos.as<int32_t>();
  a.arrow_slot = h.d_arrow_slot.as<int64_t>();
  const bool damp = h.have_D && h.beta != 0.0;
  a.Kc = h.dKs.as<cd>();
  a.Mc = h.dMs.as<cd>();
  a.Dc = damp ? h.dDs.as<cd>() : nullptr;
  a.beta = h.beta;
  a.omega = dom.as<double>();
  a.arena = arena.as<cplx<T>>();
  a.stride = S.arena;
  a.piv = piv.as<int>();
  a.n = n;
  a.tiny = sizeof(T) == 8 ? (T)h.opt.tiny_c128 : (T)h.opt.tiny_c64;
  a.nperturb = npert.as<int>();
  a.active = h.dmask.as<int>();
  sw.wstride = W;
  const int maxit = sizeof(T) == 8 ? 1 : 40;   // FP64: one refinement step
  const double tol = sizeof(T) == 8 ? 1e-15 : 1e-12;
  cudaEvent_t e0, e1, e2;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventCreate(&e2);
  double fac_ms = 0, sol_ms = 0;
  std::vector<double> hn(2 * B);
  std::vector<int> hp(B), hit(B);
  std::vector<char> conv(B);
  const unsigned vb = (unsigned)((n + 255) / 256);
  auto t_start = std::chrono::steady_clock::now();
  cudaEvent_t eall0, eall1;
  cudaEventCreate(&eall0);
  cudaEventCreate(&eall1);
  cudaEventRecord(eall0, h.stream);
  int perturbed = 0, nfail = 0;
  int64_t steps_p = 0, steps_a = 0;
  for (int c0 = 0; c0 < n_f; c0 += B) {
    const int nb = std::min(B, n_f - c0);
    SS_CK(cudaMemcpyAsync(dom.p, omega + c0, nb * sizeof(double), cudaMemcpyHostToDevice, h.stream));
    SS_CK(cudaMemsetAsync(npert.p, 0, nb * sizeof(int), h.stream));
    rhs_kernel<<<dim3(vb, nb), 256, 0, h.stream>>>(n, nb, dom.as<double>(), V, h.beta, h.dks.as<cd>(),
                                                   h.dms.as<cd>(), damp ? h.dds.as<cd>() : nullptr,
                                                   h.drow_scale.as<double>(), b.as<cd>());
    cudaEventRecord(e0, h.stream);
    int rc = sw.factor_graphed(nb);
    if (rc) return rc;
    cudaEventRecord(e1, h.stream);
    rc = sw.solve_graphed(1, nb, b.as<cd>(), x.as<cd>());
    if (rc) return rc;
    cudaEventRecord(e2, h.stream);
    SS_CK(cudaEventSynchronize(e2));
    float ms1 = 0, ms2 = 0;
    cudaEventElapsedTime(&ms1, e0, e1);
    cudaEventElapsedTime(&ms2, e1, e2);
    fac_ms += ms1;
    sol_ms += ms2;
    sw.collect(nb);
    std::fill(conv.begin(), conv.end(), 0);
    std::fill(hit.begin(), hit.end(), 0);
    const bool use_krylov = sizeof(T) == 4 || getenv("SS_FP64_KRYLOV") != nullptr;
    const MatOp opA{h.dc_ptr.as<int64_t>(), h.dc_idx.as<int64_t>(), nullptr};
    if (use_krylov) {
      // FGMRES-IR: FP64 Krylov, complex64 factors as right preconditioner
      std::vector<int> kits;
      std::vector<char> kconv;
      auto pre = [&](const cd *src, cd *dst) { return sw.solve_graphed(1, nb, src, dst); };
      rc = fgmres(h, kw, opA, nb, krylov_m, krylov_restarts, tol_p, a.Kc, a.Mc, a.Dc, dom.as<double>(), b.as<cd>(),
                  x.as<cd>(), pre, kits, kconv, h.dmask.as<int>());
      if (rc) return rc;
      for (int f = 0; f < nb; ++f) hit[f] = kits[f], conv[f] = kconv[f], steps_p += kits[f];
    }
    if (getenv("SS_DEBUG_IR")) {
      // backward error of the direct solve: |b - A x| / |b|, and the solution size
      residual_kernel<<<dim3(vb, spmv_blocks(nb)), 256, 0, h.stream>>>(n, nb, h.dc_ptr.as<int64_t>(), h.dc_idx.as<int64_t>(), nullptr,
                                                          a.Kc, a.Mc, a.Dc, dom.as<double>(), h.beta, b.as<cd>(),
                                                          x.as<cd>(), r.as<cd>());
      norm2_kernel<<<nb, 256, 0, h.stream>>>(n, r.as<cd>(), nrm.as<double>());
      norm2_kernel<<<nb, 256, 0, h.stream>>>(n, b.as<cd>(), nrm.as<double>() + nb);
      std::vector<double> q(2 * nb);
      cudaMemcpyAsync(q.data(), nrm.p, 2 * nb * sizeof(double), cudaMemcpyDeviceToHost, h.stream);
      cudaStreamSynchronize(h.stream);
      fprintf(stderr, "direct solve (%s): |r|/|b| f0 %.3e f_last %.3e\n", sizeof(T) == 8 ? "c128" : "c64",
              q[0] / q[nb], q[nb - 1] / q[2 * nb - 1]);
    }
    for (int it = 0; it < (use_krylov ? 0 : maxit); ++it) {
      residual_kernel<<<dim3(vb, spmv_blocks(nb)), 256, 0, h.stream>>>(n, nb, h.dc_ptr.as<int64_t>(), h.dc_idx.as<int64_t>(), nullptr,
                                                          a.Kc, a.Mc, a.Dc, dom.as<double>(), h.beta, b.as<cd>(),
                                                          x.as<cd>(), r.as<cd>());
      rc = sw.solve_graphed(1, nb, r.as<cd>(), dx.as<cd>());
      if (rc) return rc;
      axpy_norm_kernel<<<nb, 256, 0, h.stream>>>(n, x.as<cd>(), dx.as<cd>(), nrm.as<double>());
      SS_CK(cudaMemcpyAsync(hn.data(), nrm.p, 2 * nb * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
      SS_CK(cudaStreamSynchronize(h.stream));
      bool all = true;
      if (getenv("SS_DEBUG_IR")) {
        double mx = 0;
        for (int f = 0; f < nb; ++f) mx = std::max(mx, hn[2 * f] / hn[2 * f + 1]);
        fprintf(stderr, "IR it %d: dx/x f0 %.3e f_last %.3e max %.3e\n", it, hn[0] / hn[1],
                hn[2 * (nb - 1)] / hn[2 * nb - 1], mx);
      }
      for (int f = 0; f < nb; ++f) {
        if (!conv[f]) {
          ++hit[f];
          conv[f] = hn[2 * f] <= tol * hn[2 * f + 1];
        }
        all = all && conv[f];
      }
      if (all) break;
    }
    // adjoint of the charge functional: A'^T mu = c with c = cs * kq (Q = c^T x' + V Qz)
    std::vector<cd> corr(nb, cd{0.0, 0.0});
    std::vector<char> aconv(nb, 1);
    if (need_adjoint) {
      const MatOp opT{h.dct_ptr.as<int64_t>(), h.dct_idx.as<int64_t>(), h.dct_src.as<int64_t>()};
      charge_row_kernel<<<dim3(vb, nb), 256, 0, h.stream>>>(n, nb, h.dks.as<cd>() + n, h.dcol_scale.as<double>(),
                                                          cvec.as<cd>());
      rc = sw.solve_graphed(2, nb, cvec.as<cd>(), mu.as<cd>());
      if (rc) return rc;
      if (use_krylov) {
        std::vector<int> kits;
        std::vector<char> kconv;
        auto pre = [&](const cd *src, cd *dst) { return sw.solve_graphed(2, nb, src, dst); };
        rc = fgmres(h, kw, opT, nb, krylov_m, krylov_restarts, tol_a, a.Kc, a.Mc, a.Dc, dom.as<double>(),
                    cvec.as<cd>(), mu.as<cd>(), pre, kits, kconv, h.dmask.as<int>());
        if (rc) return rc;
        for (int f = 0; f < nb; ++f) hit[f] += kits[f], aconv[f] = kconv[f], steps_a += kits[f];
      } else {
        // one FP64 refinement step, as for the primal solution
        residual_kernel<<<dim3(vb, spmv_blocks(nb)), 256, 0, h.stream>>>(n, nb, opT.rp, opT.ci, opT.vp, a.Kc, a.Mc, a.Dc,
                                                            dom.as<double>(), h.beta, cvec.as<cd>(), mu.as<cd>(),
                                                            r.as<cd>());
        rc = sw.solve_graphed(2, nb, r.as<cd>(), dx.as<cd>());
        if (rc) return rc;
        axpy_norm_kernel<<<nb, 256, 0, h.stream>>>(n, mu.as<cd>(), dx.as<cd>(), nrm.as<double>());
      }
      if (correct) {
        // dual-weighted correction: Q = c^T x + mu^T (b - A' x) is exact up to
        // (mu_exact - mu)^T (b - A' x), the product of the two solves' errors
        residual_kernel<<<dim3(vb, spmv_blocks(nb)), 256, 0, h.stream>>>(n, nb, h.dc_ptr.as<int64_t>(), h.dc_idx.as<int64_t>(),
                                                            nullptr, a.Kc, a.Mc, a.Dc, dom.as<double>(), h.beta,
                                                            b.as<cd>(), x.as<cd>(), r.as<cd>());
        dotu_kernel<<<nb, 256, 0, h.stream>>>(n, mu.as<cd>(), r.as<cd>(), dQ.as<cd>() + B);
        SS_CK(cudaMemcpyAsync(corr.data(), dQ.as<cd>() + B, nb * sizeof(cd), cudaMemcpyDeviceToHost, h.stream));
      }
      if (ex && ex->per_chunk) {
        rc = ex->per_chunk(c0, nb, x.as<cd>(), mu.as<cd>());
        if (rc) return rc;
      }
    }
    charge_kernel<<<nb, 256, 0, h.stream>>>(n, h.dks.as<cd>() + n, h.dcol_scale.as<double>(), x.as<cd>(),
                                            h.dQz.as<cd>(), V, dQ.as<cd>());
    SS_CK(cudaGetLastError());
    SS_CK(cudaMemcpyAsync(Qout + 2 * (int64_t)c0, dQ.p, nb * sizeof(cd), cudaMemcpyDeviceToHost, h.stream));
    SS_CK(cudaMemcpyAsync(hp.data(), npert.p, nb * sizeof(int), cudaMemcpyDeviceToHost, h.stream));
    SS_CK(cudaStreamSynchronize(h.stream));
    for (int f = 0; f < nb; ++f) {
      perturbed += hp[f];
      if (correct) {
        Qout[2 * (int64_t)(c0 + f)] += corr[f].x;
        Qout[2 * (int64_t)(c0 + f) + 1] += corr[f].y;
      }
      const bool ok = !(sizeof(T) == 4 && !(conv[f] && aconv[f]));
      nfail += !ok;
      // singular: a non-finite charge, or (FP64 direct solve) statically
      // perturbed pivots whose refinement step still moves the solution by more
      // than 1e-6 of its size
      const bool finite = std::isfinite(Qout[2 * (int64_t)(c0 + f)]) && std::isfinite(Qout[2 * (int64_t)(c0 + f) + 1]);
      const bool moved = !use_krylov && hp[f] > 0 && !(hn[2 * f] <= 1e-6 * hn[2 * f + 1]);
      if (status) status[c0 + f] = (!finite || moved) ? SS_ESINGULAR : ok ? SS_OK : SS_ENOCONV;
      if (iters) iters[c0 + f] = hit[f];
    }
    if (disp) {
      std::vector<cd> y(n);
      std::vector<double> cs(n);
      SS_CK(cudaMemcpy(y.data(), x.p, n * sizeof(cd), cudaMemcpyDeviceToHost));
      SS_CK(cudaMemcpy(cs.data(), h.dcol_scale.p, n * sizeof(double), cudaMemcpyDeviceToHost));
      std::vector<cd> pre(h.gdof, cd{0, 0});
      for (int64_t Pa = 0; Pa < n; ++Pa) {
        const int64_t R = S.new_of_act[Pa];
        pre[h.active[Pa]] = y[R] * cs[R];
      }
      for (int64_t i = 0; i < h.gdof; ++i) {
        const cd v = pre[h.rep[i]];
        disp[2 * i] = v.x;
        disp[2 * i + 1] = v.y;
      }
      for (int64_t d : h.zheng) disp[2 * d] = V, disp[2 * d + 1] = 0;
      for (int64_t d : h.fu) disp[2 * d] = 0, disp[2 * d + 1] = 0;
    }
  }
  cudaEventRecord(eall1, h.stream);
  cudaEventSynchronize(eall1);
  {
    int e = 0;
    SS_CK(cudaMemcpy(&e, tcerr.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return fail(h, SS_ETIMEOUT, "sweep: a tensor-core front update timed out waiting for its MMAs");
  }
  float total_f = 0;
  cudaEventElapsedTime(&total_f, eall0, eall1);
  const double total_ms = total_f;
  cudaEventDestroy(eall0);
  cudaEventDestroy(eall1);
  const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  h.st[7] = wall;
  h.st[8] = fac_ms;
  h.st[9] = sol_ms;
  h.st[10] = B;
  h.st[11] = sw.schur_ms;
  h.st[12] = P.schur_flops * n_f;
  h.st[16] = sw.schur_launches;
  h.st[17] = total_ms;
  h.st[14] = perturbed;
  h.st[15] = sw.launches;
  h.st[30] = (double)steps_p;
  h.st[31] = (double)steps_a;
  h.st[32] = nfail;
  h.st[20] = h.st[21] = h.st[22] = h.st[36] = 0;
  h.st[23] = P.panel_cst ? 4 : P.panel_dmma;
  h.st[37] = P.panel_thin ? (double)P.thin_tasks : 0.0;
  h.st[24] = P.panel_ms[0];
  h.st[25] = std::min(std::min(P.panel_ms[1], P.panel_ms[2]), P.panel_ms[3]);
  h.st[26] = (double)P.fronts_small.size();
  h.st[27] = 0;
  for (float t : P.tune_ms) h.st[27] += t;
  for (size_t l = 0; l < P.pick.size(); ++l)
    if (P.schur_ptr[l + 1] > P.schur_ptr[l]) h.st[P.pick[l] == 3 ? 36 : 20 + P.pick[l]] += 1;
  {
    double tot = 0;
    if (iters)
      for (int i = 0; i < n_f; ++i) tot += iters[i];
    h.st[18] = tot;
  }
  return SS_OK;
}

// SS_PREC_AUTO: a probe of the mixed sweep on the band's two end points with a
// short Krylov budget (the handle's auto_probe_steps, 12 by default, for the
// primal and the adjoint); if both converge the whole sweep runs mixed, otherwise
// FP64 (the complex64 factors of a cell whose conditioning defeats FP32 would
// need many Krylov steps per point).  The decision is kept for the band's end
// points until the system or an option changes, so a repeated sweep of the same
// band probes once; the probe's device time is kept in stats slot 28.
//
// A mixed sweep whose refinement leaves points unconverged re-solves those points
// with the FP64 path in the same call (option fp64_fallback, on by default), so
// every point returned has SS_OK unless FP64 fails too.
int run_sweep(Handle &h, int n_f, const double *omega, double V, int precision, double *Q, int *status,
              int *iters, double *disp_out, const SweepExtra *ex) {
  SweepOpts opt;
  opt.krylov_m = h.opt.krylov_m;
  opt.restarts = h.opt.krylov_cycles;
  opt.tol = h.opt.krylov_tol;
  std::vector<int> st_local, it_local;
  if (!status) {
    st_local.assign(std::max(0, n_f), 0);
    status = st_local.data();
  }
  if (!iters) {
    it_local.assign(std::max(0, n_f), 0);
    iters = it_local.data();
  }
  int rc;
  double probe_ms = 0, probe_launches = 0;
  if (precision == SS_PREC_AUTO && n_f > 0 && h.auto_prec >= 0 && h.auto_w0 == omega[0] &&
      h.auto_w1 == omega[n_f - 1])
    precision = h.auto_prec;
  if (precision == SS_PREC_AUTO && n_f > 0) {
    const double ends[2] = {omega[0], omega[n_f - 1]};
    double q[4];
    int st[2] = {0, 0}, it[2] = {0, 0};
    SweepOpts probe = opt;
    probe.restarts = 1;
    probe.krylov_m = h.opt.auto_probe_m;
    rc = sweep_impl<float>(h, n_f > 1 ? 2 : 1, ends, V, q, st, it, nullptr, nullptr, probe);
    if (rc) return rc;
    precision = (st[0] == SS_OK && st[1] == SS_OK) ? SS_PREC_MIXED : SS_PREC_FP64;
    h.auto_w0 = omega[0];
    h.auto_w1 = omega[n_f - 1];
    h.auto_prec = precision;
    probe_ms = h.st[17];
    probe_launches = h.st[15];
    h.st[28] = probe_ms;
  }
  if (precision == SS_PREC_MIXED)
    rc = sweep_impl<float>(h, n_f, omega, V, Q, status, iters, disp_out, ex, opt);
  else
    rc = sweep_impl<double>(h, n_f, omega, V, Q, status, iters, disp_out, ex, opt);
  if (rc) return rc;
  h.st[19] = precision;
  h.st[29] = 0;
  h.st[33] = 0;
  if (precision == SS_PREC_MIXED && h.opt.fp64_fallback) {
    // maximal runs of consecutive unconverged points, each re-solved in FP64
    std::vector<std::pair<int, int>> runs;
    for (int i = 0; i < n_f;) {
      if (status[i] != SS_ENOCONV) {
        ++i;
        continue;
      }
      int j = i;
      while (j < n_f && status[j] == SS_ENOCONV) ++j;
      runs.emplace_back(i, j);
      i = j;
    }
    if (!runs.empty()) {
      double keep[Handle::kStats];
      std::copy(h.st, h.st + Handle::kStats, keep);
      double fb_ms = 0, fb_launches = 0;
      int resolved = 0;
      for (const auto &r : runs) {
        const int i0 = r.first, len = r.second - r.first;
        SweepExtra exr;
        if (ex && ex->per_chunk)
          exr.per_chunk = [ex, i0](int c0, int nb, const cplx<double> *x, const cplx<double> *mu) {
            return ex->per_chunk(c0 + i0, nb, x, mu);
          };
        std::vector<int> it2(len, 0);
        rc = sweep_impl<double>(h, len, omega + i0, V, Q + 2 * (int64_t)i0, status + i0, it2.data(),
                                disp_out, ex ? &exr : nullptr, opt);
        if (rc) return rc;
        for (int f = 0; f < len; ++f) iters[i0 + f] += it2[f];
        fb_ms += h.st[17];
        fb_launches += h.st[15];
        resolved += len;
      }
      std::copy(keep, keep + Handle::kStats, h.st);
      h.st[17] += fb_ms;
      h.st[15] += fb_launches;
      h.st[29] = resolved;
      h.st[33] = fb_ms;
    }
  }
  h.st[17] += probe_ms;        // the probe is part of an AUTO sweep's device time
  h.st[15] += probe_launches;
  {
    double tot = 0;
    for (int i = 0; i < n_f; ++i) tot += iters[i];
    h.st[18] = tot;
  }
  return SS_OK;
}

}  // namespace ss

namespace ss {

// deterministic pseudo-random fill of a complex buffer (values in [-1, 1))
template <class T>
__global__ void fill_hash_kernel(int64_t n, cplx<T> *x) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t z = (uint64_t)i * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull;
  z ^= z >> 29;
  z *= 0xbf58476d1ce4e5b9ull;
  z ^= z >> 32;
  const T re = (T)((double)(z & 0xffffff) / 8388608.0 - 1.0);
  const T im = (T)((double)((z >> 24) & 0xffffff) / 8388608.0 - 1.0);
  x[i] = cplx<T>{re, im};
}

// Measured ceiling of one Schur-update kernel: n_fronts dense fronts of m rows
// with k pivots (C -= A B over the (m-k) x (m-k) update block, K = k), every
// front a separate "frequency" of one launch, timed by CUDA events over `reps`
// launches after one warm-up; returns the median algorithmic rate (8 real flops
// per complex multiply-add).  kernel: 0 FP64 DMMA 64x64, 1 FP64 SIMT 128x64,
// 2 / 3 complex64 TMA + tcgen05 3xTF32 with 128 / 64-column tiles (operands
// packed once before the timed launches), 5 FP64 DMMA 64x64 with three real
// products per complex block,
// 4 complex64 SIMT FP32 128x64, 6 FP64 DMMA 64x64 with three real products and
// the C tile staged in shared memory.
template <class T>
static int measure_ceiling_impl(Handle &h, int kernel, int m, int k, int nb, int reps, double *tflops) {
  const int ld = (m + 3) / 4 * 4;
  DBuf arena, dld, doff, dtasks, derr;
  const size_t stride = (size_t)m * ld;
  SS_CK(dalloc(arena, (size_t)nb * stride * sizeof(cplx<T>)));
  std::vector<int> vld(1, ld);
  std::vector<int64_t> voff(1, 0);
  std::vector<GemmTask> tasks;
  if (kernel == 0 || kernel == 5 || kernel == 6)
    add_tiles(tasks, kSquare64, 0, k, m, k, m, 0, k);
  else
    add_tiles(tasks, kSquare, 0, k, m, k, m, 0, k);
  // TMA kernels: the front's packed operands and the tiles of 128 / 64 columns
  const int kc = (k + tc::KCH - 1) / tc::KCH, u = m - k, au = (u + tc::PADC - 1) / tc::PADC * tc::PADC;
  const int bnc = kernel == 2 ? 128 : 64;
  std::vector<tc::PackFront> pk(1, tc::PackFront{0, 0, kc, au, au});
  std::vector<int2> pitems;
  for (int c = 0; c < kc; ++c) pitems.push_back(make_int2(0, c));
  std::vector<tc::TmaTask> tt;
  for (int r0 = k; r0 < m; r0 += tc::BM)
    for (int c0 = k; c0 < m; c0 += bnc) tt.push_back(tc::TmaTask{0, 0, r0, c0, m, m, kc, au, au, r0 - k, 2 * (c0 - k)});
  const int64_t srows = tc::pack_rows(kc, au, au);
  DBuf dpk, dpi, dtt, dk, dm, dstage;
  CUtensorMap map{};
  const bool tma = kernel == 2 || kernel == 3;
  if (tma) {
    if ((int64_t)nb * srows >= ((int64_t)1 << 31)) return fail(h, SS_EINVAL, "ceiling: staging rows exceed 2^31");
    SS_CK(dupload(dpk, pk));
    SS_CK(dupload(dpi, pitems));
    SS_CK(dupload(dtt, tt));
    SS_CK(dupload(dk, std::vector<int>(1, k)));
    SS_CK(dupload(dm, std::vector<int>(1, m)));
    SS_CK(dalloc(dstage, (size_t)nb * srows * tc::ROWB));
    const int rc = encode_stage_map(h, map, dstage.p, (int64_t)nb * srows);
    if (rc) return rc;
  }
  SS_CK(dupload(dld, vld));
  SS_CK(dupload(doff, voff));
  SS_CK(dupload(dtasks, tasks));
  SS_CK(dalloc(derr, sizeof(int)));
  SS_CK(cudaMemsetAsync(derr.p, 0, sizeof(int), h.stream));
  const int64_t ne = (int64_t)nb * stride;
  fill_hash_kernel<T><<<(unsigned)((ne + 255) / 256), 256, 0, h.stream>>>(ne, arena.as<cplx<T>>());
  FrontArgs<T> a{};
  a.ld = dld.as<int>();
  a.off = doff.as<int64_t>();
  a.arena = arena.as<cplx<T>>();
  a.stride = (int64_t)stride;
  const GemmTask *tk = dtasks.as<GemmTask>();
  const unsigned nt = (unsigned)tasks.size();
  if (tma) {
    SS_CK(cudaFuncSetAttribute(tc::tma_gemm_kernel<128, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               tc::TmaCfg<128, 2>::SMEM));
    SS_CK(cudaFuncSetAttribute(tc::tma_gemm_kernel<64, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               tc::TmaCfg<64, 3>::SMEM));
    // operands packed once; the timed launches are the GEMM alone
    tc::pack_kernel<<<dim3((unsigned)pitems.size(), nb), tc::PACK_THREADS, 0, h.stream>>>(
        reinterpret_cast<const cf *>(a.arena), a.stride, a.off, a.ld, dk.as<int>(), dm.as<int>(),
        dpk.as<tc::PackFront>(), dpi.as<int2>(), dstage.as<float>(), srows);
  }
  auto launch = [&]() {
    if constexpr (sizeof(T) == 8) {
      if (kernel == 0)
        front_dmma_kernel<2, 2><<<dim3(nt, nb), 128, 0, h.stream>>>(a, tk);
      else if (kernel == 5)
        front_dmma3_kernel<2, 2><<<dim3(nt, nb), 128, 0, h.stream>>>(a, tk);
      else if (kernel == 6)
        front_dmma3_kernel<2, 2, true><<<dim3(nt, nb), 128, dmma_cst_bytes<2, 2>(), h.stream>>>(a, tk);
      else
        front_gemm_kernel<T, kSquare><<<dim3(nt, nb), 256, 0, h.stream>>>(a, tk);
    } else {
      cf *ar = reinterpret_cast<cf *>(a.arena);
      const unsigned grid = (unsigned)std::min<int64_t>((int64_t)tt.size() * nb, h.num_sms);
      if (kernel == 2)
        tc::tma_gemm_kernel<128, 2><<<grid, tc::TmaCfg<128, 2>::THREADS, tc::TmaCfg<128, 2>::SMEM, h.stream>>>(
            map, ar, a.stride, a.off, a.ld, dtt.as<tc::TmaTask>(), (int)tt.size(), nb, srows, derr.as<int>());
      else if (kernel == 3)
        tc::tma_gemm_kernel<64, 3><<<grid, tc::TmaCfg<64, 3>::THREADS, tc::TmaCfg<64, 3>::SMEM, h.stream>>>(
            map, ar, a.stride, a.off, a.ld, dtt.as<tc::TmaTask>(), (int)tt.size(), nb, srows, derr.as<int>());
      else
        front_gemm_kernel<T, kSquare><<<dim3(nt, nb), 256, 0, h.stream>>>(a, tk);
    }
  };
  launch();
  SS_CK(cudaGetLastError());
  std::vector<cudaEvent_t> ev(2 * reps);
  for (auto &e : ev) SS_CK(cudaEventCreate(&e));
  for (int r = 0; r < reps; ++r) {
    cudaEventRecord(ev[2 * r], h.stream);
    launch();
    cudaEventRecord(ev[2 * r + 1], h.stream);
  }
  SS_CK(cudaGetLastError());
  SS_CK(cudaStreamSynchronize(h.stream));
  std::vector<double> ms(reps);
  for (int r = 0; r < reps; ++r) {
    float t = 0;
    cudaEventElapsedTime(&t, ev[2 * r], ev[2 * r + 1]);
    ms[r] = t;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  int e = 0;
  SS_CK(cudaMemcpy(&e, derr.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) return fail(h, SS_ETIMEOUT, "ceiling: a tensor-core tile timed out waiting for its MMAs");
  std::sort(ms.begin(), ms.end());
  const double med = ms[reps / 2];
  const double flops = 8.0 * k * (double)(m - k) * (m - k) * nb;
  *tflops = flops / (med * 1e-3) / 1e12;
  return SS_OK;
}

int measure_ceiling(Handle &h, int kernel, int m, int k, int nb, int reps, double *tflops) {
  if (kernel <= 1 || kernel == 5 || kernel == 6) {
    cudaError_t e = cudaFuncSetAttribute(front_dmma3_kernel<2, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         dmma_cst_bytes<2, 2>());
    if (e != cudaSuccess) return cuda_fail(h, e, "ceiling: shared memory attribute");
    return measure_ceiling_impl<double>(h, kernel, m, k, nb, reps, tflops);
  }
  return measure_ceiling_impl<float>(h, kernel, m, k, nb, reps, tflops);
}

}  // namespace ss

namespace ss {
void free_plans(Handle &h) {
  h.auto_prec = -1;
  for (int i = 0; i < 2; ++i) {
    delete static_cast<Plan *>(h.plan[i]);
    h.plan[i] = nullptr;
  }
}
}  // namespace ss
