// Batched flexible GMRES in FP64 with the low-precision LU as right
// preconditioner (GMRES-based iterative refinement).  Used by the mixed-precision
// sweep: the complex64 multifrontal factors are too inexact for plain
// refinement on cells whose condition number reaches 1e8-1e9 near resonance,
// but they cluster the spectrum of A M^-1 so that a few Krylov steps recover the
// FP64 solution.  Vectors of frequency f live at base + f * n; Krylov vector j at
// base + j * nb * n.  All reductions are fixed-order trees (deterministic).
#pragma once
#include <complex>
#include <functional>

namespace ss {

// Sparse operator of the scaled condensed system: the CSR pattern (rp, ci) and,
// for the transposed operator, the value slot of each entry (vp; nullptr = the
// entry's own slot).
struct MatOp {
  const int64_t *rp, *ci, *vp;
};

// y_f = A'(w_f) x_f   (or A'(w_f)^T x_f with the transposed pattern).  A thread
// owns a row for a block of kSpmvFreqs frequencies, so that the row's K, M (and D)
// values and column indices are read once per block instead of once per
// frequency; each frequency's sum runs over the row in the same order as a
// one-frequency product.
__global__ void spmv_kernel(int64_t n, int nb, const int64_t *__restrict__ rp, const int64_t *__restrict__ ci,
                            const int64_t *__restrict__ vp, const cd *__restrict__ K, const cd *__restrict__ M,
                            const cd *__restrict__ D, const double *__restrict__ omega, double beta,
                            const cd *__restrict__ x, cd *__restrict__ y, const int *__restrict__ active = nullptr) {
  const int64_t R = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int f0 = blockIdx.y * kSpmvFreqs;
  if (R >= n || f0 >= nb) return;
  // frequencies [f0, f0 + nf) of this block; trailing ones that stopped iterating
  // are left out (a block whose frequencies have all stopped returns)
  int nf = min(kSpmvFreqs, nb - f0);
  if (active) {
    while (nf > 0 && !active[f0 + nf - 1]) --nf;
    if (nf == 0) return;
  }
  double w2[kSpmvFreqs], wb[kSpmvFreqs];
  cd acc[kSpmvFreqs];
#pragma unroll
  for (int q = 0; q < kSpmvFreqs; ++q) {
    const double w = q < nf ? omega[f0 + q] : 0.0;
    w2[q] = w * w;
    wb[q] = w * beta;
    acc[q] = cd{0.0, 0.0};
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
        acc[q] = acc[q] + cmul(a, xb[(int64_t)q * n + j]);
      }
  }
#pragma unroll
  for (int q = 0; q < kSpmvFreqs; ++q)
    if (q < nf) y[(int64_t)(f0 + q) * n + R] = acc[q];
}

__device__ inline cd block_reduce_cd(cd v, cd *red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
    __syncthreads();
  }
  const cd r = red[0];
  __syncthreads();
  return r;
}

// h[f * ldh + i] = V_i,f^H w_f for i < J;  grid (J, nb), 256 threads
__global__ void multi_dot_kernel(int64_t n, int nb, const cd *__restrict__ V, const cd *__restrict__ w,
                                 cd *__restrict__ h, int ldh, const int *__restrict__ active = nullptr) {
  __shared__ cd red[256];
  const int i = blockIdx.x, f = blockIdx.y;
  if (active && !active[f]) return;
  const cd *v = V + ((int64_t)i * nb + f) * n;
  const cd *x = w + (int64_t)f * n;
  cd acc{0.0, 0.0};
  for (int64_t R = threadIdx.x; R < n; R += blockDim.x) {
    const cd a = v[R], b = x[R];
    acc.x += a.x * b.x + a.y * b.y;   // conj(a) * b
    acc.y += a.x * b.y - a.y * b.x;
  }
  const cd r = block_reduce_cd(acc, red);
  if (threadIdx.x == 0) h[f * ldh + i] = r;
}

// w_f -= sum_{i<J} h[f*ldh+i] V_i,f
__global__ void multi_axpy_kernel(int64_t n, int nb, int J, const cd *__restrict__ V, const cd *__restrict__ h,
                                  int ldh, cd *__restrict__ w, const int *__restrict__ active = nullptr) {
  const int64_t R = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (R >= n || (active && !active[f])) return;
  cd acc = w[(int64_t)f * n + R];
  for (int i = 0; i < J; ++i) acc = acc - cmul(h[f * ldh + i], V[((int64_t)i * nb + f) * n + R]);
  w[(int64_t)f * n + R] = acc;
}

// out[f] = ||w_f||_2
__global__ void norm2_kernel(int64_t n, const cd *__restrict__ w, double *__restrict__ out,
                             const int *__restrict__ active = nullptr) {
  __shared__ cd red[256];
  const int f = blockIdx.x;
  if (active && !active[f]) return;
  const cd *x = w + (int64_t)f * n;
  double acc = 0.0;
  for (int64_t R = threadIdx.x; R < n; R += blockDim.x) acc += cabs2(x[R]);
  const cd r = block_reduce_cd(cd{acc, 0.0}, red);
  if (threadIdx.x == 0) out[f] = sqrt(r.x);
}

// out_f = w_f * s[f]
// out may be w (in-place scaling): each element is read and written by one thread
__global__ void scale_vec_kernel(int64_t n, int nb, const cd *w, const double *__restrict__ s, cd *out,
                                 const int *__restrict__ active = nullptr) {
  const int64_t R = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (R >= n || (active && !active[f])) return;
  out[(int64_t)f * n + R] = w[(int64_t)f * n + R] * s[f];
}

// x_f += sum_{i<k_f} y[f*ldy+i] Z_i,f
__global__ void combine_kernel(int64_t n, int nb, const int *__restrict__ kf, const cd *__restrict__ Z,
                               const cd *__restrict__ y, int ldy, cd *__restrict__ x) {
  const int64_t R = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (R >= n) return;
  cd acc = x[(int64_t)f * n + R];
  for (int i = 0; i < kf[f]; ++i) acc = acc + cmul(y[f * ldy + i], Z[((int64_t)i * nb + f) * n + R]);
  x[(int64_t)f * n + R] = acc;
}


// FGMRES(m) with up to `restarts` cycles; x holds the initial guess on entry.
// precond(src, dst) applies M^-1 to nb vectors.  Returns the number of
// preconditioner applications per frequency in `its`, converged flags in `conv`.
// d_active (nb ints on the device, may be null) marks the frequencies still
// iterating: the preconditioner's solve kernels, the sparse products and the
// orthogonalisation skip the others, so a chunk's cost follows each point's own
// step count rather than its slowest point's; all ones again on return.
template <class Precond>
int fgmres(Handle &h, KrylovWork &kw, const MatOp &op, int nb, int m, int restarts, double tol, const cd *Kc, const cd *Mc,
           const cd *Dc, const double *d_omega, const cd *b, cd *x, Precond precond, std::vector<int> &its,
           std::vector<char> &conv, int *d_active = nullptr) {
  const int64_t n = h.sym.n;
  const unsigned vb = (unsigned)((n + 255) / 256);
  const size_t vec = (size_t)nb * n * sizeof(cd);
  cudaError_t e;
#define KCK(x)                                          \
  if ((e = (x)) != cudaSuccess) return cuda_fail(h, e, #x)
  KCK(dalloc(kw.V, vec * (m + 1)));
  KCK(dalloc(kw.Z, vec * m));
  KCK(dalloc(kw.w, vec));
  KCK(dalloc(kw.h, sizeof(cd) * nb * (m + 1) * 2));
  KCK(dalloc(kw.hn, sizeof(double) * nb * 2));
  KCK(dalloc(kw.y, sizeof(cd) * nb * m));
  KCK(dalloc(kw.kf, sizeof(int) * nb));
  KCK(dalloc(kw.sc, sizeof(double) * nb));
  cd *V = kw.V.as<cd>(), *Z = kw.Z.as<cd>(), *w = kw.w.as<cd>(), *hd = kw.h.as<cd>();
  double *hn = kw.hn.as<double>();
  const int ldh = m + 1;
  its.assign(nb, 0);
  conv.assign(nb, 0);
  std::vector<double> bnorm(nb), nrm(nb), sc(nb);
  norm2_kernel<<<nb, 256, 0, h.stream>>>(n, b, hn);
  KCK(cudaMemcpyAsync(bnorm.data(), hn, nb * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
  KCK(cudaStreamSynchronize(h.stream));
  using C = std::complex<double>;
  std::vector<C> H((size_t)nb * (m + 1) * m), g((size_t)nb * (m + 1)), cs_s((size_t)nb * m);
  std::vector<double> cs_c((size_t)nb * m);
  std::vector<cd> hcol((size_t)nb * ldh * 2);
  std::vector<int> kf(nb);
  std::vector<char> done(nb);
  std::vector<int> act(nb, 1);
  // mirror of d_active: upload when a point stops
  auto push_active = [&]() -> cudaError_t {
    if (!d_active) return cudaSuccess;
    for (int f = 0; f < nb; ++f) act[f] = done[f] ? 0 : 1;
    return cudaMemcpyAsync(d_active, act.data(), nb * sizeof(int), cudaMemcpyHostToDevice, h.stream);
  };
  auto all_active = [&]() -> cudaError_t {
    if (!d_active) return cudaSuccess;
    std::fill(act.begin(), act.end(), 1);
    const cudaError_t r = cudaMemcpyAsync(d_active, act.data(), nb * sizeof(int), cudaMemcpyHostToDevice, h.stream);
    return r == cudaSuccess ? cudaStreamSynchronize(h.stream) : r;
  };
  for (int cyc = 0; cyc < restarts; ++cyc) {
    // r = b - A x  -> V_0
    spmv_kernel<<<dim3(vb, spmv_blocks(nb)), 256, 0, h.stream>>>(n, nb, op.rp, op.ci, op.vp, Kc, Mc,
                                                    Dc, d_omega, h.beta, x, w);
    KCK(cudaMemcpyAsync(V, b, vec, cudaMemcpyDeviceToDevice, h.stream));
    {
      std::vector<cd> one(nb, cd{1.0, 0.0});
      KCK(cudaMemcpyAsync(hd, one.data(), nb * sizeof(cd), cudaMemcpyHostToDevice, h.stream));
      multi_axpy_kernel<<<dim3(vb, nb), 256, 0, h.stream>>>(n, nb, 1, w, hd, 1, V);
    }
    norm2_kernel<<<nb, 256, 0, h.stream>>>(n, V, hn);
    KCK(cudaMemcpyAsync(nrm.data(), hn, nb * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
    KCK(cudaStreamSynchronize(h.stream));
    if (getenv("SS_DEBUG_IR"))
      fprintf(stderr, "FGMRES cycle %d: |r|/|b| f0 %.3e f_last %.3e\n", cyc, nrm[0] / bnorm[0],
              nrm[nb - 1] / bnorm[nb - 1]);
    bool all = true;
    for (int f = 0; f < nb; ++f) {
      conv[f] = nrm[f] <= tol * bnorm[f];
      all = all && conv[f];
      done[f] = conv[f];
      kf[f] = 0;
      g[(size_t)f * (m + 1)] = nrm[f];
      for (int i = 1; i <= m; ++i) g[(size_t)f * (m + 1) + i] = 0.0;
      sc[f] = nrm[f] > 0 ? 1.0 / nrm[f] : 0.0;
    }
    if (all) break;
    KCK(push_active());
    KCK(cudaMemcpyAsync(kw.sc.p, sc.data(), nb * sizeof(double), cudaMemcpyHostToDevice, h.stream));
    scale_vec_kernel<<<dim3(vb, nb), 256, 0, h.stream>>>(n, nb, V, kw.sc.as<double>(), V, d_active);
    for (int j = 0; j < m; ++j) {
      cd *Vj = V + (size_t)j * nb * n, *Zj = Z + (size_t)j * nb * n;
      int rc = precond(Vj, Zj);
      if (rc) return rc;
      spmv_kernel<<<dim3(vb, spmv_blocks(nb)), 256, 0, h.stream>>>(n, nb, op.rp, op.ci, op.vp, Kc,
                                                      Mc, Dc, d_omega, h.beta, Zj, w, d_active);
      // classical Gram-Schmidt, twice
      for (int pass = 0; pass < 2; ++pass) {
        cd *hp = hd + (size_t)pass * nb * ldh;
        multi_dot_kernel<<<dim3(j + 1, nb), 256, 0, h.stream>>>(n, nb, V, w, hp, ldh, d_active);
        multi_axpy_kernel<<<dim3(vb, nb), 256, 0, h.stream>>>(n, nb, j + 1, V, hp, ldh, w, d_active);
      }
      norm2_kernel<<<nb, 256, 0, h.stream>>>(n, w, hn, d_active);
      KCK(cudaMemcpyAsync(hcol.data(), hd, sizeof(cd) * nb * ldh * 2, cudaMemcpyDeviceToHost, h.stream));
      KCK(cudaMemcpyAsync(nrm.data(), hn, nb * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
      KCK(cudaStreamSynchronize(h.stream));
      all = true;
      bool stopped = false;
      for (int f = 0; f < nb; ++f) {
        const double hnext = nrm[f];
        sc[f] = hnext > 0 ? 1.0 / hnext : 0.0;
        if (done[f]) continue;
        C *Hc = &H[((size_t)f * m + j) * (m + 1)];
        for (int i = 0; i <= j; ++i) {
          const cd a = hcol[(size_t)f * ldh + i], c2 = hcol[(size_t)nb * ldh + (size_t)f * ldh + i];
          Hc[i] = C(a.x + c2.x, a.y + c2.y);
        }
        Hc[j + 1] = hnext;
        for (int i = 0; i < j; ++i) {
          const double c = cs_c[(size_t)f * m + i];
          const C s = cs_s[(size_t)f * m + i];
          const C t = c * Hc[i] + s * Hc[i + 1];
          Hc[i + 1] = -std::conj(s) * Hc[i] + c * Hc[i + 1];
          Hc[i] = t;
        }
        const C a = Hc[j], bb = Hc[j + 1];
        const double t = std::sqrt(std::norm(a) + std::norm(bb));
        double c;
        C s;
        if (std::abs(a) == 0.0) {
          c = 0.0;
          s = 1.0;
        } else {
          c = std::abs(a) / t;
          s = (a / std::abs(a)) * std::conj(bb) / t;
        }
        cs_c[(size_t)f * m + j] = c;
        cs_s[(size_t)f * m + j] = s;
        Hc[j] = c * a + s * bb;
        Hc[j + 1] = 0.0;
        C *gf = &g[(size_t)f * (m + 1)];
        gf[j + 1] = -std::conj(s) * gf[j];
        gf[j] = c * gf[j];
        kf[f] = j + 1;
        ++its[f];
        if (std::abs(gf[j + 1]) <= tol * bnorm[f] || hnext == 0.0) done[f] = 1, stopped = true;
        all = all && done[f];
      }
      if (all || j == m - 1) break;
      if (stopped) KCK(push_active());
      KCK(cudaMemcpyAsync(kw.sc.p, sc.data(), nb * sizeof(double), cudaMemcpyHostToDevice, h.stream));
      scale_vec_kernel<<<dim3(vb, nb), 256, 0, h.stream>>>(n, nb, w, kw.sc.as<double>(), V + (size_t)(j + 1) * nb * n,
                                                           d_active);
    }
    KCK(all_active());   // the solution update and the next cycle's residual cover every point
    // least squares: H(0:k,0:k) y = g(0:k), back substitution
    std::vector<cd> yh((size_t)nb * m, cd{0, 0});
    for (int f = 0; f < nb; ++f) {
      const int k = kf[f];
      std::vector<C> yv(k);
      for (int i = k - 1; i >= 0; --i) {
        C s = g[(size_t)f * (m + 1) + i];
        for (int q = i + 1; q < k; ++q) s -= H[((size_t)f * m + q) * (m + 1) + i] * yv[q];
        yv[i] = s / H[((size_t)f * m + i) * (m + 1) + i];
      }
      for (int i = 0; i < k; ++i) yh[(size_t)f * m + i] = cd{yv[i].real(), yv[i].imag()};
    }
    KCK(cudaMemcpyAsync(kw.y.p, yh.data(), sizeof(cd) * nb * m, cudaMemcpyHostToDevice, h.stream));
    KCK(cudaMemcpyAsync(kw.kf.p, kf.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, h.stream));
    combine_kernel<<<dim3(vb, nb), 256, 0, h.stream>>>(n, nb, kw.kf.as<int>(), Z, kw.y.as<cd>(), m, x);
    KCK(cudaGetLastError());
  }
  KCK(all_active());
  // final true residual check
  spmv_kernel<<<dim3(vb, spmv_blocks(nb)), 256, 0, h.stream>>>(n, nb, op.rp, op.ci, op.vp, Kc, Mc, Dc,
                                                  d_omega, h.beta, x, w);
  {
    std::vector<cd> one(nb, cd{1.0, 0.0});
    KCK(cudaMemcpyAsync(kw.V.p, b, vec, cudaMemcpyDeviceToDevice, h.stream));
    KCK(cudaMemcpyAsync(hd, one.data(), nb * sizeof(cd), cudaMemcpyHostToDevice, h.stream));
    multi_axpy_kernel<<<dim3(vb, nb), 256, 0, h.stream>>>(n, nb, 1, w, hd, 1, V);
  }
  norm2_kernel<<<nb, 256, 0, h.stream>>>(n, V, hn);
  KCK(cudaMemcpyAsync(nrm.data(), hn, nb * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
  KCK(cudaStreamSynchronize(h.stream));
  for (int f = 0; f < nb; ++f) conv[f] = nrm[f] <= 10.0 * tol * bnorm[f];
  return SS_OK;
#undef KCK
}

}  // namespace ss
