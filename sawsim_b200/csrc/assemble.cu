// GPU assembly of the global piezoelectric K and M.
//
// Q9 (src/sawsim/saw2d/piezo_fem.py:248-367): one warp per element computes the
// 9-point Jacobians, the gradient Grams G[d1][d2] and the mass Gram, stretches the
// element's C/e/eps/rho by the PML alphas (frozen at omega_top, centre node), and
// writes the nc x nc x 9 x 9 complex element blocks with the reference's scale
// factors (SCALE on K_uu, K_phi-u and M; -1 on K_phi-phi) to a scratch array.
// A second kernel then sums, for every node pair, its element contributions in
// ascending element order into the CSR slots: a fixed-order segmented reduction,
// so repeated assemblies are bitwise identical and no atomics are used.
#include "ss_internal.h"
#include "dev_complex.cuh"
#include "q9_element.cuh"

namespace ss {

__constant__ double c_gp[3] = {-0.774596669241483, 0.0, 0.774596669241483};
__constant__ double c_gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
// gradient-form strain rows / derivative directions per displacement component
// (piezo_fem.py:31-35): {row, dir} pairs
__constant__ int c_sel[3][2][2] = {{{0, 0}, {5, 1}}, {{1, 1}, {8, 0}}, {{6, 1}, {7, 0}}};
// PML multiplier letters of T9 (piezo_fem.py:127-142): 0 A=a2a3/a1, 1 b=a3, 2 c=a2,
// 3 D=a1a3/a2, 4 e=a1, 5 F=a1a2/a3
__constant__ unsigned char c_t9[9][9] = {
    {0, 1, 2, 2, 2, 1, 1, 0, 0}, {1, 3, 4, 4, 4, 3, 3, 1, 1}, {2, 4, 5, 5, 5, 4, 4, 2, 2},
    {2, 4, 5, 5, 5, 4, 4, 2, 2}, {2, 4, 5, 5, 5, 4, 4, 2, 2}, {1, 3, 4, 4, 4, 3, 3, 1, 1},
    {1, 3, 4, 4, 4, 3, 3, 1, 1}, {0, 1, 2, 2, 2, 1, 1, 0, 0}, {0, 1, 2, 2, 2, 1, 1, 0, 0}};
__constant__ unsigned char c_teps[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

__device__ inline void q9_shape(double x, double y, double *N, double *dx, double *dy) {
  N[0] = 0.25 * (x * y * (x - 1) * (y - 1));
  N[1] = 0.25 * (x * y * (x + 1) * (y - 1));
  N[2] = 0.25 * (x * y * (x + 1) * (y + 1));
  N[3] = 0.25 * (x * y * (x - 1) * (y + 1));
  N[4] = 0.25 * (-2 * y * (x * x - 1) * (y - 1));
  N[5] = 0.25 * (-2 * x * (x + 1) * (y * y - 1));
  N[6] = 0.25 * (-2 * y * (x * x - 1) * (y + 1));
  N[7] = 0.25 * (-2 * x * (x - 1) * (y * y - 1));
  N[8] = 0.25 * (4 * (x * x - 1) * (y * y - 1));
  dx[0] = 0.25 * (y * (2 * x - 1) * (y - 1));
  dx[1] = 0.25 * (y * (2 * x + 1) * (y - 1));
  dx[2] = 0.25 * (y * (2 * x + 1) * (y + 1));
  dx[3] = 0.25 * (y * (2 * x - 1) * (y + 1));
  dx[4] = 0.25 * (-4 * x * y * (y - 1));
  dx[5] = 0.25 * (-2 * (2 * x + 1) * (y + 1) * (y - 1));
  dx[6] = 0.25 * (-4 * x * y * (y + 1));
  dx[7] = 0.25 * (-2 * (2 * x - 1) * (y + 1) * (y - 1));
  dx[8] = 0.25 * (8 * x * (y * y - 1));
  dy[0] = 0.25 * (x * (x - 1) * (2 * y - 1));
  dy[1] = 0.25 * (x * (x + 1) * (2 * y - 1));
  dy[2] = 0.25 * (x * (x + 1) * (2 * y + 1));
  dy[3] = 0.25 * (x * (x - 1) * (2 * y + 1));
  dy[4] = 0.25 * (-2 * (x + 1) * (x - 1) * (2 * y - 1));
  dy[5] = 0.25 * (-4 * x * y * (x + 1));
  dy[6] = 0.25 * (-2 * (x + 1) * (x - 1) * (2 * y + 1));
  dy[7] = 0.25 * (-4 * x * y * (x - 1));
  dy[8] = 0.25 * (8 * y * (x * x - 1));
}

__device__ inline void stretch_codes(const cd *a, cd *s) {
  s[0] = cdiv(cmul(a[1], a[2]), a[0]);
  s[1] = a[2];
  s[2] = a[1];
  s[3] = cdiv(cmul(a[0], a[2]), a[1]);
  s[4] = a[0];
  s[5] = cdiv(cmul(a[0], a[1]), a[2]);
}

constexpr double kScaleQ9 = 6.173191780858575e-11;  // piezo_fem.py:26

// One warp per element.  Kel: [e][A][B][81] complex, Mel: [e][81] complex.
__global__ void __launch_bounds__(128) q9_element_kernel(
    int64_t ne, int nc, const double *__restrict__ pos, const int64_t *__restrict__ conn,
    const int32_t *__restrict__ emat, const double *__restrict__ rho, const double *__restrict__ Cm,
    const double *__restrict__ em, const double *__restrict__ epsm, PmlDev pml, cd *__restrict__ Kel,
    cd *__restrict__ Mel) {
  __shared__ double s_dN[4][9][9][2];   // [warp][q][node][dir]
  __shared__ double s_dV[4][9];
  __shared__ double s_N[9][9];
  __shared__ cd s_C[4][9][9], s_E[4][3][9], s_P[4][3][3];
  __shared__ cd s_rho[4];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t e = (int64_t)blockIdx.x * 4 + w;
  if (threadIdx.x < 9) {
    double N[9], dx[9], dy[9];
    q9_shape(c_gp[threadIdx.x % 3], c_gp[threadIdx.x / 3], N, dx, dy);
    for (int a = 0; a < 9; ++a) s_N[threadIdx.x][a] = N[a];
  }
  __syncthreads();
  if (e >= ne) return;
  const int64_t *cn = conn + e * 9;
  if (lane < 9) {
    const int q = lane;
    double N[9], dx[9], dy[9];
    q9_shape(c_gp[q % 3], c_gp[q / 3], N, dx, dy);
    double J00 = 0, J01 = 0, J10 = 0, J11 = 0;  // J[i][j] = sum_a xy[a][i] dN[a][j]
    for (int a = 0; a < 9; ++a) {
      const double x = pos[cn[a] * 2], y = pos[cn[a] * 2 + 1];
      J00 += x * dx[a];
      J01 += x * dy[a];
      J10 += y * dx[a];
      J11 += y * dy[a];
    }
    const double det = J00 * J11 - J01 * J10;
    const double i00 = J11 / det, i11 = J00 / det, i01 = -J01 / det, i10 = -J10 / det;
    for (int a = 0; a < 9; ++a) {
      s_dN[w][q][a][0] = dx[a] * i00 + dy[a] * i10;
      s_dN[w][q][a][1] = dx[a] * i01 + dy[a] * i11;
    }
    s_dV[w][q] = c_gw[q % 3] * c_gw[q / 3] * det;
  }
  // stretched constitutive tensors of this element
  const int mi = emat[e];
  cd alpha[3], sc[6];
  double xc[3] = {pos[cn[8] * 2], pos[cn[8] * 2 + 1], 0.0};
  pml_alpha(pml, e, xc, alpha);
  stretch_codes(alpha, sc);
  for (int t = lane; t < 81; t += 32) {
    const int r = t / 9, c = t % 9;
    const int rr = r < 6 ? r : r - 3, cc = c < 6 ? c : c - 3;  // 9x9 gradient form of C
    const double *src = Cm + ((int64_t)mi * 36 + rr * 6 + cc) * 2;
    s_C[w][r][c] = cmul(sc[c_t9[r][c]], cd{src[0], src[1]});
  }
  for (int t = lane; t < 27; t += 32) {
    const int r = t / 9, c = t % 9;
    const int cc = c < 6 ? c : c - 3;
    const double *src = em + ((int64_t)mi * 18 + r * 6 + cc) * 2;
    s_E[w][r][c] = cmul(sc[c_t9[r][c]], cd{src[0], src[1]});
  }
  if (lane < 9) {
    const int r = lane / 3, c = lane % 3;
    const double *src = epsm + ((int64_t)mi * 9 + r * 3 + c) * 2;
    s_P[w][r][c] = cmul(sc[c_teps[r][c]], cd{src[0], src[1]});
  }
  if (lane == 0) s_rho[w] = cmul(cmul(cd{rho[mi], 0.0} * alpha[0], alpha[1]), alpha[2]);
  __syncwarp();

  // ME1 component -> output component (ME0 keeps ux, uy, phi)
  const int comp_out[4] = {0, 1, nc == 3 ? -1 : 2, nc == 3 ? 2 : 3};
  const int64_t blk = 81;
  cd *Ke = Kel + e * (int64_t)nc * nc * blk;
  for (int t = lane; t < 81; t += 32) {
    const int i = t / 9, j = t % 9;
    double G[2][2] = {{0, 0}, {0, 0}}, gm = 0;
    for (int q = 0; q < 9; ++q) {
      const double dv = s_dV[w][q];
      for (int d1 = 0; d1 < 2; ++d1)
        for (int d2 = 0; d2 < 2; ++d2) G[d1][d2] += dv * s_dN[w][q][i][d1] * s_dN[w][q][j][d2];
      gm += dv * s_N[q][i] * s_N[q][j];
    }
    // K_uu (x SCALE)
    for (int a = 0; a < 3; ++a) {
      if (comp_out[a] < 0) continue;
      for (int b = 0; b < 3; ++b) {
        if (comp_out[b] < 0) continue;
        cd acc{0.0, 0.0};
        for (int s = 0; s < 2; ++s)
          for (int u = 0; u < 2; ++u)
            acc = acc + s_C[w][c_sel[a][s][0]][c_sel[b][u][0]] * G[c_sel[a][s][1]][c_sel[b][u][1]];
        Ke[(comp_out[a] * nc + comp_out[b]) * blk + t] = acc * kScaleQ9;
      }
    }
    // K_u-phi at (a, phi) unscaled, K_phi-u = SCALE * transpose
    const int fo = comp_out[3];
    for (int a = 0; a < 3; ++a) {
      if (comp_out[a] < 0) continue;
      cd uf{0.0, 0.0}, fu{0.0, 0.0};
      for (int s = 0; s < 2; ++s)
        for (int k = 0; k < 2; ++k) {
          uf = uf + s_E[w][k][c_sel[a][s][0]] * G[c_sel[a][s][1]][k];
          fu = fu + s_E[w][k][c_sel[a][s][0]] * G[k][c_sel[a][s][1]];  // (j,i) entry of K_uf
        }
      Ke[(comp_out[a] * nc + fo) * blk + t] = uf;
      Ke[(fo * nc + comp_out[a]) * blk + t] = fu * kScaleQ9;
    }
    // K_phi-phi (x -1)
    cd ff{0.0, 0.0};
    for (int j2 = 0; j2 < 2; ++j2)
      for (int k = 0; k < 2; ++k) ff = ff + s_P[w][j2][k] * G[j2][k];
    Ke[(fo * nc + fo) * blk + t] = ff * -1.0;
    Mel[e * blk + t] = (s_rho[w] * gm) * kScaleQ9;
  }
}

}  // namespace ss

namespace ss {

int64_t global_slot(const Handle &h, int64_t i, int a, int64_t r, int b);

cudaError_t launch_q9_elements(cudaStream_t s, int64_t ne, int nc, const double *pos, const int64_t *conn,
                               const int32_t *emat, const double *rho, const double *C, const double *e,
                               const double *eps, const PmlDev &pml, cd *Kel, cd *Mel) {
  if (ne <= 0) return cudaSuccess;
  q9_element_kernel<<<(unsigned)((ne + 3) / 4), 128, 0, s>>>(ne, nc, pos, conn, emat, rho, C, e, eps, pml, Kel, Mel);
  return cudaGetLastError();
}

// Sum the element contributions of every (node pair, component pair) in
// ascending element order into the global CSR values.
__global__ void gather_pairs_kernel(int64_t npairs, int nc, int npe2, int hex, int ndisp, int64_t N,
                                    const int32_t *__restrict__ pair_row, const int64_t *__restrict__ nadj_ptr,
                                    const int64_t *__restrict__ indptr, const int64_t *__restrict__ gp_ptr,
                                    const int64_t *__restrict__ gp_src, const cd *__restrict__ Kel,
                                    const cd *__restrict__ Mel, cd *__restrict__ K, cd *__restrict__ M) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ncc = (int64_t)nc * nc;
  if (t >= npairs * ncc) return;
  const int64_t p = t / ncc;
  const int A = (int)((t % ncc) / nc), B = (int)(t % nc);
  const int64_t i = pair_row[p];
  const int64_t r = p - nadj_ptr[i], d = nadj_ptr[i + 1] - nadj_ptr[i];
  int64_t row, col;
  if (hex) {
    row = A < 3 ? 3 * i + A : 3 * N + i;
    col = B < 3 ? 3 * r + B : 3 * d + r;
  } else {
    row = (int64_t)A * N + i;
    col = (int64_t)B * d + r;
  }
  const int64_t slot = indptr[row] + col;
  cd acc{0.0, 0.0}, macc{0.0, 0.0};
  const bool wantM = M && A == B && A < ndisp;
  for (int64_t q = gp_ptr[p]; q < gp_ptr[p + 1]; ++q) {
    const int64_t code = gp_src[q];
    const int64_t e = code / npe2, loc = code % npe2;
    acc = acc + Kel[(e * ncc + A * nc + B) * npe2 + loc];
    if (wantM) macc = macc + Mel[e * npe2 + loc];
  }
  K[slot] = acc;
  if (wantM) M[slot] = macc;
}

int launch_hex27_elements(Handle &h, int which, const PmlDev &pml, cd *Kel, cd *Mel, const double *dpos,
                          const int64_t *dconn, const int32_t *demat, const double *drho, const double *dC,
                          const double *de, const double *deps);

cudaError_t dalloc(DBuf &b, size_t bytes) {
  if (b.p && b.bytes >= bytes) return cudaSuccess;
  b.release();
  cudaError_t e = cudaMalloc(&b.p, bytes ? bytes : 16);
  if (e == cudaSuccess) b.bytes = bytes;
  return e;
}

int launch_assemble(Handle &h, int which) {
  const int npe = h.npe, nc = h.nc, npe2 = npe * npe;
  const int64_t ne = h.ne, N = h.N;
  // node-pair gather lists, element-ascending
  const int64_t npairs = h.nadj_ptr[N];
  std::vector<int64_t> cnt(npairs + 1, 0), src((size_t)ne * npe2);
  std::vector<int64_t> pidx((size_t)ne * npe2);
  for (int64_t e = 0; e < ne; ++e)
    for (int a = 0; a < npe; ++a) {
      const int64_t i = h.conn[e * npe + a];
      const int64_t *b0 = &h.nadj[h.nadj_ptr[i]], *b1 = &h.nadj[h.nadj_ptr[i + 1]];
      for (int b = 0; b < npe; ++b) {
        const int64_t j = h.conn[e * npe + b];
        const int64_t p = h.nadj_ptr[i] + (std::lower_bound(b0, b1, j) - b0);
        pidx[e * npe2 + a * npe + b] = p;
        ++cnt[p + 1];
      }
    }
  for (int64_t p = 0; p < npairs; ++p) cnt[p + 1] += cnt[p];
  {
    std::vector<int64_t> f(cnt.begin(), cnt.end() - 1);
    for (int64_t c = 0; c < ne * npe2; ++c) src[f[pidx[c]]++] = c;
  }
  std::vector<int32_t> prow(npairs);
  for (int64_t i = 0; i < N; ++i)
    for (int64_t p = h.nadj_ptr[i]; p < h.nadj_ptr[i + 1]; ++p) prow[p] = (int32_t)i;
  pidx.clear();

  DBuf dpos, dconn, demat, drho, dC, de, deps, dax, dnp, dreg, ddm, din, dout, dKel, dMel, dprow, dnadj, dindptr,
      dgp, dgs;
  cudaError_t err;
#define SS_TRY(x)                                   \
  do {                                              \
    if ((err = (x)) != cudaSuccess) return cuda_fail(h, err, #x); \
  } while (0)
  SS_TRY(dupload(dpos, h.pos));
  SS_TRY(dupload(dconn, h.conn));
  SS_TRY(dupload(demat, h.emat));
  const int wm = which;
  SS_TRY(dupload(drho, h.rho[wm]));
  SS_TRY(dupload(dC, h.C[wm]));
  SS_TRY(dupload(de, h.e[wm]));
  SS_TRY(dupload(deps, h.eps[wm]));
  PmlDev pml{};
  pml.clip = h.pml_clip;
  pml.omega = h.omega_top;
  if (h.npml > 0) {
    SS_TRY(dupload(dax, h.pml_axis));
    SS_TRY(dupload(dnp, h.pml_npow));
    SS_TRY(dupload(dreg, h.elem_region));
    SS_TRY(dupload(ddm, h.pml_dmax));
    SS_TRY(dupload(din, h.pml_inner));
    SS_TRY(dupload(dout, h.pml_outer));
    pml.axis = dax.as<int32_t>();
    pml.npow = dnp.as<int32_t>();
    pml.elem_region = dreg.as<int32_t>();
    pml.dmax = ddm.as<double>();
    pml.inner = din.as<double>();
    pml.outer = dout.as<double>();
  }
  SS_TRY(dalloc(dKel, (size_t)ne * nc * nc * npe2 * sizeof(cd)));
  SS_TRY(dalloc(dMel, (size_t)ne * npe2 * sizeof(cd)));
  // the element and scatter kernels are timed by events (stats slots 34 and 35)
  cudaEvent_t ev[3];
  for (auto &x : ev) SS_TRY(cudaEventCreate(&x));
  struct EvFree {
    cudaEvent_t *e;
    ~EvFree() { for (int i = 0; i < 3; ++i) cudaEventDestroy(e[i]); }
  } ev_free{ev};
  SS_TRY(cudaEventRecord(ev[0], h.stream));
  if (h.kind == SS_HEX27) {
    int rc = launch_hex27_elements(h, which, pml, dKel.as<cd>(), dMel.as<cd>(), dpos.as<double>(),
                                   dconn.as<int64_t>(), demat.as<int32_t>(), drho.as<double>(), dC.as<double>(),
                                   de.as<double>(), deps.as<double>());
    if (rc) return rc;
  } else {
    q9_element_kernel<<<(unsigned)((ne + 3) / 4), 128, 0, h.stream>>>(
        ne, nc, dpos.as<double>(), dconn.as<int64_t>(), demat.as<int32_t>(), drho.as<double>(), dC.as<double>(),
        de.as<double>(), deps.as<double>(), pml, dKel.as<cd>(), dMel.as<cd>());
    SS_TRY(cudaGetLastError());
  }
  SS_TRY(cudaEventRecord(ev[1], h.stream));
  SS_TRY(dupload(dprow, prow));
  SS_TRY(dupload(dnadj, h.nadj_ptr));
  SS_TRY(dupload(dindptr, h.indptr));
  SS_TRY(dupload(dgp, cnt));
  SS_TRY(dupload(dgs, src));
  DBuf &dst = which ? h.dD : h.dK;
  SS_TRY(dalloc(dst, (size_t)h.nnz * sizeof(cd)));
  SS_TRY(cudaMemsetAsync(dst.p, 0, (size_t)h.nnz * sizeof(cd), h.stream));
  cd *dM = nullptr;
  if (!which) {
    SS_TRY(dalloc(h.dM, (size_t)h.nnz * sizeof(cd)));
    SS_TRY(cudaMemsetAsync(h.dM.p, 0, (size_t)h.nnz * sizeof(cd), h.stream));
    dM = h.dM.as<cd>();
  }
  const int ndisp = h.kind == SS_Q9_ME0 ? 2 : 3;
  const int64_t nt = npairs * nc * nc;
  cudaEvent_t g0;
  SS_TRY(cudaEventCreate(&g0));
  SS_TRY(cudaEventRecord(g0, h.stream));
  gather_pairs_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, h.stream>>>(
      npairs, nc, npe2, h.kind == SS_HEX27, ndisp, N, dprow.as<int32_t>(), dnadj.as<int64_t>(),
      dindptr.as<int64_t>(), dgp.as<int64_t>(), dgs.as<int64_t>(), dKel.as<cd>(), dMel.as<cd>(), dst.as<cd>(), dM);
  SS_TRY(cudaGetLastError());
  SS_TRY(cudaEventRecord(ev[2], h.stream));
  SS_TRY(cudaStreamSynchronize(h.stream));
  if (!which) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    h.st[34] = ms;
    cudaEventElapsedTime(&ms, g0, ev[2]);
    h.st[35] = ms;
  }
  cudaEventDestroy(g0);
  if (which) h.have_D = true;
  else h.have_K = h.have_M = true;
  return SS_OK;
#undef SS_TRY
}

}  // namespace ss
