// Adjoint gradient of the charge: dQ/dp for parameters that move the mesh nodes
// (Q9 or Hex27), the material tensors and the PML bounds.
//
// The reference has no derivative; its charge is Q = kts . disp with
// kts = K^T s (src/sawsim/saw2d/sweep.py:303-305, :356-363) and disp[active]
// solving A_aa x = -(Km_s - w^2 Mm_s)[active] V (:337-353).  Differentiating,
//   dQ/dp = sum_e [ (s - mu)_e^T dK_e/dp d_e + w^2 mu_e^T dM_e/dp d_e ]
// with d the full DOF vector (disp), mu = T lambda the adjoint (A_aa^T lambda =
// kq, expanded to all DOFs through the master/slave fold, zero at prescribed
// DOFs) and s the + electrode indicator.  Rayleigh damping is not differentiated.
//
// dK_e/dp, dM_e/dp are recomputed on the fly by forward-mode differentiation
// (dual numbers) of the element routines: Q9 piezo_fem.py:248-367 (the
// arithmetic of q9_element_kernel) and Hex27 saw3d/assembly.py:230-327
// (hex27_tangent_kernel), seeded with the parameter's node velocities,
// material-tensor derivatives and PML-bound derivatives.  For Hex27 the charge
// is the same functional (bc_solve.py:141-175, Q from the unfolded K rows).
#include "ss_internal.h"
#include "dev_complex.cuh"
#include "q9_element.cuh"
#include "dual.cuh"

#include <vector>

namespace ss {

__constant__ double c_gpa[3] = {-0.774596669241483, 0.0, 0.774596669241483};
__constant__ double c_gwa[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
__constant__ int c_sela[3][2][2] = {{{0, 0}, {5, 1}}, {{1, 1}, {8, 0}}, {{6, 1}, {7, 0}}};
__constant__ unsigned char c_t9a[9][9] = {
    {0, 1, 2, 2, 2, 1, 1, 0, 0}, {1, 3, 4, 4, 4, 3, 3, 1, 1}, {2, 4, 5, 5, 5, 4, 4, 2, 2},
    {2, 4, 5, 5, 5, 4, 4, 2, 2}, {2, 4, 5, 5, 5, 4, 4, 2, 2}, {1, 3, 4, 4, 4, 3, 3, 1, 1},
    {1, 3, 4, 4, 4, 3, 3, 1, 1}, {0, 1, 2, 2, 2, 1, 1, 0, 0}, {0, 1, 2, 2, 2, 1, 1, 0, 0}};
__constant__ unsigned char c_tepsa[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

__device__ inline void q9_shape_a(double x, double y, double *N, double *dx, double *dy) {
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

// Tangent element matrices dKel [e][A][B][81], dMel [e][81] of ne Q9 elements,
// one warp per element (the layout of q9_element_kernel).
__global__ void __launch_bounds__(128) q9_tangent_kernel(int64_t ne, int nc, const double *__restrict__ pos,
                                                         const int64_t *__restrict__ conn,
                                                         const int32_t *__restrict__ emat,
                                                         const double *__restrict__ rho, const double *__restrict__ Cm,
                                                         const double *__restrict__ em,
                                                         const double *__restrict__ epsm, PmlDev pml, Seed sd,
                                                         cd *__restrict__ dKel, cd *__restrict__ dMel) {
  __shared__ dual s_dN[4][9][9][2];
  __shared__ dual s_dV[4][9];
  __shared__ double s_N[9][9];
  __shared__ cdu s_C[4][9][9], s_E[4][3][9], s_P[4][3][3];
  __shared__ cdu s_rho[4];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t e = (int64_t)blockIdx.x * 4 + w;
  if (threadIdx.x < 9) {
    double N[9], dx[9], dy[9];
    q9_shape_a(c_gpa[threadIdx.x % 3], c_gpa[threadIdx.x / 3], N, dx, dy);
    for (int a = 0; a < 9; ++a) s_N[threadIdx.x][a] = N[a];
  }
  __syncthreads();
  if (e >= ne) return;
  const int64_t *cn = conn + e * 9;
  auto X = [&](int a, int c) {
    return dual{pos[cn[a] * 2 + c], sd.dpos ? sd.dpos[cn[a] * 2 + c] : 0.0};
  };
  if (lane < 9) {
    const int q = lane;
    double N[9], dx[9], dy[9];
    q9_shape_a(c_gpa[q % 3], c_gpa[q / 3], N, dx, dy);
    dual J00, J01, J10, J11;
    for (int a = 0; a < 9; ++a) {
      const dual x = X(a, 0), y = X(a, 1);
      J00 = J00 + x * dual{dx[a]};
      J01 = J01 + x * dual{dy[a]};
      J10 = J10 + y * dual{dx[a]};
      J11 = J11 + y * dual{dy[a]};
    }
    const dual det = J00 * J11 - J01 * J10;
    const dual i00 = J11 / det, i11 = J00 / det, i01 = -J01 / det, i10 = -J10 / det;
    for (int a = 0; a < 9; ++a) {
      s_dN[w][q][a][0] = dual{dx[a]} * i00 + dual{dy[a]} * i10;
      s_dN[w][q][a][1] = dual{dx[a]} * i01 + dual{dy[a]} * i11;
    }
    s_dV[w][q] = dual{c_gwa[q % 3] * c_gwa[q / 3]} * det;
  }
  const int mi = emat[e];
  cdu alpha[3], sc[6];
  const dual xc[3] = {X(8, 0), X(8, 1), dual{0.0}};
  pml_alpha_dual(pml, sd, e, xc, alpha);
  sc[0] = cdiv(cmul(alpha[1], alpha[2]), alpha[0]);
  sc[1] = alpha[2];
  sc[2] = alpha[1];
  sc[3] = cdiv(cmul(alpha[0], alpha[2]), alpha[1]);
  sc[4] = alpha[0];
  sc[5] = cdiv(cmul(alpha[0], alpha[1]), alpha[2]);
  for (int t = lane; t < 81; t += 32) {
    const int r = t / 9, c = t % 9;
    const int rr = r < 6 ? r : r - 3, cc = c < 6 ? c : c - 3;
    const int64_t o = ((int64_t)mi * 36 + rr * 6 + cc) * 2;
    s_C[w][r][c] = cmul(sc[c_t9a[r][c]], cdu_of(Cm + o, sd.dC ? sd.dC + o : nullptr));
  }
  for (int t = lane; t < 27; t += 32) {
    const int r = t / 9, c = t % 9;
    const int cc = c < 6 ? c : c - 3;
    const int64_t o = ((int64_t)mi * 18 + r * 6 + cc) * 2;
    s_E[w][r][c] = cmul(sc[c_t9a[r][c]], cdu_of(em + o, sd.de ? sd.de + o : nullptr));
  }
  if (lane < 9) {
    const int r = lane / 3, c = lane % 3;
    const int64_t o = ((int64_t)mi * 9 + r * 3 + c) * 2;
    s_P[w][r][c] = cmul(sc[c_tepsa[r][c]], cdu_of(epsm + o, sd.deps ? sd.deps + o : nullptr));
  }
  if (lane == 0) {
    const dual r0{rho[mi], sd.drho ? sd.drho[mi] : 0.0};
    s_rho[w] = cmul(cmul(cmul(cdu{r0, dual{0.0}}, alpha[0]), alpha[1]), alpha[2]);
  }
  __syncwarp();
  constexpr double kScaleQ9 = 6.173191780858575e-11;   // piezo_fem.py:26
  const int comp_out[4] = {0, 1, nc == 3 ? -1 : 2, nc == 3 ? 2 : 3};
  cd *Ke = dKel + e * (int64_t)nc * nc * 81;
  for (int t = lane; t < 81; t += 32) {
    const int i = t / 9, j = t % 9;
    dual G[2][2], gm;
    for (int q = 0; q < 9; ++q) {
      const dual dv = s_dV[w][q];
      for (int d1 = 0; d1 < 2; ++d1)
        for (int d2 = 0; d2 < 2; ++d2) G[d1][d2] = G[d1][d2] + dv * s_dN[w][q][i][d1] * s_dN[w][q][j][d2];
      gm = gm + dv * dual{s_N[q][i] * s_N[q][j]};
    }
    for (int a = 0; a < 3; ++a) {
      if (comp_out[a] < 0) continue;
      for (int b = 0; b < 3; ++b) {
        if (comp_out[b] < 0) continue;
        cdu acc{dual{0.0}, dual{0.0}};
        for (int s = 0; s < 2; ++s)
          for (int u = 0; u < 2; ++u)
            acc = acc + s_C[w][c_sela[a][s][0]][c_sela[b][u][0]] * G[c_sela[a][s][1]][c_sela[b][u][1]];
        Ke[(comp_out[a] * nc + comp_out[b]) * 81 + t] = tangent(acc) * kScaleQ9;
      }
    }
    const int fo = comp_out[3];
    for (int a = 0; a < 3; ++a) {
      if (comp_out[a] < 0) continue;
      cdu uf{dual{0.0}, dual{0.0}}, fu{dual{0.0}, dual{0.0}};
      for (int s = 0; s < 2; ++s)
        for (int k = 0; k < 2; ++k) {
          uf = uf + s_E[w][k][c_sela[a][s][0]] * G[c_sela[a][s][1]][k];
          fu = fu + s_E[w][k][c_sela[a][s][0]] * G[k][c_sela[a][s][1]];
        }
      Ke[(comp_out[a] * nc + fo) * 81 + t] = tangent(uf);
      Ke[(fo * nc + comp_out[a]) * 81 + t] = tangent(fu) * kScaleQ9;
    }
    cdu ff{dual{0.0}, dual{0.0}};
    for (int j2 = 0; j2 < 2; ++j2)
      for (int k = 0; k < 2; ++k) ff = ff + s_P[w][j2][k] * G[j2][k];
    Ke[(fo * nc + fo) * 81 + t] = tangent(ff) * -1.0;
    dMel[e * 81 + t] = tangent(s_rho[w] * gm) * kScaleQ9;
  }
}

// Per-chunk full DOF vectors from the scaled solutions:
//   d[f][i]  = cs[R] x'[f][R] for R = gnew[i] >= 0, V for the + electrode (gnew = -1), else 0
//   mu[f][i] = rs[R] mu'[f][R] for R >= 0, else 0
// (sweep.py:356-362: slaves take their master's value; the prescribed values last)
__global__ void expand_kernel(int64_t gdof, int nb, int64_t n, const int64_t *__restrict__ gnew,
                              const double *__restrict__ cs, const double *__restrict__ rs,
                              const cd *__restrict__ x, const cd *__restrict__ mu, double V, cd *__restrict__ d,
                              cd *__restrict__ m) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (i >= gdof || f >= nb) return;
  const int64_t R = gnew[i];
  cd dv{0.0, 0.0}, mv{0.0, 0.0};
  if (R >= 0) {
    dv = x[(int64_t)f * n + R] * cs[R];
    mv = mu[(int64_t)f * n + R] * rs[R];
  } else if (R == -1) {
    dv = cd{V, 0.0};
  }
  d[(int64_t)f * gdof + i] = dv;
  m[(int64_t)f * gdof + i] = mv;
}

// part[f][e] = (s - mu)_e^T dK_e d_e + w_f^2 mu_e^T dM_e d_e, one CTA per element,
// frequencies of the chunk in a loop; fixed-order tree reduction inside the CTA.
__global__ void __launch_bounds__(128) contract_kernel(int64_t ne, int nc, int ndisp, int64_t N, int nb,
                                                       int64_t gdof, const int64_t *__restrict__ conn,
                                                       const cd *__restrict__ dKel, const cd *__restrict__ dMel,
                                                       const cd *__restrict__ d, const cd *__restrict__ m,
                                                       const unsigned char *__restrict__ splus,
                                                       const double *__restrict__ omega, cd *__restrict__ part) {
  __shared__ cd s_K[16 * 81];
  __shared__ cd s_M[81];
  __shared__ cd s_d[36], s_w[36], s_m[36];
  __shared__ cd red[128];
  const int64_t e = blockIdx.x;
  const int nd = nc * 9;
  for (int t = threadIdx.x; t < nc * nc * 81; t += blockDim.x) s_K[t] = dKel[e * nc * nc * 81 + t];
  for (int t = threadIdx.x; t < 81; t += blockDim.x) s_M[t] = dMel[e * 81 + t];
  const int64_t *cn = conn + e * 9;
  for (int f = 0; f < nb; ++f) {
    __syncthreads();
    if (threadIdx.x < nd) {
      const int A = threadIdx.x / 9, a = threadIdx.x % 9;
      const int64_t g = (int64_t)A * N + cn[a];
      const cd dv = d[(int64_t)f * gdof + g], mv = m[(int64_t)f * gdof + g];
      s_d[threadIdx.x] = dv;
      s_m[threadIdx.x] = mv;
      s_w[threadIdx.x] = cd{(splus[g] ? 1.0 : 0.0) - mv.x, -mv.y};
    }
    __syncthreads();
    cd acc{0.0, 0.0};
    const double w2 = omega[f] * omega[f];
    for (int r = threadIdx.x; r < nd; r += blockDim.x) {
      const int A = r / 9, a = r % 9;
      cd y{0.0, 0.0};
      for (int B = 0; B < nc; ++B)
        for (int b = 0; b < 9; ++b) y = y + cmul(s_K[(A * nc + B) * 81 + a * 9 + b], s_d[B * 9 + b]);
      acc = acc + cmul(s_w[r], y);
      if (A < ndisp) {
        cd ym{0.0, 0.0};
        for (int b = 0; b < 9; ++b) ym = ym + cmul(s_M[a * 9 + b], s_d[A * 9 + b]);
        acc = acc + cmul(s_m[r], ym) * w2;
      }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[(int64_t)f * ne + e] = red[0];
  }
}

// Hex27: part[f][e] as contract_kernel for 108 element DOFs (u interleaved 3n + c,
// phi at 3N + n).  The element's dK (16 x 729 complex) stays in global memory
// (L1/L2-resident while the CTA works); frequencies go in groups of 4 whose
// vectors are staged in shared memory; fixed-order reduction per frequency.
constexpr int kHexFG = 4;
__global__ void __launch_bounds__(256) contract_hex_kernel(int64_t ne, int64_t N, int nb, int64_t gdof,
                                                           const int64_t *__restrict__ conn,
                                                           const cd *__restrict__ dKel, const cd *__restrict__ dMel,
                                                           const cd *__restrict__ d, const cd *__restrict__ m,
                                                           const unsigned char *__restrict__ splus,
                                                           const double *__restrict__ omega, cd *__restrict__ part) {
  __shared__ cd s_d[kHexFG][108], s_w[kHexFG][108], s_m[kHexFG][108];
  __shared__ cd s_r[kHexFG][108];
  const int64_t e = blockIdx.x;
  const int64_t *cn = conn + e * 27;
  const cd *K = dKel + e * 16 * 729;
  const cd *Me = dMel + e * 729;
  for (int f0 = 0; f0 < nb; f0 += kHexFG) {
    const int nf = min(kHexFG, nb - f0);
    __syncthreads();
    for (int t = threadIdx.x; t < nf * 108; t += blockDim.x) {
      const int fi = t / 108, r = t % 108, A = r / 27, a = r % 27;
      const int64_t g = A < 3 ? 3 * cn[a] + A : 3 * N + cn[a];
      const cd dv = d[(int64_t)(f0 + fi) * gdof + g], mv = m[(int64_t)(f0 + fi) * gdof + g];
      s_d[fi][r] = dv;
      s_m[fi][r] = mv;
      s_w[fi][r] = cd{(splus[g] ? 1.0 : 0.0) - mv.x, -mv.y};
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nf * 108; t += blockDim.x) {
      const int fi = t / 108, r = t % 108, A = r / 27, a = r % 27;
      cd y{0.0, 0.0};
      for (int B = 0; B < 4; ++B) {
        const cd *row = K + (A * 4 + B) * 729 + a * 27;
        for (int b = 0; b < 27; ++b) y = y + cmul(row[b], s_d[fi][B * 27 + b]);
      }
      cd acc = cmul(s_w[fi][r], y);
      if (A < 3) {
        cd ym{0.0, 0.0};
        for (int b = 0; b < 27; ++b) ym = ym + cmul(Me[a * 27 + b], s_d[fi][A * 27 + b]);
        const double w2 = omega[f0 + fi] * omega[f0 + fi];
        acc = acc + cmul(s_m[fi][r], ym) * w2;
      }
      s_r[fi][r] = acc;
    }
    __syncthreads();
    if (threadIdx.x < nf) {
      cd acc{0.0, 0.0};
      for (int r = 0; r < 108; ++r) acc = acc + s_r[threadIdx.x][r];
      part[(int64_t)(f0 + threadIdx.x) * ne + e] = acc;
    }
  }
}

// out[f] = sum_e part[f][e], fixed-order tree per frequency
__global__ void sum_rows_kernel(int64_t ne, const cd *__restrict__ part, cd *__restrict__ out) {
  __shared__ cd red[256];
  const int f = blockIdx.x;
  cd acc{0.0, 0.0};
  for (int64_t e = threadIdx.x; e < ne; e += blockDim.x) acc = acc + part[(int64_t)f * ne + e];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[f] = red[0];
}


#define AD_CK(x)                                                 \
  do {                                                           \
    cudaError_t e_ = (x);                                        \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, #x);          \
  } while (0)

int run_adjoint_gradient(Handle &h, int n_f, const double *omega, double V, int precision, int n_params,
                         const double *dpos, const double *dC, const double *de, const double *deps,
                         const double *drho, const double *dinner, const double *douter, double *Q, double *dQ,
                         int *status) {
  if (h.have_D && h.beta != 0.0) return fail(h, SS_EINVAL, "adjoint gradient: Rayleigh damping is not differentiated");
  if (!h.have_K) return fail(h, SS_ESTATE, "adjoint gradient: assemble first");
  const bool hex = h.kind == SS_HEX27;
  const int nc = h.nc, ndisp = h.kind == SS_Q9_ME0 ? 2 : 3, nm = h.nmat[0], npml = h.npml;
  const int npe = h.npe, dim = h.dim;
  const int64_t N = h.N, ne = h.ne, G = h.gdof, n = h.sym.n;
  // device copies of the mesh, materials and PML
  DBuf dp, dcn, dem, drh, dCm, deM, depsM, dax, dnp, dreg, ddm, din, dout;
  AD_CK(dupload(dp, h.pos));
  AD_CK(dupload(dcn, h.conn));
  AD_CK(dupload(dem, h.emat));
  AD_CK(dupload(drh, h.rho[0]));
  AD_CK(dupload(dCm, h.C[0]));
  AD_CK(dupload(deM, h.e[0]));
  AD_CK(dupload(depsM, h.eps[0]));
  PmlDev pml{};
  pml.clip = h.pml_clip;
  pml.omega = h.omega_top;
  if (npml > 0) {
    AD_CK(dupload(dax, h.pml_axis));
    AD_CK(dupload(dnp, h.pml_npow));
    AD_CK(dupload(dreg, h.elem_region));
    AD_CK(dupload(ddm, h.pml_dmax));
    AD_CK(dupload(din, h.pml_inner));
    AD_CK(dupload(dout, h.pml_outer));
    pml.axis = dax.as<int32_t>();
    pml.npow = dnp.as<int32_t>();
    pml.elem_region = dreg.as<int32_t>();
    pml.dmax = ddm.as<double>();
    pml.inner = din.as<double>();
    pml.outer = dout.as<double>();
  }
  // seeds, parameter-major
  auto up = [&](DBuf &b, const double *src, size_t cnt) -> cudaError_t {
    if (!src) return cudaSuccess;
    std::vector<double> v(src, src + cnt);
    return dupload(b, v);
  };
  DBuf sp, sC, se, seps, srho, sin, sout;
  AD_CK(up(sp, dpos, (size_t)n_params * N * dim));
  AD_CK(up(sC, dC, (size_t)n_params * nm * 72));
  AD_CK(up(se, de, (size_t)n_params * nm * 36));
  AD_CK(up(seps, deps, (size_t)n_params * nm * 18));
  AD_CK(up(srho, drho, (size_t)n_params * nm));
  AD_CK(up(sin, npml ? dinner : nullptr, (size_t)n_params * npml * 3));
  AD_CK(up(sout, npml ? douter : nullptr, (size_t)n_params * npml * 3));
  // DOF maps: new index of each DOF's master, -1 on the + electrode, -2 otherwise
  std::vector<int64_t> gnew(G, -2);
  std::vector<unsigned char> splus(G, 0);
  for (int64_t i = 0; i < G; ++i) {
    const int64_t a = h.act_of_gdof[h.rep[i]];
    if (a >= 0) gnew[i] = h.sym.new_of_act[a];
  }
  for (int64_t z : h.zheng) gnew[z] = -1, splus[z] = 1;
  for (int64_t z : h.fu) gnew[z] = -2;
  DBuf dgn, dsp, dK, dM, dd, dm, dpart, dout2, dom;
  AD_CK(dupload(dgn, gnew));
  AD_CK(dupload(dsp, splus));
  AD_CK(dalloc(dK, (size_t)ne * nc * nc * npe * npe * sizeof(cd)));
  AD_CK(dalloc(dM, (size_t)ne * npe * npe * sizeof(cd)));
  SweepExtra ex;
  ex.per_chunk = [&](int c0, int nb, const cplx<double> *x, const cplx<double> *mu) -> int {
    AD_CK(dalloc(dd, (size_t)nb * G * sizeof(cd)));
    AD_CK(dalloc(dm, (size_t)nb * G * sizeof(cd)));
    AD_CK(dalloc(dpart, (size_t)nb * ne * sizeof(cd)));
    AD_CK(dalloc(dout2, (size_t)nb * sizeof(cd)));
    AD_CK(dalloc(dom, (size_t)nb * sizeof(double)));
    AD_CK(cudaMemcpyAsync(dom.p, omega + c0, nb * sizeof(double), cudaMemcpyHostToDevice, h.stream));
    expand_kernel<<<dim3((unsigned)((G + 255) / 256), nb), 256, 0, h.stream>>>(
        G, nb, n, dgn.as<int64_t>(), h.dcol_scale.as<double>(), h.drow_scale.as<double>(), x, mu, V, dd.as<cd>(),
        dm.as<cd>());
    std::vector<cd> out(nb);
    for (int p = 0; p < n_params; ++p) {
      Seed sd{};
      sd.dpos = sp.p ? sp.as<double>() + (size_t)p * N * dim : nullptr;
      sd.dC = sC.p ? sC.as<double>() + (size_t)p * nm * 72 : nullptr;
      sd.de = se.p ? se.as<double>() + (size_t)p * nm * 36 : nullptr;
      sd.deps = seps.p ? seps.as<double>() + (size_t)p * nm * 18 : nullptr;
      sd.drho = srho.p ? srho.as<double>() + (size_t)p * nm : nullptr;
      sd.dinner = sin.p ? sin.as<double>() + (size_t)p * npml * 3 : nullptr;
      sd.douter = sout.p ? sout.as<double>() + (size_t)p * npml * 3 : nullptr;
      if (hex) {
        AD_CK(launch_hex27_tangent(h.stream, ne, dp.as<double>(), dcn.as<int64_t>(), dem.as<int32_t>(),
                                   drh.as<double>(), dCm.as<double>(), deM.as<double>(), depsM.as<double>(), pml, sd,
                                   dK.as<cd>(), dM.as<cd>()));
        contract_hex_kernel<<<(unsigned)ne, 256, 0, h.stream>>>(ne, N, nb, G, dcn.as<int64_t>(), dK.as<cd>(),
                                                                dM.as<cd>(), dd.as<cd>(), dm.as<cd>(),
                                                                dsp.as<unsigned char>(), dom.as<double>(),
                                                                dpart.as<cd>());
      } else {
        q9_tangent_kernel<<<(unsigned)((ne + 3) / 4), 128, 0, h.stream>>>(
            ne, nc, dp.as<double>(), dcn.as<int64_t>(), dem.as<int32_t>(), drh.as<double>(), dCm.as<double>(),
            deM.as<double>(), depsM.as<double>(), pml, sd, dK.as<cd>(), dM.as<cd>());
        contract_kernel<<<(unsigned)ne, 128, 0, h.stream>>>(ne, nc, ndisp, N, nb, G, dcn.as<int64_t>(), dK.as<cd>(),
                                                            dM.as<cd>(), dd.as<cd>(), dm.as<cd>(),
                                                            dsp.as<unsigned char>(), dom.as<double>(),
                                                            dpart.as<cd>());
      }
      sum_rows_kernel<<<nb, 256, 0, h.stream>>>(ne, dpart.as<cd>(), dout2.as<cd>());
      AD_CK(cudaGetLastError());
      AD_CK(cudaMemcpyAsync(out.data(), dout2.p, nb * sizeof(cd), cudaMemcpyDeviceToHost, h.stream));
      AD_CK(cudaStreamSynchronize(h.stream));
      for (int f = 0; f < nb; ++f) {
        dQ[2 * ((int64_t)(c0 + f) * n_params + p)] = out[f].x;
        dQ[2 * ((int64_t)(c0 + f) * n_params + p) + 1] = out[f].y;
      }
    }
    return SS_OK;
  };
  std::vector<int> st(n_f, 0), it(n_f, 0);
  const int rc = run_sweep(h, n_f, omega, V, precision, Q, status ? status : st.data(), it.data(), nullptr, &ex);
  return rc;
}
#undef AD_CK

}  // namespace ss
