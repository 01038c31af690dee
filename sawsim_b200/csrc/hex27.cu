// Hex27 element matrices of the 2.5D periodic slab (src/sawsim/saw2d/saw3d/assembly.py:230-327,
// elements.py:63-105), one CTA per element.
//
// Per element: the H27 basis at the 27 Gauss points (products of the 1-D
// quadratics m = t(t-1), p = t(t+1), z = (t+1)(t-1), reordered by the sortSF27
// permutation; truncated Gauss literals as in elements.py:22-24), Jacobians with
// |det| weights (assembly.py:31-70), then for every node pair (a, b) the
// gradient Gram G[i][j] = sum_q w dN_a/dx_i dN_b/dx_j and the mass Gram, from
// which the 4x4 component blocks follow:
//   K_uu[c][d]  = S * sum_{(s,i) in sel(c)} sum_{(t,j) in sel(d)} C[s][t] G[i][j]
//   K_uphi[c]   =     sum_{(s,i) in sel(c)} sum_j e[j][s] G[i][j]
//   K_phiu[d]   = S * conj(K_uphi of the pair (b, a), component d)      (assembly.py:300-302)
//   K_phiphi    = -   sum_{i,j} eps[i][j] G[i][j]
//   M[c][c]     = S * rho * GM
// with S = KM_SCALE, Voigt strain order xx, yy, zz, yz, xz, xy and the strain
// selectors of the reference B matrix (assembly.py:81-101), including its quirk:
// the yz strain has only the duy/dz term (duz/dy is dropped).  PML elements
// stretch C, e, eps by the Voigt multiplier tables of assembly.py:146-179 and rho
// by a1 a2 a3, with the alphas at the centre node (node 26) and no clamp.
// Output layout matches the Q9 kernel: Kel[e][A][B][a*27+b], Mel[e][a*27+b].
#include "ss_internal.h"
#include "dev_complex.cuh"
#include "q9_element.cuh"
#include "dual.cuh"

namespace ss {

namespace h27 {

constexpr double kG = 0.774596669241483;   // elements.py:22
constexpr double kW5 = 0.555555555555556;  // elements.py:23
constexpr double kW8 = 0.888888888888889;  // elements.py:24
constexpr double kScale = 6.723363908816403e-11;   // assembly.py:24

// raw shape functions (coefficient, factor code per axis; 0 m, 1 p, 2 z) in the
// order of elements.py:28-39, and the sortSF27 permutation (elements.py:42-44)
__constant__ double c_coef[27] = {0.125, 0.125, 0.125, 0.125, 0.125, 0.125, 0.125, 0.125, -0.25, -0.25,
                                  -0.25, -0.25, -0.25, -0.25, -0.25, -0.25, -0.25, -0.25, -0.25, -0.25,
                                  0.5,   0.5,   0.5,   0.5,   0.5,   0.5,   -1.0};
__constant__ unsigned char c_fac[27][3] = {
    {0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}, {2, 0, 0},
    {1, 2, 0}, {2, 1, 0}, {0, 2, 0}, {0, 0, 2}, {1, 0, 2}, {1, 1, 2}, {0, 1, 2}, {2, 0, 1}, {1, 2, 1},
    {2, 1, 1}, {0, 2, 1}, {2, 2, 0}, {2, 0, 2}, {1, 2, 2}, {2, 1, 2}, {0, 2, 2}, {2, 2, 1}, {2, 2, 2}};
__constant__ unsigned char c_perm[27] = {6,  5,  4,  7,  2,  1,  0,  3,  17, 18, 14, 16, 13, 19,
                                         12, 15, 9,  10, 8,  11, 25, 22, 23, 21, 24, 20, 26};
// strain selectors of the reference B matrix: component c -> (strain row, derivative)
__constant__ unsigned char c_sel_n[3] = {3, 3, 2};
__constant__ unsigned char c_sel[3][3][2] = {{{0, 0}, {5, 1}, {4, 2}}, {{5, 0}, {1, 1}, {3, 2}}, {{4, 0}, {2, 2}, {0, 0}}};
// Voigt stretch multipliers: 0 r1 = a2a3/a1, 1 r2 = a1a3/a2, 2 r3 = a1a2/a3, 3 a1, 4 a2, 5 a3
__constant__ unsigned char c_cst[6][6] = {{0, 5, 4, 5, 0, 0}, {5, 1, 3, 1, 5, 5}, {4, 3, 2, 3, 4, 4},
                                          {4, 3, 2, 3, 4, 4}, {4, 3, 2, 3, 4, 4}, {5, 1, 3, 1, 5, 5}};
__constant__ unsigned char c_est[3][6] = {{0, 5, 4, 4, 4, 5}, {5, 1, 3, 3, 3, 1}, {4, 3, 2, 2, 2, 3}};
__constant__ unsigned char c_pst[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};

__device__ inline double fac(int code, double t) {
  return code == 0 ? t * (t - 1.0) : code == 1 ? t * (t + 1.0) : (t + 1.0) * (t - 1.0);
}
__device__ inline double dfac(int code, double t) { return code == 0 ? 2.0 * t - 1.0 : code == 1 ? 2.0 * t + 1.0 : 2.0 * t; }

}  // namespace h27

// Element matrices of ne Hex27 elements (the launch's first element is `e0`).
__global__ void __launch_bounds__(128) hex27_element_kernel(int64_t ne, const double *__restrict__ pos,
                                                            const int64_t *__restrict__ conn,
                                                            const int32_t *__restrict__ emat,
                                                            const double *__restrict__ rho, const double *__restrict__ Cm,
                                                            const double *__restrict__ em,
                                                            const double *__restrict__ epsm, PmlDev pml,
                                                            cd *__restrict__ Kel, cd *__restrict__ Mel) {
  using namespace h27;
  __shared__ double s_N[27][27];        // [q][a]
  __shared__ double s_dx[27][27][3];    // [q][a][i]: natural, then physical derivatives
  __shared__ double s_w[27];
  __shared__ double s_xyz[27][3];
  __shared__ cd s_C[6][6], s_E[3][6], s_P[3][3], s_rho;
  const int64_t e = blockIdx.x;
  if (e >= ne) return;
  const int tid = threadIdx.x;
  const int64_t *cn = conn + e * 27;
  if (tid < 81) s_xyz[tid / 3][tid % 3] = pos[cn[tid / 3] * 3 + tid % 3];
  // basis at the Gauss points (q = k1 + 3 k2 + 9 k3), sortSF27 order
  for (int t = tid; t < 729; t += blockDim.x) {
    const int q = t / 27, a = t % 27;
    const double g[3] = {-kG, 0.0, kG};
    const double x1 = g[q % 3], x2 = g[(q / 3) % 3], x3 = g[q / 9];
    const int r = c_perm[a];
    const int f1 = c_fac[r][0], f2 = c_fac[r][1], f3 = c_fac[r][2];
    const double a1 = fac(f1, x1), a2 = fac(f2, x2), a3 = fac(f3, x3);
    s_N[q][a] = c_coef[r] * a1 * a2 * a3;
    s_dx[q][a][0] = c_coef[r] * dfac(f1, x1) * a2 * a3;
    s_dx[q][a][1] = c_coef[r] * a1 * dfac(f2, x2) * a3;
    s_dx[q][a][2] = c_coef[r] * a1 * a2 * dfac(f3, x3);
  }
  __syncthreads();
  // Jacobian per Gauss point: J[r][c] = sum_a x_c(a) dN_a/dxi_r (assembly.py:54-60)
  if (tid < 27) {
    const int q = tid;
    double j[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int a = 0; a < 27; ++a)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) j[r][c] += s_xyz[a][c] * s_dx[q][a][r];
    const double det = j[0][0] * (j[1][1] * j[2][2] - j[2][1] * j[1][2]) -
                       j[0][1] * (j[1][0] * j[2][2] - j[1][2] * j[2][0]) +
                       j[0][2] * (j[1][0] * j[2][1] - j[1][1] * j[2][0]);
    double ji[3][3];
    ji[0][0] = (j[1][1] * j[2][2] - j[1][2] * j[2][1]) / det;
    ji[0][1] = -(j[0][1] * j[2][2] - j[0][2] * j[2][1]) / det;
    ji[0][2] = (j[0][1] * j[1][2] - j[0][2] * j[1][1]) / det;
    ji[1][0] = -(j[1][0] * j[2][2] - j[1][2] * j[2][0]) / det;
    ji[1][1] = (j[0][0] * j[2][2] - j[0][2] * j[2][0]) / det;
    ji[1][2] = -(j[0][0] * j[1][2] - j[0][2] * j[1][0]) / det;
    ji[2][0] = (j[1][0] * j[2][1] - j[1][1] * j[2][0]) / det;
    ji[2][1] = -(j[0][0] * j[2][1] - j[0][1] * j[2][0]) / det;
    ji[2][2] = (j[0][0] * j[1][1] - j[0][1] * j[1][0]) / det;
    const double wq[3] = {kW5, kW8, kW5};
    s_w[q] = ::fabs(det) * (wq[q % 3] * wq[(q / 3) % 3] * wq[q / 9]);
    for (int a = 0; a < 27; ++a) {
      const double d1 = s_dx[q][a][0], d2 = s_dx[q][a][1], d3 = s_dx[q][a][2];
      s_dx[q][a][0] = ji[0][0] * d1 + ji[0][1] * d2 + ji[0][2] * d3;
      s_dx[q][a][1] = ji[1][0] * d1 + ji[1][1] * d2 + ji[1][2] * d3;
      s_dx[q][a][2] = ji[2][0] * d1 + ji[2][1] * d2 + ji[2][2] * d3;
    }
  }
  // stretched constitutive tensors of this element
  const int mi = emat[e];
  cd alpha[3], sc[6];
  {
    const double xc[3] = {pos[cn[26] * 3], pos[cn[26] * 3 + 1], pos[cn[26] * 3 + 2]};
    pml_alpha(pml, e, xc, alpha);
    sc[0] = cdiv(cmul(alpha[1], alpha[2]), alpha[0]);
    sc[1] = cdiv(cmul(alpha[0], alpha[2]), alpha[1]);
    sc[2] = cdiv(cmul(alpha[0], alpha[1]), alpha[2]);
    sc[3] = alpha[0];
    sc[4] = alpha[1];
    sc[5] = alpha[2];
  }
  for (int t = tid; t < 36 + 18 + 9; t += blockDim.x) {
    if (t < 36) {
      const double *src = Cm + ((int64_t)mi * 36 + t) * 2;
      s_C[t / 6][t % 6] = cmul(cd{src[0], src[1]}, sc[c_cst[t / 6][t % 6]]);
    } else if (t < 54) {
      const int u = t - 36;
      const double *src = em + ((int64_t)mi * 18 + u) * 2;
      s_E[u / 6][u % 6] = cmul(cd{src[0], src[1]}, sc[c_est[u / 6][u % 6]]);
    } else {
      const int u = t - 54;
      const double *src = epsm + ((int64_t)mi * 9 + u) * 2;
      s_P[u / 3][u % 3] = cmul(cd{src[0], src[1]}, sc[c_pst[u / 3][u % 3]]);
    }
  }
  if (tid == 0) s_rho = cmul(cmul(cd{rho[mi], 0.0} * alpha[0], alpha[1]), alpha[2]);
  __syncthreads();

  constexpr int64_t blk = 729;
  cd *Ke = Kel + e * 16 * blk;
  for (int t = tid; t < 729; t += blockDim.x) {
    const int a = t / 27, b = t % 27;
    double G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, gm = 0.0;
    for (int q = 0; q < 27; ++q) {
      const double w = s_w[q];
      const double pa[3] = {w * s_dx[q][a][0], w * s_dx[q][a][1], w * s_dx[q][a][2]};
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) G[i][j] += pa[i] * s_dx[q][b][j];
      gm += w * s_N[q][a] * s_N[q][b];
    }
    // K_uu
    for (int c = 0; c < 3; ++c)
      for (int d = 0; d < 3; ++d) {
        cd acc{0.0, 0.0};
        for (int u = 0; u < c_sel_n[c]; ++u)
          for (int v = 0; v < c_sel_n[d]; ++v)
            acc = acc + s_C[c_sel[c][u][0]][c_sel[d][v][0]] * G[c_sel[c][u][1]][c_sel[d][v][1]];
        Ke[(c * 4 + d) * blk + t] = acc * kScale;
      }
    // K_u-phi (unscaled) and K_phi-u = S * conj of the (b, a) K_u-phi
    for (int c = 0; c < 3; ++c) {
      cd uf{0.0, 0.0}, fu{0.0, 0.0};
      for (int u = 0; u < c_sel_n[c]; ++u) {
        const int s = c_sel[c][u][0], i = c_sel[c][u][1];
        for (int j = 0; j < 3; ++j) {
          uf = uf + s_E[j][s] * G[i][j];
          fu = fu + s_E[j][s] * G[j][i];
        }
      }
      Ke[(c * 4 + 3) * blk + t] = uf;
      Ke[(3 * 4 + c) * blk + t] = cd{fu.x, -fu.y} * kScale;
    }
    cd ff{0.0, 0.0};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) ff = ff + s_P[i][j] * G[i][j];
    Ke[15 * blk + t] = ff * -1.0;
    Mel[e * blk + t] = (s_rho * gm) * kScale;
  }
}

// Tangent element matrices dKel [e][A][B][729], dMel [e][729] of the Hex27
// element routine above, by forward-mode dual numbers seeded with node velocities
// (N x 3), material-tensor derivatives and PML-bound derivatives (the same
// arithmetic as hex27_element_kernel, differentiated).
__global__ void __launch_bounds__(128) hex27_tangent_kernel(int64_t ne, const double *__restrict__ pos,
                                                            const int64_t *__restrict__ conn,
                                                            const int32_t *__restrict__ emat,
                                                            const double *__restrict__ rho,
                                                            const double *__restrict__ Cm, const double *__restrict__ em,
                                                            const double *__restrict__ epsm, PmlDev pml, Seed sd,
                                                            cd *__restrict__ dKel, cd *__restrict__ dMel) {
  using namespace h27;
  __shared__ double s_N[27][27];
  __shared__ dual s_dx[27][27][3];
  __shared__ dual s_w[27];
  __shared__ dual s_xyz[27][3];
  __shared__ cdu s_C[6][6], s_E[3][6], s_P[3][3], s_rho;
  const int64_t e = blockIdx.x;
  if (e >= ne) return;
  const int tid = threadIdx.x;
  const int64_t *cn = conn + e * 27;
  if (tid < 81) {
    const int64_t i = cn[tid / 3] * 3 + tid % 3;
    s_xyz[tid / 3][tid % 3] = dual{pos[i], sd.dpos ? sd.dpos[i] : 0.0};
  }
  for (int t = tid; t < 729; t += blockDim.x) {
    const int q = t / 27, a = t % 27;
    const double g[3] = {-kG, 0.0, kG};
    const double x1 = g[q % 3], x2 = g[(q / 3) % 3], x3 = g[q / 9];
    const int r = c_perm[a];
    const int f1 = c_fac[r][0], f2 = c_fac[r][1], f3 = c_fac[r][2];
    const double a1 = fac(f1, x1), a2 = fac(f2, x2), a3 = fac(f3, x3);
    s_N[q][a] = c_coef[r] * a1 * a2 * a3;
    s_dx[q][a][0] = dual{c_coef[r] * dfac(f1, x1) * a2 * a3};
    s_dx[q][a][1] = dual{c_coef[r] * a1 * dfac(f2, x2) * a3};
    s_dx[q][a][2] = dual{c_coef[r] * a1 * a2 * dfac(f3, x3)};
  }
  __syncthreads();
  if (tid < 27) {
    const int q = tid;
    dual j[3][3];
    for (int a = 0; a < 27; ++a)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) j[r][c] = j[r][c] + s_xyz[a][c] * s_dx[q][a][r];
    const dual det = j[0][0] * (j[1][1] * j[2][2] - j[2][1] * j[1][2]) -
                     j[0][1] * (j[1][0] * j[2][2] - j[1][2] * j[2][0]) +
                     j[0][2] * (j[1][0] * j[2][1] - j[1][1] * j[2][0]);
    dual ji[3][3];
    ji[0][0] = (j[1][1] * j[2][2] - j[1][2] * j[2][1]) / det;
    ji[0][1] = -(j[0][1] * j[2][2] - j[0][2] * j[2][1]) / det;
    ji[0][2] = (j[0][1] * j[1][2] - j[0][2] * j[1][1]) / det;
    ji[1][0] = -(j[1][0] * j[2][2] - j[1][2] * j[2][0]) / det;
    ji[1][1] = (j[0][0] * j[2][2] - j[0][2] * j[2][0]) / det;
    ji[1][2] = -(j[0][0] * j[1][2] - j[0][2] * j[1][0]) / det;
    ji[2][0] = (j[1][0] * j[2][1] - j[1][1] * j[2][0]) / det;
    ji[2][1] = -(j[0][0] * j[2][1] - j[0][1] * j[2][0]) / det;
    ji[2][2] = (j[0][0] * j[1][1] - j[0][1] * j[1][0]) / det;
    const double wq[3] = {kW5, kW8, kW5};
    s_w[q] = fabs(det) * dual{wq[q % 3] * wq[(q / 3) % 3] * wq[q / 9]};
    for (int a = 0; a < 27; ++a) {
      const dual d1 = s_dx[q][a][0], d2 = s_dx[q][a][1], d3 = s_dx[q][a][2];
      s_dx[q][a][0] = ji[0][0] * d1 + ji[0][1] * d2 + ji[0][2] * d3;
      s_dx[q][a][1] = ji[1][0] * d1 + ji[1][1] * d2 + ji[1][2] * d3;
      s_dx[q][a][2] = ji[2][0] * d1 + ji[2][1] * d2 + ji[2][2] * d3;
    }
  }
  const int mi = emat[e];
  cdu alpha[3], sc[6];
  {
    dual xc[3];
    for (int c = 0; c < 3; ++c) {
      const int64_t i = cn[26] * 3 + c;
      xc[c] = dual{pos[i], sd.dpos ? sd.dpos[i] : 0.0};
    }
    pml_alpha_dual(pml, sd, e, xc, alpha);
    sc[0] = cdiv(cmul(alpha[1], alpha[2]), alpha[0]);
    sc[1] = cdiv(cmul(alpha[0], alpha[2]), alpha[1]);
    sc[2] = cdiv(cmul(alpha[0], alpha[1]), alpha[2]);
    sc[3] = alpha[0];
    sc[4] = alpha[1];
    sc[5] = alpha[2];
  }
  for (int t = tid; t < 36 + 18 + 9; t += blockDim.x) {
    if (t < 36) {
      const int64_t o = ((int64_t)mi * 36 + t) * 2;
      s_C[t / 6][t % 6] = cmul(cdu_of(Cm + o, sd.dC ? sd.dC + o : nullptr), sc[c_cst[t / 6][t % 6]]);
    } else if (t < 54) {
      const int u = t - 36;
      const int64_t o = ((int64_t)mi * 18 + u) * 2;
      s_E[u / 6][u % 6] = cmul(cdu_of(em + o, sd.de ? sd.de + o : nullptr), sc[c_est[u / 6][u % 6]]);
    } else {
      const int u = t - 54;
      const int64_t o = ((int64_t)mi * 9 + u) * 2;
      s_P[u / 3][u % 3] = cmul(cdu_of(epsm + o, sd.deps ? sd.deps + o : nullptr), sc[c_pst[u / 3][u % 3]]);
    }
  }
  if (tid == 0) {
    const dual r0{rho[mi], sd.drho ? sd.drho[mi] : 0.0};
    s_rho = cmul(cmul(cmul(cdu{r0, dual{0.0}}, alpha[0]), alpha[1]), alpha[2]);
  }
  __syncthreads();
  constexpr int64_t blk = 729;
  cd *Ke = dKel + e * 16 * blk;
  for (int t = tid; t < 729; t += blockDim.x) {
    const int a = t / 27, b = t % 27;
    dual G[3][3], gm;
    for (int q = 0; q < 27; ++q) {
      const dual w = s_w[q];
      const dual pa[3] = {w * s_dx[q][a][0], w * s_dx[q][a][1], w * s_dx[q][a][2]};
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) G[i][j] = G[i][j] + pa[i] * s_dx[q][b][j];
      gm = gm + w * dual{s_N[q][a] * s_N[q][b]};
    }
    for (int c = 0; c < 3; ++c)
      for (int d = 0; d < 3; ++d) {
        cdu acc{dual{0.0}, dual{0.0}};
        for (int u = 0; u < c_sel_n[c]; ++u)
          for (int v = 0; v < c_sel_n[d]; ++v)
            acc = acc + s_C[c_sel[c][u][0]][c_sel[d][v][0]] * G[c_sel[c][u][1]][c_sel[d][v][1]];
        Ke[(c * 4 + d) * blk + t] = tangent(acc) * kScale;
      }
    for (int c = 0; c < 3; ++c) {
      cdu uf{dual{0.0}, dual{0.0}}, fu{dual{0.0}, dual{0.0}};
      for (int u = 0; u < c_sel_n[c]; ++u) {
        const int s2 = c_sel[c][u][0], i = c_sel[c][u][1];
        for (int j = 0; j < 3; ++j) {
          uf = uf + s_E[j][s2] * G[i][j];
          fu = fu + s_E[j][s2] * G[j][i];
        }
      }
      Ke[(c * 4 + 3) * blk + t] = tangent(uf);
      const cd tf = tangent(fu);
      Ke[(3 * 4 + c) * blk + t] = cd{tf.x, -tf.y} * kScale;
    }
    cdu ff{dual{0.0}, dual{0.0}};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) ff = ff + s_P[i][j] * G[i][j];
    Ke[15 * blk + t] = tangent(ff) * -1.0;
    dMel[e * blk + t] = tangent(s_rho * gm) * kScale;
  }
}

cudaError_t launch_hex27_tangent(cudaStream_t st, int64_t ne, const double *pos, const int64_t *conn,
                                 const int32_t *emat, const double *rho, const double *C, const double *e,
                                 const double *eps, const PmlDev &pml, const Seed &sd, cd *dKel, cd *dMel) {
  if (ne <= 0) return cudaSuccess;
  hex27_tangent_kernel<<<(unsigned)ne, 128, 0, st>>>(ne, pos, conn, emat, rho, C, e, eps, pml, sd, dKel, dMel);
  return cudaGetLastError();
}

int launch_hex27_elements(Handle &h, int, const PmlDev &pml, cd *Kel, cd *Mel, const double *pos, const int64_t *conn,
                          const int32_t *emat, const double *rho, const double *C, const double *e, const double *eps) {
  if (h.ne <= 0) return SS_OK;
  hex27_element_kernel<<<(unsigned)h.ne, 128, 0, h.stream>>>(h.ne, pos, conn, emat, rho, C, e, eps, pml, Kel, Mel);
  const cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? SS_OK : cuda_fail(h, err, "hex27_element_kernel");
}

}  // namespace ss
