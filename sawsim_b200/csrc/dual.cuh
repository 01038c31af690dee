// Dual numbers (value, tangent) for forward-mode derivatives of the element
// routines, and the per-parameter derivative seeds of the adjoint gradient.
#pragma once
#include <cstdint>
#include "dev_complex.cuh"
#include "q9_element.cuh"

namespace ss {

// value and tangent
struct dual {
  double v, d;
  __host__ __device__ dual(double a = 0.0, double b = 0.0) : v(a), d(b) {}
};
__device__ inline dual operator+(dual a, dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ inline dual operator-(dual a, dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ inline dual operator-(dual a) { return {-a.v, -a.d}; }
__device__ inline dual operator*(dual a, dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ inline dual operator/(dual a, dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
__device__ inline dual fabs(dual a) { return a.v < 0 ? -a : a; }
__device__ inline bool operator>=(dual a, dual b) { return a.v >= b.v; }
__device__ inline dual ipow(dual a, int n) {
  dual r{1.0, 0.0};
  for (int i = 0; i < n; ++i) r = r * a;
  return r;
}
using cdu = cplx<dual>;
__device__ inline cdu cdu_of(const double *v, const double *t) { return cdu{dual{v[0], t ? t[0] : 0.0}, dual{v[1], t ? t[1] : 0.0}}; }
__device__ inline cd tangent(cdu a) { return cd{a.x.d, a.y.d}; }

// Seeds of one parameter (device pointers, any may be null = zero).
struct Seed {
  const double *dpos;     // N x dim (metres per unit parameter)
  const double *dC, *de, *deps, *drho;   // per material, complex interleaved like ss_set_materials
  const double *dinner, *douter;         // per PML region x 3
};

// PML alphas in dual numbers (piezo_fem.py:222-242 with the clamp for Q9;
// saw3d/assembly.py:127-143 without it for Hex27), centre-node coordinate xc[3]
__device__ inline void pml_alpha_dual(const PmlDev &P, const Seed &sd, int64_t e, const dual *xc, cdu *a) {
  a[0] = a[1] = a[2] = cdu{dual{1.0}, dual{0.0}};
  if (!P.elem_region) return;
  const int r = P.elem_region[e];
  if (r < 0) return;
  for (int ax = 0; ax < 3; ++ax) {
    if (!((P.axis[r] >> ax) & 1)) continue;
    const dual o{P.outer[3 * r + ax], sd.douter ? sd.douter[3 * r + ax] : 0.0};
    const dual in{P.inner[3 * r + ax], sd.dinner ? sd.dinner[3 * r + ax] : 0.0};
    dual ratio = (xc[ax] - o) * (xc[ax] - o) / ((in - o) * (in - o));
    if (P.clip) {
      if (ratio.v < 0.0) ratio = dual{0.0};
      if (ratio.v > 1.0) ratio = dual{1.0};
    }
    const dual d = dual{P.dmax[r]} * ipow(dual{1.0} - ratio, P.npow[r]);
    // 1 + d / (i w) = 1 - i d / w
    a[ax] = cdu{dual{1.0}, -(d / dual{P.omega})};
  }
}

}  // namespace ss
