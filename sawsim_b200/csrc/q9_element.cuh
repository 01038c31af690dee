// Shared declarations of the Q9 element-assembly kernel (assemble.cu) for other
// translation units.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "dev_complex.cuh"

namespace ss {

// PML description on the device (one entry per region; elem_region per element)
struct PmlDev {
  const int32_t *axis, *npow, *elem_region;
  const double *dmax, *inner, *outer;
  int clip;
  double omega;
};

// alphas (a1, a2, a3) of one element from its centre coordinate
// (piezo_fem.py:222-242; saw3d/assembly.py:127-143)
__device__ inline void pml_alpha(const PmlDev &P, int64_t e, const double *xc, cd *a) {
  a[0] = a[1] = a[2] = cd{1.0, 0.0};
  if (!P.elem_region) return;
  const int r = P.elem_region[e];
  if (r < 0) return;
  for (int ax = 0; ax < 3; ++ax) {
    if (!((P.axis[r] >> ax) & 1)) continue;
    const double o = P.outer[3 * r + ax], in = P.inner[3 * r + ax];
    double ratio = (xc[ax] - o) * (xc[ax] - o) / ((in - o) * (in - o));
    if (P.clip) ratio = fmin(fmax(ratio, 0.0), 1.0);
    double d = P.dmax[r] * pow(1.0 - ratio, (double)P.npow[r]);
    // 1 + d / (i w) = 1 - i d / w
    a[ax] = cd{1.0, 0.0} + cdiv(cd{d, 0.0}, cd{0.0, P.omega});
  }
}

// Element matrices of ne Q9 elements: Kel [e][A][B][81], Mel [e][81] (complex),
// with the reference's scale factors applied.  conn / emat / pml.elem_region
// are indexed from the first element of this launch.
cudaError_t launch_q9_elements(cudaStream_t s, int64_t ne, int nc, const double *pos, const int64_t *conn,
                               const int32_t *emat, const double *rho, const double *C, const double *e,
                               const double *eps, const PmlDev &pml, cd *Kel, cd *Mel);

}  // namespace ss
