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

// Element matrices of ne Q9 elements: Kel [e][A][B][81], Mel [e][81] (complex),
// with the reference's scale factors applied.  conn / emat / pml.elem_region
// are indexed from the first element of this launch.
cudaError_t launch_q9_elements(cudaStream_t s, int64_t ne, int nc, const double *pos, const int64_t *conn,
                               const int32_t *emat, const double *rho, const double *C, const double *e,
                               const double *eps, const PmlDev &pml, cd *Kel, cd *Mel);

}  // namespace ss
