// Hex27 element assembly (src/sawsim/saw2d/saw3d/assembly.py:230-327).
#include "ss_internal.h"
#include "dev_complex.cuh"

namespace ss {
struct PmlDev;
int launch_hex27_elements(Handle &h, int, const PmlDev &, cd *, cd *, const double *, const int64_t *,
                          const int32_t *, const double *, const double *, const double *, const double *) {
  return fail(h, SS_EINVAL, "Hex27 element assembly is not available in this build");
}
}  // namespace ss
