// Allocation-free Q9 assembly entry point.
//
// Some callers of this library may not call cudaMalloc: a host framework that
// hands out all device memory from its own pool (a caching allocator, a serving
// runtime with a fixed memory budget) and forbids allocations behind its back.
// ss_assemble_q9_noalloc gives them the GPU Q9 assembly with no allocation at
// all: inputs and outputs are device buffers the caller already owns, and the
// element-matrix scratch lives in a fixed file-scope __device__ array below.
#include "ss_internal.h"
#include "dev_complex.cuh"
#include "q9_element.cuh"

#include <algorithm>
#include <mutex>

namespace ss {

// Elements per batch of the allocation-free path.  The scratch below holds the
// element matrices of one batch: 512 x (16 x 81 + 81) complex128 = 11.3 MB,
// resident on every GPU that loads this library until the process exits.
constexpr int kNoAllocMaxElems = 512;
constexpr int kNoAllocMaxComp = 4;

static __device__ __align__(256) cd g_noalloc_kel[kNoAllocMaxElems * kNoAllocMaxComp * kNoAllocMaxComp * 81];
static __device__ __align__(256) cd g_noalloc_mel[kNoAllocMaxElems * 81];
static __device__ __align__(256) int g_noalloc_bad[1];   // pattern-mismatch counter of the last call

namespace {
struct NoAllocPtrs {
  cd *kel = nullptr, *mel = nullptr;
  int *bad = nullptr;
  bool ready = false;
};
constexpr int kMaxDevices = 64;
NoAllocPtrs g_ptrs[kMaxDevices];
std::mutex g_mu;

// Host code must not use the arrays' names as device addresses: resolve them
// once per device, with that device current, on the first call there.  The
// addresses are kept for the life of the process (a cudaDeviceReset of the
// device would make them stale; the header tells callers not to do that).
int noalloc_setup(int dev, NoAllocPtrs &out) {
  std::lock_guard<std::mutex> lk(g_mu);
  NoAllocPtrs &p = g_ptrs[dev];
  if (!p.ready) {
    if (cudaGetSymbolAddress((void **)&p.kel, g_noalloc_kel) != cudaSuccess) return SS_ECUDA;
    if (cudaGetSymbolAddress((void **)&p.mel, g_noalloc_mel) != cudaSuccess) return SS_ECUDA;
    if (cudaGetSymbolAddress((void **)&p.bad, g_noalloc_bad) != cudaSuccess) return SS_ECUDA;
    p.ready = true;
  }
  out = p;
  return SS_OK;
}
}  // namespace

// Add one batch of element matrices into K/M (component-major Q9 CSR layout).
// Atomic adds: the result matches the ordered gather of ss_assemble to
// rounding, but the summation order of shared slots is not fixed.
__global__ void noalloc_scatter_kernel(int64_t nbatch, int nc, int ndisp, int64_t N, const int64_t *__restrict__ conn,
                                       const int64_t *__restrict__ indptr, const int64_t *__restrict__ nadj_ptr,
                                       const int64_t *__restrict__ nadj, const cd *__restrict__ Kel,
                                       const cd *__restrict__ Mel, double *__restrict__ K, double *__restrict__ M,
                                       int *bad) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbatch * 81) return;
  const int64_t e = t / 81;
  const int loc = (int)(t % 81), li = loc / 9, lj = loc % 9;
  const int64_t i = conn[e * 9 + li], j = conn[e * 9 + lj];
  int64_t lo = nadj_ptr[i], hi = nadj_ptr[i + 1], b = lo, en = hi;
  while (b < en) {
    const int64_t mid = (b + en) / 2;
    if (nadj[mid] < j) b = mid + 1; else en = mid;
  }
  if (b == hi || nadj[b] != j) {
    atomicAdd(bad, 1);
    return;
  }
  const int64_t r = b - lo, d = hi - lo;
  for (int A = 0; A < nc; ++A)
    for (int B = 0; B < nc; ++B) {
      const int64_t slot = indptr[(int64_t)A * N + i] + (int64_t)B * d + r;
      const cd v = Kel[(e * nc * nc + A * nc + B) * 81 + loc];
      atomicAdd(&K[2 * slot], v.x);
      atomicAdd(&K[2 * slot + 1], v.y);
      if (M && A == B && A < ndisp) {
        const cd mv = Mel[e * 81 + loc];
        atomicAdd(&M[2 * slot], mv.x);
        atomicAdd(&M[2 * slot + 1], mv.y);
      }
    }
}

}  // namespace ss

using namespace ss;

extern "C" int ss_assemble_q9_noalloc(int ndisp, int64_t n_nodes, const double *pos, int64_t n_elem,
                                      const int64_t *conn, const int32_t *elem_mat, const double *rho, const double *C,
                                      const double *e, const double *eps, int n_regions, const int32_t *elem_region,
                                      const int32_t *pml_axis, const double *pml_dmax, const int32_t *pml_npow,
                                      const double *pml_inner, const double *pml_outer, double omega_top,
                                      const int64_t *indptr, const int64_t *nadj_ptr, const int64_t *nadj,
                                      int64_t nnz, double *K, double *M, void *stream) {
  if (ndisp != 2 && ndisp != 3) return SS_EINVAL;
  if (n_nodes <= 0 || n_elem <= 0 || nnz <= 0) return SS_EINVAL;
  if (!pos || !conn || !elem_mat || !rho || !C || !e || !eps || !indptr || !nadj_ptr || !nadj || !K || !M)
    return SS_EINVAL;
  if (n_regions < 0 || (n_regions > 0 && (!elem_region || !pml_axis || !pml_dmax || !pml_npow || !pml_inner ||
                                          !pml_outer || !(omega_top > 0.0))))
    return SS_EINVAL;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SS_ECUDA;
  NoAllocPtrs sp;
  if (noalloc_setup(dev, sp) != SS_OK) return SS_ECUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nc = ndisp + 1;
  if (cudaMemsetAsync(K, 0, (size_t)nnz * 2 * sizeof(double), s) != cudaSuccess) return SS_ECUDA;
  if (cudaMemsetAsync(M, 0, (size_t)nnz * 2 * sizeof(double), s) != cudaSuccess) return SS_ECUDA;
  if (cudaMemsetAsync(sp.bad, 0, sizeof(int), s) != cudaSuccess) return SS_ECUDA;
  PmlDev pml{};
  pml.clip = 1;
  pml.omega = omega_top;
  if (n_regions > 0) {
    pml.axis = pml_axis;
    pml.npow = pml_npow;
    pml.dmax = pml_dmax;
    pml.inner = pml_inner;
    pml.outer = pml_outer;
  }
  // element batches in ascending element order; the scratch is reused per batch
  for (int64_t e0 = 0; e0 < n_elem; e0 += kNoAllocMaxElems) {
    const int64_t nb = std::min<int64_t>(kNoAllocMaxElems, n_elem - e0);
    pml.elem_region = n_regions > 0 ? elem_region + e0 : nullptr;
    if (launch_q9_elements(s, nb, nc, pos, conn + e0 * 9, elem_mat + e0, rho, C, e, eps, pml, sp.kel, sp.mel) !=
        cudaSuccess)
      return SS_ECUDA;
    noalloc_scatter_kernel<<<(unsigned)((nb * 81 + 255) / 256), 256, 0, s>>>(
        nb, nc, ndisp, n_nodes, conn + e0 * 9, indptr, nadj_ptr, nadj, sp.kel, sp.mel, K, M, sp.bad);
    if (cudaGetLastError() != cudaSuccess) return SS_ECUDA;
  }
  int bad = 0;
  if (cudaMemcpyAsync(&bad, sp.bad, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return SS_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return SS_ECUDA;
  return bad ? SS_EINVAL : SS_OK;
}
