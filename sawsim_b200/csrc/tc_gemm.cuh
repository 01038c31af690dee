// Complex64 front updates C -= A B on the 5th-generation tensor cores (sm_100a):
// tcgen05.mma kind::tf32 with FP32 accumulators in tensor memory, operands
// brought into 128-byte-swizzled shared memory by the Tensor Memory Accelerator
// (cp.async.bulk.tensor), one elected thread issuing the MMAs, completion
// tracked by mbarriers (tcgen05.commit, complete_tx).
//
// Complex product as one real GEMM.  A (rows x k complex, row-major, re/im
// interleaved) is read as a real K-major matrix A_il (rows x 2k).  B (k x n
// complex) becomes the real K-major operand B' (2n rows of 2k): row 2c holds
// (Br, -Bi) and row 2c+1 holds (Bi, Br) at real K positions (2j, 2j+1).  Then
// C_il = A_il B'^T is C in interleaved form: column 2c = Re(AB), 2c+1 = Im(AB).
// The flops equal the complex count.
//
// FP32 accuracy from TF32 inputs (3xTF32): every operand value v is split as
// v = hi + lo with hi = v rounded to TF32 and lo = v - hi (exact in FP32); the
// accumulator receives hi*hi + hi*lo + lo*hi.  The dropped lo*lo term and the
// truncation of lo to TF32 are at the 2^-22 relative level, the FP32 rounding
// level of the SIMT kernel this competes with.
//
// Two kernels per level:
//  * pack_kernel writes, once per level and frequency, the split operands of
//    every front in the exact shape of an MMA operand tile: rows of 128 bytes
//    (16 complex of K), K chunk by K chunk, A rows and B' rows padded to
//    multiples of 128 with zeros (A_hi, A_lo, B'_hi, B'_lo);
//  * tma_gemm_kernel, persistent and warp-specialised (one CTA per SM): warp 0
//    streams the packed tiles with TMA into a ring of shared-memory stages (the
//    tensor map's 128-byte swizzle is the layout the MMA descriptors expect),
//    warp 1 issues 12 MMAs per K chunk into one of two TMEM accumulators, warps
//    2-9 drain the other accumulator into C (two warps per TMEM lane quarter,
//    each half of the columns: TMEM -> registers -> a padded per-warp shared
//    tile -> coalesced read-modify-write rows of C with all 32 rows of a column
//    block loaded before any is stored), so one tile's epilogue overlaps the
//    next tile's loads and MMAs.
// Every mbarrier wait is bounded (kWaitNs); on time-out the CTA records the
// error, every role leaves its loop, the producer waits (bounded) for the
// copies it issued, the MMA warp waits on one final commit that tracks all of
// its MMAs (its own bound) and only then is the tensor memory freed.  The
// tensor map covers this GPU's own staging buffer; no load is multicast.
#pragma once
#include <cstdint>
#include <cuda.h>
#include "dev_complex.cuh"

namespace ss {

// One output tile of C -= A B inside front f: rows [r0, rhi), cols [c0, chi),
// contraction [kk0, kk1); A = F[:, kk], B = F[kk, :] (F = the front, row-major, ld).
struct GemmTask {
  int f, r0, c0, rhi, chi, kk0, kk1;
};

namespace tc {

constexpr int BM = 128;              // complex rows per tile (MMA M)
constexpr int KCH = 16;              // complex K per chunk (32 fp32 = one 128-byte row)
constexpr int ROWB = 128;            // bytes per packed row
constexpr int PADC = 128;            // packed A rows and B' columns: multiples of 128
constexpr uint64_t kWaitNs = 200000000ull;   // 0.2 s bound on any mbarrier wait

// Packed operands of one front at one level, in rows of 128 bytes counted from
// the frequency's block of the staging buffer: with kc K chunks, au padded A
// rows and bu padded B columns (complex),
//   A_hi chunk c row r     base + c au + r
//   A_lo chunk c row r     base + (kc + c) au + r
//   B'_hi chunk c row q    base + 2 kc au + 2 c bu + q        (q < 2 bu)
//   B'_lo chunk c row q    base + 2 kc au + 2 (kc + c) bu + q
// 2 kc (au + 2 bu) rows in all.
struct PackFront {
  int64_t base;
  int f, kc, au, bu;
};
__host__ __device__ inline int64_t pack_rows(int kc, int au, int bu) { return 2 * (int64_t)kc * (au + 2 * (int64_t)bu); }

// One output tile of the TMA kernel: rows [r0, rhi) and columns [c0, chi) of
// front f (front coordinates, r0, c0 >= k), with the front's packed operands
// (base, kc, au, bu) and the tile's offsets into them: A row ra = r0 - k, B'
// row cb = 2 (c0 - k).
struct TmaTask {
  int64_t base;
  int f, r0, c0, rhi, chi, kc, au, bu, ra, cb;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// tf32 round-to-nearest (ties away) of an fp32 value, low 13 mantissa bits zero
__device__ __forceinline__ float tf32_hi(float v) {
  uint32_t u = __float_as_uint(v);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
  return __uint_as_float(u);
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3fff);          // start address
  d |= (uint64_t)1 << 16;                          // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;                // stride byte offset
  d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                          // 128-byte swizzle
  return d;
}

// instruction descriptor: kind::tf32, FP32 accumulate, K-major A and B, M = 128, N real columns
__host__ __device__ constexpr uint32_t idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

template <uint32_t IDESC>
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(IDESC), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar) : "memory");
}

// the producer's arrival on a stage's full barrier, announcing `bytes` of copies
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(bar),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait for the mbarrier phase with parity `parity` to complete (at most
// kWaitNs of wall time); false on time-out
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = global_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (global_ns() - t0 > kWaitNs) return false;
  }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 2D tiled TMA load of one box (32 fp32 x 128 rows) at (x, y) into shared memory,
// completing on the mbarrier `bar`
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *tmap, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

// 32 consecutive fp32 columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------------------
// Pack: one CTA per (front, K chunk, frequency).  A rows are copied straight
// (a row of the chunk is 16 complex = 128 contiguous bytes of the front row);
// B' rows are built from 16 x 64 complex blocks of U12 staged in shared memory
// (rows padded to 65 complex: the column-wise reads hit 32 distinct banks).
constexpr int PACK_THREADS = 256;

__global__ void __launch_bounds__(PACK_THREADS) pack_kernel(const cf *__restrict__ arena, int64_t stride,
                                                            const int64_t *__restrict__ off, const int *__restrict__ ldv,
                                                            const int *__restrict__ kv, const int *__restrict__ mv,
                                                            const PackFront *__restrict__ fronts,
                                                            const int2 *__restrict__ items, float *__restrict__ stage,
                                                            int64_t stage_rows) {
  __shared__ float2 T[KCH][65];
  const int2 it = items[blockIdx.x];
  const PackFront P = fronts[it.x];
  const int c = it.y, fq = blockIdx.y;
  const int f = P.f, k = kv[f], m = mv[f], ld = ldv[f], u = m - k;
  const cf *F = arena + (int64_t)fq * stride + off[f];
  float *S = stage + ((int64_t)fq * stage_rows + P.base) * 32;
  float *Ahi = S + (int64_t)c * P.au * 32, *Alo = S + (int64_t)(P.kc + c) * P.au * 32;
  const int j0 = KCH * c;
  for (int t = threadIdx.x; t < P.au * 32; t += PACK_THREADS) {
    const int r = t >> 5, q = t & 31, j = j0 + (q >> 1);
    float v = 0.f;
    if (r < u && j < k) {
      const cf a = F[(int64_t)(k + r) * ld + j];
      v = (q & 1) ? a.y : a.x;
    }
    const float hi = tf32_hi(v);
    Ahi[t] = hi;
    Alo[t] = v - hi;
  }
  float *Bhi = S + (2 * (int64_t)P.kc * P.au + 2 * (int64_t)c * P.bu) * 32;
  float *Blo = S + (2 * (int64_t)P.kc * P.au + 2 * (int64_t)(P.kc + c) * P.bu) * 32;
  for (int cc0 = 0; cc0 < P.bu; cc0 += 64) {
    // U12 rows j0 .. j0 + 15, columns k + cc0 .. + 63 (zero outside the front)
    for (int t = threadIdx.x; t < KCH * 64; t += PACK_THREADS) {
      const int jj = t >> 6, cc = t & 63, j = j0 + jj, col = cc0 + cc;
      float2 b = make_float2(0.f, 0.f);
      if (j < k && col < u) {
        const cf x = F[(int64_t)j * ld + k + col];
        b = make_float2(x.x, x.y);
      }
      T[jj][cc] = b;
    }
    __syncthreads();
    // 128 packed rows (2 per column) x 32 fp32: row 2cc = (Br, -Bi), row 2cc+1 = (Bi, Br)
    for (int t = threadIdx.x; t < 128 * 32; t += PACK_THREADS) {
      const int qr = t >> 5, p = t & 31, cc = qr >> 1, s = qr & 1, jj = p >> 1, e = p & 1;
      const float2 b = T[jj][cc];
      const float v = s == 0 ? (e == 0 ? b.x : -b.y) : (e == 0 ? b.y : b.x);
      const float hi = tf32_hi(v);
      const int64_t o = (int64_t)(2 * cc0 + qr) * 32 + p;
      Bhi[o] = hi;
      Blo[o] = v - hi;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Persistent TMA + tcgen05 GEMM.  BNC complex columns per tile (MMA N = 2 BNC
// real), STG shared-memory stages.
template <int BNC, int STG>
struct TmaCfg {
  static constexpr int NR = 2 * BNC;                      // real MMA N
  static constexpr int A_BYTES = BM * ROWB;               // one A operand (hi or lo) of a chunk
  static constexpr int B_BYTES = NR * ROWB;               // one B' operand of a chunk
  static constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES; // A hi, A lo, B' hi, B' lo
  static constexpr int EPI_WARPS = 8;                     // two per TMEM lane quarter
  static constexpr int EPI_FLOATS = 32 * 33;              // per epilogue warp: 32 rows x 33 fp32
  static constexpr int SMEM = STG * STAGE + EPI_WARPS * EPI_FLOATS * 4;
  static constexpr int TMEM_COLS = 2 * NR;                // two accumulators
  static constexpr int THREADS = 64 + 32 * EPI_WARPS;     // producer, MMA, epilogue warps
  static constexpr uint32_t IDESC = idesc_tf32(NR);
  static_assert(NR % 128 == 0 && NR <= 256, "B' loads are 128-row boxes; N <= 256");
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

template <int BNC, int STG>
__global__ void __launch_bounds__(TmaCfg<BNC, STG>::THREADS, 1)
    tma_gemm_kernel(const __grid_constant__ CUtensorMap tmap, cf *__restrict__ arena, int64_t stride,
                    const int64_t *__restrict__ off, const int *__restrict__ ldv, const TmaTask *__restrict__ tasks,
                    int ntasks, int nb, int64_t stage_rows, int *__restrict__ err) {
  using Cfg = TmaCfg<BNC, STG>;
  constexpr int NR = Cfg::NR;
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  __shared__ __align__(8) uint64_t full[STG], empty[STG], acc_full[2], acc_empty[2], drain;
  __shared__ uint32_t tmem_base_s;
  __shared__ volatile int abort_s;
  // the 128-byte-swizzled stages need 1024-byte alignment, which the declaration
  // gives; a base that lacked it would be reported, not used
  unsigned char *smem = tc_smem_raw;
  float *epi = reinterpret_cast<float *>(smem + STG * Cfg::STAGE);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n_items = (int64_t)ntasks * nb;
  if (threadIdx.x == 0) {
    abort_s = *reinterpret_cast<volatile int *>(err);
    if (smem_u32(smem) & 1023u) {
      abort_s = 1;
      atomicExch(err, 1);
    }
    for (int s = 0; s < STG; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(smem_u32(&acc_full[a]), 1);
      mbar_init(smem_u32(&acc_empty[a]), 32 * Cfg::EPI_WARPS);
    }
    mbar_init(smem_u32(&drain), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmap)) : "memory");
  }
  __syncthreads();
  if (abort_s) return;      // an earlier launch timed out: do nothing (uniform)
  if (wid == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(Cfg::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;

  if (wid == 0) {
    // ---------------- TMA producer (one lane): A hi/lo and B' hi/lo of each K chunk
    if (lane == 0) {
      int64_t gc = 0;
      for (int64_t it = blockIdx.x; it < n_items && !abort_s; it += gridDim.x) {
        const TmaTask tk = tasks[it % ntasks];
        const int64_t fb = (it / ntasks) * stage_rows + tk.base;   // this frequency's packed front
        const int64_t bofs = fb + 2 * (int64_t)tk.kc * tk.au;
        for (int c = 0; c < tk.kc; ++c) {
          const int s = (int)(gc % STG);
          if (gc >= STG && !mbar_wait(smem_u32(&empty[s]), (uint32_t)(((gc / STG) - 1) & 1))) {
            abort_s = 1;
            break;
          }
          const uint32_t st = smem_u32(smem + s * Cfg::STAGE), bar = smem_u32(&full[s]);
          mbar_expect_tx(bar, (uint32_t)Cfg::STAGE);
          tma_load_2d(st, &tmap, bar, 0, (int)(fb + (int64_t)c * tk.au + tk.ra));
          tma_load_2d(st + Cfg::A_BYTES, &tmap, bar, 0, (int)(fb + (int64_t)(tk.kc + c) * tk.au + tk.ra));
#pragma unroll
          for (int h = 0; h < NR / 128; ++h) {
            tma_load_2d(st + 2 * Cfg::A_BYTES + h * 128 * ROWB, &tmap, bar, 0,
                        (int)(bofs + 2 * (int64_t)c * tk.bu + tk.cb + 128 * h));
            tma_load_2d(st + 2 * Cfg::A_BYTES + Cfg::B_BYTES + h * 128 * ROWB, &tmap, bar, 0,
                        (int)(bofs + 2 * (int64_t)(tk.kc + c) * tk.bu + tk.cb + 128 * h));
          }
          ++gc;
        }
      }
      // no copy may still be writing shared memory when the CTA ends: wait
      // (bounded) for the full barriers of the last chunks issued
      for (int64_t g = gc - 1; g >= 0 && g >= gc - STG; --g)
        if (!mbar_wait(smem_u32(&full[g % STG]), (uint32_t)((g / STG) & 1))) abort_s = 1;
    }
    __syncwarp();
  } else if (wid == 1) {
    // ---------------- MMA issuer (one lane)
    if (lane == 0) {
      int64_t gc = 0, ac = 0;
      bool issued = false;
      for (int64_t it = blockIdx.x; it < n_items && !abort_s; it += gridDim.x) {
        const TmaTask tk = tasks[it % ntasks];
        const int a = (int)(ac & 1);
        if (ac >= 2 && !mbar_wait(smem_u32(&acc_empty[a]), (uint32_t)(((ac / 2) - 1) & 1))) {
          abort_s = 1;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(a * NR);
        bool ok = true;
        for (int c = 0; c < tk.kc; ++c) {
          const int s = (int)(gc % STG);
          if (!mbar_wait(smem_u32(&full[s]), (uint32_t)((gc / STG) & 1))) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t base = smem_u32(smem + s * Cfg::STAGE);
          const uint32_t ahi = base, alo = base + Cfg::A_BYTES, bhi = base + 2 * Cfg::A_BYTES,
                         blo = base + 2 * Cfg::A_BYTES + Cfg::B_BYTES;
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {   // K = 8 fp32 = 32 bytes per MMA
            const uint32_t ko = 32u * ks;
            mma_tf32<Cfg::IDESC>(d, sw128_desc(ahi + ko), sw128_desc(bhi + ko), (c > 0 || ks > 0) ? 1u : 0u);
            mma_tf32<Cfg::IDESC>(d, sw128_desc(ahi + ko), sw128_desc(blo + ko), 1u);
            mma_tf32<Cfg::IDESC>(d, sw128_desc(alo + ko), sw128_desc(bhi + ko), 1u);
          }
          mma_commit(smem_u32(&empty[s]));
          issued = true;
          ++gc;
        }
        if (!ok) {
          abort_s = 1;
          break;
        }
        mma_commit(smem_u32(&acc_full[a]));
        ++ac;
      }
      // every MMA of this CTA complete before the tensor memory is freed: one
      // final commit tracks all of them (its own bound, apart from the handoffs)
      if (issued) {
        mma_commit(smem_u32(&drain));
        if (!mbar_wait(smem_u32(&drain), 0u)) abort_s = 1;
      }
    }
    __syncwarp();
  } else {
    // ---------------- epilogue warps 2-9: TMEM lane quarter q = warp % 4, column
    // blocks of 32 fp32 with parity h = (warp - 2) / 4
    const int q = wid & 3, h = (wid - 2) >> 2;
    float *stg = epi + (wid - 2) * Cfg::EPI_FLOATS;
    int64_t ac = 0;
    for (int64_t it = blockIdx.x; it < n_items; it += gridDim.x) {
      if (__any_sync(0xffffffffu, abort_s != 0)) break;      // warp-uniform (tcgen05.ld is .sync.aligned)
      const TmaTask tk = tasks[it % ntasks];
      const int fq = (int)(it / ntasks);
      const int ld = ldv[tk.f];
      float *F = reinterpret_cast<float *>(arena + (int64_t)fq * stride + off[tk.f]);
      const int a = (int)(ac & 1);
      const bool ok = mbar_wait(smem_u32(&acc_full[a]), (uint32_t)((ac / 2) & 1));
      if (__any_sync(0xffffffffu, !ok)) {
        abort_s = 1;
        break;
      }
      tc_fence_after();
      const int rbase = tk.r0 + 32 * q;
      const int nrow = min(32, tk.rhi - rbase);                // rows of this quarter inside the tile
#pragma unroll 1
      for (int blk = h; blk < NR / 32; blk += 2) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(a * NR + 32 * blk), v);
#pragma unroll
        for (int i = 0; i < 32; ++i) stg[lane * 33 + i] = v[i];
        __syncwarp();
        // rows of the block: 32 consecutive fp32 (16 complex columns) each; every
        // row's load is issued before any store
        const int c = tk.c0 + 16 * blk + (lane >> 1);
        if (nrow > 0 && c < tk.chi) {
          float *p0 = F + 2 * ((int64_t)rbase * ld + tk.c0 + 16 * blk) + lane;
          const int64_t rs = 2 * (int64_t)ld;
          float cur[32];
#pragma unroll
          for (int rr = 0; rr < 32; ++rr) cur[rr] = rr < nrow ? p0[rr * rs] : 0.f;
#pragma unroll
          for (int rr = 0; rr < 32; ++rr)
            if (rr < nrow) p0[rr * rs] = cur[rr] - stg[rr * 33 + lane];
        }
        __syncwarp();
      }
      tc_fence_before();
      mbar_arrive(smem_u32(&acc_empty[a]));
      ++ac;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && abort_s) atomicExch(err, 1);   // after every role has finished
  if (wid == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::TMEM_COLS) : "memory");
  }
}

}  // namespace tc
}  // namespace ss
