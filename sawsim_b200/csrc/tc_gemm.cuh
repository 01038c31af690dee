// Complex64 front updates C -= A B on the 5th-generation tensor cores (sm_100a):
// tcgen05.mma kind::tf32 with FP32 accumulators in tensor memory, operands
// staged in 128-byte-swizzled shared memory, one elected thread issuing the MMAs,
// completion tracked by an mbarrier (tcgen05.commit).
//
// Complex product as one real GEMM.  A (rows x k complex, row-major, re/im
// interleaved) is read as a real K-major matrix A_il (rows x 2k).  B (k x n
// complex) is expanded in shared memory into the real K-major operand B'
// (2n rows of 2k): row 2c holds (Br, -Bi) and row 2c+1 holds (Bi, Br) at real K
// positions (2j, 2j+1).  Then C_il = A_il B'^T is C in interleaved form:
// column 2c = Re(AB), 2c+1 = Im(AB).  The flops equal the complex count.
//
// FP32 accuracy from TF32 inputs (3xTF32): every operand value v is split as
// v = hi + lo with hi = v rounded to TF32 and lo = v - hi (exact in FP32); the
// accumulator receives hi*hi + hi*lo + lo*hi.  The dropped lo*lo term and the
// truncation of lo to TF32 are at the 2^-22 relative level, the FP32 rounding
// level of the SIMT kernel this replaces.
//
// Tile: 128 complex rows x 64 complex columns (M = 128, N = 128 real) per CTA,
// K in chunks of 16 complex (one 128-byte swizzle row of fp32).  Raw tiles
// stream in with cp.async three chunks deep (24 KB each); 256 threads convert
// each into the split, swizzled operands (2 stages of 64 KB: A hi/lo, B' hi/lo);
// thread 0 issues 12 MMAs of 128x128x8 per chunk.  Every mbarrier wait is bounded: on time-out the
// CTA records the error, drains its own MMAs (bounded), frees its tensor memory
// and returns without touching C.
#pragma once
#include <cstdint>
#include "dev_complex.cuh"

namespace ss {

// One output tile of C -= A B inside front f: rows [r0, rhi), cols [c0, chi),
// contraction [kk0, kk1); A = F[:, kk], B = F[kk, :] (F = the front, row-major, ld).
struct GemmTask {
  int f, r0, c0, rhi, chi, kk0, kk1;
};

namespace tc {

constexpr int BM = 128;              // complex rows per tile (MMA M)
constexpr int BN = 64;               // complex columns per tile (MMA N = 128 real)
constexpr int BKC = 16;              // complex K per chunk (32 fp32 = one 128-byte row)
constexpr int STAGES = 2;                             // operand stages (MMA side)
constexpr int RAW_STAGES = 3;                         // raw tile stages (cp.async side)
constexpr int THREADS = 256;
constexpr int OPER_BYTES = 128 * 128;                 // 128 rows x 128 bytes
constexpr int STAGE_BYTES = 4 * OPER_BYTES;           // A hi, A lo, B hi, B lo
constexpr int RAW_A_BYTES = BM * BKC * 8;             // 128 rows x 16 complex
constexpr int RAW_B_STRIDE = BN * 8 + 32;             // bytes per raw B row (+32: conflict-free reads)
constexpr int RAW_B_BYTES = BKC * RAW_B_STRIDE;       // 16 rows x 64 complex
constexpr int RAW_BYTES = RAW_A_BYTES + RAW_B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + RAW_STAGES * RAW_BYTES + 1024;   // + alignment slack
constexpr int TMEM_COLS = 128;
constexpr uint64_t kWaitNs = 200000000ull;           // 0.2 s bound on any mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// tf32 round-to-nearest (ties away) of an fp32 value, low 13 mantissa bits zero
__device__ __forceinline__ float tf32_hi(float v) {
  uint32_t u = __float_as_uint(v);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
  return __uint_as_float(u);
}

// asynchronous global -> shared copies; src_bytes < size zero-fills the rest
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void *src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

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

// instruction descriptor: kind::tf32, FP32 accumulate, K-major A and B, M=128, N=128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(128 >> 3) << 17) |
                            ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
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

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

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

// byte offset of 16-byte chunk q of row r in a 128-byte-swizzled K-major operand
__device__ __forceinline__ uint32_t sw_off(int r, int q) { return (uint32_t)(r * 128 + ((q ^ (r & 7)) << 4)); }

// Raw tiles of one K chunk into shared memory with cp.async: A 128 rows x 16
// complex (16-byte pieces: two complex, aligned because ld, the front offsets
// and the chunk start are even), B 16 rows x 64 complex (8-byte pieces: the
// column start k + 64 t may be odd).  Out-of-range pieces are zero-filled.
template <int NT = THREADS>
__device__ __forceinline__ void issue_chunk(unsigned char *raw, const cf *F, int ld, const GemmTask &tk, int kb) {
  const int t = threadIdx.x;
  const uint32_t ra = smem_u32(raw), rb = ra + RAW_A_BYTES;
#pragma unroll
  for (int i = 0; i < 1024 / NT; ++i) {
    const int idx = t + NT * i;             // 0..1023
    const int row = idx >> 3, q = idx & 7;  // q: pair of complex K columns
    const int r = tk.r0 + row, c = kb + 2 * q;
    const int valid = (r < tk.rhi) ? max(0, min(2, tk.kk1 - c)) : 0;
    const cf *src = valid ? F + (int64_t)r * ld + c : F;
    cp_async16(ra + (uint32_t)(row * 128 + q * 16), src, (uint32_t)(valid * 8));
  }
#pragma unroll
  for (int i = 0; i < 1024 / NT; ++i) {
    const int idx = t + NT * i;             // 0..1023
    const int j = idx >> 6, cc = idx & 63;  // complex k-row, complex column
    const int r = kb + j, c = tk.c0 + cc;
    const bool ok = r < tk.kk1 && c < tk.chi;
    cp_async8(rb + (uint32_t)(j * RAW_B_STRIDE + cc * 8), ok ? F + (int64_t)r * ld + c : F, ok ? 8u : 0u);
  }
}

// Raw tiles -> the four MMA operands (A hi/lo, B' hi/lo) in 128-byte swizzle.
template <int NT = THREADS>
__device__ __forceinline__ void convert_chunk(const unsigned char *raw, unsigned char *stage) {
  unsigned char *ahi = stage, *alo = stage + OPER_BYTES, *bhi = stage + 2 * OPER_BYTES, *blo = stage + 3 * OPER_BYTES;
  const int t = threadIdx.x;
  constexpr int NW = NT / 32;
#pragma unroll
  for (int i = 0; i < 1024 / NT; ++i) {
    const int idx = t + NT * i;
    const int row = idx >> 3, q = idx & 7;
    const float4 v = *reinterpret_cast<const float4 *>(raw + row * 128 + q * 16);
    const float4 h = make_float4(tf32_hi(v.x), tf32_hi(v.y), tf32_hi(v.z), tf32_hi(v.w));
    const float4 l = make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w);
    *reinterpret_cast<float4 *>(ahi + sw_off(row, q)) = h;
    *reinterpret_cast<float4 *>(alo + sw_off(row, q)) = l;
  }
  // B: a warp takes 8 k-rows x 4 columns per step, so that its stores cover every
  // (swizzle slot, half) pair of the rows 2cc / 2cc+1 twice (two wavefronts)
  const int lane = t & 31, wrp = t >> 5;
#pragma unroll
  for (int i = 0; i < 1024 / NT; ++i) {
    const int j = 8 * (i & 1) + (lane & 7);
    const int cc = 4 * (wrp + NW * (i >> 1)) + (lane >> 3);
    const float2 v = *reinterpret_cast<const float2 *>(raw + RAW_A_BYTES + j * RAW_B_STRIDE + cc * 8);
    const float hr = tf32_hi(v.x), hi = tf32_hi(v.y), nhi = tf32_hi(-v.y);
    const float lr = v.x - hr, li = v.y - hi, nli = -v.y - nhi;
    // real K positions (2j, 2j+1) = byte 8j of the row: chunk j/2, half j%2
    const uint32_t o0 = sw_off(2 * cc, j >> 1) + ((j & 1) << 3);
    const uint32_t o1 = sw_off(2 * cc + 1, j >> 1) + ((j & 1) << 3);
    *reinterpret_cast<float2 *>(bhi + o0) = make_float2(hr, nhi);
    *reinterpret_cast<float2 *>(bhi + o1) = make_float2(hi, hr);
    *reinterpret_cast<float2 *>(blo + o0) = make_float2(lr, nli);
    *reinterpret_cast<float2 *>(blo + o1) = make_float2(li, lr);
  }
}

// grid (tasks, frequencies); C -= A B for every task tile of every frequency
__global__ void __launch_bounds__(THREADS, 1)
    front_tc_gemm_kernel(cf *__restrict__ arena, int64_t stride, const int64_t *__restrict__ off,
                         const int *__restrict__ ldv, const GemmTask *__restrict__ tasks, int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  __shared__ __align__(8) uint64_t bars[STAGES + 1];
  __shared__ uint32_t tmem_base_s;
  __shared__ int abort_s;
  unsigned char *smem = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  const GemmTask tk = tasks[blockIdx.x];
  const int fq = blockIdx.y;
  const int ld = ldv[tk.f];
  cf *F = arena + (int64_t)fq * stride + off[tk.f];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = (tk.kk1 - tk.kk0 + BKC - 1) / BKC;
  if (nk <= 0) return;
  // an earlier tile timed out: the whole CTA does nothing (one read, shared)
  if (threadIdx.x == 0) abort_s = *reinterpret_cast<volatile int *>(err);
  __syncthreads();
  if (abort_s) return;
  __syncthreads();

  if (threadIdx.x == 0) {
    for (int s = 0; s <= STAGES; ++s) mbar_init(smem_u32(&bars[s]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (wid == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;

  unsigned char *raw0 = smem + STAGES * STAGE_BYTES;
  // prologue: the first RAW_STAGES - 1 chunks in flight
#pragma unroll
  for (int c = 0; c < RAW_STAGES - 1; ++c) {
    if (c < nk) issue_chunk(raw0 + c * RAW_BYTES, F, ld, tk, tk.kk0 + c * BKC);
    cp_async_commit();
  }
  bool ok = true;
  for (int kc = 0; kc < nk; ++kc) {
    const int s = kc % STAGES;
    unsigned char *stage = smem + s * STAGE_BYTES;
    // chunk kc + RAW_STAGES - 1 into the raw stage that held chunk kc - 1 (converted
    // in the previous iteration, before its closing barrier)
    const int cn = kc + RAW_STAGES - 1;
    if (cn < nk) issue_chunk(raw0 + (cn % RAW_STAGES) * RAW_BYTES, F, ld, tk, tk.kk0 + cn * BKC);
    cp_async_commit();
    cp_async_wait<RAW_STAGES - 1>();                 // this thread's pieces of chunk kc landed
    // the MMAs that read this operand stage two chunks ago must be complete
    if (kc >= STAGES) {
      if (!mbar_wait(smem_u32(&bars[s]), (uint32_t)((kc / STAGES - 1) & 1))) abort_s = 1;
    }
    __syncthreads();
    if (abort_s) {
      ok = false;
      break;
    }
    convert_chunk(raw0 + (kc % RAW_STAGES) * RAW_BYTES, stage);
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      const uint32_t base = smem_u32(stage);
      const uint32_t ahi = base, alo = base + OPER_BYTES, bhi = base + 2 * OPER_BYTES, blo = base + 3 * OPER_BYTES;
#pragma unroll
      for (int k = 0; k < 4; ++k) {   // K = 8 fp32 = 32 bytes per MMA
        const uint32_t ko = 32u * k;
        mma_tf32(tmem, sw128_desc(ahi + ko), sw128_desc(bhi + ko), (kc > 0 || k > 0) ? 1u : 0u);
        mma_tf32(tmem, sw128_desc(ahi + ko), sw128_desc(blo + ko), 1u);
        mma_tf32(tmem, sw128_desc(alo + ko), sw128_desc(bhi + ko), 1u);
      }
      mma_commit(smem_u32(&bars[s]));
    }
  }
  cp_async_wait<0>();                                // no copy outlives the CTA
  // all MMAs of this CTA complete (the last commit tracks every earlier MMA)
  if (threadIdx.x == 0) {
    if (ok) {
      mma_commit(smem_u32(&bars[STAGES]));
      if (!mbar_wait(smem_u32(&bars[STAGES]), 0u)) abort_s = 1;
    } else {
      // drain: the stages' last commits, bounded
      for (int kc = nk - 1; kc >= 0 && kc >= nk - STAGES; --kc)
        mbar_wait(smem_u32(&bars[kc % STAGES]), (uint32_t)((kc / STAGES) & 1));
    }
    if (abort_s) atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (!abort_s) {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +32 (tile rows) and real
    // columns 64 (w / 4) .. +64 (32 complex columns) into a padded row-major
    // staging tile in the (now idle) operand stages; then every warp updates
    // whole rows of C with coalesced loads and stores
    constexpr int SROW = BN * 8 + 8;                  // staging row stride (bytes)
    unsigned char *stg = smem;
    const int row = 32 * (wid & 3) + lane;
    const int cb = 32 * (wid >> 2);
    float v[32];
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const uint32_t taddr = tmem + ((uint32_t)(32 * (wid & 3)) << 16) + (uint32_t)(64 * (wid >> 2) + 32 * half);
      tmem_ld32(taddr, v);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        *reinterpret_cast<float2 *>(stg + row * SROW + (cb + 16 * half + j) * 8) = make_float2(v[2 * j], v[2 * j + 1]);
    }
    __syncthreads();
    for (int rr = wid; rr < BM; rr += THREADS / 32) {
      const int r = tk.r0 + rr;
      if (r >= tk.rhi) break;
      cf *crow = F + (int64_t)r * ld + tk.c0;
#pragma unroll
      for (int h2 = 0; h2 < 2; ++h2) {
        const int c = lane + 32 * h2;
        if (tk.c0 + c < tk.chi) {
          const float2 acc = *reinterpret_cast<const float2 *>(stg + rr * SROW + c * 8);
          cf d = crow[c];
          d.x -= acc.x;
          d.y -= acc.y;
          crow[c] = d;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (wid == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}


// ---------------------------------------------------------------------------
// Persistent, warp-specialised version: one CTA per SM walks the (tile,
// frequency) items of a launch.  Warps 0-3 stream and convert operands (the
// per-chunk pipeline above), warp 8 issues the MMAs, warps 4-7 drain the
// accumulator.  Two TMEM accumulators (2 x 128 columns) let one tile's epilogue
// overlap the next tile's loads and MMAs.  Handoffs are mbarriers:
//   op_full[s]   producers -> MMA   (stage s converted)
//   op_empty[s]  MMA -> producers   (tcgen05.commit: the MMAs reading s are done)
//   acc_full[a]  MMA -> epilogue    (tcgen05.commit after an item's last chunk)
//   acc_empty[a] epilogue -> MMA    (128 arrivals: accumulator a read out)
// Every wait is bounded; on time-out the CTA records the error and every role
// leaves its loop (bounded), the MMA role drains its commits, TMEM is freed.
constexpr int P_THREADS = 288;
constexpr int P_TMEM_COLS = 256;

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void producers_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }
// barrier of the 128 producer threads that also ORs a flag across them, so that a
// decision to stop is taken by all of them together
__device__ __forceinline__ bool producers_sync_or(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, 1, 128, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ int item_chunks(const GemmTask &tk) { return (tk.kk1 - tk.kk0 + BKC - 1) / BKC; }

__global__ void __launch_bounds__(P_THREADS, 1)
    front_tc_gemm_persistent(cf *__restrict__ arena, int64_t stride, const int64_t *__restrict__ off,
                             const int *__restrict__ ldv, const GemmTask *__restrict__ tasks, int ntasks, int nb,
                             int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  __shared__ __align__(8) uint64_t op_full[STAGES], op_empty[STAGES], acc_full[2], acc_empty[2], drain;
  __shared__ uint32_t tmem_base_s;
  __shared__ volatile int abort_s;
  unsigned char *smem = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  unsigned char *raw0 = smem + STAGES * STAGE_BYTES;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n_items = (int64_t)ntasks * nb;
  if (threadIdx.x == 0) {
    abort_s = *reinterpret_cast<volatile int *>(err);
    for (int s2 = 0; s2 < STAGES; ++s2) {
      mbar_init(smem_u32(&op_full[s2]), 1);
      mbar_init(smem_u32(&op_empty[s2]), 1);
    }
    for (int a2 = 0; a2 < 2; ++a2) {
      mbar_init(smem_u32(&acc_full[a2]), 1);
      mbar_init(smem_u32(&acc_empty[a2]), 128);
    }
    mbar_init(smem_u32(&drain), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (abort_s) return;
  if (wid == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(P_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;

  if (wid < 4) {
    // ---------------- producers: raw tiles by cp.async, conversion into the operand stages
    int64_t gc = 0;   // chunks converted by this CTA
    bool stop = false;
    for (int64_t it = blockIdx.x; it < n_items && !stop; it += gridDim.x) {
      const GemmTask tk = tasks[it % ntasks];
      const int fq = (int)(it / ntasks);
      const int ld = ldv[tk.f];
      const cf *F = arena + (int64_t)fq * stride + off[tk.f];
      const int nk = item_chunks(tk);
      for (int c = 0; c < RAW_STAGES - 1; ++c) {
        if (c < nk) issue_chunk<128>(raw0 + c * RAW_BYTES, F, ld, tk, tk.kk0 + c * BKC);
        cp_async_commit();
      }
      for (int kc = 0; kc < nk; ++kc) {
        const int cn = kc + RAW_STAGES - 1;
        if (cn < nk) issue_chunk<128>(raw0 + (cn % RAW_STAGES) * RAW_BYTES, F, ld, tk, tk.kk0 + cn * BKC);
        cp_async_commit();
        cp_async_wait<RAW_STAGES - 1>();
        const int s2 = (int)(gc % STAGES);
        bool late = gc >= STAGES && !mbar_wait(smem_u32(&op_empty[s2]), (uint32_t)(((gc / STAGES) - 1) & 1));
        // chunk kc in shared memory and stage s2 free, or every producer stops
        if (producers_sync_or(late || abort_s)) {
          abort_s = 1;
          stop = true;
          break;
        }
        convert_chunk<128>(raw0 + (kc % RAW_STAGES) * RAW_BYTES, smem + s2 * STAGE_BYTES);
        fence_async_smem();
        producers_sync();
        if (threadIdx.x == 0) mbar_arrive(smem_u32(&op_full[s2]));
        ++gc;
      }
      cp_async_wait<0>();
      // raw stages free before the next item's prologue; stop together
      if (producers_sync_or(stop || abort_s)) stop = true;
    }
    cp_async_wait<0>();
  } else if (wid == 8) {
    // ---------------- MMA issuer (one lane)
    if (lane == 0) {
      int64_t gc = 0, ac = 0;
      bool issued = false;
      for (int64_t it = blockIdx.x; it < n_items && !abort_s; it += gridDim.x) {
        const GemmTask tk = tasks[it % ntasks];
        const int nk = item_chunks(tk);
        if (nk <= 0) continue;
        const int a2 = (int)(ac & 1);
        if (ac >= 2 && !mbar_wait(smem_u32(&acc_empty[a2]), (uint32_t)(((ac / 2) - 1) & 1))) {
          abort_s = 1;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(a2 * 128);
        for (int kc = 0; kc < nk; ++kc) {
          const int s2 = (int)(gc % STAGES);
          if (!mbar_wait(smem_u32(&op_full[s2]), (uint32_t)((gc / STAGES) & 1))) {
            abort_s = 1;
            break;
          }
          tc_fence_after();
          const uint32_t base = smem_u32(smem + s2 * STAGE_BYTES);
          const uint32_t ahi = base, alo = base + OPER_BYTES, bhi = base + 2 * OPER_BYTES, blo = base + 3 * OPER_BYTES;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const uint32_t ko = 32u * k;
            mma_tf32(d, sw128_desc(ahi + ko), sw128_desc(bhi + ko), (kc > 0 || k > 0) ? 1u : 0u);
            mma_tf32(d, sw128_desc(ahi + ko), sw128_desc(blo + ko), 1u);
            mma_tf32(d, sw128_desc(alo + ko), sw128_desc(bhi + ko), 1u);
          }
          mma_commit(smem_u32(&op_empty[s2]));
          issued = true;
          ++gc;
        }
        if (abort_s) break;
        mma_commit(smem_u32(&acc_full[a2]));
        ++ac;
      }
      if (issued) {   // every MMA of this CTA complete before TMEM is freed
        mma_commit(smem_u32(&drain));
        if (!mbar_wait(smem_u32(&drain), 0u)) abort_s = 1;
      }
    }
    __syncwarp();
  } else {
    // ---------------- epilogue warps 4-7: TMEM lanes 32 (wid - 4) .. +32, all 128 columns
    const int q = wid - 4;
    const int row = 32 * q + lane;
    int64_t ac = 0;
    for (int64_t it = blockIdx.x; it < n_items; it += gridDim.x) {
      if (__any_sync(0xffffffffu, abort_s != 0)) break;     // warp-uniform (tcgen05.ld is .sync.aligned)
      const GemmTask tk = tasks[it % ntasks];
      if (item_chunks(tk) <= 0) continue;
      const int fq = (int)(it / ntasks);
      const int ld = ldv[tk.f];
      cf *F = arena + (int64_t)fq * stride + off[tk.f];
      const int a2 = (int)(ac & 1);
      const bool ok = mbar_wait(smem_u32(&acc_full[a2]), (uint32_t)((ac / 2) & 1));
      if (__any_sync(0xffffffffu, !ok)) {
        abort_s = 1;
        break;
      }
      tc_fence_after();
      const int r = tk.r0 + row;
      float v[32];
#pragma unroll
      for (int cb = 0; cb < 4; ++cb) {
        const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(a2 * 128 + 32 * cb);
        tmem_ld32(taddr, v);
        if (r < tk.rhi) {
          cf *crow = F + (int64_t)r * ld;
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int c = tk.c0 + 16 * cb + j;
            if (c < tk.chi) {
              cf dv = crow[c];
              dv.x -= v[2 * j];
              dv.y -= v[2 * j + 1];
              crow[c] = dv;
            }
          }
        }
      }
      tc_fence_before();
      mbar_arrive(smem_u32(&acc_empty[a2]));
      ++ac;
    }
  }
  if (abort_s && threadIdx.x == 0) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  if (wid == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P_TMEM_COLS) : "memory");
  }
}

}  // namespace tc
}  // namespace ss
