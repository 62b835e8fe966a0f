// S/H contraction on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// For every tile job (A panel of 128 V rows, B panel of 32 V rows, walker
// split) the kernel accumulates
//   D[r][h*32 + c] = sum_w V[a0+r][w] * W_h(w) * V[b0+c][w],   h = 0,1,2
// with W_0 = w1, W_1 = w1 sum|z|^2, W_2 = w1 sum|z|^4: one M=128 x N=96 MMA
// produces the S, H2 and H4 blocks at once.  Complex Gram entries are
// recovered from the real products of the [Re; Im] row planes afterwards.
//
// Precision: each FP32 operand x is split x = hi + lo with hi = bf16(x),
// lo = bf16(x - hi) (kind::f16) or hi = tf32_rn(x), lo = tf32_rn(x - hi)
// (kind::tf32).  Each accumulator buffer holds 192 FP32 columns: hi*hi in the
// first 96 and the correction products hi*lo + lo*hi (+ lo*lo) in the next 96.
// One M=128 x N=192 MMA multiplies A_hi by the stacked [B_hi; B_lo] operand
// (both products at once) and one N=96 MMA adds A_lo * B_hi to the
// corrections.  A tcgen05.mma of kind::tf32 with K=8 costs about 97 cycles for
// any N up to 128 and 106 cycles at N=192 (measured on B200), so this takes
// 203 cycles per K step where three N=96 MMAs took 290.  The tensor core's
// accumulation truncates (a relative bias of about -4e-8 per MMA step), so
// every `flush_every` K-chunks the epilogue warps move both halves of the
// buffer out of tensor memory into FP32 register sums (round-to-nearest; two
// buffers let the MMAs continue meanwhile).  At the end each job adds its
// sums, in FP64, to its private slot in global memory.
//
// Operand placement.  The A operand (hi and lo, 128 rows x one K-chunk) lives
// in tensor memory: the A converters write it with tcgen05.st and the MMAs
// read it from there, so shared memory only carries the raw TMA stages and
// the (weighted, split) B operand.
//
// Pipeline (608 threads, one CTA per SM):
//   warp 17      loader: tiled TMA loads per K-chunk (A panel 128 x KC in
//                128-byte-swizzled boxes of 32 samples, B panel 32 x KC,
//                weight planes 3 x KC; rows past the end are zero-filled by
//                the TMA unit) into a ring of raw FP32 stages;
//   warps 8-11   A converters: thread = A row (TMEM lane); raw FP32 -> hi/lo,
//                stored to the tensor-memory A stage with tcgen05.st;
//   warps 12-15  B converters: raw FP32 -> weighted, split hi/lo B operands in
//                128-byte-swizzled K-major shared-memory layout;
//   warp 16      allocates 512 TMEM columns, one lane issues tcgen05.mma;
//   warp 18      scheduler: makes the issuer's barrier waits and hands each
//                K-chunk to it through a named barrier;
// (Doubling the converter warps to 864 threads held the kernel to 72
// registers and ran slower: 0.321 against 0.266 ms at the mixed-precision
// workload.)
//   warps 0-7    epilogue: TMEM lane quarter = warp % 4, column half =
//                warp / 4, 48 FP32 accumulators per thread.
// Tensor memory columns: accumulator buffers at 0 and 192 (hi*hi at +0,
// corrections at +96), A stages at 384 and 448 (hi at +0, lo at +32).
// No load uses cluster multicast; every source is this GPU's own memory.
// Every mbarrier wait is bounded in time; on expiry the kernel records
// LEMC_ERR_TIMEOUT in the error word, skips its output and unwinds: the loader
// first waits (bounded) for the TMA copies it has in flight and the issuer for
// the MMAs it has committed, then the CTA frees its tensor memory and exits.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "lemc_internal.h"

namespace lemc {
namespace {

constexpr int kM = 128;            // A panel rows (MMA M)
constexpr int kNB = 32;            // B panel rows per weight
constexpr int kN = 3 * kNB;        // MMA N
constexpr int kOpRowBytes = 128;   // one swizzle-128B row of split operands
constexpr int kBTileBytes = kN * kOpRowBytes;  // 12 KB
constexpr int kOpStages = 2;
constexpr int kEpiWarps = 8;
constexpr int kAConvWarp0 = 8;     // warps 8-11: A converters (lane quarter = warp % 4)
constexpr int kBConvWarp0 = 12;    // warps 12-15: B converters
constexpr int kBConvThreads = 4 * 32;
constexpr int kConvThreads = 8 * 32;
constexpr int kEpiCols = kN / (kEpiWarps / 4);  // accumulator columns per epilogue thread
constexpr int kMmaWarp = 16;
constexpr int kLoadWarp = 17;
constexpr int kSchedWarp = 18;     // does the issuer's barrier waits (see the MMA issuer)
constexpr int kThreads = 19 * 32;
constexpr int kTmemCols = 512;
constexpr uint32_t kColBuf = 0;    // accumulator buffers at 0 and 192 (hi*hi +0, corrections +96)
constexpr uint32_t kBufCols = 2 * kN;
constexpr uint32_t kColA = 384;    // A stages at 384 + 64 s (hi +0, lo +32)
static_assert(2 * kBufCols <= kColA, "accumulator buffers overlap the A stages");
constexpr long long kWaitCycles = 4000000000LL;  // default wait bound, ~2 s at 1.9 GHz

template <bool TF32>
struct Cfg {
  static constexpr int KC = TF32 ? 32 : 64;           // samples per K-chunk
  static constexpr int RAW_ROW = KC * 4;              // bytes of one raw FP32 row segment
  static constexpr int A_BOXES = KC / 32;             // 128-byte-wide swizzled A boxes
  static constexpr int A_BYTES = kM * RAW_ROW;        // raw A (all boxes)
  static constexpr int B_BYTES = kNB * RAW_ROW;
  static constexpr int W_BYTES = 3 * KC * 4;
  static constexpr int RAW_STAGE = A_BYTES + B_BYTES + 1024;  // weights padded to 1 KB
  static constexpr int RAW_STAGES = TF32 ? 6 : 3;
};

template <bool TF32>
struct Smem {
  uint8_t raw[Cfg<TF32>::RAW_STAGES][Cfg<TF32>::RAW_STAGE];  // 1024-aligned stages
  uint8_t bop[kOpStages][2 * kBTileBytes];                    // B hi | B lo
  uint64_t raw_full[Cfg<TF32>::RAW_STAGES];
  uint64_t raw_empty[Cfg<TF32>::RAW_STAGES];
  uint64_t op_full[kOpStages];
  uint64_t op_empty[kOpStages];
  uint64_t acc_full[2];
  uint64_t acc_empty[2];
  uint64_t done;
  uint32_t tmem_base;
  int abort_flag;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// CTA named barriers (0 is __syncthreads), 64 threads each: ids 1/2 hand
// K-chunk c (by parity) from the scheduler warp to the MMA warp ("ready"),
// ids 3/4 return it ("issued"), so neither warp can run two chunks ahead of
// the other and every barrier completes with exactly 32 + 32 threads.
__device__ __forceinline__ void named_arrive(int id) {
  asm volatile("bar.arrive %0, 64;" ::"r"(id) : "memory");
}
__device__ __forceinline__ void named_sync(int id) {
  asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait; returns false (raising the CTA abort flag and the global error
// word) when the phase does not complete within `limit` cycles or another
// role gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* abort_flag, int* err,
                                          long long limit) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (*(volatile int*)abort_flag) return false;
    if (clock64() - t0 > limit) {
      *(volatile int*)abort_flag = 1;
      if (err) atomicExch(err, LEMC_ERR_TIMEOUT);
      return false;
    }
  }
  return true;
}

// Bounded wait for this CTA's own asynchronous work (its TMA copies, its
// committed MMAs) that does not give up when another role aborted: those
// operations complete by themselves, and the CTA must not release shared or
// tensor memory while they are in flight.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity, int* err, long long limit) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (clock64() - t0 > limit) {
      if (err) atomicExch(err, LEMC_ERR_TIMEOUT);
      return;
    }
  }
}

// Tiled 2D TMA load (no multicast) completing on an mbarrier transaction count.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), LBO 1 (unused for swizzled K-major), version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFF);
  d |= uint64_t(1) << 16;
  d |= uint64_t((1024 >> 4) & 0x3FFF) << 32;
  d |= uint64_t(1) << 46;
  d |= uint64_t(2) << 61;
  return d;
}

// Instruction descriptor: dense, FP32 accumulate, A/B K-major, M=128, N=n.
__host__ __device__ constexpr uint32_t make_idesc(uint32_t ab_format, int n) {
  return (1u << 4) | (ab_format << 7) | (ab_format << 10) | (uint32_t(n >> 3) << 17) |
         (uint32_t(kM >> 4) << 24);
}

// D (TMEM) += A (TMEM, 128 lanes x K) * B (shared memory descriptor)
template <bool TF32>
__device__ __forceinline__ void mma_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  if (TF32) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(tmem_d),
        "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(tmem_d),
        "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate));
  }
}

// 16 consecutive 32-bit columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t* r) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15])
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// byte offset of 16-byte chunk `c` of row `r` in a 128B-swizzled K-major tile
__device__ __forceinline__ uint32_t sw128_off(int r, int c) {
  return uint32_t((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4));
}

__device__ __forceinline__ void split_bf16x8(const float* x, uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const __nv_bfloat162 hb = __floats2bfloat162_rn(x[2 * q], x[2 * q + 1]);
    const float2 hf = __bfloat1622float2(hb);
    const __nv_bfloat162 lb = __floats2bfloat162_rn(x[2 * q] - hf.x, x[2 * q + 1] - hf.y);
    h[q] = *reinterpret_cast<const uint32_t*>(&hb);
    l[q] = *reinterpret_cast<const uint32_t*>(&lb);
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// x rounded to the nearest TF32 value (ties away from zero), as a 32-bit
// pattern whose 13 low mantissa bits are zero.  Adding half a TF32 ulp to the
// magnitude bits and truncating is that rounding for every finite x (a carry
// into the exponent is the correct round-up; overflow gives infinity) and
// runs as two integer ops at full ALU rate.
__device__ __forceinline__ uint32_t to_tf32_rn(float x) {
  return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u;
}

// hi = x rounded to nearest TF32, lo = (x - hi) rounded to nearest TF32: both
// roundings are unbiased (the tensor core would otherwise truncate the low 13
// bits of each operand, a systematic -2^-22 relative bias on every product).
__device__ __forceinline__ void split_tf32x4(const float* x, uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    h[q] = to_tf32_rn(x[q]);
    l[q] = to_tf32_rn(x[q] - __uint_as_float(h[q]));
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

struct TcArgs {
  const float* V;
  int ldv;
  int total_rows;
  const float* rec_w;   // weight planes, stride ldw (256-byte aligned rows)
  int ldw;
  const TcTile* tiles;
  double* partials;
  int n_chunks_total;   // K-chunks over the padded walker range
  int n_splits;
  int flush_every;
  int passes;           // 3 or 4
  int* err;
  long long wait_cycles;  // bound of every mbarrier wait
  int hold_loads;         // test hook: the loader issues nothing (the waits then expire)
};

template <bool TF32>
__global__ void __launch_bounds__(kThreads, 1)
gram_tc_kernel(const TcArgs a, const __grid_constant__ CUtensorMap tmA,
               const __grid_constant__ CUtensorMap tmB, const __grid_constant__ CUtensorMap tmW) {
  using C = Cfg<TF32>;
  constexpr int KC = C::KC;
  constexpr int EPC = TF32 ? 4 : 8;          // elements per 16-byte B operand chunk
  constexpr int NKSTEP = kOpRowBytes / 32;   // one MMA consumes 32 bytes of K
  constexpr uint32_t IDESC = make_idesc(TF32 ? 2u : 1u, kN);          // N=96
  constexpr uint32_t IDESC2 = make_idesc(TF32 ? 2u : 1u, 2 * kN);     // N=192: [B_hi; B_lo]
  constexpr int RS = C::RAW_STAGES;

  extern __shared__ __align__(1024) uint8_t smem_raw[];
  Smem<TF32>* sm = reinterpret_cast<Smem<TF32>*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));

  const TcTile tile = a.tiles[blockIdx.x];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int per = (a.n_chunks_total + a.n_splits - 1) / a.n_splits;
  const int c_beg = tile.ksplit * per;
  const int c_end = min(a.n_chunks_total, c_beg + per);
  const int nch = max(0, c_end - c_beg);
  const int F = a.flush_every;
  const int nint = (nch + F - 1) / F;

  if (threadIdx.x == 0) {
    for (int s = 0; s < RS; ++s) {
      mbar_init(&sm->raw_full[s], 1);
      mbar_init(&sm->raw_empty[s], kConvThreads);
    }
    for (int s = 0; s < kOpStages; ++s) {
      mbar_init(&sm->op_full[s], kConvThreads);
      mbar_init(&sm->op_empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sm->acc_full[b], 1);
      mbar_init(&sm->acc_empty[b], kEpiWarps * 32);
    }
    mbar_init(&sm->done, 1);
    sm->abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&sm->tmem_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm->tmem_base;
  int* abort_flag = &sm->abort_flag;

  if (warp == kLoadWarp) {
    // ------------------------------- loader --------------------------------
    if (lane == 0) {
      const uint32_t tx_bytes = uint32_t(C::A_BYTES + C::B_BYTES + C::W_BYTES);
      int issued = 0;
      for (int c = 0; c < nch && !a.hold_loads; ++c) {
        const int s = c % RS;
        if (!mbar_wait(&sm->raw_empty[s], (uint32_t(c / RS) & 1u) ^ 1u, abort_flag, a.err, a.wait_cycles)) break;
        const int k0 = (c_beg + c) * KC;
        uint8_t* dst = sm->raw[s];
        mbar_arrive_tx(&sm->raw_full[s], tx_bytes);
#pragma unroll
        for (int j = 0; j < C::A_BOXES; ++j)
          tma_load_2d(dst + j * (kM * 128), &tmA, k0 + 32 * j, tile.row0, &sm->raw_full[s]);
        tma_load_2d(dst + C::A_BYTES, &tmB, k0, tile.col0, &sm->raw_full[s]);
        tma_load_2d(dst + C::A_BYTES + C::B_BYTES, &tmW, k0, 0, &sm->raw_full[s]);
        ++issued;
      }
      // the copies still in flight land before the CTA may exit, whatever the
      // other roles did: the last one issued into each stage
      for (int c = max(0, issued - RS); c < issued; ++c)
        mbar_drain(&sm->raw_full[c % RS], uint32_t(c / RS) & 1u, a.err, a.wait_cycles);
    }
    __syncwarp();
  } else if (warp >= kAConvWarp0 && warp < kBConvWarp0) {
    // ---------------------------- A converters -----------------------------
    // Thread = A row r = TMEM lane; its raw row segment sits in 128-byte
    // swizzled boxes (16-byte chunk j of row r at r*128 + ((j ^ (r & 7)) << 4)).
    const int quarter = warp & 3;
    const int r = quarter * 32 + lane;
    const uint32_t lane_base = uint32_t(quarter * 32) << 16;
    for (int c = 0; c < nch; ++c) {
      const int rs = c % RS, os = c % kOpStages;
      if (!mbar_wait(&sm->raw_full[rs], uint32_t(c / RS) & 1u, abort_flag, a.err, a.wait_cycles)) break;
      if (!mbar_wait(&sm->op_empty[os], (uint32_t(c / kOpStages) & 1u) ^ 1u, abort_flag, a.err, a.wait_cycles)) break;
      tc_fence_after();
      const uint8_t* raw = sm->raw[rs];
      const uint32_t a_hi = tmem + lane_base + kColA + uint32_t(os * 64);
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        // 16 TMEM columns: TF32 -> 16 samples, BF16 -> 32 samples (2 per column)
        uint32_t hv[16], lv[16];
        if (TF32) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int j = half * 4 + q;
            const float4 f = *reinterpret_cast<const float4*>(raw + r * 128 + ((j ^ (r & 7)) << 4));
            const float x[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              hv[4 * q + e] = to_tf32_rn(x[e]);
              lv[4 * q + e] = to_tf32_rn(x[e] - __uint_as_float(hv[4 * q + e]));
            }
          }
        } else {
          const uint8_t* box = raw + half * (kM * 128);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const float4 f = *reinterpret_cast<const float4*>(box + r * 128 + ((q ^ (r & 7)) << 4));
            const float x[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const __nv_bfloat162 hb = __floats2bfloat162_rn(x[2 * e], x[2 * e + 1]);
              const float2 hf = __bfloat1622float2(hb);
              const __nv_bfloat162 lb = __floats2bfloat162_rn(x[2 * e] - hf.x, x[2 * e + 1] - hf.y);
              hv[2 * q + e] = *reinterpret_cast<const uint32_t*>(&hb);
              lv[2 * q + e] = *reinterpret_cast<const uint32_t*>(&lb);
            }
          }
        }
        tmem_st16(a_hi + half * 16, hv);
        tmem_st16(a_hi + 32 + half * 16, lv);
      }
      tmem_wait_st();
      tc_fence_before();
      mbar_arrive(&sm->op_full[os]);
      mbar_arrive(&sm->raw_empty[rs]);
    }
  } else if (warp >= kBConvWarp0 && warp < kBConvWarp0 + 4) {
    // ---------------------------- B converters -----------------------------
    const int t = threadIdx.x - kBConvWarp0 * 32;
    for (int c = 0; c < nch; ++c) {
      const int rs = c % RS, os = c % kOpStages;
      if (!mbar_wait(&sm->raw_full[rs], uint32_t(c / RS) & 1u, abort_flag, a.err, a.wait_cycles)) break;
      if (!mbar_wait(&sm->op_empty[os], (uint32_t(c / kOpStages) & 1u) ^ 1u, abort_flag, a.err, a.wait_cycles)) break;
      const uint8_t* rawb = sm->raw[rs] + C::A_BYTES;
      const float* rw = reinterpret_cast<const float*>(sm->raw[rs] + C::A_BYTES + C::B_BYTES);
      uint8_t* b_hi = sm->bop[os];
      uint8_t* b_lo = b_hi + kBTileBytes;
      // 32 rows x 8 operand chunks x 3 weight planes.  A thread's chunks share
      // one column range (ch = t % 8), so the weight products are formed once
      // per K-chunk and the independent chunks are interleaved.
      constexpr int kItems = (kNB * 8) / kBConvThreads;
      const int ch = t & 7;
      float ww[3][EPC];
#pragma unroll
      for (int e = 0; e < EPC; ++e) {
        const float one = rw[ch * EPC + e];
        ww[0][e] = one;
        ww[1][e] = one * rw[KC + ch * EPC + e];
        ww[2][e] = one * rw[2 * KC + ch * EPC + e];
      }
      float x[kItems][EPC];
#pragma unroll
      for (int q = 0; q < kItems; ++q) {
        const int rb = (q * kBConvThreads + t) >> 3;
        const float4* src = reinterpret_cast<const float4*>(rawb + rb * C::RAW_ROW + ch * EPC * 4);
#pragma unroll
        for (int v = 0; v < EPC / 4; ++v) {
          const float4 f = src[v];
          x[q][4 * v] = f.x; x[q][4 * v + 1] = f.y; x[q][4 * v + 2] = f.z; x[q][4 * v + 3] = f.w;
        }
      }
#pragma unroll
      for (int h = 0; h < 3; ++h) {
#pragma unroll
        for (int q = 0; q < kItems; ++q) {
          const int rb = (q * kBConvThreads + t) >> 3;
          float y[EPC];
#pragma unroll
          for (int e = 0; e < EPC; ++e) y[e] = x[q][e] * ww[h][e];
          uint4 hi, lo;
          if (TF32) split_tf32x4(y, hi, lo); else split_bf16x8(y, hi, lo);
          const uint32_t off = sw128_off(h * kNB + rb, ch);
          *reinterpret_cast<uint4*>(b_hi + off) = hi;
          *reinterpret_cast<uint4*>(b_lo + off) = lo;
        }
      }
      fence_async_smem();
      mbar_arrive(&sm->op_full[os]);
      mbar_arrive(&sm->raw_empty[rs]);
    }
  } else if (warp == kSchedWarp) {
    // ------------------------------ scheduler -------------------------------
    // An mbarrier test made by the thread that has just issued tcgen05.commit
    // stalls until the committed MMAs retire, which drains the tensor pipe every
    // K-chunk.  So this warp makes the issuer's waits (operand stage full;
    // hi*hi buffer empty at the start of a flush group) and hands each chunk
    // over through a named barrier, which needs no shared-memory access.  It
    // arrives once per chunk whatever happens (after an abort without
    // waiting), so the issuer's barrier always completes.
    int s = 0, b = 0, f = 0;
    uint32_t ph_op = 0, ph_acc = 0;
    for (int c = 0; c < nch; ++c) {
      if (c >= 2) named_sync(3 + (c & 1));  // chunk c-2 issued: ids 1/2 are free again
      if (lane == 0 && !*(volatile int*)abort_flag) {
        bool ok = true;
        if (f == 0) {
          ok = mbar_wait(&sm->acc_empty[b], ((ph_acc >> b) & 1u) ^ 1u, abort_flag, a.err, a.wait_cycles);
          ph_acc ^= 1u << b;
        }
        if (ok) mbar_wait(&sm->op_full[s], ph_op, abort_flag, a.err, a.wait_cycles);
      }
      __syncwarp();
      named_arrive(1 + (c & 1));
      if (++f == F || c == nch - 1) {
        f = 0;
        b ^= 1;
      }
      if (++s == kOpStages) {
        s = 0;
        ph_op ^= 1u;
      }
    }
    for (int c = max(0, nch - 2); c < nch; ++c) named_sync(3 + (c & 1));
  } else if (warp == kMmaWarp) {
    // ------------------------------ MMA issuer -----------------------------
    // One thread issues every MMA, so its per-MMA instruction count bounds the
    // tensor-core issue rate: all descriptors and TMEM addresses are formed
    // once per stage, a K step only adds a constant, and the flush schedule is
    // kept in counters.  Its waits are made by the scheduler warp.
    const bool four = a.passes > 3;
    static_assert(kOpStages == 2, "the issuer keeps one descriptor per operand stage");
    const uint64_t bdesc0 = sw128_desc(smem_u32(sm->bop[0]));
    const uint64_t bdesc1 = sw128_desc(smem_u32(sm->bop[1]));
    constexpr uint64_t kLoDesc = uint64_t(kBTileBytes >> 4);  // B lo tile, in descriptor units
    int s = 0, b = 0, f = 0;          // operand stage, hi*hi buffer, chunk within flush group
    int issued = 0;
    for (int c = 0; c < nch; ++c) {
      named_sync(1 + (c & 1));
      const bool go = !*(volatile int*)abort_flag;
      if (lane == 0 && go) {
        tc_fence_after();
        const uint64_t bh = s ? bdesc1 : bdesc0, bl = bh + kLoDesc;
        const uint32_t ahi = tmem + kColA + uint32_t(s * 64), alo = ahi + 32;
        const uint32_t d = tmem + kColBuf + uint32_t(b) * kBufCols;  // hi*hi | corrections
        const uint32_t dc = d + kN;
        // the first MMA of a flush group overwrites both halves of the buffer
        const uint32_t acc_d = f == 0 ? 0u : 1u;
        // K step ks: B advances 32 bytes (2 descriptor units), A 8 TMEM columns;
        // the B hi and lo tiles are contiguous, so bh with N=192 spans both
        mma_ts<TF32>(d, ahi, bh, IDESC2, acc_d);
        mma_ts<TF32>(dc, alo, bh, IDESC, 1u);
        if (four) mma_ts<TF32>(dc, alo, bl, IDESC, 1u);
#pragma unroll
        for (int ks = 1; ks < NKSTEP; ++ks) {
          mma_ts<TF32>(d, ahi + 8 * ks, bh + 2 * ks, IDESC2, 1u);
          mma_ts<TF32>(dc, alo + 8 * ks, bh + 2 * ks, IDESC, 1u);
          if (four) mma_ts<TF32>(dc, alo + 8 * ks, bl + 2 * ks, IDESC, 1u);
        }
        umma_commit(&sm->op_empty[s]);
        if (f + 1 == F || c == nch - 1) umma_commit(&sm->acc_full[b]);
        ++issued;
      }
      __syncwarp();
      named_arrive(3 + (c & 1));
      if (++f == F || c == nch - 1) {
        f = 0;
        b ^= 1;
      }
      if (++s == kOpStages) s = 0;
    }
    if (lane == 0 && issued > 0) {
      // every issued MMA must retire before TMEM is released
      umma_commit(&sm->done);
      mbar_drain(&sm->done, 0u, a.err, a.wait_cycles);
    }
    __syncwarp();
  } else if (warp < kEpiWarps) {
    // ------------------------------- epilogue ------------------------------
    const int quarter = warp & 3;
    const int part0 = (warp >> 2) * kEpiCols;  // first accumulator column of this thread
    // Plain FP32 running sums (round-to-nearest, unbiased): over n flushes the
    // relative rounding error is ~2^-24 sqrt(n) / 3 per split, and the FP64
    // sum over splits averages it down further.  Columns are read eight at a
    // time to stay within the register budget.
    float sum[kEpiCols];
#pragma unroll
    for (int i = 0; i < kEpiCols; ++i) sum[i] = 0.f;
    const uint32_t lane_base = uint32_t(quarter * 32) << 16;
    bool ok = true;
    for (int q = 0; q < nint; ++q) {
      const int b = q & 1;
      if (!mbar_wait(&sm->acc_full[b], uint32_t(q >> 1) & 1u, abort_flag, a.err, a.wait_cycles)) {
        ok = false;
        break;
      }
      tc_fence_after();
      // hi*hi column j and its correction column j + 96 belong to one sum
      const uint32_t ta = tmem + lane_base + kColBuf + uint32_t(b) * kBufCols + uint32_t(part0);
#pragma unroll
      for (int part = 0; part < kEpiCols / 8; ++part) {
        uint32_t v0[8], v1[8];
        tmem_ld8(ta + part * 8, v0);
        tmem_ld8(ta + kN + part * 8, v1);
        tmem_wait_ld();
        if (part == kEpiCols / 8 - 1) {
          // every column of this buffer is in registers: the MMAs may reuse it
          tc_fence_before();
          mbar_arrive(&sm->acc_empty[b]);
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          sum[part * 8 + i] += __uint_as_float(v0[i]);
          sum[part * 8 + i] += __uint_as_float(v1[i]);
        }
      }
    }
    if (ok && nch > 0) {
      if (!*(volatile int*)abort_flag) {
        double* slot = a.partials + (size_t)tile.slot * (kM * kN) +
                       (size_t)(quarter * 32 + lane) * kN + part0;
#pragma unroll
        for (int i = 0; i < kEpiCols; ++i) slot[i] += double(sum[i]);
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

// Fold the partial slots into the per-sector complex Gram planes:
//   G_h[a][b] += sum_splits [C(re a, re b) + C(im a, im b)]
//              + i [C(re a, im b) - C(im a, re b)]
// with C(r1, r2) read from the tile that covers A row r1 and B row r2, or
// from the tile of C(r2, r1) when that one was skipped by symmetry.  Each
// sector knows its tiles: first tile index, A/B row origins and the number
// of B panels (TcSector); A slice x of a sector holds B panels 4x .. nb-1.
__global__ void gram_tc_reduce_kernel(const double* __restrict__ partials,
                                      const TcTile* __restrict__ tiles,
                                      const TcSector* __restrict__ secs, int n_sec, int n_tiles,
                                      int n_splits, double* __restrict__ gram, size_t plane) {
  const int s = blockIdx.y;
  if (s >= n_sec) return;
  const TcSector sc = secs[s];
  const int D = sc.dim;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= D * D) return;
  const int a = idx / D, b = idx % D;
  auto C = [&](int r1, int r2, int h) {
    // A slice x holds B panels y >= 4 x only (the others are transposes)
    if ((r2 - sc.b_base) / kNB < 4 * ((r1 - sc.a_base) / kM)) {
      const int r = r1;
      r1 = r2;
      r2 = r;
    }
    const int x = (r1 - sc.a_base) / kM, y = (r2 - sc.b_base) / kNB;
    const int t = sc.tile0 + x * sc.n_bpanels - 2 * x * (x - 1) + (y - 4 * x);
    double v = 0.0;
    if (t < 0 || t >= n_tiles) return v;
    const TcTile tl = tiles[t];
    const int i = r1 - tl.row0, j = r2 - tl.col0;
    if (i < 0 || i >= kM || j < 0 || j >= kNB) return v;
    for (int sp = 0; sp < n_splits; ++sp) {
      const double* slot = partials + (size_t)(sp * n_tiles + t) * (kM * kN);
      v += slot[i * kN + h * kNB + j];
    }
    return v;
  };
  const int ra = sc.row + a, ia = sc.row + D + a, rb = sc.row + b, ib = sc.row + D + b;
  for (int h = 0; h < 3; ++h) {
    const double re = C(ra, rb, h) + C(ia, ib, h);
    const double im = C(ra, ib, h) - C(ia, rb, h);
    const size_t o = 2 * ((size_t)sc.goff + (size_t)a * D + b) + 2 * plane * h;
    gram[o] += re;
    gram[o + 1] += im;
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 2D FP32 map over a row-major [rows][ld] array, box = box_x samples x box_y rows,
// rows past `rows` read as zero; swizzle128 stores each 128-byte box row with
// its 16-byte chunks XOR-permuted by (row % 8) (box_x must then be 32).
bool make_map(CUtensorMap* m, const float* base, int ld, int rows, int box_x, int box_y,
              bool swizzle128) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {cuuint64_t(ld), cuuint64_t(rows)};
  const cuuint64_t strides[1] = {cuuint64_t(ld) * sizeof(float)};
  const cuuint32_t box[2] = {cuuint32_t(box_x), cuuint32_t(box_y)};
  const cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <bool TF32>
int launch_t(const TcArgs& a, int n_jobs, cudaStream_t st) {
  const size_t smem = sizeof(Smem<TF32>) + 1024;
  if (smem > 227 * 1024) return LEMC_ERR_CAPACITY;
  constexpr int KC = Cfg<TF32>::KC;
  CUtensorMap tmA, tmB, tmW;
  if (!make_map(&tmA, a.V, a.ldv, a.total_rows, 32, kM, true) ||
      !make_map(&tmB, a.V, a.ldv, a.total_rows, KC, kNB, false) ||
      !make_map(&tmW, a.rec_w, a.ldw, 3, KC, 3, false))
    return LEMC_ERR_CUDA;
  if (cudaFuncSetAttribute(gram_tc_kernel<TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(smem)) != cudaSuccess)
    return LEMC_ERR_CUDA;
  gram_tc_kernel<TF32><<<n_jobs, kThreads, smem, st>>>(a, tmA, tmB, tmW);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

// Host-side settings of the bounded waits (lemc_debug_gram_wait).
long long g_wait_cycles = kWaitCycles;
int g_hold_loads = 0;

}  // namespace

int set_gram_wait(long long cycles, int hold_loads) {
  if (cycles < 0) return LEMC_ERR_ARG;
  g_wait_cycles = cycles > 0 ? cycles : kWaitCycles;
  g_hold_loads = hold_loads != 0;
  return LEMC_OK;
}

int launch_gram_tc_rows(const float* V, int ldv, int total_rows, const float* rec_w, int ldw,
                        int Wpad, const TcTile* tiles, int n_jobs, int n_splits, double* partials,
                        int mode, int flush_every, int* err, cudaStream_t st) {
  if (mode != LEMC_GRAM_BF16X3 && mode != LEMC_GRAM_BF16X4 && mode != LEMC_GRAM_TF32X3)
    return LEMC_ERR_ARG;
  if (ldv % 64 != 0 || ldw % 64 != 0 || Wpad % 64 != 0 || n_jobs <= 0 || Wpad > ldv || Wpad > ldw)
    return LEMC_ERR_ARG;
  if (reinterpret_cast<uintptr_t>(V) % 256 != 0 || reinterpret_cast<uintptr_t>(rec_w) % 256 != 0)
    return LEMC_ERR_ARG;
  const bool tf32 = (mode == LEMC_GRAM_TF32X3);
  TcArgs a;
  a.V = V;
  a.ldv = ldv;
  a.total_rows = total_rows;
  a.rec_w = rec_w;
  a.ldw = ldw;
  a.tiles = tiles;
  a.partials = partials;
  a.n_chunks_total = Wpad / (tf32 ? Cfg<true>::KC : Cfg<false>::KC);
  a.n_splits = n_splits;
  // The tensor core's FP32 accumulation truncates: the relative bias grows by
  // ~4e-8 per MMA step into one accumulator, so TF32 hi/lo flushes every two
  // K-chunks (8 steps); the BF16 split is limited by its 16-bit representation,
  // so a longer interval costs nothing there
  a.flush_every = flush_every > 0 ? flush_every : (tf32 ? 2 : 4);
  a.passes = (mode == LEMC_GRAM_BF16X4) ? 4 : 3;
  a.err = err;
  a.wait_cycles = g_wait_cycles;
  a.hold_loads = g_hold_loads;
  return tf32 ? launch_t<true>(a, n_jobs, st) : launch_t<false>(a, n_jobs, st);
}

int launch_gram_tc_reduce(const double* partials, const TcTile* tiles, const TcSector* secs,
                          int n_sec, int n_tiles, int n_splits, int max_dim, double* gram,
                          size_t plane, cudaStream_t st) {
  dim3 grid((max_dim * max_dim + 255) / 256, n_sec);
  gram_tc_reduce_kernel<<<grid, 256, 0, st>>>(partials, tiles, secs, n_sec, n_tiles, n_splits,
                                              gram, plane);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

size_t gram_tc_smem_bytes(int mode) {
  return mode == LEMC_GRAM_TF32X3 ? sizeof(Smem<true>) + 1024 : sizeof(Smem<false>) + 1024;
}

}  // namespace lemc
