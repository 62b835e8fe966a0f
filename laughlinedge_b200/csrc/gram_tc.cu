// S/H contraction on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// For every tile job (A panel of 128 V rows, B panel of 32 V rows, walker
// split) the kernel accumulates
//   D[r][h*32 + c] = sum_w V[row0+r][w] * W_h(w) * V[col0+c][w],   h = 0,1,2
// with W_0 = w1, W_1 = w1 sum|z|^2, W_2 = w1 sum|z|^4: one M=128 x N=96 MMA
// produces the S, H2 and H4 blocks at once.  Complex Gram entries are
// recovered from the real products of the [Re; Im] row planes afterwards.
//
// Precision: each FP32 operand x is split x = hi + lo with hi = bf16(x),
// lo = bf16(x - hi) (kind::f16) or hi = x truncated to TF32, lo = x - hi
// (kind::tf32).  The products hi*hi + hi*lo + lo*hi (+ lo*lo) accumulate in
// FP32 in tensor memory, hi*hi in one accumulator and the (2^-8 smaller)
// correction products in a second one, so the FP32 rounding of the corrections
// does not reach the result; every `flush_every` K-chunks the epilogue warps
// move both accumulators into an FP64 tile in shared memory (double-buffered
// TMEM so the MMAs continue meanwhile); at the end the FP64 tile is added to
// the job's private FP64 slot in global memory.
//
// Warp roles (288 threads): warps 0-3 producers (global FP32 -> split
// operands, 128B-swizzled K-major shared memory), warps 4-7 epilogue (TMEM
// lane quarter = warp % 4), warp 8 allocates TMEM and one lane issues the
// MMAs.  Every mbarrier wait is bounded in time; on expiry the kernel records
// LEMC_ERR_TIMEOUT in the error word and unwinds.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "lemc_internal.h"

namespace lemc {
namespace {

constexpr int kM = 128;            // A panel rows (MMA M)
constexpr int kNB = 32;            // B panel rows per weight
constexpr int kN = 3 * kNB;        // MMA N
constexpr int kRowBytes = 128;     // one swizzle-128B row = one K-chunk
constexpr int kATileBytes = kM * kRowBytes;   // 16 KB
constexpr int kBTileBytes = kN * kRowBytes;   // 12 KB
constexpr int kStageBytes = 2 * kATileBytes + 2 * kBTileBytes;  // hi + lo
constexpr int kStages = 2;
constexpr int kAccLd = kN + 1;     // FP64 accumulator row stride (doubles)
constexpr int kThreads = 288;
constexpr int kTmemCols = 512;     // two buffers x (hi*hi accumulator, correction accumulator)
constexpr int kBufCols = 256;      // buffer b: hi*hi at b*256, corrections at b*256 + 128
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz

struct Smem {
  // operand stages first (1024-byte aligned by construction)
  uint8_t stage[kStages][kStageBytes];
  double acc[kM * kAccLd];
  uint64_t full[kStages];
  uint64_t empty[kStages];
  uint64_t tfull[2];
  uint64_t tempty[2];
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

// Bounded wait; returns false (and raises the CTA abort flag and the global
// error word) when the phase does not complete in time or another role gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, Smem* sm, int* err) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (*(volatile int*)&sm->abort_flag) return false;
    if (clock64() - t0 > kWaitCycles) {
      *(volatile int*)&sm->abort_flag = 1;
      if (err) atomicExch(err, LEMC_ERR_TIMEOUT);
      return false;
    }
  }
  return true;
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), version 1 (sm_100).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFF);
  d |= uint64_t(1) << 16;                 // LBO (unused for swizzled K-major)
  d |= uint64_t((1024 >> 4) & 0x3FFF) << 32;  // SBO
  d |= uint64_t(1) << 46;                 // descriptor version
  d |= uint64_t(2) << 61;                 // SWIZZLE_128B
  return d;
}

// Instruction descriptor: dense, FP32 accumulate, A/B K-major, M=128, N=96.
__host__ __device__ constexpr uint32_t make_idesc(uint32_t ab_format) {
  return (1u << 4) | (ab_format << 7) | (ab_format << 10) | (uint32_t(kN >> 3) << 17) |
         (uint32_t(kM >> 4) << 24);
}

template <bool TF32>
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                    uint32_t accumulate) {
  if (TF32) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
  }
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

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// byte offset of 16-byte chunk `c` of row `r` in a 128B-swizzled K-major tile
__device__ __forceinline__ uint32_t sw128_off(int r, int c) {
  return uint32_t((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4));
}

// split 8 consecutive FP32 values into bf16 hi and lo 16-byte chunks
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

// split 4 FP32 values into TF32 hi (truncated) and FP32 lo = x - hi
__device__ __forceinline__ void split_tf32x4(const float* x, uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t hb = __float_as_uint(x[q]) & 0xFFFFE000u;
    h[q] = hb;
    l[q] = __float_as_uint(x[q] - __uint_as_float(hb));
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

struct TcArgs {
  const float* V;
  int ldv;
  int total_rows;
  const float* rec_w;
  int W;
  const TcTile* tiles;
  double* partials;
  int n_chunks_total;   // K-chunks over the padded walker range
  int n_splits;
  int flush_every;
  int passes;           // 3 or 4
  int* err;
};

template <bool TF32>
__global__ void __launch_bounds__(kThreads, 1) gram_tc_kernel(const TcArgs a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // align the Smem struct to 1024 bytes for the swizzle atoms
  Smem* sm = reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));

  constexpr int KC = TF32 ? 32 : 64;          // samples per K-chunk (one 128-byte row)
  constexpr int EPC = TF32 ? 4 : 8;           // elements per 16-byte chunk
  constexpr int KSTEP_BYTES = 32;             // one MMA consumes 32 bytes of K
  constexpr int NKSTEP = kRowBytes / KSTEP_BYTES;
  constexpr uint32_t IDESC = make_idesc(TF32 ? 2u : 1u);

  const TcTile tile = a.tiles[blockIdx.x];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int per = (a.n_chunks_total + a.n_splits - 1) / a.n_splits;
  const int c_beg = tile.ksplit * per;
  const int c_end = min(a.n_chunks_total, c_beg + per);
  const int nch = max(0, c_end - c_beg);
  const int F = a.flush_every;
  const int nint = (nch + F - 1) / F;  // accumulation intervals

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&sm->full[s], 128);
      mbar_init(&sm->empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sm->tfull[b], 1);
      mbar_init(&sm->tempty[b], 128);
    }
    mbar_init(&sm->done, 1);
    sm->abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 8) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&sm->tmem_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (warp >= 4 && warp < 8) {
    for (int i = threadIdx.x - 128; i < kM * kAccLd; i += 128) sm->acc[i] = 0.0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm->tmem_base;

  if (warp < 4) {
    // ------------------------------ producers ------------------------------
    const int t = threadIdx.x;
    for (int c = 0; c < nch; ++c) {
      const int s = c % kStages;
      const uint32_t ph = uint32_t(c / kStages) & 1u;
      if (!mbar_wait(&sm->empty[s], ph ^ 1u, sm, a.err)) break;
      uint8_t* st = sm->stage[s];
      uint8_t* a_hi = st;
      uint8_t* a_lo = st + kATileBytes;
      uint8_t* b_hi = st + 2 * kATileBytes;
      uint8_t* b_lo = st + 2 * kATileBytes + kBTileBytes;
      const int k0 = (c_beg + c) * KC;
      // A: 128 rows x 8 chunks, unweighted
#pragma unroll 2
      for (int q = 0; q < 8; ++q) {
        const int id = q * 128 + t;
        const int r = id >> 3, ch = id & 7;
        const int row = tile.row0 + r;
        float x[EPC];
        if (row < a.total_rows) {
          const float4* src = reinterpret_cast<const float4*>(a.V + (size_t)row * a.ldv + k0 + ch * EPC);
#pragma unroll
          for (int v = 0; v < EPC / 4; ++v) {
            const float4 f = __ldg(src + v);
            x[4 * v] = f.x; x[4 * v + 1] = f.y; x[4 * v + 2] = f.z; x[4 * v + 3] = f.w;
          }
        } else {
#pragma unroll
          for (int e = 0; e < EPC; ++e) x[e] = 0.f;
        }
        uint4 hi, lo;
        if (TF32) split_tf32x4(x, hi, lo); else split_bf16x8(x, hi, lo);
        const uint32_t off = sw128_off(r, ch);
        *reinterpret_cast<uint4*>(a_hi + off) = hi;
        *reinterpret_cast<uint4*>(a_lo + off) = lo;
      }
      // B: 32 rows x 8 chunks, three weight planes
#pragma unroll 1
      for (int q = 0; q < 2; ++q) {
        const int id = q * 128 + t;
        const int r = id >> 3, ch = id & 7;
        const int row = tile.col0 + r;
        float x[EPC], w0[EPC], w1[EPC], w2[EPC];
        const int kk = k0 + ch * EPC;
#pragma unroll
        for (int e = 0; e < EPC; ++e) {
          const int wi = kk + e;
          const bool ok = (wi < a.W);
          const float one = ok ? __ldg(a.rec_w + (size_t)LEMC_W_ONE * a.W + wi) : 0.f;
          w0[e] = one;
          w1[e] = ok ? one * __ldg(a.rec_w + (size_t)LEMC_W_R2 * a.W + wi) : 0.f;
          w2[e] = ok ? one * __ldg(a.rec_w + (size_t)LEMC_W_R4 * a.W + wi) : 0.f;
        }
        if (row < a.total_rows) {
          const float4* src = reinterpret_cast<const float4*>(a.V + (size_t)row * a.ldv + kk);
#pragma unroll
          for (int v = 0; v < EPC / 4; ++v) {
            const float4 f = __ldg(src + v);
            x[4 * v] = f.x; x[4 * v + 1] = f.y; x[4 * v + 2] = f.z; x[4 * v + 3] = f.w;
          }
        } else {
#pragma unroll
          for (int e = 0; e < EPC; ++e) x[e] = 0.f;
        }
#pragma unroll
        for (int h = 0; h < 3; ++h) {
          float y[EPC];
#pragma unroll
          for (int e = 0; e < EPC; ++e) y[e] = x[e] * (h == 0 ? w0[e] : (h == 1 ? w1[e] : w2[e]));
          uint4 hi, lo;
          if (TF32) split_tf32x4(y, hi, lo); else split_bf16x8(y, hi, lo);
          const uint32_t off = sw128_off(h * kNB + r, ch);
          *reinterpret_cast<uint4*>(b_hi + off) = hi;
          *reinterpret_cast<uint4*>(b_lo + off) = lo;
        }
      }
      fence_async_smem();
      mbar_arrive(&sm->full[s]);
    }
  } else if (warp < 8) {
    // ------------------------------ epilogue -------------------------------
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    for (int q = 0; q < nint; ++q) {
      const int b = q & 1;
      if (!mbar_wait(&sm->tfull[b], uint32_t(q >> 1) & 1u, sm, a.err)) break;
      tc_fence_after();
#pragma unroll 1
      for (int cc = 0; cc < kN / 32; ++cc) {
        float v[32], u[32];
        const uint32_t ta = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(b * kBufCols + cc * 32);
        tmem_ld32(ta, v);
        tmem_ld32(ta + 128, u);
        double* dst = sm->acc + row * kAccLd + cc * 32;
#pragma unroll
        for (int i = 0; i < 32; ++i) dst[i] += double(v[i]) + double(u[i]);
      }
      tc_fence_before();
      mbar_arrive(&sm->tempty[b]);
    }
  } else if (lane == 0) {
    // ------------------------------ MMA issuer -----------------------------
    bool ok = true;
    for (int c = 0; c < nch && ok; ++c) {
      const int s = c % kStages;
      const int q = c / F;
      const int b = q & 1;
      if (c % F == 0) {
        // the epilogue must have drained this accumulator buffer
        if (!mbar_wait(&sm->tempty[b], (uint32_t(q >> 1) & 1u) ^ 1u, sm, a.err)) { ok = false; break; }
        tc_fence_after();
      }
      if (!mbar_wait(&sm->full[s], uint32_t(c / kStages) & 1u, sm, a.err)) { ok = false; break; }
      tc_fence_after();
      const uint32_t base = smem_u32(sm->stage[s]);
      const uint32_t ahi = base, alo = base + kATileBytes;
      const uint32_t bhi = base + 2 * kATileBytes, blo = bhi + kBTileBytes;
      const uint32_t d = tmem + uint32_t(b * kBufCols);   // hi*hi
      const uint32_t dc = d + 128u;                          // corrections
#pragma unroll
      for (int ks = 0; ks < NKSTEP; ++ks) {
        const uint32_t o = ks * KSTEP_BYTES;
        const uint32_t first = (c % F == 0 && ks == 0) ? 0u : 1u;
        mma<TF32>(d, sw128_desc(ahi + o), sw128_desc(bhi + o), IDESC, first);
        mma<TF32>(dc, sw128_desc(ahi + o), sw128_desc(blo + o), IDESC, first);
        mma<TF32>(dc, sw128_desc(alo + o), sw128_desc(bhi + o), IDESC, 1u);
        if (a.passes > 3) mma<TF32>(dc, sw128_desc(alo + o), sw128_desc(blo + o), IDESC, 1u);
      }
      umma_commit(&sm->empty[s]);
      if (c % F == F - 1 || c == nch - 1) umma_commit(&sm->tfull[b]);
    }
    if (nch > 0) {
      // all issued MMAs must retire before TMEM is released
      umma_commit(&sm->done);
      mbar_wait(&sm->done, 0u, sm, a.err);
    }
  }

  __syncthreads();
  // epilogue warps add the FP64 tile to the job's private slot
  if (warp >= 4 && warp < 8 && !sm->abort_flag) {
    double* slot = a.partials + (size_t)tile.slot * (kM * kN);
    for (int i = threadIdx.x - 128; i < kM * kN; i += 128) {
      const int r = i / kN, cidx = i % kN;
      slot[i] += sm->acc[r * kAccLd + cidx];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 8) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
}

// Fold the partial slots into the per-sector complex Gram planes:
//   G_h[a][b] += sum_splits [C(re a, re b) + C(im a, im b)]
//              + i [C(re a, im b) - C(im a, re b)]
__global__ void gram_tc_reduce_kernel(const double* __restrict__ partials,
                                      const int* __restrict__ tile_of, int n_pi, int n_pj,
                                      int n_tiles, int n_splits, const int32_t* __restrict__ sec_row,
                                      const int32_t* __restrict__ sec_dim,
                                      const int32_t* __restrict__ sec_goff, int n_sec,
                                      double* __restrict__ gram, size_t plane) {
  const int s = blockIdx.y;
  if (s >= n_sec) return;
  const int D = sec_dim[s];
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= D * D) return;
  const int a = idx / D, b = idx % D;
  const int r0 = sec_row[s];
  auto C = [&](int r1, int r2, int h) {
    const int t = tile_of[(r1 / kM) * n_pj + (r2 / kNB)];
    double v = 0.0;
    if (t < 0) return v;
    for (int sp = 0; sp < n_splits; ++sp) {
      const double* slot = partials + (size_t)(sp * n_tiles + t) * (kM * kN);
      v += slot[(r1 % kM) * kN + h * kNB + (r2 % kNB)];
    }
    return v;
  };
  const int ra = r0 + a, ia = r0 + D + a, rb = r0 + b, ib = r0 + D + b;
  for (int h = 0; h < 3; ++h) {
    const double re = C(ra, rb, h) + C(ia, ib, h);
    const double im = C(ra, ib, h) - C(ia, rb, h);
    const size_t o = 2 * ((size_t)sec_goff[s] + (size_t)a * D + b) + 2 * plane * h;
    gram[o] += re;
    gram[o + 1] += im;
  }
}

}  // namespace

int launch_gram_tc_rows(const float* V, int ldv, int total_rows, const float* rec_w, int W,
                        int Wpad, const TcTile* tiles, int n_jobs, int n_splits, double* partials,
                        int mode, int flush_every, int* err, cudaStream_t st) {
  if (mode != LEMC_GRAM_BF16X3 && mode != LEMC_GRAM_BF16X4 && mode != LEMC_GRAM_TF32X3)
    return LEMC_ERR_ARG;
  if (ldv % 64 != 0 || Wpad % 64 != 0 || n_jobs <= 0 || Wpad > ldv) return LEMC_ERR_ARG;
  if (reinterpret_cast<uintptr_t>(V) % 16 != 0) return LEMC_ERR_ARG;
  const bool tf32 = (mode == LEMC_GRAM_TF32X3);
  const int KC = tf32 ? 32 : 64;
  TcArgs a;
  a.V = V;
  a.ldv = ldv;
  a.total_rows = total_rows;
  a.rec_w = rec_w;
  a.W = W;
  a.tiles = tiles;
  a.partials = partials;
  a.n_chunks_total = Wpad / KC;
  a.n_splits = n_splits;
  // TF32 hi/lo reaches ~1e-6 only with a flush per K-chunk; the BF16 split is
  // limited by its 16-bit representation, so a longer FP32 interval costs nothing
  a.flush_every = flush_every > 0 ? flush_every : (tf32 ? 1 : 4);
  a.passes = (mode == LEMC_GRAM_BF16X4) ? 4 : 3;
  a.err = err;
  const size_t smem = sizeof(Smem) + 1024;
  if (tf32) {
    if (cudaFuncSetAttribute(gram_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem)) != cudaSuccess)
      return LEMC_ERR_CUDA;
    gram_tc_kernel<true><<<n_jobs, kThreads, smem, st>>>(a);
  } else {
    if (cudaFuncSetAttribute(gram_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem)) != cudaSuccess)
      return LEMC_ERR_CUDA;
    gram_tc_kernel<false><<<n_jobs, kThreads, smem, st>>>(a);
  }
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

int launch_gram_tc_reduce(const double* partials, const int* tile_of, int n_pi, int n_pj,
                          int n_tiles, int n_splits, const int32_t* sec_row,
                          const int32_t* sec_dim, const int32_t* sec_goff, int n_sec,
                          int max_dim, double* gram, size_t plane, cudaStream_t st) {
  dim3 grid((max_dim * max_dim + 255) / 256, n_sec);
  gram_tc_reduce_kernel<<<grid, 256, 0, st>>>(partials, tile_of, n_pi, n_pj, n_tiles, n_splits,
                                              sec_row, sec_dim, sec_goff, n_sec, gram, plane);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

size_t gram_tc_smem_bytes() { return sizeof(Smem) + 1024; }

}  // namespace lemc
