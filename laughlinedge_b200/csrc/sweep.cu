// Metropolis sweep over |P_guide Psi_m|^2 on sm_100a.
//
// Target density (z in units of l_B):
//   |Psi_m|^2 = prod_{i<j} |z_i - z_j|^{2m} exp(-sum_i |z_i|^2 / 2)
// optionally multiplied by |P_a(z)|^2, P_a = prod_k p_k^{r_k}, for the
// per-row guide of the reference estimator (reference
// modules/edge_mc/em_markovchain.cu:266-334 and em_spectrum.cu:49-97).
//
// Layout: a walker is a group of G consecutive lanes (G in {1,..,32}; G = 32
// is one walker per warp).  The walker's coordinates live in shared memory;
// lane l of the group owns particles j = l, l+G, l+2G, ... (slots 0, 1, 2,
// ...), stored as 16-byte records of two slots {x, x', y, y'}.  For a move of
// particle i every lane accumulates the products prod |z'-z_j|^2 and
// prod |z-z_j|^2 over its particles with packed FP32x2 arithmetic, even and
// odd slots in the two halves (one log2 per chain every 16 slots keeps FP32
// in range); the G partial log-ratios are combined with a butterfly of
// __shfl_xor_sync (all lanes end with bitwise identical sums, hence identical
// accept decisions), and the owner lane commits the move.  The row-guide
// state exists only in the row-guide instantiation (kRowGuide), so the
// Laughlin-guide kernel keeps its register count, and occupancy, low.
//
// Random numbers: one Philox-4x32-10 call per proposed move,
// counter = {i, sweep, walker, 0}: (u1, u2) -> Box-Muller step, u3 -> the
// Metropolis test log2(u3) <= log2(acceptance ratio).  Lane l of the group
// draws the randoms of particle i0 + l of each block of G moves and hands
// them to the group with three shuffles.
#include <cuda_runtime.h>

#include "lemc_internal.h"
#include "lemc_rng.h"

namespace lemc {
namespace {

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kTiny = 0x1p-64f;  // added to every squared pair distance

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// z^k for 1 <= k by binary powering (k < 64).
__device__ __forceinline__ float2 cpowi(float2 z, int k) {
  float2 r = make_float2(1.f, 0.f);
  float2 b = z;
  while (k) {
    if (k & 1) r = cmul(r, b);
    k >>= 1;
    if (k) b = cmul(b, b);
  }
  return r;
}

__device__ __forceinline__ double2 cpowi_d(float2 z, int k) {
  double2 r = make_double2(1.0, 0.0);
  double2 b = make_double2(z.x, z.y);
  while (k) {
    if (k & 1) r = make_double2(r.x * b.x - r.y * b.y, r.x * b.y + r.y * b.x);
    k >>= 1;
    if (k) b = make_double2(b.x * b.x - b.y * b.y, 2.0 * b.x * b.y);
  }
  return r;
}

template <int G>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
  for (int off = G / 2; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off, G);
  return v;
}

template <int G, bool kRowGuide>
__global__ void __launch_bounds__(kSweepThreads)
sweep_kernel(const SweepArgs a) {
  constexpr int WPW = 32 / G;           // walkers per warp
  constexpr int WPB = (kSweepThreads / 32) * WPW;
  constexpr int GPL = (kMaxGuideParts + G - 1) / G;  // guide slots per lane
  extern __shared__ __align__(16) float2 sm_pos[];  // 16-byte slot-pair records

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int gl = lane % G;
  const int wl = warp * WPW + lane / G;
  const int w = blockIdx.x * WPB + wl;
  const bool live = w < a.W;
  const int N = a.N;
  const int T2 = a.T2;  // particle slots per lane, rounded up to even
  // Walker layout: lane gl owns particles j = gl + t G (slot t); slots 2q and
  // 2q+1 of a lane form one 16-byte record {x_2q, x_2q+1, y_2q, y_2q+1} at
  // float4 index q G + gl, so one load gives the x pair and the y pair.
  float* zf = reinterpret_cast<float*>(sm_pos + (size_t)wl * a.Npad);
  const float4* zs4 = reinterpret_cast<const float4*>(zf);
  auto zoff = [](int j) {  // float offset of x_j (y_j at +2)
    const int t = j / G;
    return (((t >> 1) * G + (j % G)) << 2) + (t & 1);
  };
  auto ldz = [&](int j) {
    const int o = zoff(j);
    return make_float2(zf[o], zf[o + 2]);
  };
  auto stz = [&](int j, float2 z) {
    const int o = zoff(j);
    zf[o] = z.x;
    zf[o + 2] = z.y;
  };

  for (int j = gl; j < T2 * G; j += G)
    stz(j, (live && j < N) ? a.pos[(size_t)w * N + j] : make_float2(3.f * j + 1.f, 0.25f * j));
  __syncwarp();

  // ---- guide state: the distinct parts of the walker's guide partition ----
  constexpr bool row_guide = kRowGuide;  // a.guide == LEMC_GUIDE_ROW
  int gk[GPL], gr[GPL];
  double2 gp[GPL];
#pragma unroll
  for (int t = 0; t < GPL; ++t) { gk[t] = 0; gr[t] = 0; gp[t] = make_double2(0.0, 0.0); }
  if (row_guide && live) {
    const int row = a.walker_row[w];
    const int np = a.guide_npairs[row];
#pragma unroll
    for (int t = 0; t < GPL; ++t) {
      const int slot = gl + t * G;
      if (slot < np) {
        gk[t] = a.guide_pairs[row * 2 * kMaxGuideParts + 2 * slot];
        gr[t] = a.guide_pairs[row * 2 * kMaxGuideParts + 2 * slot + 1];
      }
    }
  }

  // Slot pairs q < qfull hold particles in both slots in every lane; pair
  // qfull (if any lane has a particle there) is masked per slot.
  const int tfull = N / G;                   // slots that hold a particle in every lane
  const int qfull = tfull >> 1;
  const bool rem_lane = gl < N - tfull * G;  // slot tfull holds a particle in this lane
  const bool tail0 = 2 * qfull < tfull || (2 * qfull == tfull && rem_lane);
  const bool tail1 = 2 * qfull + 1 == tfull && rem_lane;
  const bool tail = (tfull & 1) || tfull * G < N;  // lane 0 has a particle in pair qfull
  const float sigma = a.sigma;
  const float invR = a.invR;
  const float mf = float(a.m);
  uint32_t nacc = 0;
  const uint32_t sweep_base = a.sweep0 + (a.sweep_ctr ? *a.sweep_ctr : 0u);

  for (int s = 0; s < a.n_sweeps; ++s) {
    const uint32_t sweep = sweep_base + uint32_t(s);
    // refresh the guide power sums from the positions (bounds FP drift)
    if (row_guide) {
#pragma unroll
      for (int t = 0; t < GPL; ++t) {
        if (gk[t] > 0) {
          double2 acc = make_double2(0.0, 0.0);
          for (int j = 0; j < N; ++j) {
            const float2 z = ldz(j);
            const double2 v = cpowi_d(make_float2(z.x * invR, z.y * invR), gk[t]);
            acc.x += v.x;
            acc.y += v.y;
          }
          gp[t] = acc;
        }
      }
    }

    for (int i0 = 0; i0 < N; i0 += G) {
      // lane gl draws the randoms of particle i0 + gl
      float pzx = 0.f, pzy = 0.f, plu = 0.f;
      {
        const int i = i0 + gl;
        if (i < N) {
          const U4 r = philox4x32_10(U4{uint32_t(i), sweep, uint32_t(w), kTagMove}, a.seed_lo,
                                     a.seed_hi);
          const float u1 = u01(r.x), u2 = u01(r.y), u3 = u01(r.z);
          const float rad = sqrtf(-2.f * logf(u1));
          float sn, cs;
          sincospif(2.f * u2, &sn, &cs);
          const float2 zi = ldz(i);
          pzx = zi.x + sigma * (rad * cs);
          pzy = zi.y + sigma * (rad * sn);
          plu = log2f(u3);
        }
      }
      const int nb = min(G, N - i0);
      for (int b = 0; b < nb; ++b) {
        const int im = i0 + b;
        const float2 zo = ldz(im);
        const float xn = __shfl_sync(0xffffffffu, pzx, b, G);
        const float yn = __shfl_sync(0xffffffffu, pzy, b, G);
        const float lu = __shfl_sync(0xffffffffu, plu, b, G);

        // Jastrow log2-ratio over this lane's particles j = gl + t G: packed
        // FP32x2 arithmetic on slot pairs, two product chains (even and odd
        // slots), one log2 per chain every 16 slots (keeps FP32 in range).  No
        // per-pair masks: every squared distance carries + 2^-64, which leaves
        // any distance above 2^-40 unchanged and turns the self pair j == im
        // into the factors (s + 2^-64) / 2^-64, removed once after the loop;
        // the slots past the last full pair are masked outside the loop.
        float part = 0.f;
        {
          const float2 XN = make_float2(xn, xn), YN = make_float2(yn, yn);
          const float2 XO = make_float2(zo.x, zo.x), YO = make_float2(zo.y, zo.y);
          const float2 M1 = make_float2(-1.f, -1.f), TN = make_float2(kTiny, kTiny);
          auto factors = [&](int q, float2& pn, float2& po) {
            const float4 P = zs4[q * G + gl];
            const float2 X = make_float2(P.x, P.y), Y = make_float2(P.z, P.w);
            const float2 ax = __ffma2_rn(X, M1, XN), ay = __ffma2_rn(Y, M1, YN);
            const float2 ex = __ffma2_rn(X, M1, XO), ey = __ffma2_rn(Y, M1, YO);
            pn = __ffma2_rn(ax, ax, __ffma2_rn(ay, ay, TN));
            po = __ffma2_rn(ex, ex, __ffma2_rn(ey, ey, TN));
          };
          float2 n2 = make_float2(1.f, 1.f), d2 = n2;
          if (tail) {  // slot pair qfull: a full slot and/or the partly filled slot
            float2 pn, po;
            factors(qfull, pn, po);
            n2 = make_float2(tail0 ? pn.x : 1.f, tail1 ? pn.y : 1.f);
            d2 = make_float2(tail0 ? po.x : 1.f, tail1 ? po.y : 1.f);
          }
          for (int q0 = 0; q0 < qfull || q0 == 0; q0 += 8) {
            const int qend = min(qfull, q0 + 8);
            for (int q = q0; q < qend; ++q) {
              float2 pn, po;
              factors(q, pn, po);
              n2 = __fmul2_rn(n2, pn);
              d2 = __fmul2_rn(d2, po);
            }
            part += (__log2f(n2.x) + __log2f(n2.y)) - (__log2f(d2.x) + __log2f(d2.y));
            n2 = d2 = make_float2(1.f, 1.f);
          }
        }
        {
          const float sx = xn - zo.x, sy = yn - zo.y;
          const float self = fmaf(sx, sx, fmaf(sy, sy, kTiny));
          if (gl == im % G) part -= __log2f(self) + 64.f;  // log2(2^-64) = -64
        }
        part *= mf;

        // guide polynomial ratio |P_a(z')/P_a(z)|^2 (row guide)
        double2 gnew[GPL];
        if (row_guide) {
          const float2 wo = make_float2(zo.x * invR, zo.y * invR);
          const float2 wn = make_float2(xn * invR, yn * invR);
#pragma unroll
          for (int t = 0; t < GPL; ++t) {
            gnew[t] = gp[t];
            if (gk[t] > 0) {
              const double2 po = cpowi_d(wo, gk[t]);
              const double2 pn = cpowi_d(wn, gk[t]);
              gnew[t].x = gp[t].x - po.x + pn.x;
              gnew[t].y = gp[t].y - po.y + pn.y;
              const double n1 = gnew[t].x * gnew[t].x + gnew[t].y * gnew[t].y;
              const double n0 = gp[t].x * gp[t].x + gp[t].y * gp[t].y;
              part += float(gr[t]) * (__log2f(float(n1)) - __log2f(float(n0)));
            }
          }
        }

        const float tot = group_sum<G>(part);
        const float gauss = (fmaf(zo.x, zo.x, zo.y * zo.y) - fmaf(xn, xn, yn * yn)) * (0.5f * kLog2e);
        const bool accept = (tot + gauss) >= lu;
        if (accept) {
          if (gl == b) stz(im, make_float2(xn, yn));
          ++nacc;
          if (row_guide) {
#pragma unroll
            for (int t = 0; t < GPL; ++t) gp[t] = gnew[t];
          }
        }
        __syncwarp();
      }
    }
  }

  if (live) {
    for (int j = gl; j < N; j += G) a.pos[(size_t)w * N + j] = ldz(j);
    if (gl == 0 && a.accepted) a.accepted[w] += nacc;
  }

  if (!a.measure) return;

  // ---- measurement record: p_k = sum_i (z_i / R)^k, k = 1..K, and weights ----
  // kPassDeg degrees per pass over the particles (w^k by the same sequence of
  // multiplications in every pass; two passes for K = 12), then r^2 / r^4,
  // then one pass per probe: few live registers, so the kernel's register
  // count is set by the sweep.
  constexpr int kPassDeg = 6;
  const int K = a.K;
  for (int k0 = 0; k0 < K; k0 += kPassDeg) {
    float2 acc[kPassDeg];
#pragma unroll
    for (int k = 0; k < kPassDeg; ++k) acc[k] = make_float2(0.f, 0.f);
    for (int j = gl; j < N; j += G) {
      const float2 z = ldz(j);
      const float2 wv = make_float2(z.x * invR, z.y * invR);
      float2 pw = wv;
      for (int k = 0; k < k0; ++k) pw = cmul(pw, wv);
#pragma unroll
      for (int k = 0; k < kPassDeg; ++k) {
        acc[k].x += pw.x;
        acc[k].y += pw.y;
        pw = cmul(pw, wv);
      }
    }
#pragma unroll
    for (int k = 0; k < kPassDeg; ++k) {
      const float sx = group_sum<G>(acc[k].x), sy = group_sum<G>(acc[k].y);
      if (live && k0 + k < K && ((k0 + k) % G) == gl)
        a.rec_p[(size_t)(k0 + k) * a.W + w] = make_float2(sx, sy);
    }
  }
  const size_t ldw = a.ldw;
  {
    float h2 = 0.f, h4 = 0.f;
    for (int j = gl; j < N; j += G) {
      const float2 z = ldz(j);
      const float r2 = fmaf(z.x, z.x, z.y * z.y);
      h2 += r2;
      h4 = fmaf(r2, r2, h4);
    }
    h2 = group_sum<G>(h2);
    h4 = group_sum<G>(h4);
    if (live && gl == 0) {
      a.rec_w[LEMC_W_ONE * ldw + w] = 1.f;
      a.rec_w[LEMC_W_R2 * ldw + w] = h2;
      a.rec_w[LEMC_W_R4 * ldw + w] = h4;
      a.rec_w[LEMC_W_USER * ldw + w] = 0.f;
    }
  }
#pragma unroll
  for (int q = 0; q < LEMC_MAX_PROBES; ++q) {  // constant indices into the argument struct
    if (q >= a.n_probes) break;
    const int l = a.probes[q];
    float hc = 0.f, hs = 0.f;
    for (int j = gl; j < N; j += G) {
      const float2 z = ldz(j);
      const float rinv = rsqrtf(fmaf(z.x, z.x, z.y * z.y));
      const float2 e = cpowi(make_float2(z.x * rinv, z.y * rinv), l);
      hc += e.x;
      hs += e.y;
    }
    hc = group_sum<G>(hc);
    hs = group_sum<G>(hs);
    if (live && gl == 0) {
      a.rec_w[(LEMC_W_PROBE0 + 2 * q) * ldw + w] = hc;
      a.rec_w[(LEMC_W_PROBE0 + 2 * q + 1) * ldw + w] = hs;
    }
  }
}

// Uniform initial positions in a disk, Philox counter {i, 0, w, 1}.
__global__ void init_walkers_kernel(float2* pos, int W, int N, float radius, uint32_t k0,
                                    uint32_t k1) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)W * N) return;
  const uint32_t w = uint32_t(t / N), i = uint32_t(t % N);
  const U4 r = philox4x32_10(U4{i, 0u, w, kTagInit}, k0, k1);
  const float rho = radius * sqrtf(u01(r.x));
  float sn, cs;
  sincospif(2.f * u01(r.y), &sn, &cs);
  pos[t] = make_float2(rho * cs, rho * sn);
}

template <int G, bool kRowGuide>
int launch_gr(const SweepArgs& a, cudaStream_t st) {
  constexpr int WPB = (kSweepThreads / 32) * (32 / G);
  const size_t smem = size_t(WPB) * a.Npad * sizeof(float2);
  if (smem > 227 * 1024) return LEMC_ERR_CAPACITY;
  if (smem > 48 * 1024) {
    if (cudaFuncSetAttribute(sweep_kernel<G, kRowGuide>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
      return LEMC_ERR_CUDA;
  }
  const int blocks = (a.W + WPB - 1) / WPB;
  sweep_kernel<G, kRowGuide><<<blocks, kSweepThreads, smem, st>>>(a);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

// the row-guide state (guide parts, power sums) only exists in the row-guide
// instantiation, so the Laughlin-guide kernel runs with fewer registers
template <int G>
int launch_g(const SweepArgs& a, cudaStream_t st) {
  return a.guide == LEMC_GUIDE_ROW ? launch_gr<G, true>(a, st) : launch_gr<G, false>(a, st);
}

}  // namespace

void sweep_layout(int G, int N, int* T2, int* Npad) {
  int t = (N + G - 1) / G;
  t += (t & 1);
  int np = t * G;  // even: the 16-byte slot-pair records stay aligned
  // For G < 8 a quarter-warp's 16-byte loads span 8 / G walkers of G * 16
  // bytes each; a walker stride of 2G float2 mod 16 puts them in disjoint banks.
  if (G < 8) np += ((2 * G - np) % 16 + 16) % 16;
  *T2 = t;
  *Npad = np;
}

size_t sweep_smem_bytes(int G, int Npad) {
  return size_t((kSweepThreads / 32) * (32 / G)) * Npad * sizeof(float2);
}

bool sweep_config_ok(int G, int N) {
  if (G != 1 && G != 2 && G != 4 && G != 8 && G != 16 && G != 32) return false;
  int t2, np;
  sweep_layout(G, N, &t2, &np);
  return sweep_smem_bytes(G, np) <= 227 * 1024;
}

int launch_sweep(const SweepArgs& a_in, int G, cudaStream_t st) {
  if (a_in.K > kMaxDegree || a_in.N <= 1 || a_in.W <= 0) return LEMC_ERR_ARG;
  SweepArgs a = a_in;
  sweep_layout(G, a.N, &a.T2, &a.Npad);
  switch (G) {
    case 1: return launch_g<1>(a, st);
    case 2: return launch_g<2>(a, st);
    case 4: return launch_g<4>(a, st);
    case 8: return launch_g<8>(a, st);
    case 16: return launch_g<16>(a, st);
    case 32: return launch_g<32>(a, st);
    default: return LEMC_ERR_ARG;
  }
}

int launch_init_walkers(float2* pos, int W, int N, float radius, uint32_t k0, uint32_t k1,
                        cudaStream_t st) {
  const size_t n = size_t(W) * N;
  const int threads = 256;
  const unsigned blocks = unsigned((n + threads - 1) / threads);
  init_walkers_kernel<<<blocks, threads, 0, st>>>(pos, W, N, radius, k0, k1);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

namespace {
__global__ void advance_counters_kernel(uint32_t* ctr) {
  ctr[0] += 1u;
  ctr[1] += 1u;
}
}  // namespace

int launch_advance_counters(uint32_t* ctr, cudaStream_t st) {
  advance_counters_kernel<<<1, 1, 0, st>>>(ctr);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

}  // namespace lemc
