// Orbital occupation numbers <f_L| a^dagger_l a_l |f_R> with the two-state
// walker (reference modules/green_function/green_function.cu:199-373 and
// gf_occupation_numbers.cu:16-239), all (L, R) pairs of a sector in one launch.
//
// A walker carries N+1 particles z_0..z_N: f_L depends on z_0..z_{N-1}, f_R
// on z_1..z_N, and the walker samples |f_L| |f_R| with
// f = P_row(z) prod_{i<j} (z_i - z_j)^m exp(-sum |z|^2 / 4).  One sweep moves
// particle 0, then 1..N-1, then N, each with its own Metropolis test:
//   0:      |J_0|^m |P_L'/P_L| exp((|z|^2 - |z'|^2)/4)
//   1..N-1: |c|^m |P_L'/P_L| |P_R'/P_R| |J|^{2m} exp((|z|^2 - |z'|^2)/2),
//           c = (z'-z_0)(z'-z_N) / ((z-z_0)(z-z_N))
//   N:      |J_N|^m |P_R'/P_R| exp((|z|^2 - |z'|^2)/4)
// evaluated as log-ratios.  After every sweep the estimator
//   sum_l exp(-ln(2 pi l!) + l ln(z_0 conj(z_N)/2) - (|z_0|^2+|z_N|^2)/4 + i phase),
//   phase = arg(P_R/P_L) + m arg prod_{i=1}^{N-1} (z_i - z_N)/(z_0 - z_i),
// is accumulated per walker in FP64 (magnitudes by a log-domain recurrence,
// so nothing under- or overflows for large N), and reduced per pair at the end.
//
// One thread per walker; positions in shared memory, interleaved by thread.
// Random numbers: Philox counter {particle, sweep, walker, 2}, init tag 3.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "lemc_internal.h"
#include "lemc_rng.h"
#include "partitions.hpp"

namespace lemc {
namespace {

constexpr uint32_t kTagOccMove = 2u, kTagOccInit = 3u;

struct OccArgs {
  int W, N, m, D, Lc;
  float sigma;
  float invR;
  uint32_t k0, k1;
  int burn, sweeps;
  const int32_t* pairs;   // [D][2*kMaxGuideParts] (part, mult)
  const int32_t* npairs;  // [D]
  double2* acc;           // [Lc][W] per-walker sums
  uint32_t* accepted;     // [W]
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ double2 cpow_d(double2 z, int k) {
  double2 r = make_double2(1.0, 0.0), b = z;
  while (k) {
    if (k & 1) r = cmul(r, b);
    k >>= 1;
    if (k) b = cmul(b, b);
  }
  return r;
}

struct Guide {
  int k[kMaxGuideParts], r[kMaxGuideParts], n;
  double2 p[kMaxGuideParts];
};

// log|P'/P| after replacing particle position zo by zn in the guide's power sums
__device__ __forceinline__ double guide_delta(const Guide& g, float2 zo, float2 zn, float invR,
                                              double2* pn) {
  double d = 0.0;
  const double2 wo = make_double2(zo.x * invR, zo.y * invR), wn = make_double2(zn.x * invR, zn.y * invR);
  for (int q = 0; q < g.n; ++q) {
    pn[q] = g.p[q];
    if (g.k[q] == 0) continue;
    const double2 a = cpow_d(wo, g.k[q]), b = cpow_d(wn, g.k[q]);
    pn[q].x += b.x - a.x;
    pn[q].y += b.y - a.y;
    // ln of the ratio of squared moduli: formed in FP64, its log in FP32
    // (the ratio of two moduli of the same power sum before and after one
    // particle moved; an infinite or zero ratio gives +-inf as the FP64 log did)
    const double ratio = (pn[q].x * pn[q].x + pn[q].y * pn[q].y) /
                         (g.p[q].x * g.p[q].x + g.p[q].y * g.p[q].y);
    d += 0.5 * 0.6931471805599453 * g.r[q] * double(__log2f(float(ratio)));
  }
  return d;
}

__device__ __forceinline__ double guide_arg(const Guide& g) {
  double a = 0.0;
  for (int q = 0; q < g.n; ++q)
    if (g.k[q] > 0) a += g.r[q] * atan2(g.p[q].y, g.p[q].x);
  return a;
}

// G lanes per walker (one walker group of G consecutive lanes of a warp):
// lane gl owns the shared particles j = 1 + gl + tG of the Jastrow sums, the
// estimator's partial products over the same particles and the orbitals
// l = gl + tG of the estimator; xor-butterfly reductions within the group give
// every lane bit-identical sums, hence the same accept decision.  Every
// shuffle sits in control flow that is uniform over the warp (the guide loops
// run over all kMaxGuideParts slots, the walkers beyond W compute and do not
// write), so full-warp masks are exact.
constexpr int kOccLanesThreads = 128;

template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
  return v;
}

template <int G>
__device__ __forceinline__ float group_sumf(float v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
  return v;
}

// power sums of the guide parts over particles [j0, j1) of the walker, every
// lane of the group ending with the same values
template <int G>
__device__ __forceinline__ void guide_refresh(Guide& g, const float2* zs, int j0, int j1, float invR,
                                              int gl) {
#pragma unroll
  for (int q = 0; q < kMaxGuideParts; ++q) {
    double re = 0.0, im = 0.0;
    if (q < g.n && g.k[q] > 0)
      for (int j = j0 + gl; j < j1; j += G) {
        const double2 v = cpow_d(make_double2(zs[j].x * invR, zs[j].y * invR), g.k[q]);
        re += v.x;
        im += v.y;
      }
    g.p[q] = make_double2(group_sum<G>(re), group_sum<G>(im));
  }
}

template <int G>
__global__ void __launch_bounds__(kOccLanesThreads) occupation_kernel(const OccArgs a) {
  extern __shared__ double occ_smem[];
  constexpr int WPB = kOccLanesThreads / G;
  const int t = threadIdx.x;
  const int gl = t % G, wl = t / G;
  const int w = blockIdx.x * WPB + wl;
  const bool live = w < a.W;
  const int N = a.N, NP = a.N + 1;
  // ln(l!) for the estimator's orbitals, then the walkers' positions
  double* lnfact = occ_smem;
  float2* zs = reinterpret_cast<float2*>(occ_smem + a.Lc) + size_t(wl) * NP;
  for (int l = t; l < a.Lc; l += kOccLanesThreads) lnfact[l] = lgamma(double(l) + 1.0);

  const int wr = live ? w : a.W - 1;  // walkers beyond W compute, never write
  const int pair = int((int64_t(wr) * a.D * a.D) / a.W);
  const int rowL = pair / a.D, rowR = pair % a.D;
  Guide gL, gR;
  gL.n = a.npairs[rowL];
  gR.n = a.npairs[rowR];
  for (int q = 0; q < kMaxGuideParts; ++q) {
    gL.k[q] = q < gL.n ? a.pairs[rowL * 2 * kMaxGuideParts + 2 * q] : 0;
    gL.r[q] = q < gL.n ? a.pairs[rowL * 2 * kMaxGuideParts + 2 * q + 1] : 0;
    gR.k[q] = q < gR.n ? a.pairs[rowR * 2 * kMaxGuideParts + 2 * q] : 0;
    gR.r[q] = q < gR.n ? a.pairs[rowR * 2 * kMaxGuideParts + 2 * q + 1] : 0;
  }
  // initial positions: uniform in the disk of radius sqrt(2 m N)
  const float r0 = sqrtf(2.f * a.m * N);
  for (int j = gl; j < NP; j += G) {
    const U4 r = philox4x32_10(U4{uint32_t(j), 0u, uint32_t(w), kTagOccInit}, a.k0, a.k1);
    const float rho = r0 * sqrtf(u01(r.x));
    float sn, cs;
    sincospif(2.f * u01(r.y), &sn, &cs);
    zs[j] = make_float2(rho * cs, rho * sn);
  }
  __syncthreads();
  uint32_t nacc = 0;
  const float sigma = a.sigma;
  const double mm = double(a.m);
  for (int s = 0; s < a.burn + a.sweeps; ++s) {
    // refresh guide power sums: left over 0..N-1, right over 1..N
    guide_refresh<G>(gL, zs, 0, N, a.invR, gl);
    guide_refresh<G>(gR, zs, 1, NP, a.invR, gl);
    float dx_l = 0.f, dy_l = 0.f;
    double lu_l = 0.0;
    for (int i = 0; i < NP; ++i) {
      // the randoms of move i, Philox {i, sweep, walker, 2}: lane gl draws
      // those of move i0 + gl for the block of G moves starting at i0
      if (i % G == 0) {
        const U4 r = philox4x32_10(U4{uint32_t(i + gl), uint32_t(s), uint32_t(w), kTagOccMove},
                                   a.k0, a.k1);
        const float rad = sqrtf(-2.f * logf(u01(r.x)));
        float sn, cs;
        sincospif(2.f * u01(r.y), &sn, &cs);
        dx_l = sigma * (rad * cs);
        dy_l = sigma * (rad * sn);
        lu_l = log(double(u01(r.z)));
      }
      const float ddx = __shfl_sync(0xffffffffu, dx_l, i % G, G);
      const float ddy = __shfl_sync(0xffffffffu, dy_l, i % G, G);
      const double lu = __shfl_sync(0xffffffffu, lu_l, i % G, G);
      const float2 zo = zs[i];
      const float2 zn = make_float2(zo.x + ddx, zo.y + ddy);
      // Jastrow log|ratio| over the shared particles 1..N-1: FP32 products of
      // the squared distances, four terms at a time, one log2 per product
      float lj2 = 0.f;
      {
        float pn = 1.f, po = 1.f;
        int c = 0;
        for (int j = 1 + gl; j < N; j += G) {
          if (j == i) continue;
          const float2 zj = zs[j];
          const float dx = zn.x - zj.x, dy = zn.y - zj.y, ex = zo.x - zj.x, ey = zo.y - zj.y;
          pn *= fmaf(dx, dx, dy * dy);
          po *= fmaf(ex, ex, ey * ey);
          if (++c == 4) {
            lj2 += __log2f(pn) - __log2f(po);
            pn = po = 1.f;
            c = 0;
          }
        }
        if (c) lj2 += __log2f(pn) - __log2f(po);
      }
      const double lj = 0.5 * 0.6931471805599453 * double(group_sumf<G>(lj2));
      const double gz = double(zo.x) * zo.x + double(zo.y) * zo.y - (double(zn.x) * zn.x + double(zn.y) * zn.y);
      double delta;
      double2 pl[kMaxGuideParts], pr[kMaxGuideParts];
      if (i == 0) {
        delta = mm * lj + guide_delta(gL, zo, zn, a.invR, pl) + 0.25 * gz;
      } else if (i == N) {
        delta = mm * lj + guide_delta(gR, zo, zn, a.invR, pr) + 0.25 * gz;
      } else {
        const float2 z0 = zs[0], zN = zs[N];
        // ln|z' - z_0| - ln|z - z_0| and the same for z_N, in FP32 like the
        // Jastrow chains
        const float c02 = __log2f(fmaf(zn.x - z0.x, zn.x - z0.x, (zn.y - z0.y) * (zn.y - z0.y))) -
                          __log2f(fmaf(zo.x - z0.x, zo.x - z0.x, (zo.y - z0.y) * (zo.y - z0.y)));
        const float cN2 = __log2f(fmaf(zn.x - zN.x, zn.x - zN.x, (zn.y - zN.y) * (zn.y - zN.y))) -
                          __log2f(fmaf(zo.x - zN.x, zo.x - zN.x, (zo.y - zN.y) * (zo.y - zN.y)));
        const double c0 = 0.5 * 0.6931471805599453 * double(c02);
        const double cN = 0.5 * 0.6931471805599453 * double(cN2);
        delta = mm * (c0 + cN) + guide_delta(gL, zo, zn, a.invR, pl) +
                guide_delta(gR, zo, zn, a.invR, pr) + 2.0 * mm * lj + 0.5 * gz;
      }
      const bool acc = delta >= lu;
      __syncwarp();
      if (acc) {
        if (gl == 0) zs[i] = zn;
        ++nacc;
        if (i < N)
          for (int q = 0; q < gL.n; ++q) gL.p[q] = pl[q];
        if (i > 0)
          for (int q = 0; q < gR.n; ++q) gR.p[q] = pr[q];
      }
      __syncwarp();
    }
    if (s < a.burn) continue;
    // estimator: u = prod_{i=1}^{N-1} (z_i - z_N) conj(z_0 - z_i), kept at unit
    // modulus, as group partial products combined by the butterfly
    const float2 z0 = zs[0], zN = zs[N];
    double2 u = make_double2(1.0, 0.0);
    for (int i = 1 + gl; i < N; i += G) {
      const float2 zi = zs[i];
      const double2 num = make_double2(zi.x - zN.x, zi.y - zN.y);
      const double2 den = make_double2(z0.x - zi.x, z0.y - zi.y);
      u = cmul(u, make_double2(num.x * den.x + num.y * den.y, num.y * den.x - num.x * den.y));
      const double nu = sqrt(u.x * u.x + u.y * u.y);
      if (nu > 0) {
        u.x /= nu;
        u.y /= nu;
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      const double2 v = make_double2(__shfl_xor_sync(0xffffffffu, u.x, o, G),
                                     __shfl_xor_sync(0xffffffffu, u.y, o, G));
      u = cmul(u, v);
      const double nu = sqrt(u.x * u.x + u.y * u.y);
      if (nu > 0) {
        u.x /= nu;
        u.y /= nu;
      }
    }
    const double phase = guide_arg(gR) - guide_arg(gL) + mm * atan2(u.y, u.x);
    const double2 q0 = make_double2(0.5 * (double(z0.x) * zN.x + double(z0.y) * zN.y),
                                    0.5 * (double(z0.y) * zN.x - double(z0.x) * zN.y));  // z0 conj(zN) / 2
    const double lx = 0.5 * log(q0.x * q0.x + q0.y * q0.y);
    const double phi = atan2(q0.y, q0.x);
    const double base = -0.25 * (double(z0.x) * z0.x + double(z0.y) * z0.y + double(zN.x) * zN.x +
                                 double(zN.y) * zN.y) - log(2.0 * 3.14159265358979323846);
    if (!live) continue;
    for (int l = gl; l < a.Lc; l += G) {
      // log magnitude of term l: base + l ln|z_0 conj(z_N)/2| - ln l!
      const double la = base + double(l) * lx - lnfact[l];
      if (la > -700.0) {
        const double mag = exp(la);
        double sn2, cs2;
        sincos(l * phi + phase, &sn2, &cs2);
        double2* p = a.acc + size_t(l) * a.W + w;
        p->x += mag * cs2;
        p->y += mag * sn2;
      }
    }
  }
  if (live && gl == 0) a.accepted[w] = nacc;
}

// Lanes per walker for N + 1 particles: about eight particles per lane.
int occupation_lanes(int N) {
  int G = 4;
  while (G < 32 && (N + G - 1) / G > 8) G *= 2;
  return G;
}

size_t occupation_smem(int N, int Lc) {
  const int G = occupation_lanes(N);
  return sizeof(double) * size_t(Lc) + sizeof(float2) * size_t(kOccLanesThreads / G) * (N + 1);
}

template <int G>
int launch_occ_g(const OccArgs& a, cudaStream_t st) {
  const size_t smem = occupation_smem(a.N, a.Lc);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(occupation_kernel<G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(smem)) != cudaSuccess)
    return LEMC_ERR_CUDA;
  constexpr int WPB = kOccLanesThreads / G;
  occupation_kernel<G><<<(a.W + WPB - 1) / WPB, kOccLanesThreads, smem, st>>>(a);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

int launch_occupation(const OccArgs& a, cudaStream_t st) {
  if (occupation_smem(a.N, a.Lc) > 227 * 1024) return LEMC_ERR_CAPACITY;
  switch (occupation_lanes(a.N)) {
    case 4: return launch_occ_g<4>(a, st);
    case 8: return launch_occ_g<8>(a, st);
    case 16: return launch_occ_g<16>(a, st);
    default: return launch_occ_g<32>(a, st);
  }
}

__global__ void occupation_reduce(const double2* acc, int W, int D, int Lc, double2* out) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  const int pair = blockIdx.y;
  if (l >= Lc) return;
  const int w0 = int((int64_t(pair) * W + (int64_t(D) * D) - 1) / (int64_t(D) * D));
  const int w1 = int((int64_t(pair + 1) * W + (int64_t(D) * D) - 1) / (int64_t(D) * D));
  double2 s = make_double2(0.0, 0.0);
  for (int w = w0; w < w1; ++w) {
    s.x += acc[size_t(l) * W + w].x;
    s.y += acc[size_t(l) * W + w].y;
  }
  out[size_t(pair) * Lc + l] = s;
}

}  // namespace
}  // namespace lemc

using namespace lemc;

extern "C" int lemc_occupation(const lemc_occupation_config* cfg, double* out, double* acceptance) {
  if (!cfg || !out) return LEMC_ERR_ARG;
  const int N = cfg->particles, m = cfg->inverse_filling, W = cfg->n_walkers, Lc = cfg->l_cutoff;
  if (N < 2 || m < 1 || W < 1 || Lc < 1 || cfg->dL < 0 || cfg->dL > kMaxDegree || cfg->sweeps < 1 ||
      cfg->burn_in < 0 || !(cfg->step_sigma > 0.f))
    return LEMC_ERR_ARG;
  if (occupation_smem(N, Lc) > 227 * 1024) return LEMC_ERR_CAPACITY;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return LEMC_ERR_NODEVICE;
  }
  const Basis B = build_basis(N, {cfg->dL});
  const int D = int(B.rows.size());
  if (W < D * D) return LEMC_ERR_ARG;  // at least one walker per pair
  std::vector<int32_t> pairs(size_t(D) * 2 * kMaxGuideParts, 0), np(D, 0);
  for (int r = 0; r < D; ++r) {
    const auto& pr = B.rows[r].pairs;
    if (int(pr.size()) > kMaxGuideParts) return LEMC_ERR_CAPACITY;
    np[r] = int(pr.size());
    for (size_t q = 0; q < pr.size(); ++q) {
      pairs[size_t(r) * 2 * kMaxGuideParts + 2 * q] = pr[q].part;
      pairs[size_t(r) * 2 * kMaxGuideParts + 2 * q + 1] = pr[q].part > 0 ? pr[q].mult : 0;
    }
  }
  int32_t *d_pairs = nullptr, *d_np = nullptr;
  double2 *d_acc = nullptr, *d_out = nullptr;
  uint32_t* d_accp = nullptr;
  int st = LEMC_OK;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && st == LEMC_OK) st = LEMC_ERR_CUDA;
    return st == LEMC_OK;
  };
  ok(cudaMalloc(&d_pairs, pairs.size() * 4));
  ok(cudaMalloc(&d_np, np.size() * 4));
  ok(cudaMalloc(&d_acc, sizeof(double2) * size_t(Lc) * W));
  ok(cudaMalloc(&d_out, sizeof(double2) * size_t(D) * D * Lc));
  ok(cudaMalloc(&d_accp, sizeof(uint32_t) * W));
  if (st == LEMC_OK) {
    ok(cudaMemcpy(d_pairs, pairs.data(), pairs.size() * 4, cudaMemcpyHostToDevice));
    ok(cudaMemcpy(d_np, np.data(), np.size() * 4, cudaMemcpyHostToDevice));
    ok(cudaMemset(d_acc, 0, sizeof(double2) * size_t(Lc) * W));
  }
  if (st == LEMC_OK) {
    OccArgs a;
    a.W = W;
    a.N = N;
    a.m = m;
    a.D = D;
    a.Lc = Lc;
    a.sigma = cfg->step_sigma;
    a.invR = float(1.0 / std::sqrt(2.0 * m * N));
    a.k0 = uint32_t(cfg->seed);
    a.k1 = uint32_t(cfg->seed >> 32);
    a.burn = cfg->burn_in;
    a.sweeps = cfg->sweeps;
    a.pairs = d_pairs;
    a.npairs = d_np;
    a.acc = d_acc;
    a.accepted = d_accp;
    if (st == LEMC_OK) {
      const int ls = launch_occupation(a, nullptr);
      if (ls != LEMC_OK && st == LEMC_OK) st = ls;
      occupation_reduce<<<dim3((Lc + 127) / 128, D * D), 128>>>(d_acc, W, D, Lc, d_out);
      ok(cudaPeekAtLastError());
      ok(cudaDeviceSynchronize());
    }
  }
  if (st == LEMC_OK) {
    std::vector<double2> h(size_t(D) * D * Lc);
    std::vector<uint32_t> acc(W);
    ok(cudaMemcpy(h.data(), d_out, sizeof(double2) * h.size(), cudaMemcpyDeviceToHost));
    ok(cudaMemcpy(acc.data(), d_accp, sizeof(uint32_t) * W, cudaMemcpyDeviceToHost));
    if (st == LEMC_OK) {
      double tot = 0;
      for (uint32_t v : acc) tot += v;
      if (acceptance)
        *acceptance = tot / (double(W) * (N + 1) * (cfg->burn_in + cfg->sweeps));
      for (int pr = 0; pr < D * D; ++pr) {
        const int w0 = int((int64_t(pr) * W + (int64_t(D) * D) - 1) / (int64_t(D) * D));
        const int w1 = int((int64_t(pr + 1) * W + (int64_t(D) * D) - 1) / (int64_t(D) * D));
        const double n = double(w1 - w0) * cfg->sweeps;
        for (int l = 0; l < Lc; ++l) {
          out[2 * (size_t(pr) * Lc + l)] = h[size_t(pr) * Lc + l].x / n;
          out[2 * (size_t(pr) * Lc + l) + 1] = h[size_t(pr) * Lc + l].y / n;
        }
      }
    }
  }
  cudaFree(d_pairs);
  cudaFree(d_np);
  cudaFree(d_acc);
  cudaFree(d_out);
  cudaFree(d_accp);
  return st;
}

// ---- allocation-free variant ----------------------------------------------
// lemc_occupation_static runs the same two kernels as lemc_occupation, but all
// device memory beyond the caller's host buffers comes from one fixed,
// file-scope device array instead of cudaMalloc: the row table, the per-walker
// accumulators, the per-pair sums and the acceptance counters.  It is for
// callers that must not allocate device memory during the call: a process
// whose device memory is already handed to a caching allocator (so cudaMalloc
// would fail or fragment it), or a loop that cannot afford the implicit device
// synchronisation of cudaFree.
namespace lemc {
namespace {

constexpr size_t kOccStaticBytes = size_t(LEMC_OCC_STATIC_SCRATCH_BYTES);
constexpr int kOccStaticDevices = 64;

static __device__ __align__(256) unsigned char g_occ_scratch[kOccStaticBytes];

std::mutex g_occ_scratch_mu;
void* g_occ_scratch_ptr[kOccStaticDevices] = {};

// Address of g_occ_scratch on the current device, resolved once per device
// with that device current.
int occ_scratch_address(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return LEMC_ERR_NODEVICE;
  }
  if (dev < 0 || dev >= kOccStaticDevices) return LEMC_ERR_CAPACITY;
  std::lock_guard<std::mutex> lock(g_occ_scratch_mu);
  if (!g_occ_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_occ_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return LEMC_ERR_CUDA;
    }
    g_occ_scratch_ptr[dev] = p;
  }
  *out = g_occ_scratch_ptr[dev];
  return LEMC_OK;
}

constexpr size_t occ_align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace
}  // namespace lemc

extern "C" int lemc_occupation_static(const lemc_occupation_config* cfg, double* out,
                                      double* acceptance) {
  if (!cfg || !out) return LEMC_ERR_ARG;
  const int N = cfg->particles, m = cfg->inverse_filling, W = cfg->n_walkers, Lc = cfg->l_cutoff;
  if (N < 2 || m < 1 || W < 1 || Lc < 1 || cfg->dL < 0 || cfg->dL > kMaxDegree || cfg->sweeps < 1 ||
      cfg->burn_in < 0 || !(cfg->step_sigma > 0.f))
    return LEMC_ERR_ARG;
  if (occupation_smem(N, Lc) > 227 * 1024) return LEMC_ERR_CAPACITY;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return LEMC_ERR_NODEVICE;
  }
  const Basis B = build_basis(N, {cfg->dL});
  const int D = int(B.rows.size());
  if (W < D * D) return LEMC_ERR_ARG;  // at least one walker per pair
  std::vector<int32_t> table(size_t(D) * 2 * kMaxGuideParts + D, 0);
  int32_t* pairs = table.data();
  int32_t* np = table.data() + size_t(D) * 2 * kMaxGuideParts;
  for (int r = 0; r < D; ++r) {
    const auto& pr = B.rows[r].pairs;
    if (int(pr.size()) > kMaxGuideParts) return LEMC_ERR_CAPACITY;
    np[r] = int(pr.size());
    for (size_t q = 0; q < pr.size(); ++q) {
      pairs[size_t(r) * 2 * kMaxGuideParts + 2 * q] = pr[q].part;
      pairs[size_t(r) * 2 * kMaxGuideParts + 2 * q + 1] = pr[q].part > 0 ? pr[q].mult : 0;
    }
  }
  // scratch layout: [row table][accepted W][acc Lc x W][out D*D x Lc], 256-B aligned parts
  const size_t b_table = occ_align256(table.size() * sizeof(int32_t));
  const size_t b_accp = occ_align256(sizeof(uint32_t) * size_t(W));
  const size_t b_acc = occ_align256(sizeof(double2) * size_t(Lc) * W);
  const size_t b_out = occ_align256(sizeof(double2) * size_t(D) * D * Lc);
  if (b_table + b_accp + b_acc + b_out > kOccStaticBytes) return LEMC_ERR_CAPACITY;
  void* base = nullptr;
  int st = occ_scratch_address(&base);
  if (st != LEMC_OK) return st;
  unsigned char* s = static_cast<unsigned char*>(base);
  int32_t* d_table = reinterpret_cast<int32_t*>(s);
  uint32_t* d_accp = reinterpret_cast<uint32_t*>(s + b_table);
  double2* d_acc = reinterpret_cast<double2*>(s + b_table + b_accp);
  double2* d_out = reinterpret_cast<double2*>(s + b_table + b_accp + b_acc);
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && st == LEMC_OK) st = LEMC_ERR_CUDA;
    return st == LEMC_OK;
  };
  // Only the per-walker accumulators must start at zero: the kernel adds
  // into them.  The table is copied, and the counters and per-pair sums are
  // written in full by the kernels.
  ok(cudaMemcpy(d_table, table.data(), table.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  ok(cudaMemset(d_acc, 0, sizeof(double2) * size_t(Lc) * W));
  if (st == LEMC_OK) {
    OccArgs a;
    a.W = W;
    a.N = N;
    a.m = m;
    a.D = D;
    a.Lc = Lc;
    a.sigma = cfg->step_sigma;
    a.invR = float(1.0 / std::sqrt(2.0 * m * N));
    a.k0 = uint32_t(cfg->seed);
    a.k1 = uint32_t(cfg->seed >> 32);
    a.burn = cfg->burn_in;
    a.sweeps = cfg->sweeps;
    a.pairs = d_table;
    a.npairs = d_table + size_t(D) * 2 * kMaxGuideParts;
    a.acc = d_acc;
    a.accepted = d_accp;
    if (st == LEMC_OK) {
      const int ls = launch_occupation(a, nullptr);
      if (ls != LEMC_OK && st == LEMC_OK) st = ls;
      occupation_reduce<<<dim3((Lc + 127) / 128, D * D), 128>>>(d_acc, W, D, Lc, d_out);
      ok(cudaPeekAtLastError());
      ok(cudaDeviceSynchronize());
    }
  }
  if (st == LEMC_OK) {
    std::vector<double2> h(size_t(D) * D * Lc);
    std::vector<uint32_t> acc(W);
    ok(cudaMemcpy(h.data(), d_out, sizeof(double2) * h.size(), cudaMemcpyDeviceToHost));
    ok(cudaMemcpy(acc.data(), d_accp, sizeof(uint32_t) * W, cudaMemcpyDeviceToHost));
    if (st == LEMC_OK) {
      double tot = 0;
      for (uint32_t v : acc) tot += v;
      if (acceptance)
        *acceptance = tot / (double(W) * (N + 1) * (cfg->burn_in + cfg->sweeps));
      for (int pr = 0; pr < D * D; ++pr) {
        const int w0 = int((int64_t(pr) * W + (int64_t(D) * D) - 1) / (int64_t(D) * D));
        const int w1 = int((int64_t(pr + 1) * W + (int64_t(D) * D) - 1) / (int64_t(D) * D));
        const double n = double(w1 - w0) * cfg->sweeps;
        for (int l = 0; l < Lc; ++l) {
          out[2 * (size_t(pr) * Lc + l)] = h[size_t(pr) * Lc + l].x / n;
          out[2 * (size_t(pr) * Lc + l) + 1] = h[size_t(pr) * Lc + l].y / n;
        }
      }
    }
  }
  return st;
}
