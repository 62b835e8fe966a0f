// Counter-based random numbers shared by host and device code.
//
// Philox-4x32-10 as published in Salmon, Moraes, Dror & Shaw, "Parallel
// random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of two 32x32->64
// multiplications with the round constants 0xD2511F53 / 0xCD9E8D57 and the
// Weyl key increments 0x9E3779B9 / 0xBB67AE85.
//
// Stream layout used by every sampler in this library (the oracle restates
// the same layout):
//   counter = { particle index i, sweep index, walker index, stream tag }
//   key     = { seed low 32 bits, seed high 32 bits }
// Tags: 0 = Metropolis moves, 1 = walker initialisation.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define LEMC_HD __host__ __device__ __forceinline__
#else
#define LEMC_HD inline
#endif

namespace lemc {

enum : uint32_t { kTagMove = 0u, kTagInit = 1u };

struct U4 {
  uint32_t x, y, z, w;
};

LEMC_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#if defined(__CUDA_ARCH__)
  lo = a * b;
  hi = __umulhi(a, b);
#else
  uint64_t p = uint64_t(a) * uint64_t(b);
  lo = uint32_t(p);
  hi = uint32_t(p >> 32);
#endif
}

LEMC_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c.x, hi0, lo0);
    mulhilo32(0xCD9E8D57u, c.z, hi1, lo1);
    U4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// Uniform in (0, 1), exactly representable in FP32: ((x >> 9) + 1/2) * 2^-23.
LEMC_HD float u01(uint32_t x) {
  return (float(x >> 9) + 0.5f) * 1.1920928955078125e-07f;
}

}  // namespace lemc
