// Basis build: v_lambda = prod_j p_{lambda_j} for every basis row of the
// selected sectors, one thread per walker sample (reference: symPol_construct
// and the ek/ekr tables, modules/edge_mc/em_markovchain.cu:120-183).
//
// The rows are produced by a depth-first program over the partition trie:
// node t multiplies its parent (the node one level up on the DFS stack) by a
// single power sum, so every v costs one complex multiplication.  Outputs are
// written as FP32 planes V[row][w] (Re rows, then Im rows of each sector),
// walker-contiguous so that consecutive threads write consecutive addresses.
// The same pass reduces Re/Im p_1..p_4 over the block into the walker-mean
// series used for the integrated autocorrelation time.
#include <cuda_runtime.h>

#include "lemc_internal.h"

namespace lemc {
namespace {

__global__ void __launch_bounds__(256)
basis_kernel(const float2* __restrict__ rec_p, int W, int K, float pN,
             const BasisNode* __restrict__ prog, int n_nodes, float* __restrict__ V, int ldv,
             double* __restrict__ series, const uint32_t* __restrict__ series_idx) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = w < W;
  float2 p[kMaxDegree + 1];
  p[0] = make_float2(pN, 0.f);
#pragma unroll
  for (int k = 0; k < kMaxDegree; ++k)
    p[k + 1] = (live && k < K) ? rec_p[(size_t)k * W + w] : make_float2(0.f, 0.f);

  if (series) {
    if (series_idx) series += 8 * size_t(*series_idx);
    __shared__ double red[8][8];
    float o[8];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      o[2 * k] = (k < K) ? p[k + 1].x : 0.f;
      o[2 * k + 1] = (k < K) ? p[k + 1].y : 0.f;
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      double v = o[c];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
      double v = 0.0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) v += red[q][threadIdx.x];
      atomicAdd(&series[threadIdx.x], v);
    }
  }
  if (!live) return;

  float2 stack[kMaxDegree + 2];
  stack[0] = make_float2(1.f, 0.f);
  for (int t = 0; t < n_nodes; ++t) {
    const BasisNode nd = prog[t];
    const float2 a = stack[nd.depth - 1];
    const float2 b = p[nd.part];
    const float2 v = make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
    stack[nd.depth] = v;
    if (nd.row_re >= 0) {
      V[(size_t)nd.row_re * ldv + w] = v.x;
      V[(size_t)nd.row_im * ldv + w] = v.y;
    }
  }
}

}  // namespace

int launch_basis(const float2* rec_p, int W, int K, int N, const BasisNode* prog, int n_nodes,
                 float* V, int ldv, double* series, const uint32_t* series_idx, cudaStream_t st) {
  if (K > kMaxDegree) return LEMC_ERR_CAPACITY;
  const int threads = 256;
  const int blocks = (W + threads - 1) / threads;
  basis_kernel<<<blocks, threads, 0, st>>>(reinterpret_cast<const float2*>(rec_p), W, K,
                                           float(N), prog, n_nodes, V, ldv, series,
                                           series_idx);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

}  // namespace lemc
