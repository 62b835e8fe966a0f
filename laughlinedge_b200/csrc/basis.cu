// Basis build: v_lambda = prod_j p_{lambda_j} for every basis row of the
// selected sectors, one thread per (walker sample, program segment)
// (reference: symPol_construct and the ek/ekr tables,
// modules/edge_mc/em_markovchain.cu:120-183).
//
// The rows are produced by a depth-first program over the partition trie:
// node t multiplies its parent (the node one level up on the DFS stack) by a
// single power sum, so every v costs one complex multiplication.  The program
// is cut at depth-1 nodes into segments that run as separate blocks
// (blockIdx.y), so a launch holds several threads per walker.  A block first
// copies its walkers' p_0..p_K into shared memory; each node then reads its p
// from there one node ahead.  A node's parent is the previous node on a
// descent (kept in a register); on a backtrack it is an ancestor whose value
// sits on the thread's stack in shared memory, and that load is also issued
// one node ahead.  Outputs are written as FP32 planes V[row][w] (Re rows,
// then Im rows of each sector), walker-contiguous so that consecutive threads
// write consecutive addresses, each multiplied by its row's range factor when
// the program carries one (the sampling context sets them so that the values
// of every state are O(1) on a geometric mean over walkers).  Segment-0 blocks
// also reduce Re/Im p_1..p_4 into the walker-mean series used for the
// integrated autocorrelation time.
#include <cuda_runtime.h>

#include "lemc_internal.h"

namespace lemc {
namespace {

constexpr int kBasisThreads = 128;

// P complex values of P consecutive walkers, kept together in shared memory
// so that one vector access moves all of them.
template <int P>
struct Vals {
  float2 c[P];
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

template <int P>
__device__ __forceinline__ Vals<P> vload(const float2* p) {
  Vals<P> r;
  if constexpr (P == 1) {
    r.c[0] = *p;
  } else {
    const float4 q = *reinterpret_cast<const float4*>(p);
    r.c[0] = make_float2(q.x, q.y);
    r.c[1] = make_float2(q.z, q.w);
  }
  return r;
}

template <int P>
__device__ __forceinline__ void vstore(float2* p, const Vals<P>& v) {
  if constexpr (P == 1)
    *p = v.c[0];
  else
    *reinterpret_cast<float4*>(p) = make_float4(v.c[0].x, v.c[0].y, v.c[1].x, v.c[1].y);
}

template <int P>
__device__ __forceinline__ Vals<P> vmul(const Vals<P>& a, const Vals<P>& b) {
  Vals<P> r;
#pragma unroll
  for (int i = 0; i < P; ++i) r.c[i] = cmul(a.c[i], b.c[i]);
  return r;
}

// Re (part 0) or Im (part 1) of the P values to P consecutive floats of a row
template <int P>
__device__ __forceinline__ void row_store(float* p, const Vals<P>& v, bool im) {
  if constexpr (P == 1)
    *p = im ? v.c[0].y : v.c[0].x;
  else
    *reinterpret_cast<float2*>(p) = im ? make_float2(v.c[0].y, v.c[1].y)
                                       : make_float2(v.c[0].x, v.c[1].x);
}

// One thread per P consecutive walkers and program segment (blockIdx.y).
template <int P>
__global__ void __launch_bounds__(kBasisThreads)
basis_kernel(const float2* __restrict__ rec_p, int W, int K, float pN, BasisProgram prog,
             float* __restrict__ V, int ldv, double* __restrict__ series,
             const uint32_t* __restrict__ series_idx) {
  // Shared memory, one column of P values per thread (no thread reads
  // another's column):
  //   ps[k][thread]  = p_k of the thread's walkers, k = 0..K (p_0 = N)
  //   stk[d][thread] = value of the depth-d node on the current DFS path, d < K
  // followed by the block's program segment and the two nodes after it, and
  // their range factors.
  extern __shared__ float4 smem_basis[];
  constexpr int T = kBasisThreads;
  constexpr int R = T * P;  // row stride in float2
  const int tid = threadIdx.x;
  float2* ps = reinterpret_cast<float2*>(smem_basis) + tid * P;
  float2* stk = ps + (K + 1) * R;
  const int w0 = (blockIdx.x * T + tid) * P;  // W is a multiple of P
  const bool live = w0 < W;
  const int t0 = __ldg(prog.seg_dev + blockIdx.y);
  const int t1 = __ldg(prog.seg_dev + blockIdx.y + 1);
  int4* snodes = reinterpret_cast<int4*>(smem_basis) + (2 * K + 1) * R / 2;
  float* sscale = reinterpret_cast<float*>(snodes + prog.max_seg + 2);
  const bool scaled = prog.node_scale != nullptr;
  for (int i = tid; i < t1 - t0 + 2; i += T) {
    snodes[i] = __ldg(reinterpret_cast<const int4*>(prog.nodes) + t0 + i);
    if (scaled) sscale[i] = __ldg(prog.node_scale + t0 + i);
  }
  Vals<P> v0;
#pragma unroll
  for (int i = 0; i < P; ++i) v0.c[i] = make_float2(pN, 0.f);
  vstore<P>(ps, v0);
  for (int k = 1; k <= K; ++k) {
    Vals<P> q;
    if (live) {
      q = vload<P>(rec_p + (size_t)(k - 1) * W + w0);
    } else {
#pragma unroll
      for (int i = 0; i < P; ++i) q.c[i] = make_float2(0.f, 0.f);
    }
    vstore<P>(ps + k * R, q);
  }

  if (series && blockIdx.y == 0) {
    if (series_idx) series += 8 * size_t(*series_idx);
    __shared__ double red[T / 32][8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int k = 1 + (c >> 1);
      double v = 0.0;
      if (k <= K) {
        const Vals<P> pk = vload<P>(ps + k * R);
#pragma unroll
        for (int i = 0; i < P; ++i) v += (c & 1) ? pk.c[i].y : pk.c[i].x;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if ((tid & 31) == 0) red[tid >> 5][c] = v;
    }
    __syncthreads();
    if (tid < 8) {
      double v = 0.0;
      for (int q = 0; q < T / 32; ++q) v += red[q][tid];
      atomicAdd(&series[tid], v);
    }
  }
  __syncthreads();  // the program segment is in shared memory
  if (!live) return;

  // node = {depth, part, row_re, row_im}; the device array ends with two
  // sentinel nodes {0, 0, -1, -1}, so nodes t + 1 and t + 2 always exist.
  const int4* nodes = snodes - t0;
  const float* nscale = sscale - t0;
  float* __restrict__ Vw = V + w0;
  Vals<P> one;
#pragma unroll
  for (int i = 0; i < P; ++i) one.c[i] = make_float2(1.f, 0.f);
  // Software pipeline over three node slots that rotate roles, so no values
  // are copied between iterations.  At step t the slot of node t holds
  // (node, parent value, p); the slot of node t + 1 gets its p and, on a
  // backtrack, its parent's value from the stack; node t + 2 is loaded.
  int4 n0 = nodes[t0], n1 = nodes[t0 + 1], n2;
  Vals<P> a0 = one, a1, a2;  // segments start at depth 1: parent value 1
  Vals<P> b0 = vload<P>(ps + n0.y * R), b1, b2;
  auto step = [&](const int t, const int4& nd, const Vals<P>& a, const Vals<P>& b,
                  const int4& nx, Vals<P>& ax, Vals<P>& bx, int4& nn) {
    nn = nodes[t + 2];
    bx = vload<P>(ps + nx.y * R);
    const bool descend = nx.x == nd.x + 1;  // nx is this node's first child
    Vals<P> an = one;
    if (!descend && nx.x > 1) an = vload<P>(stk + (nx.x - 1) * R);  // an ancestor of this node
    const Vals<P> v = vmul<P>(a, b);
    if (descend) vstore<P>(stk + nd.x * R, v);
    if (nd.z >= 0) {
      Vals<P> out = v;
      if (scaled) {
        const float sc = nscale[t];
#pragma unroll
        for (int i = 0; i < P; ++i) out.c[i] = make_float2(sc * v.c[i].x, sc * v.c[i].y);
      }
      row_store<P>(Vw + (size_t)nd.z * ldv, out, false);
      row_store<P>(Vw + (size_t)nd.w * ldv, out, true);
    }
    ax = descend ? v : an;
  };
  for (int t = t0; t < t1; t += 3) {
    step(t, n0, a0, b0, n1, a1, b1, n2);
    if (t + 1 >= t1) break;
    step(t + 1, n1, a1, b1, n2, a2, b2, n0);
    if (t + 2 >= t1) break;
    step(t + 2, n2, a2, b2, n0, a0, b0, n1);
  }
}

template <int P>
int launch_p(const float2* rec_p, int W, int K, int N, const BasisProgram& prog, float* V,
             int ldv, double* series, const uint32_t* series_idx, cudaStream_t st) {
  const size_t smem = sizeof(float2) * size_t(2 * K + 1) * kBasisThreads * P +
                      (sizeof(BasisNode) + sizeof(float)) * size_t(prog.max_seg + 2);
  if (smem > 40 * 1024) {  // the static reduction buffer shares the 48 KiB default
    if (cudaFuncSetAttribute(basis_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(smem)) != cudaSuccess)
      return LEMC_ERR_CUDA;
  }
  // segment-major block order: the blocks in flight write the same rows of V
  // at neighbouring walkers
  const int per_block = kBasisThreads * P;
  const dim3 grid((W + per_block - 1) / per_block, prog.n_seg);
  basis_kernel<P><<<grid, kBasisThreads, smem, st>>>(rec_p, W, K, float(N), prog, V, ldv,
                                                     series, series_idx);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

// USER plane of a multipole potential U = amp sum_i r_i^k cos(k theta_i)
// = amp R^k Re p_k, from the recorded (z/R)^k power sums.
__global__ void multipole_plane_kernel(const float2* __restrict__ rec_p, int W, int k, float scale,
                                       float* __restrict__ plane) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w < W) plane[w] = scale * rec_p[size_t(k - 1) * W + w].x;
}

}  // namespace

int launch_multipole_plane(const float2* rec_p, int W, int K, int k, double scale, float* plane,
                           cudaStream_t st) {
  if (k < 1 || k > K || W <= 0) return LEMC_ERR_ARG;
  multipole_plane_kernel<<<(W + 255) / 256, 256, 0, st>>>(rec_p, W, k, float(scale), plane);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

int launch_basis(const float2* rec_p, int W, int K, int N, const BasisProgram& prog, float* V,
                 int ldv, double* series, const uint32_t* series_idx, cudaStream_t st) {
  if (K > kMaxDegree || prog.max_part > K || prog.max_depth > K || prog.n_seg < 1 ||
      prog.n_seg > kMaxBasisSegments)
    return LEMC_ERR_CAPACITY;
  // two walkers per thread when the vector accesses are aligned: 16-byte p_k
  // pairs, 8-byte pairs of V entries
  const bool pairs = W % 2 == 0 && ldv % 2 == 0 &&
                     reinterpret_cast<uintptr_t>(rec_p) % 16 == 0 &&
                     reinterpret_cast<uintptr_t>(V) % 8 == 0;
  return pairs ? launch_p<2>(rec_p, W, K, N, prog, V, ldv, series, series_idx, st)
               : launch_p<1>(rec_p, W, K, N, prog, V, ldv, series, series_idx, st);
}

}  // namespace lemc
