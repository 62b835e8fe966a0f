// FP64 accumulation of the weighted Gram matrices (SIMT, exact products).
//
//   G_h[a][b] += sum_w  W_h(w) * conj(v_a(w)) * v_b(w)
//
// for three weight planes h at once.  The FP32 inputs are widened to FP64
// before multiplying, so each product is exact and the only rounding is the
// FP64 summation.  This is the reference accumulation the tensor-core path is
// checked against, and the production path for LEMC_GRAM_FP64.
//
// Also here: the row sums of the reference estimator (LEMC_GUIDE_ROW),
// fg[a][b] = sum v_b/v_a, gg = sum |v_b/v_a|^2, and V-weighted sums, over the
// walkers guided by row a (reference em_spectrum.cu:99-115).
#include <cuda_runtime.h>

#include "lemc_internal.h"

namespace lemc {
namespace {

constexpr int TS = 16;     // 16 x 16 output tile
constexpr int CH = 64;     // walkers per staged chunk

__global__ void __launch_bounds__(256)
gram_simt_kernel(const float* __restrict__ V, int ldv, const float* __restrict__ rec_w, int ldw,
                 int W,
                 const GramJob* __restrict__ jobs, int n_splits, double* __restrict__ out0,
                 size_t plane0, double* __restrict__ out1, size_t plane1) {
  // plane[h] < 0 disables sum h
  const GramJob jb = jobs[blockIdx.x];
  const int split = blockIdx.y;
  const int per = (W + n_splits - 1) / n_splits;
  const int wbeg = split * per;
  const int wend = min(W, wbeg + per);

  __shared__ float are[TS][CH + 1], aim[TS][CH + 1], bre[TS][CH + 1], bim[TS][CH + 1];
  __shared__ float wt[3][CH];

  const int tx = threadIdx.x % TS, ty = threadIdx.x / TS;
  const int a = jb.a0 + ty, b = jb.b0 + tx;
  double acc[6] = {0, 0, 0, 0, 0, 0};

  for (int c0 = wbeg; c0 < wend; c0 += CH) {
    for (int e = threadIdx.x; e < TS * CH; e += blockDim.x) {
      const int r = e / CH, s = e % CH;
      const int wi = c0 + s;
      const bool ok = wi < wend;
      const int ra = jb.a0 + r, rb = jb.b0 + r;
      are[r][s] = (ok && ra < jb.Da) ? V[(size_t)(jb.row_a + ra) * ldv + wi] : 0.f;
      aim[r][s] = (ok && ra < jb.Da) ? V[(size_t)(jb.row_a + jb.Da + ra) * ldv + wi] : 0.f;
      bre[r][s] = (ok && rb < jb.Db) ? V[(size_t)(jb.row_b + rb) * ldv + wi] : 0.f;
      bim[r][s] = (ok && rb < jb.Db) ? V[(size_t)(jb.row_b + jb.Db + rb) * ldv + wi] : 0.f;
    }
    for (int e = threadIdx.x; e < 3 * CH; e += blockDim.x) {
      const int h = e / CH, s = e % CH;
      const int wi = c0 + s;
      float v = 0.f;
      const int pl = jb.plane[h];
      if (wi < wend && pl >= 0) {
        const float one = rec_w[(size_t)LEMC_W_ONE * ldw + wi];
        v = (pl == LEMC_W_ONE) ? one : one * rec_w[(size_t)pl * ldw + wi];
      }
      wt[h][s] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int s = 0; s < CH; ++s) {
      const double ar = are[ty][s], ai = aim[ty][s];
      const double br = bre[tx][s], bi = bim[tx][s];
      const double pr = ar * br + ai * bi;  // conj(a) * b
      const double pi = ar * bi - ai * br;
      const double w0 = wt[0][s], w1 = wt[1][s], w2 = wt[2][s];
      acc[0] += w0 * pr;
      acc[1] += w0 * pi;
      acc[2] += w1 * pr;
      acc[3] += w1 * pi;
      acc[4] += w2 * pr;
      acc[5] += w2 * pi;
    }
    __syncthreads();
  }
  if (a < jb.Da && b < jb.Db) {
    // three weight planes, each `plane` complex entries apart
    double* out = (jb.buf == 0) ? out0 : out1;
    const size_t plane = (jb.buf == 0) ? plane0 : plane1;
    if (!out) return;
    const size_t idx = 2 * ((size_t)jb.out + (size_t)a * jb.Db + b);
    atomicAdd(out + idx, acc[0]);
    atomicAdd(out + idx + 1, acc[1]);
    atomicAdd(out + idx + 2 * plane, acc[2]);
    atomicAdd(out + idx + 2 * plane + 1, acc[3]);
    atomicAdd(out + idx + 4 * plane, acc[4]);
    atomicAdd(out + idx + 4 * plane + 1, acc[5]);
  }
}

// Row sums of the reference estimator.  Block (row a, 32-column tile);
// 256 threads = 32 columns x 8 walker lanes.  Accumulators per (a, b):
//   [0,1] sum v_b/v_a      [2] sum |v_b/v_a|^2
//   [3,4] sum r2 v_b/v_a   [5,6] sum r4 v_b/v_a
//   [7,8] sum cos v_b/v_a  [9,10] sum sin v_b/v_a   [11,12] sum U v_b/v_a
// (cos/sin of the first angular probe)
constexpr int NROWACC = 13;

__global__ void __launch_bounds__(256)
row_accumulate_kernel(const float* __restrict__ V, int ldv, const float* __restrict__ rec_w,
                      int ldw, const int32_t* __restrict__ row_first, int D,
                      const int32_t* __restrict__ row_re, const int32_t* __restrict__ row_im,
                      double* __restrict__ acc_out) {
  const int a = blockIdx.x;
  const int b = blockIdx.y * 32 + (threadIdx.x & 31);
  const int lanew = threadIdx.x >> 5;
  const int w0 = row_first[a], w1 = row_first[a + 1];
  double acc[NROWACC];
#pragma unroll
  for (int q = 0; q < NROWACC; ++q) acc[q] = 0.0;
  if (b < D) {
    const size_t ra = row_re[a], ia = row_im[a], rb = row_re[b], ib = row_im[b];
    for (int w = w0 + lanew; w < w1; w += 8) {
      const double var = V[ra * ldv + w], vai = V[ia * ldv + w];
      const double vbr = V[rb * ldv + w], vbi = V[ib * ldv + w];
      const double den = var * var + vai * vai;
      // v_b / v_a = v_b conj(v_a) / |v_a|^2
      const double rr = (vbr * var + vbi * vai) / den;
      const double ri = (vbi * var - vbr * vai) / den;
      const double one = rec_w[(size_t)LEMC_W_ONE * ldw + w];
      const double h2 = rec_w[(size_t)LEMC_W_R2 * ldw + w];
      const double h4 = rec_w[(size_t)LEMC_W_R4 * ldw + w];
      const double hc = rec_w[(size_t)LEMC_W_PROBE0 * ldw + w];
      const double hs = rec_w[(size_t)(LEMC_W_PROBE0 + 1) * ldw + w];
      const double hu = rec_w[(size_t)LEMC_W_USER * ldw + w];
      acc[0] += one * rr;
      acc[1] += one * ri;
      acc[2] += one * (rr * rr + ri * ri);
      acc[3] += h2 * rr;
      acc[4] += h2 * ri;
      acc[5] += h4 * rr;
      acc[6] += h4 * ri;
      acc[7] += hc * rr;
      acc[8] += hc * ri;
      acc[9] += hs * rr;
      acc[10] += hs * ri;
      acc[11] += hu * rr;
      acc[12] += hu * ri;
    }
  }
  __shared__ double red[8][32][NROWACC + 1];
#pragma unroll
  for (int q = 0; q < NROWACC; ++q) red[lanew][threadIdx.x & 31][q] = acc[q];
  __syncthreads();
  if (lanew == 0 && b < D) {
    for (int q = 0; q < NROWACC; ++q) {
      double v = 0.0;
      for (int l = 0; l < 8; ++l) v += red[l][threadIdx.x & 31][q];
      acc_out[((size_t)a * D + b) * NROWACC + q] += v;
    }
  }
}

}  // namespace

int launch_gram_simt(const float* V, int ldv, const float* rec_w, int ldw, int W, const GramJob* jobs,
                     int n_jobs, int n_splits, double* out0, size_t plane0, double* out1,
                     size_t plane1, cudaStream_t st) {
  if (n_jobs <= 0) return LEMC_OK;
  dim3 grid(n_jobs, n_splits);
  gram_simt_kernel<<<grid, 256, 0, st>>>(V, ldv, rec_w, ldw, W, jobs, n_splits, out0, plane0, out1,
                                         plane1);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

int launch_row_accumulate(const float* V, int ldv, const float* rec_w, int ldw, int W,
                          const int32_t* row_first, int n_rows, int D, const int32_t* row_re,
                          const int32_t* row_im, double* acc, cudaStream_t st) {
  if (n_rows <= 0 || D <= 0) return LEMC_OK;
  (void)W;
  dim3 grid(n_rows, (D + 31) / 32);
  row_accumulate_kernel<<<grid, 256, 0, st>>>(V, ldv, rec_w, ldw, row_first, D, row_re, row_im,
                                              acc);
  return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

}  // namespace lemc
