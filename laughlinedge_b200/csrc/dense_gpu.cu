// FP64 dense tail on the GPU: the generalized edge spectrum of one sector for
// many confinement strengths (the kappa sweep of the batched form).
//
// Reference: ges::generalizedEigenproblem (modules/eigensolver/
// generalized_eigenproblem.cpp:38-95) solves H c = E M c once per call on the
// host through a Cholesky of M.  Here M is factorised once per sector on the
// device by canonical orthogonalisation, which tolerates the near-singular
// metric of power-sum states at large dL:
//   M = U diag(m) U^H,  keep m_k > eps * max(m)  (rank r),  X = U_r diag(m_r^-1/2),
//   E_j = eig(X^H H_j X),  H_j = omega_j H2 + kappa_j H4   (all normalised).
// The eigen decompositions are cuSOLVER's Hermitian divide-and-conquer solver,
// the two products per strength cuBLAS ZGEMMs; everything stays in FP64.
//
// Row-major complex input is read as column-major, i.e. as the conjugate
// matrices; the generalized eigenvalues of (conj H, conj M) are those of (H, M).
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cmath>
#include <limits>
#include <vector>

#include "lemc_internal.h"

namespace lemc {
namespace {

// Normalise and Hermitise: X[a][b] = (Y[a][b] + conj(Y[b][a])) / 2 / sqrt(S_aa S_bb)
__global__ void normalise_kernel(int D, const double2* __restrict__ S, const double2* __restrict__ Y,
                                 double2* __restrict__ X) {
  const int a = blockIdx.y * blockDim.y + threadIdx.y;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= D || b >= D) return;
  const double n = sqrt(S[size_t(a) * D + a].x * S[size_t(b) * D + b].x);
  const double2 y = Y[size_t(a) * D + b], yt = Y[size_t(b) * D + a];
  X[size_t(a) * D + b] = make_double2(0.5 * (y.x + yt.x) / n, 0.5 * (y.y - yt.y) / n);
}

// column k of U (of the kept r) scaled by 1/sqrt(m), into X (D x r, column-major)
__global__ void scale_columns_kernel(int D, int r, int first, const double2* __restrict__ U,
                                     const double* __restrict__ m, double2* __restrict__ X) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (i >= D || k >= r) return;
  const double s = 1.0 / sqrt(m[first + k]);
  const double2 u = U[size_t(first + k) * D + i];
  X[size_t(k) * D + i] = make_double2(u.x * s, u.y * s);
}

__global__ void combine_kernel(int n, double w2, const double2* __restrict__ H2, double w4,
                               const double2* __restrict__ H4, double2* __restrict__ H) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  H[i] = make_double2(w2 * H2[i].x + w4 * H4[i].x, w2 * H2[i].y + w4 * H4[i].y);
}

struct Gpu {
  cusolverDnHandle_t sol = nullptr;
  cublasHandle_t blas = nullptr;
  std::vector<void*> bufs;
  ~Gpu() {
    for (void* p : bufs) cudaFree(p);
    if (blas) cublasDestroy(blas);
    if (sol) cusolverDnDestroy(sol);
  }
  template <class T>
  T* alloc(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
    bufs.push_back(p);
    return static_cast<T*>(p);
  }
};

}  // namespace
}  // namespace lemc

using namespace lemc;

extern "C" int lemc_geneig_sweep(int D, const double* S, const double* H2, const double* H4,
                                 const double* omega, const double* kappa, int n, double eps,
                                 double* evals, int* rank) {
  if (D <= 0 || n <= 0 || !S || !H2 || !H4 || !omega || !kappa || !evals || !(eps >= 0.0))
    return LEMC_ERR_ARG;
  for (int a = 0; a < D; ++a)
    if (!(S[2 * (size_t(a) * D + a)] > 0.0)) return LEMC_ERR_NUMERIC;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return LEMC_ERR_NODEVICE;
  }
  Gpu g;
  if (cusolverDnCreate(&g.sol) != CUSOLVER_STATUS_SUCCESS) return LEMC_ERR_CUDA;
  if (cublasCreate(&g.blas) != CUBLAS_STATUS_SUCCESS) return LEMC_ERR_CUDA;
  const size_t DD = size_t(D) * D;
  double2 *dS = g.alloc<double2>(DD), *dH2 = g.alloc<double2>(DD), *dH4 = g.alloc<double2>(DD);
  double2 *M = g.alloc<double2>(DD), *N2 = g.alloc<double2>(DD), *N4 = g.alloc<double2>(DD);
  double2 *X = g.alloc<double2>(DD), *H = g.alloc<double2>(DD), *T = g.alloc<double2>(DD);
  double2* A = g.alloc<double2>(DD);
  double* w = g.alloc<double>(D);
  int* info = g.alloc<int>(1);
  if (!dS || !dH2 || !dH4 || !M || !N2 || !N4 || !X || !H || !T || !A || !w || !info)
    return LEMC_ERR_CUDA;
  if (cudaMemcpy(dS, S, DD * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dH2, H2, DD * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dH4, H4, DD * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess)
    return LEMC_ERR_CUDA;
  const dim3 tb(16, 16), gb((D + 15) / 16, (D + 15) / 16);
  normalise_kernel<<<gb, tb>>>(D, dS, dS, M);
  normalise_kernel<<<gb, tb>>>(D, dS, dH2, N2);
  normalise_kernel<<<gb, tb>>>(D, dS, dH4, N4);
  if (cudaPeekAtLastError() != cudaSuccess) return LEMC_ERR_CUDA;

  // M = U diag(m) U^H (eigenvalues ascending, U overwrites M)
  int lwork = 0;
  if (cusolverDnZheevd_bufferSize(g.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, D,
                                  reinterpret_cast<cuDoubleComplex*>(M), D, w, &lwork) !=
      CUSOLVER_STATUS_SUCCESS)
    return LEMC_ERR_CUDA;
  double2* work = g.alloc<double2>(size_t(std::max(1, lwork)));
  if (!work) return LEMC_ERR_CUDA;
  if (cusolverDnZheevd(g.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, D,
                       reinterpret_cast<cuDoubleComplex*>(M), D, w,
                       reinterpret_cast<cuDoubleComplex*>(work), lwork, info) !=
      CUSOLVER_STATUS_SUCCESS)
    return LEMC_ERR_CUDA;
  std::vector<double> m(D);
  int h_info = 0;
  if (cudaMemcpy(m.data(), w, D * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return LEMC_ERR_CUDA;
  if (h_info != 0) return LEMC_ERR_NUMERIC;
  const double mmax = m[D - 1];
  if (!(mmax > 0.0)) return LEMC_ERR_NUMERIC;
  int first = 0;
  while (first < D && !(m[first] > eps * mmax)) ++first;
  const int r = D - first;
  if (rank) *rank = r;
  scale_columns_kernel<<<dim3((D + 127) / 128, r), 128>>>(D, r, first, M, w, X);
  if (cudaPeekAtLastError() != cudaSuccess) return LEMC_ERR_CUDA;

  int lwork2 = 0;
  if (cusolverDnZheevd_bufferSize(g.sol, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_LOWER, r,
                                  reinterpret_cast<cuDoubleComplex*>(A), r, w, &lwork2) !=
      CUSOLVER_STATUS_SUCCESS)
    return LEMC_ERR_CUDA;
  double2* work2 = g.alloc<double2>(size_t(std::max(1, lwork2)));
  if (!work2) return LEMC_ERR_CUDA;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  std::vector<double> e(r);
  for (int j = 0; j < n; ++j) {
    combine_kernel<<<(int(DD) + 255) / 256, 256>>>(int(DD), omega[j], N2, kappa[j], N4, H);
    if (cudaPeekAtLastError() != cudaSuccess) return LEMC_ERR_CUDA;
    // T = H X (D x r), A = X^H T (r x r)
    if (cublasZgemm(g.blas, CUBLAS_OP_N, CUBLAS_OP_N, D, r, D, &one,
                    reinterpret_cast<cuDoubleComplex*>(H), D, reinterpret_cast<cuDoubleComplex*>(X),
                    D, &zero, reinterpret_cast<cuDoubleComplex*>(T), D) != CUBLAS_STATUS_SUCCESS ||
        cublasZgemm(g.blas, CUBLAS_OP_C, CUBLAS_OP_N, r, r, D, &one,
                    reinterpret_cast<cuDoubleComplex*>(X), D, reinterpret_cast<cuDoubleComplex*>(T),
                    D, &zero, reinterpret_cast<cuDoubleComplex*>(A), r) != CUBLAS_STATUS_SUCCESS)
      return LEMC_ERR_CUDA;
    if (cusolverDnZheevd(g.sol, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_LOWER, r,
                         reinterpret_cast<cuDoubleComplex*>(A), r, w,
                         reinterpret_cast<cuDoubleComplex*>(work2), lwork2, info) !=
        CUSOLVER_STATUS_SUCCESS)
      return LEMC_ERR_CUDA;
    if (cudaMemcpy(e.data(), w, r * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      return LEMC_ERR_CUDA;
    if (h_info != 0) return LEMC_ERR_NUMERIC;
    for (int k = 0; k < D; ++k)
      evals[size_t(j) * D + k] = k < r ? e[k] : std::numeric_limits<double>::quiet_NaN();
  }
  return cudaDeviceSynchronize() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
}

// ---- time evolution in the S-orthonormal basis ------------------------------
// Reference: timeEvolution::edgeDensityResponse_compute (modules/dynamics/
// dynamics.cpp:24-53, :149-308) integrates M dC/dt = -i (H + f(t) U) C on the
// host with an adaptive Cash-Karp pair.  Here, on the GPU in FP64: with the
// canonical orthogonalisation X of M (X^H M X = 1), C = X y and
//   dy/dt = -i (H' + f(t) U') y,   H' = X^H H X - e I,  U' = X^H U X,
// e = tr(H')/r removed as a global phase (no observable depends on it, and it
// keeps h |H'| small).  Classical RK4 with h = save_step / substeps; every
// stage is one fused kernel (axpy + the two matrix-vector products, one warp
// per row).  Observables C^H rho_l C = y^H (X^H rho_l X) y and C^H M C = y^H y
// are recorded on the device at every save point.
namespace lemc {
namespace {

// row-major complex input -> column-major device layout (a transpose)
__global__ void to_colmajor_kernel(int D, const double2* __restrict__ in, double2* __restrict__ out) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < D && j < D) out[size_t(j) * D + i] = in[size_t(i) * D + j];
}

// column-major r x r -> row-major, minus e on the diagonal
__global__ void to_rowmajor_shift_kernel(int r, const double2* __restrict__ in, double e,
                                         double2* __restrict__ out) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < r && j < r) {
    double2 v = in[size_t(j) * r + i];
    if (i == j) v.x -= e;
    out[size_t(i) * r + j] = v;
  }
}

__global__ void diag_mean_kernel(int r, const double2* __restrict__ A, double* __restrict__ out) {
  __shared__ double s[256];
  double v = 0.0;
  for (int i = threadIdx.x; i < r; i += blockDim.x) v += A[size_t(i) * r + i].x;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0] / r;
}

__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}

// k_out = -i (H + f U) (y + a k_in), one warp per row; rows row-major.
__global__ void rk_stage_kernel(int r, const double2* __restrict__ Hr, const double2* __restrict__ Ur,
                                const double2* __restrict__ y, const double2* __restrict__ kin,
                                double a, double f, double2* __restrict__ kout) {
  const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= r) return;
  double2 sh = make_double2(0.0, 0.0), su = make_double2(0.0, 0.0);
  for (int j = lane; j < r; j += 32) {
    double2 v = y[j];
    if (kin) v = make_double2(fma(a, kin[j].x, v.x), fma(a, kin[j].y, v.y));
    sh = cfma(Hr[size_t(row) * r + j], v, sh);
    su = cfma(Ur[size_t(row) * r + j], v, su);
  }
  for (int o = 16; o > 0; o >>= 1) {
    sh.x += __shfl_xor_sync(0xffffffffu, sh.x, o);
    sh.y += __shfl_xor_sync(0xffffffffu, sh.y, o);
    su.x += __shfl_xor_sync(0xffffffffu, su.x, o);
    su.y += __shfl_xor_sync(0xffffffffu, su.y, o);
  }
  if (lane == 0) {
    const double2 t = make_double2(sh.x + f * su.x, sh.y + f * su.y);
    kout[row] = make_double2(t.y, -t.x);  // -i t
  }
}

__global__ void rk_update_kernel(int r, double h, double2* __restrict__ y, const double2* __restrict__ k1,
                                 const double2* __restrict__ k2, const double2* __restrict__ k3,
                                 const double2* __restrict__ k4) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r) return;
  const double c = h / 6.0;
  y[i].x += c * (k1[i].x + 2.0 * k2[i].x + 2.0 * k3[i].x + k4[i].x);
  y[i].y += c * (k1[i].y + 2.0 * k2[i].y + 2.0 * k3[i].y + k4[i].y);
}

// out[l] = y^H R_l y for the L row-major r x r matrices R, and nrm = y^H y;
// one block per l (block L computes the norm).
__global__ void observe_kernel(int r, int L, const double2* __restrict__ R, const double2* __restrict__ y,
                               double2* __restrict__ out, double* __restrict__ nrm) {
  __shared__ double2 red[256];
  const int l = blockIdx.x;
  double2 acc = make_double2(0.0, 0.0);
  if (l < L) {
    const double2* A = R + size_t(l) * r * r;
    for (int i = threadIdx.x; i < r; i += blockDim.x) {
      double2 row = make_double2(0.0, 0.0);
      for (int j = 0; j < r; ++j) row = cfma(A[size_t(i) * r + j], y[j], row);
      const double2 yc = make_double2(y[i].x, -y[i].y);
      acc = cfma(yc, row, acc);
    }
  } else {
    for (int i = threadIdx.x; i < r; i += blockDim.x) acc.x += y[i].x * y[i].x + y[i].y * y[i].y;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[threadIdx.x].x += red[threadIdx.x + o].x;
      red[threadIdx.x].y += red[threadIdx.x + o].y;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (l < L) out[l] = red[0];
    else *nrm = red[0].x;
  }
}

}  // namespace
}  // namespace lemc

extern "C" int lemc_evolve_device(int D, const double* M, const double* H, const double* U, int L,
                                  const double* rho, lemc_profile_fn f, void* user,
                                  double end_time, double save_step, int substeps, double eps,
                                  double* out, double* norms, int* n_save, int* rank) {
  if (D <= 0 || !M || !H || !U || L < 0 || (L > 0 && !rho) || !(save_step > 0) ||
      !(end_time > 0) || substeps < 1 || !(eps >= 0.0))
    return LEMC_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return LEMC_ERR_NODEVICE;
  }
  const int ns = int(std::ceil(end_time / save_step));
  if (n_save) *n_save = ns;
  Gpu g;
  if (cusolverDnCreate(&g.sol) != CUSOLVER_STATUS_SUCCESS) return LEMC_ERR_CUDA;
  if (cublasCreate(&g.blas) != CUBLAS_STATUS_SUCCESS) return LEMC_ERR_CUDA;
  const size_t DD = size_t(D) * D;
  const int NM = 3 + L;  // M, H, U, rho_0..rho_{L-1}
  double2* raw = g.alloc<double2>(DD);
  double2* cm = g.alloc<double2>(DD * NM);  // column-major copies
  double2* X = g.alloc<double2>(DD);
  double2* T = g.alloc<double2>(DD);
  double2* P = g.alloc<double2>(DD);
  double* w = g.alloc<double>(D);
  int* info = g.alloc<int>(1);
  if (!raw || !cm || !X || !T || !P || !w || !info) return LEMC_ERR_CUDA;
  const dim3 tb(16, 16), gb((D + 15) / 16, (D + 15) / 16);
  for (int q = 0; q < NM; ++q) {
    const double* src = q == 0 ? M : q == 1 ? H : q == 2 ? U : rho + size_t(2) * DD * (q - 3);
    if (cudaMemcpy(raw, src, DD * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess)
      return LEMC_ERR_CUDA;
    to_colmajor_kernel<<<gb, tb>>>(D, raw, cm + DD * q);
  }
  // canonical orthogonalisation of M (column-major copy 0 is overwritten by U)
  if (cudaMemcpy(P, cm, DD * sizeof(double2), cudaMemcpyDeviceToDevice) != cudaSuccess)
    return LEMC_ERR_CUDA;
  int lwork = 0;
  if (cusolverDnZheevd_bufferSize(g.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, D,
                                  reinterpret_cast<cuDoubleComplex*>(P), D, w, &lwork) !=
      CUSOLVER_STATUS_SUCCESS)
    return LEMC_ERR_CUDA;
  double2* work = g.alloc<double2>(size_t(std::max(1, lwork)));
  if (!work) return LEMC_ERR_CUDA;
  if (cusolverDnZheevd(g.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, D,
                       reinterpret_cast<cuDoubleComplex*>(P), D, w,
                       reinterpret_cast<cuDoubleComplex*>(work), lwork, info) != CUSOLVER_STATUS_SUCCESS)
    return LEMC_ERR_CUDA;
  std::vector<double> m(D);
  int h_info = 0;
  if (cudaMemcpy(m.data(), w, D * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return LEMC_ERR_CUDA;
  if (h_info != 0 || !(m[D - 1] > 0.0)) return LEMC_ERR_NUMERIC;
  int first = 0;
  while (first < D && !(m[first] > eps * m[D - 1])) ++first;
  const int r = D - first;
  if (rank) *rank = r;
  scale_columns_kernel<<<dim3((D + 127) / 128, r), 128>>>(D, r, first, P, w, X);
  // projected matrices, row-major on the device: H', U', rho'_l
  const size_t RR = size_t(r) * r;
  double2* Hr = g.alloc<double2>(RR);
  double2* Ur = g.alloc<double2>(RR);
  double2* Rr = g.alloc<double2>(RR * std::max(1, L));
  double2* A = g.alloc<double2>(RR);
  double* emean = g.alloc<double>(1);
  double2 *y = g.alloc<double2>(r), *k1 = g.alloc<double2>(r), *k2 = g.alloc<double2>(r),
          *k3 = g.alloc<double2>(r), *k4 = g.alloc<double2>(r);
  double2* obs = g.alloc<double2>(size_t(ns) * std::max(1, L));
  double* nrm = g.alloc<double>(ns);
  if (!Hr || !Ur || !Rr || !A || !emean || !y || !k1 || !k2 || !k3 || !k4 || !obs || !nrm)
    return LEMC_ERR_CUDA;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  auto project = [&](const double2* Bcm) -> bool {  // A = X^H B X (column-major r x r)
    return cublasZgemm(g.blas, CUBLAS_OP_N, CUBLAS_OP_N, D, r, D, &one,
                       reinterpret_cast<const cuDoubleComplex*>(Bcm), D,
                       reinterpret_cast<const cuDoubleComplex*>(X), D, &zero,
                       reinterpret_cast<cuDoubleComplex*>(T), D) == CUBLAS_STATUS_SUCCESS &&
           cublasZgemm(g.blas, CUBLAS_OP_C, CUBLAS_OP_N, r, r, D, &one,
                       reinterpret_cast<const cuDoubleComplex*>(X), D,
                       reinterpret_cast<const cuDoubleComplex*>(T), D, &zero,
                       reinterpret_cast<cuDoubleComplex*>(A), r) == CUBLAS_STATUS_SUCCESS;
  };
  const dim3 gr((r + 15) / 16, (r + 15) / 16);
  if (!project(cm + DD)) return LEMC_ERR_CUDA;
  diag_mean_kernel<<<1, 256>>>(r, A, emean);
  double e = 0.0;
  if (cudaMemcpy(&e, emean, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return LEMC_ERR_CUDA;
  to_rowmajor_shift_kernel<<<gr, tb>>>(r, A, e, Hr);
  if (!project(cm + 2 * DD)) return LEMC_ERR_CUDA;
  to_rowmajor_shift_kernel<<<gr, tb>>>(r, A, 0.0, Ur);
  for (int l = 0; l < L; ++l) {
    if (!project(cm + DD * (3 + l))) return LEMC_ERR_CUDA;
    to_rowmajor_shift_kernel<<<gr, tb>>>(r, A, 0.0, Rr + RR * l);
  }
  // y(0) = X^H M e_0 (C(0) = e_0)
  if (cublasZgemv(g.blas, CUBLAS_OP_C, D, r, &one, reinterpret_cast<const cuDoubleComplex*>(X), D,
                  reinterpret_cast<const cuDoubleComplex*>(cm), 1, &zero,
                  reinterpret_cast<cuDoubleComplex*>(y), 1) != CUBLAS_STATUS_SUCCESS)
    return LEMC_ERR_CUDA;
  if (cudaPeekAtLastError() != cudaSuccess) return LEMC_ERR_CUDA;
  // profile values at every stage time, evaluated on the host
  const double h = save_step / substeps;
  const size_t nsteps = size_t(ns > 1 ? ns - 1 : 0) * substeps;
  std::vector<double> fv(3 * nsteps);
  for (size_t k = 0; k < nsteps; ++k) {
    const double t = double(k) * h;
    fv[3 * k] = f ? f(t, user) : 0.0;
    fv[3 * k + 1] = f ? f(t + 0.5 * h, user) : 0.0;
    fv[3 * k + 2] = f ? f(t + h, user) : 0.0;
  }
  const int wpb = 8, sblocks = (r + wpb - 1) / wpb, ublocks = (r + 255) / 256;
  observe_kernel<<<L + 1, 256>>>(r, L, Rr, y, obs, nrm);
  size_t k = 0;
  for (int s = 1; s < ns; ++s) {
    for (int q = 0; q < substeps; ++q, ++k) {
      rk_stage_kernel<<<sblocks, 32 * wpb>>>(r, Hr, Ur, y, nullptr, 0.0, fv[3 * k], k1);
      rk_stage_kernel<<<sblocks, 32 * wpb>>>(r, Hr, Ur, y, k1, 0.5 * h, fv[3 * k + 1], k2);
      rk_stage_kernel<<<sblocks, 32 * wpb>>>(r, Hr, Ur, y, k2, 0.5 * h, fv[3 * k + 1], k3);
      rk_stage_kernel<<<sblocks, 32 * wpb>>>(r, Hr, Ur, y, k3, h, fv[3 * k + 2], k4);
      rk_update_kernel<<<ublocks, 256>>>(r, h, y, k1, k2, k3, k4);
    }
    observe_kernel<<<L + 1, 256>>>(r, L, Rr, y, obs + size_t(s) * std::max(1, L), nrm + s);
  }
  if (cudaPeekAtLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
    return LEMC_ERR_CUDA;
  if (L > 0 && out) {
    std::vector<double2> all(size_t(ns) * L);
    if (cudaMemcpy(all.data(), obs, all.size() * sizeof(double2), cudaMemcpyDeviceToHost) != cudaSuccess)
      return LEMC_ERR_CUDA;
    for (size_t q = 0; q < all.size(); ++q) {
      out[2 * q] = all[q].x;
      out[2 * q + 1] = all[q].y;
    }
  }
  if (norms && cudaMemcpy(norms, nrm, ns * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return LEMC_ERR_CUDA;
  return LEMC_OK;
}

// Edge density on an angular grid from its Fourier components (reference
// observer::edgeDensity_reconstruct, dynamics.cpp:110-125, gives the
// components <rho_l>(t) = C^H rho_l C; the density itself is
// n(theta) = (1/2pi) [<rho_0> + 2 Re sum_{l>0} e^{-i l theta} <rho_l>]).
namespace lemc {
namespace {

__global__ void density_grid_kernel(int L, const int* __restrict__ ls, int n_times,
                                    const double2* __restrict__ rho, const double2* __restrict__ ref,
                                    int n_theta, double* __restrict__ out) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = blockIdx.y;
  if (g >= n_theta || t >= n_times) return;
  const double theta = 2.0 * M_PI * double(g) / double(n_theta);
  double acc = 0.0;
  for (int q = 0; q < L; ++q) {
    const double2 r = rho[size_t(t) * L + q];
    const double2 r0 = ref[q];
    const double dr = r.x - r0.x, di = r.y - r0.y;
    const int l = ls[q];
    if (l == 0) {
      acc += dr;
    } else {
      double s, c;
      sincos(double(l) * theta, &s, &c);
      acc += 2.0 * (dr * c + di * s);  // 2 Re(e^{-i l theta} (dr + i di))
    }
  }
  out[size_t(t) * n_theta + g] = acc / (2.0 * M_PI);
}

}  // namespace
}  // namespace lemc

extern "C" int lemc_edge_density_grid(int L, const int32_t* l, int n_times, const double* rho_t,
                                      const double* rho_ref, int n_theta, double* out) {
  using namespace lemc;
  if (L <= 0 || !l || n_times <= 0 || !rho_t || n_theta <= 0 || !out) return LEMC_ERR_ARG;
  for (int q = 0; q < L; ++q)
    if (l[q] < 0) return LEMC_ERR_ARG;
  int* d_l = nullptr;
  double2 *d_rho = nullptr, *d_ref = nullptr;
  double* d_out = nullptr;
  int st = LEMC_OK;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && st == LEMC_OK) st = LEMC_ERR_CUDA;
    return st == LEMC_OK;
  };
  const size_t nr = size_t(n_times) * L;
  if (ok(cudaMalloc(&d_l, sizeof(int) * L)) && ok(cudaMalloc(&d_rho, sizeof(double2) * nr)) &&
      ok(cudaMalloc(&d_ref, sizeof(double2) * L)) &&
      ok(cudaMalloc(&d_out, sizeof(double) * size_t(n_times) * n_theta)) &&
      ok(cudaMemcpy(d_l, l, sizeof(int) * L, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(d_rho, rho_t, sizeof(double2) * nr, cudaMemcpyHostToDevice)) &&
      ok(cudaMemcpy(d_ref, rho_ref ? rho_ref : rho_t, sizeof(double2) * L, cudaMemcpyHostToDevice))) {
    const dim3 grid((n_theta + 127) / 128, n_times);
    density_grid_kernel<<<grid, 128>>>(L, d_l, n_times, d_rho, d_ref, n_theta, d_out);
    if (ok(cudaGetLastError()))
      ok(cudaMemcpy(out, d_out, sizeof(double) * size_t(n_times) * n_theta, cudaMemcpyDeviceToHost));
  }
  cudaFree(d_l);
  cudaFree(d_rho);
  cudaFree(d_ref);
  cudaFree(d_out);
  return st;
}
