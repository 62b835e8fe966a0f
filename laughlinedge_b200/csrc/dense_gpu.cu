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
