// edgeMC: spectrum, metric, dynamic structure factor and excitation response
// of Laughlin edge states (drop-in for the reference's modules/edge_montecarlo.h,
// edgeMC::spectrum_compute :209-211, metric_compute :199-201, dsf_compute
// :220-222, excitationResponse_compute :233-237).
//
// Sampling runs on the B200 through liblemc.so: all basis rows of the
// requested sectors share one set of walkers (shared |Psi_m|^2 guide) and
// the S, H2, H4 Gram matrices are contracted on the tensor cores; set
// params.setEstimator(LEMC_GUIDE_ROW) for the reference's per-row guides.
#ifndef LAUGHLINEDGE_EDGE_MONTECARLO_H
#define LAUGHLINEDGE_EDGE_MONTECARLO_H

#include <type_traits>
#include <utility>
#include <vector>

#include "complex_numbers.h"
#include "integer_partitions.h"
#include "lemc_api_core.h"
#include "sys_params_bridge.h"
#include "tensors.h"

#if defined(__CUDACC__)
#include <cuda_runtime.h>
#endif

namespace edgeMC {
using namespace iparts;

inline std::vector<double> spectrum_compute(monteCarloParameters& params, int angular_momentum_sector,
                                            bool saveOutput = false, int fileNumber = 0) {
  return spectrum_compute_rt(lemc_api::physics_from_sys_params(), params, angular_momentum_sector,
                             saveOutput, fileNumber);
}

inline cmatrix<double> metric_compute(monteCarloParameters& params, int angular_momentum_sector,
                                      bool saveOutput = false, int fileNumber = 0) {
  return metric_compute_rt(lemc_api::physics_from_sys_params(), params, angular_momentum_sector,
                           saveOutput, fileNumber);
}

inline std::vector<std::pair<double, double>> dsf_compute(monteCarloParameters& params,
                                                          int angular_momentum_sector,
                                                          bool saveOutput = false,
                                                          int fileNumber = 0) {
  return dsf_compute_rt(lemc_api::physics_from_sys_params(), params, angular_momentum_sector,
                        saveOutput, fileNumber);
}

#if defined(__CUDACC__)
namespace detail {
// U(z) of every walker into the user weight plane; z points at the walker's
// N positions (complex<float> has the layout of the library's float2 pairs).
template <typename Func>
__global__ void apply_excitation_potential(Func U, const float* xy, float* out, int W, int N) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  complex<float>* z = reinterpret_cast<complex<float>*>(const_cast<float*>(xy)) + size_t(w) * N;
  out[w] = float(U(z));
}

template <typename Func>
struct PotentialHook {
  Func U;
  static int call(void* self, const float* xy, float* out, int W, int N, void* stream) {
    auto* h = static_cast<PotentialHook*>(self);
    apply_excitation_potential<<<(W + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        h->U, xy, out, W, N);
    return cudaPeekAtLastError() == cudaSuccess ? LEMC_OK : LEMC_ERR_CUDA;
  }
};
}  // namespace detail

// U is a __device__ (extended) lambda double(complex<float>*) evaluated on
// every walker after every measured sweep.  Writes the H, M, U and edge
// density Fourier matrices as .tsv files under
// ../output/N={N}_m={m}/ExternalExcitation/Statistics/ exactly like the
// reference (em_edgeResponse.tpp:540-594).
template <typename Func>
void excitationResponse_compute(monteCarloParameters& params, vector<int>& angular_momentum_sectors,
                                Func excitation_potential, int fileNumber) {
  static_assert(std::is_invocable_r_v<double, Func, complex<float>*>,
                "The excitation potential provided should be a __device__ function taking "
                "complex<float>* and returning double");
  detail::PotentialHook<Func> hook{excitation_potential};
  excitationResponse_compute_rt(lemc_api::physics_from_sys_params(), params,
                                angular_momentum_sectors.vec_pointer(),
                                angular_momentum_sectors.size(), &detail::PotentialHook<Func>::call,
                                &hook, fileNumber);
}
#endif

}  // namespace edgeMC

#endif
