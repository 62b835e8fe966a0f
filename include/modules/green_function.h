// greenFunctionMC: orbital occupation numbers <f_L| a^dagger_l a_l |f_R> of edge
// states (drop-in for the reference's modules/green_function.h:169-183).
#ifndef LAUGHLINEDGE_GREEN_FUNCTION_H
#define LAUGHLINEDGE_GREEN_FUNCTION_H

#include "integer_partitions.h"
#include "lemc_api_core.h"
#include "sys_params_bridge.h"
#include "tensors.h"

namespace greenFunctionMC {
using namespace iparts;

// Un-normalised occupation numbers (sum_l n_l = N per pair).
inline void occupation_numbers_compute(monteCarloParameters& params, int angular_momentum_sector,
                                       int fileNumber = 0) {
  occupation_numbers_compute_rt(lemc_api::physics_from_sys_params(), params,
                                angular_momentum_sector, nullptr, fileNumber);
}

// Normalised with the metric: n(L, R, l) * M(L, R).
inline void occupation_numbers_compute(monteCarloParameters& params, int angular_momentum_sector,
                                       cmatrix<double>& metric, int fileNumber = 0) {
  occupation_numbers_compute_rt(lemc_api::physics_from_sys_params(), params,
                                angular_momentum_sector, &metric, fileNumber);
}

}  // namespace greenFunctionMC

#endif
