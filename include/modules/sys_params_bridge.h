// Reads the compile-time constants of sys_params.h into the runtime Physics
// record of the B200 engine.
#ifndef LAUGHLINEDGE_SYS_PARAMS_BRIDGE_H
#define LAUGHLINEDGE_SYS_PARAMS_BRIDGE_H

#include "lemc_api_core.h"
#include "sys_params.h"

namespace lemc_api {
inline Physics physics_from_sys_params() {
  Physics p;
  p.N = sys_params::particlesNumber;
  p.m = sys_params::inverseFilling;
  p.conf_exponent = sys_params::confinementExponent;
  p.conf_strength = sys_params::confinementStrength;
  p.omega = sys_params::confinementOmega;
  p.kappa = sys_params::confinementKappa;
  p.ansatz_max_degree = sys_params::ansatzExtendedMaxDegree - 1;
  p.ansatz_max_partition = sys_params::ansatzMaxPartitionSize;
  p.ansatz_subspace = sys_params::ansatzSubspaceDimension;
  p.ansatz_multiplet = sys_params::ansatzMultipletSize;
  p.ansatz_max_L = sys_params::ansatzMaxAngularMomentum;
  return p;
}
}  // namespace lemc_api

#endif
