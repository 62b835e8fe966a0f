// timeEvolution: edge-density response of the Laughlin droplet to a
// space-time dependent excitation (drop-in for the reference's
// modules/dynamics.h:75-79).  Reads the matrices written by
// edgeMC::excitationResponse_compute and integrates in FP64.
#ifndef LAUGHLINEDGE_DYNAMICS_H
#define LAUGHLINEDGE_DYNAMICS_H

#include <functional>
#include <vector>

#include "lemc_api_core.h"

namespace timeEvolution {

inline void edgeDensityResponse_compute(unsigned particlesNumber, unsigned inverseFilling,
                                        std::vector<int> angular_momenta,
                                        std::function<double(double)> temporal_excitation_profile,
                                        double end_time, double save_step, int fileNumber = 0) {
  edgeDensityResponse_compute_rt(particlesNumber, inverseFilling, std::move(angular_momenta),
                                 std::move(temporal_excitation_profile), end_time, save_step,
                                 fileNumber);
}

}  // namespace timeEvolution

#endif
