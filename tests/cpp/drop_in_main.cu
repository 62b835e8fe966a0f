// Drop-in check: the usage snippets of the reference's main.cu (spectrum, DSF,
// excitation response with a device lambda, time evolution, occupation
// numbers) compiled unchanged against include/modules and linked to
// liblemc.so.  Prints machine-readable lines "KEY value ..." for the tests.
#include <cmath>
#include <cstdio>
#include <vector>

#include "complex_numbers.h"
#include "dynamics.h"
#include "edge_montecarlo.h"
#include "green_function.h"
#include "sys_params.h"
#include "tensors.h"

int main() {
  // SPECTRUM (reference main.cu:37-52)
  {
    int angularMomentumSector = 3;
    edgeMC::monteCarloParameters simulationParameters;
    simulationParameters.setMCSamples(800);
    simulationParameters.setBurnIn(300);
    simulationParameters.setSeed(7);
    simulationParameters.setRandomStep(0.3f);
    simulationParameters.setAcceptanceBisectionParams(100, 0.5f, 1.0f);
    std::vector<double> evals = edgeMC::spectrum_compute(simulationParameters, angularMomentumSector, true, 0);
    std::printf("SPECTRUM");
    for (double e : evals) std::printf(" %.10f", e);
    std::printf("\n");
  }
  // DSF (reference main.cu:55-66)
  {
    edgeMC::monteCarloParameters simulationParameters;
    simulationParameters.setMCSamples(800);
    simulationParameters.setBurnIn(300);
    simulationParameters.setSeed(11);
    simulationParameters.setRandomStep(0.3f);
    simulationParameters.setAcceptanceBisectionParams(100, 0.5f, 1.0f);
    std::vector<std::pair<double, double>> e_dsf = edgeMC::dsf_compute(simulationParameters, 2, true, 0);
    std::printf("DSF");
    for (auto elem : e_dsf) std::printf(" %.10f %.10e", elem.first, elem.second);
    std::printf("\n");
  }
  // EXCITATION MATRIX ELEMENTS AND DYNAMICS (reference main.cu:69-107)
  {
    auto spatial_profile = [] __device__(complex<float>* position) {
      double U = 0;
      for (int i = 0; i < sys_params::particlesNumber; i++) {
        U += pow(re(position[i]) / sys_params::RCl, 2);
      }
      return U;
    };
    vector<int> angular_momenta = {0, 2, 4};
    edgeMC::monteCarloParameters simulationParameters;
    simulationParameters.setMCSamples(600);
    simulationParameters.setBurnIn(300);
    simulationParameters.setSeed(13);
    simulationParameters.setRandomStep(0.3f);
    simulationParameters.setAcceptanceBisectionParams(100, 0.5f, 1.0f);
    edgeMC::excitationResponse_compute(simulationParameters, angular_momenta, spatial_profile, 0);
    double TMax = 40;
    double save_step = 0.5;
    double excitation_strength = 0.1;
    double t0 = 10.;
    double tau = 3.;
    auto temporal_profile = [&](double t) {
      double z = (t - t0) / tau;
      return excitation_strength * std::exp(-z * z);
    };
    timeEvolution::edgeDensityResponse_compute(sys_params::particlesNumber, sys_params::inverseFilling,
                                               {0, 2, 4}, temporal_profile, TMax, save_step);
    std::printf("DYNAMICS done\n");
  }
  // OCCUPATION NUMBERS (reference main.cu:110-121)
  {
    greenFunctionMC::monteCarloParameters sp2;
    sp2.setMCSamples(400);
    sp2.setBurnIn(200);
    sp2.setSeed(17);
    sp2.setRandomStep(0.3f);
    sp2.setAcceptanceBisectionParams(100, 0.5f, 1.0f);
    greenFunctionMC::occupation_numbers_compute(sp2, 0, 0);
    std::printf("OCCUPATION done\n");
  }
  return 0;
}
