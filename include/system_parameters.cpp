// Generates ./modules/sys_params.h (run from the directory that holds modules/).
//
// Same constants and names as the reference's generator
// (system_parameters.cpp:9-66): particle number, filling, the single power-law
// confinement strength * sum (r/R_cl)^exponent, the classical radius and the
// ansatz capacity bounds.  Added: the two-term confinement
// V = confinementOmega r^2 + confinementKappa r^4 (l_B units) that the B200
// engine samples; leave both at 0 to use the power law.  Values are printed
// with full precision (max_digits10) instead of 6 decimals.
#include <cmath>
#include <fstream>
#include <iomanip>
#include <limits>

int particlesNumber = 8;        // N
int inverseFilling = 3;         // nu = 1/m

int confinementExponent = 2;    // V = confinementStrength * sum (r / R_cl)^exponent
double confinementStrength = 1.;
double confinementOmega = 1e-2; // V = omega r^2 + kappa r^4 (takes precedence when non-zero)
double confinementKappa = 1e-4;

int ansatzMaxDegree = 24;            // capacity bounds (the B200 engine only needs <= 24)
int ansatzMaxPartitionSize = 8;
int ansatzSubspaceDimension = 4096;
int ansatzMultipletSize = 8;
int ansatzMaxAngularMomentum = 15;

int main() {
  std::ofstream out("./modules/sys_params.h");
  const double RCl = std::sqrt(2. * inverseFilling * particlesNumber);
  const int angularMomentumCutoff = inverseFilling * (particlesNumber - 1) + ansatzMaxAngularMomentum;
  out << std::setprecision(std::numeric_limits<double>::max_digits10);
  out << "#ifndef SYSPARAMS_H\n#define SYSPARAMS_H\n\n";
  out << "#ifndef __CUDACC__\n#ifndef __device__\n#define __device__\n#endif\n#endif\n\n";
  out << "namespace sys_params {\n";
  out << "    __device__ constexpr int particlesNumber = " << particlesNumber << ";\n";
  out << "    __device__ constexpr int inverseFilling = " << inverseFilling << ";\n\n";
  out << "    __device__ constexpr int confinementExponent = " << confinementExponent << ";\n";
  out << "    __device__ constexpr float confinementStrength = " << confinementStrength << ";\n";
  out << "    __device__ constexpr double confinementOmega = " << confinementOmega << ";\n";
  out << "    __device__ constexpr double confinementKappa = " << confinementKappa << ";\n\n";
  out << "    __device__ constexpr float RCl = " << RCl << ";\n";
  out << "    __device__ constexpr float DCl = " << 2. * RCl << ";\n";
  out << "    __device__ constexpr float RCl_reciprocal = " << 1. / RCl << ";\n";
  out << "    __device__ constexpr float R0_reciprocal = " << 2. / RCl << ";\n\n";
  out << "    __device__ constexpr int ansatzExtendedMaxDegree = " << ansatzMaxDegree + 1 << ";\n";
  out << "    __device__ constexpr int ansatzMaxPartitionSize = " << ansatzMaxPartitionSize << ";\n";
  out << "    __device__ constexpr int ansatzSubspaceDimension = " << ansatzSubspaceDimension << ";\n\n";
  out << "    __device__ constexpr int ansatzMultipletSize = " << ansatzMultipletSize << ";\n\n";
  out << "    __device__ constexpr int ansatzMaxAngularMomentum = " << ansatzMaxAngularMomentum << ";\n";
  out << "    __device__ constexpr int angularMomentumCutoff = " << angularMomentumCutoff << ";\n\n";
  out << "}\n\n#endif\n";
  return 0;
}
