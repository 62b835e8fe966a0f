// Core of the LaughlinEdge C++ drop-in API (host code), independent of the
// compile-time sys_params.h: the parameter classes, the partition basis, the
// generalized eigenproblem, and the runtime-physics entry points that the
// header wrappers in edge_montecarlo.h / green_function.h / dynamics.h call
// with the values of sys_params.h.  Implemented in liblemc.so on top of the
// C-ABI of lemc.h.
#ifndef LAUGHLINEDGE_LEMC_API_CORE_H
#define LAUGHLINEDGE_LEMC_API_CORE_H

#include <cstddef>
#include <functional>
#include <string>
#include <utility>
#include <vector>

#include "../lemc.h"
#include "complex_numbers.h"
#include "tensors.h"

#if defined(__GNUC__)
#define LEMC_CXX_API __attribute__((visibility("default")))
#else
#define LEMC_CXX_API
#endif

namespace lemc_api {

// Physics and capacity values taken from sys_params.h by the header wrappers.
struct Physics {
  int N;                   // particlesNumber
  int m;                   // inverseFilling
  int conf_exponent;       // confinementExponent (power-law form)
  double conf_strength;    // confinementStrength
  double omega, kappa;     // V = omega r^2 + kappa r^4; both 0 selects the power law
  int ansatz_max_degree;   // ansatzExtendedMaxDegree - 1
  int ansatz_max_partition;
  int ansatz_subspace;
  int ansatz_multiplet;
  int ansatz_max_L;        // ansatzMaxAngularMomentum
};

// Confinement coefficients (omega, kappa) in l_B units for the sampler's
// H2 = sum r^2 and H4 = sum r^4 planes; the reference's single power law
// strength * sum (r / R_cl)^e maps onto them for e = 2 and e = 4.
LEMC_CXX_API bool confinement_coefficients(const Physics& ph, double* omega, double* kappa);

}  // namespace lemc_api

namespace iparts {

// Basis enumeration (reference modules/integer_partitions.h:25-93), host
// only: the partitions of each dL with at most N parts, compressed to
// (number, repetitions) pairs ordered by ascending repetitions.
class LEMC_CXX_API integer_partitions {
 public:
  struct partition_element {
    int number;
    int repetitions;
  };
  struct partition {
    int dM;
    int subspaceSize;
    int size;
    partition_element* partitionArray;
  };

  int subspaceDimension = 0;
  int maximalDegree = 0;
  int longestPartitionLenght = 0;

  integer_partitions() = default;
  integer_partitions(int particles_number, vector<int>& angular_momenta_list);
  integer_partitions(const integer_partitions&) = delete;
  integer_partitions& operator=(const integer_partitions&) = delete;
  ~integer_partitions();

  void printEdgePartition(int subspace_row) const;
  partition* getHostPartitions() const { return host_; }
  // The B200 engine keeps the basis as a device-side multiplication program
  // owned by the sampling context; no pointer-of-pointers copy exists.
  partition* getDevPartitions() const { return nullptr; }
  vector<int> getAngularMomenta() const;

 private:
  partition* host_ = nullptr;
  std::vector<partition_element> elems_;
};

}  // namespace iparts

namespace ges {

// Generalized Hermitian eigenproblem H c = E M c in FP64
// (reference modules/generalized_eigenproblem.h:12-30).
class LEMC_CXX_API generalizedEigenproblem {
 public:
  generalizedEigenproblem(cmatrix<double>& H, cmatrix<double>& M);
  std::vector<double> extract_spectrum();
  // Drops row/column 0 (the Laughlin state), solves the dL block with
  // M-normalised eigenvectors and returns (E_j, |(VC - i VS)(0, 1:) c_j|^2).
  std::vector<std::pair<double, double>> extract_dsf_coefficients(cmatrix<double>& VC,
                                                                  cmatrix<double>& VS);

 private:
  cmatrix<double> H0_, M0_;
};

}  // namespace ges

namespace edgeMC {

// Reference modules/edge_montecarlo.h:44-88 and em_parameters.cu:9-79, same
// fields, defaults and setters; the B200 engine adds the walker count, the
// Philox seed, the estimator and the contraction precision.
class LEMC_CXX_API monteCarloParameters {
 public:
  int maxDegree = 0;
  int extendedMaxDegree = 1;
  int subspaceDimension = -1;
  int injectedAngularMomentum = 0;
  int* injectedAngularMomenta = nullptr;
  int numberOfSectors = 0;
  int mesh_points_number = 200;
  float dr = 0.f;
  float randomStep = 0.8f;
  unsigned burnInMoves = 1000;
  unsigned MCSamples = 50000;
  unsigned threadsPerBlock = 128;
  unsigned nBlocks = 32;
  unsigned gridSize = 128 * 32;
  size_t totalSamplesNumber = size_t(50000) * 128 * 32;
  unsigned targetAcceptanceMoves = 100;
  float targetAcceptance = 0.50f;
  float acceptance_tol = 0.01f;
  // B200 engine
  unsigned long long seed = 0;   // 0: seeded from the clock, as the reference
  int estimator = LEMC_GUIDE_LAUGHLIN;
  int precision = -1;            // enum lemc_gram_mode; -1 picks by basis size
  int outputDigits = 6;          // decimals in the .tsv files (reference: 6)

  monteCarloParameters() = default;
  void setEdgeSpaceInfo(int maxPolyDegree, int subDim);
  void setMesh(int new_mesh_points_number);
  void setBurnIn(unsigned newBurnInMoves);
  void setMCSamples(unsigned newMCSamples);
  void setGPU_threads_blocks(unsigned newThreadsPerBlock, unsigned newNBlocks);
  void setAcceptanceBisectionParams(unsigned newTargetAcceptanceMoves, float newTargetAcceptance,
                                    float newAcceptance_tol);
  void setRandomStep(float newRandomStep);
  void setWalkers(unsigned walkers);
  void setSeed(unsigned long long s);
  void setEstimator(int guide);
  void setPrecision(int gram_mode);
  void setOutputDigits(int digits);
};

LEMC_CXX_API std::vector<double> spectrum_compute_rt(const lemc_api::Physics& ph,
                                                     monteCarloParameters& params, int dL,
                                                     bool saveOutput, int fileNumber);
LEMC_CXX_API cmatrix<double> metric_compute_rt(const lemc_api::Physics& ph,
                                               monteCarloParameters& params, int dL,
                                               bool saveOutput, int fileNumber);
LEMC_CXX_API std::vector<std::pair<double, double>> dsf_compute_rt(const lemc_api::Physics& ph,
                                                                   monteCarloParameters& params,
                                                                   int dL, bool saveOutput,
                                                                   int fileNumber);
LEMC_CXX_API void excitationResponse_compute_rt(const lemc_api::Physics& ph,
                                                monteCarloParameters& params,
                                                const int* sectors, int n_sectors,
                                                lemc_step_hook hook, void* user, int fileNumber);

}  // namespace edgeMC

namespace greenFunctionMC {

// Reference modules/green_function.h:36-69 and gf_parameters.cu:9-68.
class LEMC_CXX_API monteCarloParameters {
 public:
  int maxDegree = 0;
  int extendedMaxDegree = 1;
  int subspaceDimension = -1;
  int injectedAngularMomentum = 0;
  float randomStep = 0.8f;
  unsigned burnInMoves = 1000;
  unsigned MCSamples = 50000;
  unsigned threadsPerBlock = 128;
  unsigned nBlocks = 32;
  unsigned gridSize = 128 * 32;
  size_t totalSamplesNumber = size_t(50000) * 128 * 32;
  unsigned targetAcceptanceMoves = 100;
  float targetAcceptance = 0.50f;
  float acceptance_tol = 0.01f;
  unsigned long long seed = 0;
  int outputDigits = 6;

  monteCarloParameters() = default;
  void setEdgeSpaceInfo(int maxPolyDegree, int subDim);
  void setBurnIn(unsigned newBurnInMoves);
  void setMCSamples(unsigned newMCSamples);
  void setGPU_threads_blocks(unsigned newThreadsPerBlock, unsigned newNBlocks);
  void setAcceptanceBisectionParams(unsigned newTargetAcceptanceMoves, float newTargetAcceptance,
                                    float newAcceptance_tol);
  void setRandomStep(float newRandomStep);
  void setSeed(unsigned long long s);
  void setOutputDigits(int digits);
};

LEMC_CXX_API void occupation_numbers_compute_rt(const lemc_api::Physics& ph,
                                                monteCarloParameters& params, int dL,
                                                cmatrix<double>* metric, int fileNumber);

}  // namespace greenFunctionMC

namespace timeEvolution {

LEMC_CXX_API void edgeDensityResponse_compute_rt(unsigned particlesNumber, unsigned inverseFilling,
                                                 std::vector<int> angular_momenta,
                                                 std::function<double(double)> profile,
                                                 double end_time, double save_step,
                                                 int fileNumber);

}  // namespace timeEvolution

#endif
