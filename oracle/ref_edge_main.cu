// ref_edge: drives the reference's own sampler -- edgeMC::spectrum_compute,
// edgeMC::dsf_compute and greenFunctionMC::occupation_numbers_compute,
// compiled from the reference's sources by oracle/Makefile (target refmc) with
// the Eigen stand-in of oracle/eigen_shim -- and writes its outputs as JSON.
//
// TEST INFRASTRUCTURE ONLY: the fixtures it writes (tests/golden/) pin the
// oracle and the CUDA path to the reference itself, and its kernel times are
// the reference's own CUDA sampler timed on the same GPU.
//
//   ref_edge spectrum|dsf|occupation <dL,dL,...> <burn> <samples> <reps> <sigma>
//            <clock0> <blocks> <out.json> [workdir]
//
// Seeding: the reference seeds cuRAND from srand(time(NULL)) at every call
// (em_spectrum.cu:218-220, em_dsf.cu, gf_occupation_numbers.cu).  This program
// supplies that clock: repetition r of a run reads clock0 + r, so repetitions
// are distinct and a whole run is reproducible.
// Step: setRandomStep(sigma) with setAcceptanceBisectionParams(100, 0.5, 1.0),
// which makes optimal_step keep sigma (em_bisection.cu:85-88).
// Timing: every cudaEventElapsedTime the reference makes around its sampler
// launches (em_spectrum.cu:273-287 and its counterparts) is recorded through
// the shared CUDA runtime and reported per row.
#include <dlfcn.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "edge_montecarlo.h"
#include "green_function.h"

#include <Eigen/Dense>

static time_t g_clock = 0;
extern "C" time_t time(time_t* t) noexcept {
  if (t) *t = g_clock;
  return g_clock;
}

static std::vector<float> g_event_ms;
extern "C" cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t start, cudaEvent_t end) {
  using Fn = cudaError_t (*)(float*, cudaEvent_t, cudaEvent_t);
  static Fn real = reinterpret_cast<Fn>(dlsym(RTLD_NEXT, "cudaEventElapsedTime"));
  if (!real) return cudaErrorUnknown;
  const cudaError_t e = real(ms, start, end);
  if (e == cudaSuccess && ms) g_event_ms.push_back(*ms);
  return e;
}

namespace {

std::string num(double x) {
  char b[64];
  std::snprintf(b, sizeof b, "%.17g", x);
  return std::isfinite(x) ? std::string(b) : std::string("null");
}

std::string cmat(const Eigen::MatrixXcd& A) {
  std::ostringstream o;
  o << "[";
  for (int i = 0; i < A.rows(); ++i) {
    o << (i ? ",[" : "[");
    for (int j = 0; j < A.cols(); ++j)
      o << (j ? "," : "") << "[" << num(A(i, j).real()) << "," << num(A(i, j).imag()) << "]";
    o << "]";
  }
  o << "]";
  return o.str();
}

std::string fvec(const std::vector<float>& v) {
  std::ostringstream o;
  o << "[";
  for (size_t i = 0; i < v.size(); ++i) o << (i ? "," : "") << num(v[i]);
  o << "]";
  return o.str();
}

std::vector<int> parse_list(const char* s) {
  std::vector<int> out;
  std::stringstream ss(s);
  std::string tok;
  while (std::getline(ss, tok, ',')) out.push_back(std::atoi(tok.c_str()));
  return out;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 10) {
    std::fprintf(stderr,
                 "usage: %s spectrum|dsf|occupation <dL,..> <burn> <samples> <reps> <sigma> "
                 "<clock0> <blocks> <out.json> [workdir]\n",
                 argv[0]);
    return 2;
  }
  const std::string mode = argv[1];
  const std::vector<int> sectors = parse_list(argv[2]);
  const unsigned burn = unsigned(std::atoi(argv[3]));
  const unsigned samples = unsigned(std::atoi(argv[4]));
  const int reps = std::atoi(argv[5]);
  const float sigma = float(std::atof(argv[6]));
  const long clock0 = std::atol(argv[7]);
  const unsigned blocks = unsigned(std::atoi(argv[8]));
  std::string out_path = argv[9];
  if (!out_path.empty() && out_path[0] != '/') {  // relative to the starting directory
    char cwd[4096];
    if (getcwd(cwd, sizeof cwd)) out_path = std::string(cwd) + "/" + out_path;
  }
  // the reference writes its .tsv files under ../output relative to the
  // working directory
  const std::string work = argc > 10 ? argv[10] : "ref_edge_work/run";
  std::string mk = "mkdir -p '" + work + "'";
  if (std::system(mk.c_str()) != 0 || chdir(work.c_str()) != 0) {
    std::fprintf(stderr, "cannot enter %s\n", work.c_str());
    return 2;
  }
  if (samples < 100 || blocks == 0) {
    std::fprintf(stderr, "samples must be >= 100 (progress-bar interval) and blocks >= 1\n");
    return 2;
  }

  std::ostringstream js;
  js << "{\"mode\":\"" << mode << "\",\"particles\":" << sys_params::particlesNumber
     << ",\"inverse_filling\":" << sys_params::inverseFilling
     << ",\"confinement_exponent\":" << sys_params::confinementExponent
     << ",\"confinement_strength\":" << num(sys_params::confinementStrength)
     << ",\"RCl\":" << num(sys_params::RCl) << ",\"RCl_reciprocal\":" << num(sys_params::RCl_reciprocal)
     << ",\"burn_in\":" << burn << ",\"samples\":" << samples << ",\"sigma\":" << num(sigma)
     << ",\"walkers\":" << blocks * 128 << ",\"clock0\":" << clock0
     << ",\"angular_momentum_cutoff\":" << sys_params::angularMomentumCutoff << ",\"runs\":[";
  bool first = true;
  for (int dL : sectors) {
    for (int r = 0; r < reps; ++r) {
      g_clock = time_t(clock0 + r);
      g_event_ms.clear();
      lemc_eigen_shim::captured().clear();
      std::ostringstream run;
      run << "{\"dL\":" << dL << ",\"rep\":" << r << ",\"clock\":" << (clock0 + r);
      if (mode == "spectrum" || mode == "dsf") {
        edgeMC::monteCarloParameters p;
        p.setGPU_threads_blocks(128, blocks);
        p.setBurnIn(burn);
        p.setMCSamples(samples);
        p.setRandomStep(sigma);
        p.setAcceptanceBisectionParams(100, 0.5f, 1.0f);
        if (mode == "spectrum") {
          std::vector<double> ev = edgeMC::spectrum_compute(p, dL, false, r);
          run << ",\"evals\":[";
          for (size_t i = 0; i < ev.size(); ++i) run << (i ? "," : "") << num(ev[i]);
          run << "]";
        } else {
          std::vector<std::pair<double, double>> es = edgeMC::dsf_compute(p, dL, false, r);
          run << ",\"energy_dsf\":[";
          for (size_t i = 0; i < es.size(); ++i)
            run << (i ? "," : "") << "[" << num(es[i].first) << "," << num(es[i].second) << "]";
          run << "]";
        }
        if (!lemc_eigen_shim::captured().empty()) {
          const auto& pr = lemc_eigen_shim::captured().back();
          run << ",\"H\":" << cmat(pr.A) << ",\"M\":" << cmat(pr.B);
        }
      } else if (mode == "occupation") {
        greenFunctionMC::monteCarloParameters p;
        p.setGPU_threads_blocks(128, blocks);
        p.setBurnIn(burn);
        p.setMCSamples(samples);
        p.setRandomStep(sigma);
        p.setAcceptanceBisectionParams(100, 0.5f, 1.0f);
        greenFunctionMC::occupation_numbers_compute(p, dL, r);
        char path[512];
        std::snprintf(path, sizeof path,
                      "../output/N=%d_m=%d/dL=%d/Statistics/OccupationNumbers_not_normalized/%d.tsv",
                      sys_params::particlesNumber, sys_params::inverseFilling, dL, r);
        std::ifstream f(path);
        if (!f) {
          std::fprintf(stderr, "missing %s\n", path);
          return 3;
        }
        run << ",\"occupation\":[";
        int a, b, l;
        double re, im;
        bool f1 = true;
        while (f >> a >> b >> l >> re >> im) {
          run << (f1 ? "" : ",") << "[" << a << "," << b << "," << l << "," << num(re) << ","
              << num(im) << "]";
          f1 = false;
        }
        run << "]";
      } else {
        std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
        return 2;
      }
      run << ",\"kernel_ms\":" << fvec(g_event_ms) << "}";
      js << (first ? "" : ",") << run.str();
      first = false;
      std::fflush(stdout);
    }
  }
  js << "]}\n";
  std::ofstream o(out_path);
  o << js.str();
  return o.good() ? 0 : 4;
}
