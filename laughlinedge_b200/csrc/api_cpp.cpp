// C++ drop-in API of LaughlinEdge implemented on the C-ABI (lemc.h).
//
// Reference correspondence (file:line of the LaughlinEdge project):
//   edgeMC::spectrum_compute            modules/edge_mc/em_spectrum.cu:210-422
//   edgeMC::metric_compute              modules/edge_mc/em_metric.cu:200-392
//   edgeMC::dsf_compute                 modules/edge_mc/em_dsf.cu:235-500
//   edgeMC::excitationResponse_compute  modules/edge_mc/em_edgeResponse.tpp:284-601
//   edgeMC::optimal_step                modules/edge_mc/em_bisection.cu:49-153
//   greenFunctionMC::occupation_numbers_compute  modules/green_function/gf_occupation_numbers.cu:309-566
//   timeEvolution::edgeDensityResponse_compute   modules/dynamics/dynamics.cpp:149-308
//   ges::generalizedEigenproblem        modules/eigensolver/generalized_eigenproblem.cpp:17-95
// Behaviour kept: argument meaning, returned values, Hermitisation, output
// directories and .tsv layouts, exit(1) on configuration/capacity errors.
// Changed by design: all rows of a call are sampled in the same device
// launches (one shared guide by default), the seed is settable, and CUDA
// errors abort instead of printing and continuing.
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/lemc.h"
#include "../../include/modules/lemc_api_core.h"

namespace {

[[noreturn]] void die(const std::string& msg) {
  std::fprintf(stderr, "%s\n", msg.c_str());
  std::fflush(stderr);
  std::exit(1);
}

void check(int status, const char* where) {
  if (status != LEMC_OK) {
    std::ostringstream os;
    os << "LaughlinEdge: " << where << " failed: " << lemc_status_string(status);
    die(os.str());
  }
}

unsigned long long pick_seed(unsigned long long s) {
  if (s) return s;
  return static_cast<unsigned long long>(
      std::chrono::high_resolution_clock::now().time_since_epoch().count());
}

std::string fmtnum(double v, int digits) {
  char b[64];
  std::snprintf(b, sizeof(b), "%.*f", digits, v);
  return b;
}

void write_matrix(const std::string& dir, int fileNumber, const cmatrix<double>& X, int digits) {
  std::filesystem::create_directories(dir);
  std::ofstream out(dir + "/" + std::to_string(fileNumber) + ".tsv");
  for (int i = 0; i < X.rows(); ++i)
    for (int j = 0; j < X.cols(); ++j)
      out << i << "\t" << j << "\t" << fmtnum(re(X(i, j)), digits) << "\t"
          << fmtnum(im(X(i, j)), digits) << "\n";
}

cmatrix<double> hermitise(const cmatrix<double>& X) {
  cmatrix<double> t = (X + X.adjoint()) / 2.0;
  return t;
}

int basis_rows(int N, const std::vector<int>& sectors, std::vector<int>* dL_of_row,
               int* max_degree, int* longest) {
  int nr = 0, ni = 0;
  check(lemc_partitions(N, sectors.data(), int(sectors.size()), nullptr, 0, nullptr, 0, &nr, &ni,
                        max_degree, longest),
        "lemc_partitions");
  std::vector<lemc_partition_row> rows(std::max(1, nr));
  std::vector<int32_t> pairs(std::max(1, ni));
  check(lemc_partitions(N, sectors.data(), int(sectors.size()), rows.data(), nr, pairs.data(), ni,
                        &nr, &ni, nullptr, nullptr),
        "lemc_partitions");
  if (dL_of_row) {
    dL_of_row->clear();
    for (int r = 0; r < nr; ++r) dL_of_row->push_back(rows[r].dL);
  }
  return nr;
}

void capacity_checks(const lemc_api::Physics& ph, int max_degree, int longest, int dim) {
  if (max_degree > ph.ansatz_max_degree) {
    std::ostringstream os;
    os << "\nWith this angular momentum choice,\nthe maximal singe-coordinate degree is " << max_degree
       << "\nThe upper bound is set to " << ph.ansatz_max_degree
       << " in sys_params.h. It should be at least as large\n"
          "Consider re-generating sys_params.h by running an updated system_parameters.cpp";
    die(os.str());
  }
  if (longest > ph.ansatz_max_partition) {
    std::ostringstream os;
    os << "\nWith this angular momentum choice,\nthe length of the longest (compressed) partition is "
       << longest << "\nThe upper bound is set to " << ph.ansatz_max_partition
       << " in sys_params.h. It should be at least as large";
    die(os.str());
  }
  if (dim > ph.ansatz_subspace) {
    std::ostringstream os;
    os << "\nWith this angular momentum choice,\nthe edge Hilbert space size is " << dim
       << "\nThe upper bound is set to " << ph.ansatz_subspace
       << " in sys_params.h. It should be at least as large";
    die(os.str());
  }
}

// One sampling job: context set-up, step tuning, burn-in and measurement.
struct Job {
  lemc_ctx* ctx = nullptr;
  std::vector<int> sectors, dims, dL_of_row;
  int D = 0;
  double omega = 0, kappa = 0;
  ~Job() {
    if (ctx) lemc_destroy(ctx);
  }
};

// Step search for the target acceptance, bounded in iterations (reference
// em_bisection.cu:49-153): lemc_tune_step on the live chain.
void optimal_step(lemc_ctx* ctx, edgeMC::monteCarloParameters& p) {
  if (!(p.acceptance_tol < 1.0f)) return;
  check(lemc_set_step(ctx, p.randomStep), "lemc_set_step");
  float sigma = p.randomStep;
  const int st = lemc_tune_step(ctx, p.targetAcceptance, p.acceptance_tol,
                                int(std::max(1u, p.targetAcceptanceMoves)), &sigma, nullptr);
  if (st == LEMC_ERR_NUMERIC)
    die("\nSomething went wrong with the bisection search for the optimal Markov-Chain step\nCheck the code");
  check(st, "lemc_tune_step");
  p.randomStep = sigma;
}

int default_precision(const Job& j, unsigned walkers) {
  double sd2 = 0;
  for (int d : j.dims) sd2 += double(d) * d;
  // the exact FP64 accumulation is cheap for small bases
  return (sd2 * walkers < 2e8) ? LEMC_GRAM_FP64 : LEMC_GRAM_TF32X3;
}

void start_job(Job& j, const lemc_api::Physics& ph, edgeMC::monteCarloParameters& p,
               const std::vector<int>& sectors, const std::vector<int>& probes, int guide) {
  if (!lemc_api::confinement_coefficients(ph, &j.omega, &j.kappa))
    die("LaughlinEdge: confinementExponent must be 2 or 4 (or set confinementOmega/Kappa)");
  int max_degree = 0, longest = 0;
  j.sectors = sectors;
  j.D = basis_rows(ph.N, sectors, &j.dL_of_row, &max_degree, &longest);
  capacity_checks(ph, max_degree, longest, j.D);
  j.dims.clear();
  for (int s : sectors) {
    int d = 0;
    for (int r : j.dL_of_row) d += (r == s);
    j.dims.push_back(d);
  }
  p.setEdgeSpaceInfo(max_degree, j.D);
  lemc_config cfg{};
  cfg.particles = ph.N;
  cfg.inverse_filling = ph.m;
  cfg.n_walkers = int(p.gridSize);
  cfg.lanes_per_walker = -1;
  cfg.step_sigma = p.randomStep;
  cfg.guide = guide;
  cfg.seed = pick_seed(p.seed);
  cfg.gram_mode = (p.precision >= 0) ? p.precision : default_precision(j, p.gridSize);
  check(lemc_create(&cfg, &j.ctx), "lemc_create");
  if (!probes.empty()) check(lemc_set_probes(j.ctx, probes.data(), int(probes.size())), "lemc_set_probes");
  check(lemc_set_sectors(j.ctx, sectors.data(), int(sectors.size())), "lemc_set_sectors");
  check(lemc_init_walkers(j.ctx, nullptr), "lemc_init_walkers");
  std::printf("\tDetermining the optimal Markov-Chain random step to achieve %.2f acceptance rate.",
              p.targetAcceptance);
  optimal_step(j.ctx, p);
  std::printf(" Optimal step: %g\n", p.randomStep);
  check(lemc_run(j.ctx, int(p.burnInMoves), 0), "lemc_run (burn-in)");
  check(lemc_reset_accumulators(j.ctx), "lemc_reset_accumulators");
}

void finish_print(Job& j, const edgeMC::monteCarloParameters& p, double seconds) {
  lemc_stats st;
  check(lemc_read_stats(j.ctx, &st), "lemc_read_stats");
  std::printf("\tFinished. Total number of samples: %zu. Elapsed time: %.1fs\n",
              size_t(p.MCSamples) * p.gridSize, seconds);
  std::printf("\tAverage acceptance\t%.2f\n\n", st.acceptance);
}

// Normalised blocks (reference convention) of a shared-guide job:
// same-sector S/H blocks into the full D x D matrices.
void gram_blocks(Job& j, cmatrix<double>& M, cmatrix<double>& H) {
  int first = 0;
  for (size_t s = 0; s < j.sectors.size(); ++s) {
    const int d = j.dims[s];
    std::vector<double> S(2 * d * d), H2(2 * d * d), H4(2 * d * d), Mn(2 * d * d), Hn(2 * d * d);
    double n = 0;
    check(lemc_read_gram(j.ctx, int(s), S.data(), H2.data(), H4.data(), &n), "lemc_read_gram");
    check(lemc_normalise(d, S.data(), H2.data(), H4.data(), j.omega, j.kappa, Mn.data(), Hn.data()),
          "lemc_normalise");
    for (int a = 0; a < d; ++a)
      for (int b = 0; b < d; ++b) {
        const size_t o = 2 * (size_t(a) * d + b);
        M(first + a, first + b) = complex<double>(Mn[o], Mn[o + 1]);
        H(first + a, first + b) = complex<double>(Hn[o], Hn[o + 1]);
      }
    first += d;
  }
}

// Diagonal norms sqrt(S_aa) of every row (shared guide).
std::vector<double> row_norms(Job& j) {
  std::vector<double> nrm;
  for (size_t s = 0; s < j.sectors.size(); ++s) {
    const int d = j.dims[s];
    std::vector<double> S(2 * d * d);
    check(lemc_read_gram(j.ctx, int(s), S.data(), nullptr, nullptr, nullptr), "lemc_read_gram");
    for (int a = 0; a < d; ++a) nrm.push_back(std::sqrt(S[2 * (size_t(a) * d + a)]));
  }
  return nrm;
}

// Row-estimator matrices (reference normalisation x / sqrt(gg)), full D x D.
void row_blocks(Job& j, cmatrix<double>& M, cmatrix<double>& H, cmatrix<double>* Vc,
                cmatrix<double>* Vs, bool same_sector_only) {
  const int D = j.D;
  std::vector<double> fg(2 * D * D), gg(D * D), fh(2 * D * D), fc(2 * D * D), fs(2 * D * D);
  check(lemc_read_rows(j.ctx, j.omega, j.kappa, fg.data(), gg.data(), fh.data(), fc.data(),
                       fs.data(), nullptr, nullptr),
        "lemc_read_rows");
  for (int a = 0; a < D; ++a)
    for (int b = 0; b < D; ++b) {
      const size_t o = size_t(a) * D + b;
      const double sq = std::sqrt(gg[o]);
      const bool same = j.dL_of_row[a] == j.dL_of_row[b];
      if (same || !same_sector_only) {
        M(a, b) = complex<double>(fg[2 * o], fg[2 * o + 1]) / sq;
        H(a, b) = complex<double>(fh[2 * o], fh[2 * o + 1]) / sq;
      } else {
        if (Vc) (*Vc)(a, b) = complex<double>(fc[2 * o], fc[2 * o + 1]) / sq;
        if (Vs) (*Vs)(a, b) = complex<double>(fs[2 * o], fs[2 * o + 1]) / sq;
      }
    }
}

// Normalised cross blocks Cuser/Ccos/Csin between sectors si, sj (shared guide).
void cross_block(Job& j, int si, int sj, const std::vector<double>& nrm, cmatrix<double>* U,
                 cmatrix<double>* C, cmatrix<double>* S) {
  const int da = j.dims[si], db = j.dims[sj];
  int fa = 0, fb = 0;
  for (int s = 0; s < si; ++s) fa += j.dims[s];
  for (int s = 0; s < sj; ++s) fb += j.dims[s];
  std::vector<double> cu(2 * da * db), cc(2 * da * db), cs(2 * da * db);
  check(lemc_read_cross(j.ctx, si, sj, cu.data(), cc.data(), cs.data()), "lemc_read_cross");
  for (int a = 0; a < da; ++a)
    for (int b = 0; b < db; ++b) {
      const size_t o = 2 * (size_t(a) * db + b);
      const double den = nrm[fa + a] * nrm[fb + b];
      if (U) (*U)(fa + a, fb + b) = complex<double>(cu[o], cu[o + 1]) / den;
      if (C) (*C)(fa + a, fb + b) = complex<double>(cc[o], cc[o + 1]) / den;
      if (S) (*S)(fa + a, fb + b) = complex<double>(cs[o], cs[o + 1]) / den;
    }
}

std::string out_root(int N, int m) {
  return "../output/N=" + std::to_string(N) + "_m=" + std::to_string(m);
}

}  // namespace

// ---------------------------------------------------------------------------
namespace lemc_api {

bool confinement_coefficients(const Physics& ph, double* omega, double* kappa) {
  if (ph.omega != 0.0 || ph.kappa != 0.0) {
    *omega = ph.omega;
    *kappa = ph.kappa;
    return true;
  }
  const double rcl = std::sqrt(2.0 * ph.m * ph.N);
  if (ph.conf_exponent == 2) {
    *omega = ph.conf_strength / (rcl * rcl);
    *kappa = 0.0;
    return true;
  }
  if (ph.conf_exponent == 4) {
    *omega = 0.0;
    *kappa = ph.conf_strength / (rcl * rcl * rcl * rcl);
    return true;
  }
  return false;
}

}  // namespace lemc_api

// ---------------------------------------------------------------------------
namespace iparts {

integer_partitions::integer_partitions(int particles_number, vector<int>& angular_momenta_list) {
  std::vector<int> sec(angular_momenta_list.begin(), angular_momenta_list.end());
  int nr = 0, ni = 0;
  check(lemc_partitions(particles_number, sec.data(), int(sec.size()), nullptr, 0, nullptr, 0, &nr,
                        &ni, &maximalDegree, &longestPartitionLenght),
        "lemc_partitions");
  std::vector<lemc_partition_row> rows(std::max(1, nr));
  std::vector<int32_t> pairs(std::max(1, ni));
  check(lemc_partitions(particles_number, sec.data(), int(sec.size()), rows.data(), nr, pairs.data(),
                        ni, &nr, &ni, nullptr, nullptr),
        "lemc_partitions");
  subspaceDimension = nr;
  elems_.resize(std::max(1, ni / 2));
  for (int k = 0; k < ni / 2; ++k) elems_[k] = {pairs[2 * k], pairs[2 * k + 1]};
  host_ = new partition[std::max(1, nr)];
  for (int r = 0; r < nr; ++r)
    host_[r] = {rows[r].dL, rows[r].sector_size, rows[r].n_pairs, elems_.data() + rows[r].pairs_off / 2};
  std::printf("Generating the partitions (cutoff at %d parts): %d states\n", particles_number, nr);
}

integer_partitions::~integer_partitions() { delete[] host_; }

void integer_partitions::printEdgePartition(int row) const {
  for (int k = 0; k < host_[row].size; ++k)
    std::printf("%d(x%d) ", host_[row].partitionArray[k].number, host_[row].partitionArray[k].repetitions);
}

vector<int> integer_partitions::getAngularMomenta() const {
  vector<int> v(subspaceDimension);
  for (int r = 0; r < subspaceDimension; ++r) v[r] = host_[r].dM;
  return v;
}

}  // namespace iparts

// ---------------------------------------------------------------------------
namespace ges {

generalizedEigenproblem::generalizedEigenproblem(cmatrix<double>& H, cmatrix<double>& M)
    : H0_(H), M0_(M) {}

std::vector<double> generalizedEigenproblem::extract_spectrum() {
  const int D = H0_.rows();
  std::vector<double> ev(D);
  int rank = 0;
  check(lemc_geneig(D, reinterpret_cast<const double*>(H0_.data()),
                    reinterpret_cast<const double*>(M0_.data()), 1e-12, ev.data(), nullptr, &rank),
        "lemc_geneig");
  ev.resize(rank);
  return ev;
}

std::vector<std::pair<double, double>> generalizedEigenproblem::extract_dsf_coefficients(
    cmatrix<double>& VC, cmatrix<double>& VS) {
  const int D = H0_.rows();
  std::vector<std::pair<double, double>> out;
  if (D < 2) return out;
  std::vector<double> h(2 * D * D), m(2 * D * D), vc(2 * D * D), vs(2 * D * D), e(D), w(D);
  for (int a = 0; a < D; ++a)
    for (int b = 0; b < D; ++b) {
      const size_t o = 2 * (size_t(a) * D + b);
      h[o] = re(H0_(a, b));
      h[o + 1] = im(H0_(a, b));
      m[o] = re(M0_(a, b));
      m[o + 1] = im(M0_(a, b));
      vc[o] = re(VC(a, b));
      vc[o + 1] = im(VC(a, b));
      vs[o] = re(VS(a, b));
      vs[o + 1] = im(VS(a, b));
    }
  int rank = 0;
  check(lemc_dsf_weights(D, h.data(), m.data(), vc.data(), vs.data(), 1e-12, e.data(), w.data(),
                         &rank),
        "lemc_dsf_weights");
  for (int j = 0; j < rank; ++j) out.push_back({e[j], w[j]});
  return out;
}

}  // namespace ges

// ---------------------------------------------------------------------------
namespace edgeMC {

void monteCarloParameters::setEdgeSpaceInfo(int maxPolyDegree, int subDim) {
  maxDegree = maxPolyDegree;
  extendedMaxDegree = maxDegree + 1;
  subspaceDimension = subDim;
}
void monteCarloParameters::setMesh(int n) { mesh_points_number = n; }
void monteCarloParameters::setBurnIn(unsigned n) { burnInMoves = n; }
void monteCarloParameters::setMCSamples(unsigned n) {
  MCSamples = n;
  totalSamplesNumber = size_t(MCSamples) * gridSize;
}
void monteCarloParameters::setGPU_threads_blocks(unsigned t, unsigned b) {
  threadsPerBlock = t;
  nBlocks = b;
  gridSize = t * b;
  totalSamplesNumber = size_t(MCSamples) * gridSize;
}
void monteCarloParameters::setAcceptanceBisectionParams(unsigned moves, float target, float tol) {
  targetAcceptanceMoves = moves;
  targetAcceptance = target;
  acceptance_tol = tol;
}
void monteCarloParameters::setRandomStep(float s) { randomStep = s; }
void monteCarloParameters::setWalkers(unsigned w) { setGPU_threads_blocks(w, 1); }
void monteCarloParameters::setSeed(unsigned long long s) { seed = s; }
void monteCarloParameters::setEstimator(int g) { estimator = g; }
void monteCarloParameters::setPrecision(int p) { precision = p; }
void monteCarloParameters::setOutputDigits(int d) { outputDigits = d; }

static void sample_matrices(const lemc_api::Physics& ph, monteCarloParameters& p, int dL,
                            cmatrix<double>& H, cmatrix<double>& M) {
  Job j;
  std::printf("Sampling the dL = %d sector\n", dL);
  start_job(j, ph, p, {dL}, {}, p.estimator);
  const auto t0 = std::chrono::steady_clock::now();
  check(lemc_run(j.ctx, int(p.MCSamples), 1), "lemc_run");
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  H = cmatrix<double>(j.D, j.D, complex<double>(0.0));
  M = cmatrix<double>(j.D, j.D, complex<double>(0.0));
  if (p.estimator == LEMC_GUIDE_ROW)
    row_blocks(j, M, H, nullptr, nullptr, false);
  else
    gram_blocks(j, M, H);
  finish_print(j, p, secs);
  H = hermitise(H);
  M = hermitise(M);
}

std::vector<double> spectrum_compute_rt(const lemc_api::Physics& ph, monteCarloParameters& p, int dL,
                                        bool saveOutput, int fileNumber) {
  cmatrix<double> H, M;
  sample_matrices(ph, p, dL, H, M);
  if (saveOutput) {
    const std::string base = out_root(ph.N, ph.m) + "/dL=" + std::to_string(dL) + "/Statistics/";
    write_matrix(base + "Hamiltonian", fileNumber, H, p.outputDigits);
    write_matrix(base + "Metric", fileNumber, M, p.outputDigits);
  }
  ges::generalizedEigenproblem eig(H, M);
  return eig.extract_spectrum();
}

cmatrix<double> metric_compute_rt(const lemc_api::Physics& ph, monteCarloParameters& p, int dL,
                                  bool saveOutput, int fileNumber) {
  cmatrix<double> H, M;
  sample_matrices(ph, p, dL, H, M);
  if (saveOutput)
    write_matrix(out_root(ph.N, ph.m) + "/dL=" + std::to_string(dL) + "/Statistics/Metric",
                 fileNumber, M, p.outputDigits);
  return M;
}

std::vector<std::pair<double, double>> dsf_compute_rt(const lemc_api::Physics& ph,
                                                      monteCarloParameters& p, int dL,
                                                      bool saveOutput, int fileNumber) {
  if (dL == 0) die("Select dL>0");
  p.injectedAngularMomentum = dL;
  Job j;
  std::printf("Sampling the dL = {0, %d} sectors\n", dL);
  start_job(j, ph, p, {0, dL}, {dL}, p.estimator);
  const auto t0 = std::chrono::steady_clock::now();
  check(lemc_run(j.ctx, int(p.MCSamples), 1), "lemc_run");
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  const int D = j.D;
  cmatrix<double> H(D, D, complex<double>(0.0)), M(D, D, complex<double>(0.0)),
      Vc(D, D, complex<double>(0.0)), Vs(D, D, complex<double>(0.0));
  if (p.estimator == LEMC_GUIDE_ROW) {
    row_blocks(j, M, H, &Vc, &Vs, true);
  } else {
    gram_blocks(j, M, H);
    const std::vector<double> nrm = row_norms(j);
    cross_block(j, 0, 1, nrm, nullptr, &Vc, &Vs);
    cross_block(j, 1, 0, nrm, nullptr, &Vc, &Vs);
  }
  finish_print(j, p, secs);
  H = hermitise(H);
  M = hermitise(M);
  Vc = hermitise(Vc);
  Vs = hermitise(Vs);
  if (saveOutput) {
    const std::string base = out_root(ph.N, ph.m) + "/dL=" + std::to_string(dL) + "/Statistics/";
    write_matrix(base + "Hamiltonian", fileNumber, H, p.outputDigits);
    write_matrix(base + "Metric", fileNumber, M, p.outputDigits);
    write_matrix(base + "cosine_excitation", fileNumber, Vc, p.outputDigits);
    write_matrix(base + "sine_excitation", fileNumber, Vs, p.outputDigits);
  }
  ges::generalizedEigenproblem eig(H, M);
  return eig.extract_dsf_coefficients(Vc, Vs);
}

void excitationResponse_compute_rt(const lemc_api::Physics& ph, monteCarloParameters& p,
                                   const int* sectors, int n_sectors, lemc_step_hook hook,
                                   void* user, int fileNumber) {
  std::vector<int> sec(sectors, sectors + n_sectors);
  if (n_sectors > ph.ansatz_multiplet || n_sectors > LEMC_MAX_PROBES) {
    std::ostringstream os;
    os << "\nYou chose " << n_sectors << " different angular momenta.\nThe upper bound is set to "
       << std::min(ph.ansatz_multiplet, LEMC_MAX_PROBES) << ". It should be at least as large";
    die(os.str());
  }
  p.numberOfSectors = n_sectors;
  Job j;
  std::printf("Sampling the excitation response in %d sectors\n", n_sectors);
  // the excitation potential and the edge-density Fourier sums couple
  // sectors, which only the shared guide samples in one chain
  start_job(j, ph, p, sec, sec, LEMC_GUIDE_LAUGHLIN);
  const auto t0 = std::chrono::steady_clock::now();
  check(lemc_run_hooked(j.ctx, int(p.MCSamples), hook, user), "lemc_run_hooked");
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  const int D = j.D;
  cmatrix<double> H(D, D, complex<double>(0.0)), M(D, D, complex<double>(0.0)),
      U(D, D, complex<double>(0.0));
  gram_blocks(j, M, H);
  const std::vector<double> nrm = row_norms(j);
  std::vector<cmatrix<double>> RC(n_sectors, cmatrix<double>(D, D, complex<double>(0.0)));
  std::vector<cmatrix<double>> RS(n_sectors, cmatrix<double>(D, D, complex<double>(0.0)));
  for (int si = 0; si < n_sectors; ++si)
    for (int sj = 0; sj < n_sectors; ++sj) {
      cmatrix<double> C(D, D, complex<double>(0.0)), S(D, D, complex<double>(0.0));
      cross_block(j, si, sj, nrm, &U, &C, &S);
      const int l = std::abs(sec[sj] - sec[si]);
      for (int J = 0; J < n_sectors; ++J) {
        if (sec[J] != l) continue;
        for (int a = 0; a < D; ++a)
          for (int b = 0; b < D; ++b) {
            if (re(C(a, b)) != 0.0 || im(C(a, b)) != 0.0) RC[J](a, b) = C(a, b);
            if (re(S(a, b)) != 0.0 || im(S(a, b)) != 0.0) RS[J](a, b) = S(a, b);
          }
      }
    }
  finish_print(j, p, secs);
  H = hermitise(H);
  M = hermitise(M);
  U = hermitise(U);
  for (int J = 0; J < n_sectors; ++J) {
    RC[J] = hermitise(RC[J]);
    RS[J] = hermitise(RS[J]);
  }
  std::printf("Saving the matrices (you can post-process to compute statistical errorbars)\n");
  const std::string base = out_root(ph.N, ph.m) + "/ExternalExcitation/Statistics/";
  write_matrix(base + "Hamiltonian", fileNumber, H, p.outputDigits);
  write_matrix(base + "Metric", fileNumber, M, p.outputDigits);
  write_matrix(base + "ExcitationPotential", fileNumber, U, p.outputDigits);
  for (int J = 0; J < n_sectors; ++J) {
    const std::string dir = base + "EdgeDenstiy_FourierTransform/dL=" + std::to_string(sec[J]);
    std::filesystem::create_directories(dir);
    std::ofstream out(dir + "/" + std::to_string(fileNumber) + ".tsv");
    for (int a = 0; a < D; ++a)
      for (int b = 0; b < D; ++b)
        out << a << "\t" << b << "\t" << fmtnum(re(RC[J](a, b)), p.outputDigits) << "\t"
            << fmtnum(im(RC[J](a, b)), p.outputDigits) << "\t"
            << fmtnum(re(RS[J](a, b)), p.outputDigits) << "\t"
            << fmtnum(im(RS[J](a, b)), p.outputDigits) << "\n";
  }
}

}  // namespace edgeMC

// ---------------------------------------------------------------------------
namespace greenFunctionMC {

void monteCarloParameters::setEdgeSpaceInfo(int maxPolyDegree, int subDim) {
  maxDegree = maxPolyDegree;
  extendedMaxDegree = maxDegree + 1;
  subspaceDimension = subDim;
}
void monteCarloParameters::setBurnIn(unsigned n) { burnInMoves = n; }
void monteCarloParameters::setMCSamples(unsigned n) {
  MCSamples = n;
  totalSamplesNumber = size_t(MCSamples) * gridSize;
}
void monteCarloParameters::setGPU_threads_blocks(unsigned t, unsigned b) {
  threadsPerBlock = t;
  nBlocks = b;
  gridSize = t * b;
  totalSamplesNumber = size_t(MCSamples) * gridSize;
}
void monteCarloParameters::setAcceptanceBisectionParams(unsigned moves, float target, float tol) {
  targetAcceptanceMoves = moves;
  targetAcceptance = target;
  acceptance_tol = tol;
}
void monteCarloParameters::setRandomStep(float s) { randomStep = s; }
void monteCarloParameters::setSeed(unsigned long long s) { seed = s; }
void monteCarloParameters::setOutputDigits(int d) { outputDigits = d; }

void occupation_numbers_compute_rt(const lemc_api::Physics& ph, monteCarloParameters& p, int dL,
                                   cmatrix<double>* metric, int fileNumber) {
  if (dL > ph.ansatz_max_L)
    die("The defined parameter ansatzMaxAngularMomentum is smaller than dL. Modify and re-run "
        "system_parameters.cpp");
  p.injectedAngularMomentum = dL;
  int max_degree = 0, longest = 0;
  std::vector<int> dls;
  const int D = basis_rows(ph.N, {dL}, &dls, &max_degree, &longest);
  capacity_checks(ph, max_degree, longest, D);
  p.setEdgeSpaceInfo(max_degree, D);
  const int Lc = ph.m * (ph.N - 1) + ph.ansatz_max_L;
  lemc_occupation_config oc{};
  oc.particles = ph.N;
  oc.inverse_filling = ph.m;
  oc.dL = dL;
  oc.l_cutoff = Lc;
  oc.n_walkers = int(p.gridSize);
  oc.step_sigma = p.randomStep;
  oc.seed = pick_seed(p.seed);
  oc.burn_in = int(p.burnInMoves);
  oc.sweeps = int(p.MCSamples);
  std::vector<double> occ(size_t(2) * D * D * Lc);
  double acc = 0;
  const auto t0 = std::chrono::steady_clock::now();
  check(lemc_occupation(&oc, occ.data(), &acc), "lemc_occupation");
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::printf("\tFinished %d x %d pairs. Elapsed time: %.1fs, average acceptance %.2f\n", D, D, secs, acc);
  rank3tensor<complex<double>> on(D, D, Lc, complex<double>(0.0));
  for (int a = 0; a < D; ++a)
    for (int b = 0; b < D; ++b) {
      complex<double> sum(0.0);
      for (int l = 0; l < Lc; ++l) {
        const size_t o = 2 * ((size_t(a) * D + b) * Lc + l);
        sum += complex<double>(occ[o], occ[o + 1]);
      }
      const complex<double> scale = metric ? (*metric)(a, b) : complex<double>(1.0);
      for (int l = 0; l < Lc; ++l) {
        const size_t o = 2 * ((size_t(a) * D + b) * Lc + l);
        on(a, b, l) = complex<double>(occ[o], occ[o + 1]) / sum * double(ph.N) * scale;
      }
    }
  // Hermitise per l (reference gf_occupation_numbers.cu:490-512)
  for (int l = 0; l < Lc; ++l)
    for (int a = 0; a < D; ++a)
      for (int b = a; b < D; ++b) {
        const complex<double> v = (on(a, b, l) + conj(on(b, a, l))) / 2.0;
        on(a, b, l) = v;
        on(b, a, l) = conj(v);
      }
  const std::string dir = out_root(ph.N, ph.m) + "/dL=" + std::to_string(dL) + "/Statistics/" +
                          (metric ? "OccupationNumbers_normalized" : "OccupationNumbers_not_normalized");
  std::filesystem::create_directories(dir);
  std::ofstream out(dir + "/" + std::to_string(fileNumber) + ".tsv");
  for (int a = 0; a < D; ++a)
    for (int b = 0; b < D; ++b) {
      for (int l = 0; l < Lc; ++l)
        out << a << "\t" << b << "\t" << l << "\t" << fmtnum(re(on(a, b, l)), p.outputDigits) << "\t"
            << fmtnum(im(on(a, b, l)), p.outputDigits) << "\n";
      out << "\n";
    }
}

}  // namespace greenFunctionMC

// ---------------------------------------------------------------------------
namespace timeEvolution {

namespace {

std::map<std::pair<int, int>, std::complex<double>> read_tsv(const std::string& path, int* dim,
                                                             bool six_cols,
                                                             std::map<std::pair<int, int>, std::complex<double>>* second) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("Cannot open file: " + path);
  std::map<std::pair<int, int>, std::complex<double>> m;
  int i, j, mx = -1;
  double a, b, c, d;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty()) continue;
    std::istringstream ls(line);
    if (six_cols) {
      if (!(ls >> i >> j >> a >> b >> c >> d)) throw std::runtime_error("Parsing error in " + path);
      (*second)[{i, j}] = {c, d};
    } else if (!(ls >> i >> j >> a >> b)) {
      throw std::runtime_error("Parsing error in " + path);
    }
    m[{i, j}] = {a, b};
    mx = std::max(mx, std::max(i, j));
  }
  *dim = mx + 1;
  return m;
}

std::vector<double> dense(const std::map<std::pair<int, int>, std::complex<double>>& m, int D) {
  std::vector<double> x(2 * size_t(D) * D, 0.0);
  for (const auto& [k, v] : m) {
    x[2 * (size_t(k.first) * D + k.second)] = v.real();
    x[2 * (size_t(k.first) * D + k.second) + 1] = v.imag();
  }
  return x;
}

double profile_trampoline(double t, void* user) {
  return (*static_cast<std::function<double(double)>*>(user))(t);
}

}  // namespace

void edgeDensityResponse_compute_rt(unsigned N, unsigned m, std::vector<int> am,
                                    std::function<double(double)> f, double end_time,
                                    double save_step, int fileNumber) {
  const std::string base = out_root(int(N), int(m)) + "/ExternalExcitation/Statistics/";
  const std::string fn = std::to_string(fileNumber) + ".tsv";
  int D = 0, d2 = 0, d3 = 0;
  const auto Mm = read_tsv(base + "Metric/" + fn, &D, false, nullptr);
  const auto Hm = read_tsv(base + "Hamiltonian/" + fn, &d2, false, nullptr);
  const auto Um = read_tsv(base + "ExcitationPotential/" + fn, &d3, false, nullptr);
  std::printf("Time-evolution in the [ ");
  for (int l : am) std::printf("%d ", l);
  std::printf("] angular momentum subspaces. Number of edge states: %d\n", D);
  if (am.empty() || am[0] != 0)
    die("The Laughlin state (assumed to be the initial state) is not included in the subspace!");
  std::vector<double> rho;
  for (int l : am) {
    std::map<std::pair<int, int>, std::complex<double>> sn;
    int dl = 0;
    const auto cs = read_tsv(base + "EdgeDenstiy_FourierTransform/dL=" + std::to_string(l) + "/" + fn,
                             &dl, true, &sn);
    std::vector<double> r(2 * size_t(D) * D, 0.0);
    for (const auto& [k, v] : cs) {
      const std::complex<double> s = sn[k];
      const std::complex<double> val = v + std::complex<double>(0, 1) * s;  // cos + i sin
      r[2 * (size_t(k.first) * D + k.second)] = val.real();
      r[2 * (size_t(k.first) * D + k.second) + 1] = val.imag();
    }
    rho.insert(rho.end(), r.begin(), r.end());
  }
  const std::vector<double> M = dense(Mm, D), H = dense(Hm, D), U = dense(Um, D);
  const int ns = int(std::ceil(end_time / save_step));
  std::vector<double> out(2 * size_t(ns) * am.size()), norms(ns);
  int n_save = 0;
  std::printf("\tSetting up the Schrodinger system...\n");
  check(lemc_evolve(D, M.data(), H.data(), U.data(), int(am.size()), rho.data(), &profile_trampoline,
                    &f, end_time, save_step, out.data(), norms.data(), &n_save),
        "lemc_evolve");
  std::printf("\tDone (final norm %.6f). Saving...\n", norms.empty() ? 0.0 : norms.back());
  for (size_t l = 0; l < am.size(); ++l) {
    const std::string dir = base + "edgeDynamics/dL=" + std::to_string(am[l]);
    std::filesystem::create_directories(dir);
    std::ofstream o(dir + "/" + fn);
    for (int s = 0; s < n_save; ++s) {
      const size_t q = 2 * (size_t(s) * am.size() + l);
      o << fmtnum(s * save_step, 6) << "\t" << fmtnum(out[q], 6) << "\t" << fmtnum(out[q + 1], 6) << "\n";
    }
  }
}

}  // namespace timeEvolution
