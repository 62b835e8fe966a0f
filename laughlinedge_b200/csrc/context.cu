// C-ABI context: owns the device buffers of one sampling job and drives the
// sweep -> basis -> Gram pipeline on its own CUDA stream.
//
// Reference correspondence: this replaces the host drivers *_compute
// (modules/edge_mc/em_spectrum.cu:210-422, em_metric.cu:200-392,
// em_dsf.cu:235-500): where the reference launches one <<<32,128>>> kernel
// per basis row and reduces per-block partial sums on the host, one context
// here samples every row of every selected sector in the same launches and
// keeps FP64 accumulators resident on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "lemc_internal.h"
#include "partitions.hpp"

using namespace lemc;

namespace {

constexpr int kRowAcc = 13;  // accumulators per (row, column) of the row estimator

#define LEMC_CUDA(call)                                 \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) {                            \
      last_cuda_error() = e_;                           \
      return LEMC_ERR_CUDA;                             \
    }                                                   \
  } while (0)

#define LEMC_TRY(call)      \
  do {                      \
    int s_ = (call);        \
    if (s_ != LEMC_OK) return s_; \
  } while (0)

cudaError_t& last_cuda_error() {
  static thread_local cudaError_t e = cudaSuccess;
  return e;
}

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  int alloc(size_t count) {
    if (count <= n && p) return LEMC_OK;
    release();
    if (count == 0) return LEMC_OK;
    if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) {
      p = nullptr;
      n = 0;
      return LEMC_ERR_CUDA;
    }
    n = count;
    return LEMC_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// Sokal's automatic windowing estimate of the integrated autocorrelation time
// of one series (A. D. Sokal, "Monte Carlo methods in statistical mechanics",
// 1997): tau(M) = 1/2 + sum_{t=1..M} rho(t), smallest window M with
// M >= c tau(M).  NaN when no window up to T/2 satisfies the condition, when
// the series is shorter than 100 or than 50 max(tau, 1) (below that the estimate is biased low by
// the subtracted sample mean and a self-consistent window can appear
// spuriously), or when the series is constant.
double tau_int_sokal(const double* x, size_t T, double c = 5.0) {
  if (T < 8) return NAN;
  double mean = 0;
  for (size_t i = 0; i < T; ++i) mean += x[i];
  mean /= T;
  double c0 = 0;
  for (size_t i = 0; i < T; ++i) c0 += (x[i] - mean) * (x[i] - mean);
  c0 /= T;
  if (!(c0 > 0)) return NAN;
  double tau = 0.5;
  for (size_t t = 1; t < T / 2; ++t) {
    double ct = 0;
    for (size_t s = 0; s + t < T; ++s) ct += (x[s] - mean) * (x[s + t] - mean);
    ct /= T;
    tau += ct / c0;
    if (double(t) >= c * tau) return (T >= 100 && double(T) >= 50.0 * std::max(tau, 1.0)) ? tau : NAN;
  }
  return NAN;
}

// Binning analysis (H. Flyvbjerg and H. G. Petersen, J. Chem. Phys. 91, 461
// (1989)): at bin length b = 2^k the variance of the bin means s_b^2 gives
// tau(b) = b s_b^2 / (2 s_1^2), which rises to the integrated autocorrelation
// time once b is well above it.  Levels run while at least min_bins bins
// remain; the estimate is the last level, its error tau(b) sqrt(2 / (n_b - 1)),
// and the plateau is declared when the last two levels agree within twice
// that error (or 5 %).
int binning(const double* x, size_t T, int min_bins, double* tau, double* tau_err,
            double* err_of_mean, int* converged) {
  if (T < size_t(2 * std::max(2, min_bins))) return LEMC_ERR_ARG;
  double mean = 0;
  for (size_t i = 0; i < T; ++i) mean += x[i];
  mean /= T;
  double v1 = 0;
  for (size_t i = 0; i < T; ++i) v1 += (x[i] - mean) * (x[i] - mean);
  v1 /= double(T - 1);
  double prev = NAN, last = NAN, last_err = NAN, last_em = NAN;
  for (size_t b = 1;; b *= 2) {
    const size_t nb = T / b;
    if (nb < size_t(std::max(2, min_bins))) break;
    double mb = 0;
    std::vector<double> means(nb);
    for (size_t j = 0; j < nb; ++j) {
      double sm = 0;
      for (size_t i = 0; i < b; ++i) sm += x[j * b + i];
      means[j] = sm / b;
      mb += means[j];
    }
    mb /= nb;
    double sb = 0;
    for (double m : means) sb += (m - mb) * (m - mb);
    sb /= double(nb - 1);
    prev = last;
    last = v1 > 0 ? 0.5 * b * sb / v1 : NAN;
    last_err = last * std::sqrt(2.0 / double(nb - 1));
    last_em = std::sqrt(sb / nb);
  }
  if (tau) *tau = last;
  if (tau_err) *tau_err = last_err;
  if (err_of_mean) *err_of_mean = last_em;
  if (converged)
    *converged = (std::isfinite(prev) && std::isfinite(last) &&
                  std::fabs(last - prev) <= std::max(2.0 * last_err, 0.05 * last)) ? 1 : 0;
  return LEMC_OK;
}

}  // namespace

struct lemc_ctx {
  lemc_config cfg{};
  int G = 8;
  int N = 0, m = 0, W = 0, Wpad = 0;
  float R = 1.f;
  cudaStream_t stream = nullptr;
  bool profile = false;

  // basis
  bool has_basis = false;
  Basis basis;
  int K = 0;              // power sums recorded (>= 4 for the series)
  int D = 0;              // total rows
  std::vector<int> sec_row;   // first V row of each sector (Re rows)
  std::vector<int> sec_goff;  // offset (complex entries) of each sector's D x D block
  size_t gram_plane = 0;      // sum_s D_s^2
  std::vector<std::pair<int, int>> cross_pairs;
  std::vector<size_t> cross_off;
  size_t cross_plane = 0;
  int n_gram_jobs = 0, n_cross_jobs = 0;
  std::vector<int> row_vre, row_vim;  // V rows of each basis row
  // Range factors: V holds c_r v_r, so the FP32 products and the tensor-core
  // accumulation of every state stay O(1); the FP64 sums are divided by
  // c_a c_b when read.  Set once per basis, from the walkers at the first
  // measured sweep (Laughlin guide; 1 for the row guide, whose ratios v_b/v_a
  // are formed from V directly).
  // bins: FP64 Gram sums (device layout, range factors included) of each
  // closed bin, and the cumulative sums at the last close
  std::vector<std::vector<double>> bins;
  std::vector<double> bin_samples;
  std::vector<double> bin_last;
  uint64_t bin_last_meas = 0;
  std::vector<double> row_scale;      // per basis row
  std::vector<BasisNode> prog_host;   // the basis program (with its sentinels)
  DevBuf<float> d_node_scale;         // per program node
  bool scale_pending = false;
  bool gram_tune_pending = false;  // autotune the contraction's walker split
  int gram_splits = 0;             // the tuned split (0: one-wave rule)

  std::vector<int> probes;  // angular probes l_q
  // guide rows
  std::vector<int32_t> walker_row;
  std::vector<int32_t> row_first;  // walkers of row a: [row_first[a], row_first[a+1])

  // device buffers
  DevBuf<float2> pos;
  DevBuf<float2> rec_p;
  DevBuf<float> rec_w;
  DevBuf<float> V;
  DevBuf<uint32_t> accepted;
  DevBuf<BasisNode> prog;
  DevBuf<int> prog_seg;
  BasisProgram bprog;
  DevBuf<GramJob> jobs;
  DevBuf<double> gram;      // 3 planes x gram_plane complex
  DevBuf<double> cross;     // 3 planes x cross_plane complex
  DevBuf<double> series;
  DevBuf<int32_t> d_walker_row, d_guide_pairs, d_guide_npairs, d_row_first, d_row_re, d_row_im;
  DevBuf<double> rowacc;
  DevBuf<int> err;
  // tcgen05 path
  std::vector<TcTile> tc_tiles;
  int tc_ntiles = 0, tc_maxdim = 0;
  DevBuf<TcSector> d_tc_secs;
  DevBuf<TcTile> d_tc_tiles;
  DevBuf<double> tc_partials;
  int tc_splits = 1;

  bool walkers_ready = false;
  bool hooked = false;  // a user-potential hook fills the USER plane
  int multipole_k = 0;  // > 0: the USER plane is multipole_amp * sum_i r_i^k cos(k theta_i)
  double multipole_amp = 0;
  uint64_t sweeps = 0, meas = 0, sweeps_at_reset = 0;
  std::vector<double> host_series;  // [meas][8]
  double ms_sweep = 0, ms_basis = 0, ms_gram = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> pev;  // per-step profiling events (profile mode)
  // graph replay of measured sweeps (cfg.graph_batch > 0): device counters
  // {sweep index, measurement index} advanced inside the graph, and the
  // instantiated graph with the state it was captured for
  DevBuf<uint32_t> d_ctr;
  const lemc_proposal* prop = nullptr;  // learned proposal (null: Gaussian step)
  cudaGraphExec_t gexec = nullptr;
  uint64_t version = 0;          // bumped by every setter that changes launch arguments
  uint64_t graph_version = ~uint64_t(0);
  int graph_steps = 0;
  const double* graph_series = nullptr;
};

namespace {

int pick_lanes(int N) {
  // walker width: aim for about 6-12 particles per lane
  int G = 1;
  while (G < 32 && (N + G - 1) / G > 16) G *= 2;
  while (G > 1 && !sweep_config_ok(G, N)) G /= 2;
  while (G < 32 && !sweep_config_ok(G, N)) G *= 2;
  return G;
}

int build_program(lemc_ctx* c) {
  // DFS over non-increasing part sequences with sum <= max sector and at most
  // N parts.  Node value = parent value * p_part.
  const Basis& B = c->basis;
  std::map<std::vector<int>, int> key_to_row;
  for (size_t r = 0; r < B.rows.size(); ++r) {
    std::vector<int> parts;
    for (const auto& pp : B.rows[r].pairs)
      for (int q = 0; q < pp.mult; ++q) parts.push_back(pp.part);
    std::sort(parts.begin(), parts.end(), std::greater<int>());
    key_to_row[parts] = int(r);
  }
  int smax = 0;
  bool want0 = false;
  for (int s : B.sectors) {
    smax = std::max(smax, s);
    if (s == 0) want0 = true;
  }
  std::vector<BasisNode> prog;
  if (want0) {
    auto it = key_to_row.find(std::vector<int>{0});
    if (it != key_to_row.end())
      prog.push_back({1, 0, c->row_vre[it->second], c->row_vim[it->second]});
  }
  std::vector<int> seq;
  // iterative DFS
  struct Frame { int sum, maxpart, next; };
  std::vector<Frame> st;
  st.push_back({0, smax, 1});
  while (!st.empty()) {
    Frame& f = st.back();
    const int part = f.next;
    if (part > f.maxpart || f.sum + part > smax || int(seq.size()) >= c->N) {
      st.pop_back();
      if (!seq.empty()) seq.pop_back();
      continue;
    }
    f.next++;
    seq.push_back(part);
    std::vector<int> key(seq.begin(), seq.end());
    std::sort(key.begin(), key.end(), std::greater<int>());
    auto it = key_to_row.find(key);
    BasisNode nd{int(seq.size()), part, -1, -1};
    if (it != key_to_row.end()) {
      nd.row_re = c->row_vre[it->second];
      nd.row_im = c->row_vim[it->second];
    }
    prog.push_back(nd);
    st.push_back({f.sum + part, part, 1});
  }
  // the DFS above extends sequences with parts <= previous part, i.e. each
  // multiset exactly once, ordered non-increasingly.
  const int n = int(prog.size());
  int max_depth = 0, max_part = 0;
  for (const BasisNode& nd : prog) {
    max_depth = std::max(max_depth, nd.depth);
    max_part = std::max(max_part, nd.part);
  }
  prog.push_back({0, 0, -1, -1});  // two sentinels: the kernel reads up to two nodes ahead
  prog.push_back({0, 0, -1, -1});
  c->prog_host = prog;
  LEMC_TRY(c->prog.alloc(prog.size()));
  LEMC_CUDA(cudaMemcpy(c->prog.p, prog.data(), prog.size() * sizeof(BasisNode),
                       cudaMemcpyHostToDevice));
  // Segments: cut at the depth-1 node nearest to each of the kMaxBasisSegments
  // equal shares of the program.
  BasisProgram& bp = c->bprog;
  bp = BasisProgram{};
  bp.nodes = c->prog.p;
  bp.n_nodes = n;
  bp.max_depth = max_depth;
  bp.max_part = max_part;
  std::vector<int> roots;
  for (int t = 1; t < n; ++t)
    if (prog[t].depth == 1) roots.push_back(t);
  std::vector<int> cuts{0};
  for (int k = 1; k < kMaxBasisSegments; ++k) {
    const long ideal = long(k) * n / kMaxBasisSegments;
    int best = -1;
    for (int r : roots)
      if (r > cuts.back() && (best < 0 || std::labs(r - ideal) < std::labs(best - ideal))) best = r;
    if (best > cuts.back()) cuts.push_back(best);
  }
  cuts.push_back(n);
  bp.n_seg = int(cuts.size()) - 1;
  for (int j = 0; j < bp.n_seg; ++j) bp.max_seg = std::max(bp.max_seg, cuts[j + 1] - cuts[j]);
  LEMC_TRY(c->prog_seg.alloc(cuts.size()));
  LEMC_CUDA(cudaMemcpy(c->prog_seg.p, cuts.data(), cuts.size() * sizeof(int),
                       cudaMemcpyHostToDevice));
  bp.seg_dev = c->prog_seg.p;
  return LEMC_OK;
}

int alloc_records(lemc_ctx* c) {
  LEMC_TRY(c->rec_p.alloc(size_t(c->K) * c->W));
  LEMC_TRY(c->rec_w.alloc(size_t(LEMC_N_WEIGHTS) * c->Wpad));
  LEMC_CUDA(cudaMemsetAsync(c->rec_w.p, 0, sizeof(float) * LEMC_N_WEIGHTS * c->Wpad, c->stream));
  if (c->D > 0) {
    LEMC_TRY(c->V.alloc(size_t(2) * c->D * c->Wpad));
    LEMC_CUDA(cudaMemsetAsync(c->V.p, 0, sizeof(float) * 2 * c->D * c->Wpad, c->stream));
  }
  return LEMC_OK;
}

int setup_tc(lemc_ctx* c, int force_splits = 0);

// SIMT job list: same-sector Gram tiles {ONE, R2, R4} and, for every ordered
// pair of sectors (diagonal pairs included), cross tiles {USER, COS_l, SIN_l}
// with l = |dL_j - dL_i| (cos/sin disabled unless l is a probe).
int build_jobs(lemc_ctx* c) {
  const auto& sec = c->basis.sectors;
  std::vector<GramJob> jobs;
  for (size_t s = 0; s < sec.size(); ++s) {
    const int dim = c->basis.sector_dim[s];
    for (int a0 = 0; a0 < dim; a0 += 16)
      for (int b0 = 0; b0 < dim; b0 += 16)
        jobs.push_back({c->sec_row[s], dim, c->sec_row[s], dim, a0, b0,
                        {LEMC_W_ONE, LEMC_W_R2, LEMC_W_R4}, 0, c->sec_goff[s]});
  }
  c->n_gram_jobs = int(jobs.size());
  c->cross_pairs.clear();
  c->cross_off.clear();
  size_t coff = 0;
  for (size_t i = 0; i < sec.size(); ++i)
    for (size_t j = 0; j < sec.size(); ++j) {
      const int l = std::abs(sec[j] - sec[i]);
      int pc = -1, ps = -1;
      for (size_t q = 0; q < c->probes.size(); ++q)
        if (c->probes[q] == l) {
          pc = LEMC_W_PROBE0 + 2 * int(q);
          ps = pc + 1;
        }
      c->cross_pairs.push_back({int(i), int(j)});
      c->cross_off.push_back(coff);
      const int da = c->basis.sector_dim[i], db = c->basis.sector_dim[j];
      for (int a0 = 0; a0 < da; a0 += 16)
        for (int b0 = 0; b0 < db; b0 += 16)
          jobs.push_back({c->sec_row[i], da, c->sec_row[j], db, a0, b0, {LEMC_W_USER, pc, ps}, 1,
                          int(coff)});
      coff += size_t(da) * db;
    }
  c->cross_plane = coff;
  c->n_cross_jobs = int(jobs.size()) - c->n_gram_jobs;
  LEMC_TRY(c->jobs.alloc(std::max<size_t>(1, jobs.size())));
  if (!jobs.empty())
    LEMC_CUDA(cudaMemcpy(c->jobs.p, jobs.data(), jobs.size() * sizeof(GramJob), cudaMemcpyHostToDevice));
  LEMC_TRY(c->cross.alloc(6 * std::max<size_t>(1, c->cross_plane)));
  LEMC_CUDA(cudaMemsetAsync(c->cross.p, 0, sizeof(double) * c->cross.n, c->stream));
  return LEMC_OK;
}

int upload_guide(lemc_ctx* c) {
  if (c->cfg.guide != LEMC_GUIDE_ROW || !c->has_basis) return LEMC_OK;
  const int R = int(c->basis.rows.size());
  std::vector<int32_t> pairs(size_t(R) * 2 * kMaxGuideParts, 0), np(R, 0);
  for (int r = 0; r < R; ++r) {
    const auto& pr = c->basis.rows[r].pairs;
    if (int(pr.size()) > kMaxGuideParts) return LEMC_ERR_CAPACITY;
    np[r] = int(pr.size());
    for (size_t q = 0; q < pr.size(); ++q) {
      // part 0 (the dL = 0 row) is the constant p_0 = N: no guide factor
      pairs[size_t(r) * 2 * kMaxGuideParts + 2 * q] = pr[q].part;
      pairs[size_t(r) * 2 * kMaxGuideParts + 2 * q + 1] = pr[q].part > 0 ? pr[q].mult : 0;
    }
  }
  LEMC_TRY(c->d_guide_pairs.alloc(pairs.size()));
  LEMC_TRY(c->d_guide_npairs.alloc(np.size()));
  LEMC_CUDA(cudaMemcpy(c->d_guide_pairs.p, pairs.data(), pairs.size() * 4, cudaMemcpyHostToDevice));
  LEMC_CUDA(cudaMemcpy(c->d_guide_npairs.p, np.data(), np.size() * 4, cudaMemcpyHostToDevice));
  if (c->walker_row.empty()) {
    // default: every row, walkers split into contiguous equal blocks
    std::vector<int32_t> rows(R);
    for (int r = 0; r < R; ++r) rows[r] = r;
    c->walker_row.assign(c->W, 0);
    c->row_first.assign(R + 1, 0);
    for (int w = 0; w < c->W; ++w) c->walker_row[w] = int32_t((int64_t(w) * R) / c->W);
  }
  // row_first from walker_row (walker blocks must be contiguous per row)
  c->row_first.assign(R + 1, 0);
  for (int w = 0; w < c->W; ++w) c->row_first[c->walker_row[w] + 1]++;
  for (int r = 0; r < R; ++r) c->row_first[r + 1] += c->row_first[r];
  for (int w = 1; w < c->W; ++w)
    if (c->walker_row[w] < c->walker_row[w - 1]) return LEMC_ERR_ARG;
  LEMC_TRY(c->d_walker_row.alloc(c->W));
  LEMC_TRY(c->d_row_first.alloc(R + 1));
  LEMC_CUDA(cudaMemcpy(c->d_walker_row.p, c->walker_row.data(), 4 * c->W, cudaMemcpyHostToDevice));
  LEMC_CUDA(cudaMemcpy(c->d_row_first.p, c->row_first.data(), 4 * (R + 1), cudaMemcpyHostToDevice));
  LEMC_TRY(c->d_row_re.alloc(R));
  LEMC_TRY(c->d_row_im.alloc(R));
  LEMC_CUDA(cudaMemcpy(c->d_row_re.p, c->row_vre.data(), 4 * R, cudaMemcpyHostToDevice));
  LEMC_CUDA(cudaMemcpy(c->d_row_im.p, c->row_vim.data(), 4 * R, cudaMemcpyHostToDevice));
  LEMC_TRY(c->rowacc.alloc(size_t(R) * R * kRowAcc));
  LEMC_CUDA(cudaMemset(c->rowacc.p, 0, sizeof(double) * R * R * kRowAcc));
  return LEMC_OK;
}

SweepArgs sweep_args(const lemc_ctx* c, int n_sweeps, int measure) {
  SweepArgs a{};
  a.pos = c->pos.p;
  a.rec_p = c->rec_p.p;
  a.rec_w = c->rec_w.p;
  a.accepted = c->accepted.p;
  a.reverse_evals = c->accepted.p + c->W;
  a.walker_row = c->d_walker_row.p;
  a.guide_pairs = c->d_guide_pairs.p;
  a.guide_npairs = c->d_guide_npairs.p;
  a.err = c->err.p;
  a.W = c->W;
  a.ldw = c->Wpad;
  a.N = c->N;
  a.Npad = c->N;
  a.m = c->m;
  a.K = c->K;
  a.sigma = c->cfg.step_sigma;
  a.invR = 1.f / c->R;
  a.seed_lo = uint32_t(c->cfg.seed);
  a.seed_hi = uint32_t(c->cfg.seed >> 32);
  a.sweep0 = uint32_t(c->sweeps);
  a.n_sweeps = n_sweeps;
  a.measure = measure;
  a.guide = c->cfg.guide;
  a.n_probes = int(c->probes.size());
  for (int q = 0; q < a.n_probes; ++q) a.probes[q] = c->probes[q];
  return a;
}

int launch_sweep_for(lemc_ctx* c, const SweepArgs& a) {
  if (c->prop) return launch_learned_sweep(a, lemc_proposal_weights(c->prop), c->stream);
  return launch_sweep(a, c->G, c->stream);
}

int sweep_once(lemc_ctx* c, int n_sweeps, int measure) {
  return launch_sweep_for(c, sweep_args(c, n_sweeps, measure));
}

int gram_step(lemc_ctx* c, const float* V, const float* rec_w, int ldw, int W, int mode) {
  if (c->cfg.guide == LEMC_GUIDE_ROW) {
    return launch_row_accumulate(V, c->Wpad, rec_w, ldw, W, c->d_row_first.p,
                                 int(c->basis.rows.size()), c->D, c->d_row_re.p, c->d_row_im.p,
                                 c->rowacc.p, c->stream);
  }
  const bool cross =
      c->n_cross_jobs > 0 && (c->hooked || c->multipole_k > 0 || !c->probes.empty());
  if (mode == LEMC_GRAM_FP64) {
    const int splits = std::max(1, std::min(64, W / 1024));
    return launch_gram_simt(V, c->Wpad, rec_w, ldw, W, c->jobs.p,
                            c->n_gram_jobs + (cross ? c->n_cross_jobs : 0), splits, c->gram.p,
                            c->gram_plane, c->cross.p, c->cross_plane, c->stream);
  }
  if (c->tc_tiles.empty()) LEMC_TRY(setup_tc(c, c->gram_splits));
  int s = launch_gram_tc_rows(V, c->Wpad, 2 * c->D, rec_w, ldw, c->Wpad, c->d_tc_tiles.p,
                              int(c->tc_tiles.size()), c->tc_splits, c->tc_partials.p, mode,
                              c->cfg.flush_every, c->err.p, c->stream);
  if (s != LEMC_OK) return s;
  // cross-sector planes (user potential, cos/sin probes): FP64 path
  if (cross) {
    const int splits = std::max(1, std::min(64, W / 1024));
    s = launch_gram_simt(V, c->Wpad, rec_w, ldw, W, c->jobs.p + c->n_gram_jobs, c->n_cross_jobs,
                         splits, c->gram.p, c->gram_plane, c->cross.p, c->cross_plane, c->stream);
  }
  return s;
}

// Walker split of the contraction's jobs (tiles x splits, one CTA per SM, each
// split a contiguous walker range): the smallest split whose jobs fill at
// least 95 % of the SM slots of the waves they take, else the best filling one,
// among 1..max(8, sm / tiles).  A split that adds waves keeps at least 8192
// walkers (256 K-chunks) per job, so a job's start-up and its partial-slot
// traffic stay small against its work.  E.g. 604 tiles on 148 SMs at 65536
// walkers: split 1 fills 4.08 of 5 waves (82 %), split 4 fills 16.3 of 17
// (96 %); at 8192 walkers it stays 1; 20 tiles: split 7 gives 140 jobs (95 %);
// one tile: 141 jobs.
int wave_split(int nt, int sm, int smax, int wpad) {
  int best = 1;
  double best_fill = 0.0;
  const int top = std::min(smax, std::max(8, sm / std::max(1, nt)));
  for (int s = 1; s <= top; ++s) {
    if (long(std::max(1, nt)) * s > sm && s > 1 && wpad / s < 8192) break;
    const long jobs = long(std::max(1, nt)) * s;
    const long waves = (jobs + sm - 1) / sm;
    const double fill = double(jobs) / double(waves * sm);
    if (fill >= 0.95) return s;
    if (fill > best_fill + 1e-9) {
      best_fill = fill;
      best = s;
    }
  }
  return best;
}

int setup_tc(lemc_ctx* c, int force_splits) {
  // Sector-aligned panels: consecutive sectors of at most 128 V rows are packed
  // into one 128-row A panel with 32-row B panels over the group's rows; a
  // larger sector gets its own 128-row A slices x 32-row B panels.
  const int ns = int(c->sec_row.size());
  std::vector<std::pair<int, int>> tiles;
  std::vector<TcSector> secs(ns);
  for (int i = 0; i < ns;) {
    const int r0 = c->sec_row[i], d0 = 2 * c->basis.sector_dim[i];
    if (d0 > 128) {
      // The real Gram block is symmetric: a tile whose B panel lies wholly
      // above its A slice (32 (y + 1) <= 128 x) is the transpose of a kept
      // tile and is skipped; A slice x keeps B panels y >= 4 x.
      const int na = (d0 + 127) / 128, nb = (d0 + 31) / 32;
      const int t0 = int(tiles.size());
      for (int x = 0; x < na; ++x)
        for (int y = 4 * x; y < nb; ++y) tiles.push_back({r0 + 128 * x, r0 + 32 * y});
      secs[i] = {r0, c->basis.sector_dim[i], c->sec_goff[i], t0, r0, r0, nb};
      ++i;
      continue;
    }
    int j = i, g1 = r0;
    while (j < ns && 2 * c->basis.sector_dim[j] <= 128 &&
           c->sec_row[j] + 2 * c->basis.sector_dim[j] - r0 <= 128) {
      g1 = c->sec_row[j] + 2 * c->basis.sector_dim[j];
      ++j;
    }
    const int nb = (g1 - r0 + 31) / 32;
    const int t0 = int(tiles.size());
    for (int y = 0; y < nb; ++y) tiles.push_back({r0, r0 + 32 * y});
    for (int q = i; q < j; ++q)
      secs[q] = {c->sec_row[q], c->basis.sector_dim[q], c->sec_goff[q], t0, r0, r0, nb};
    i = j;
  }
  int sm = 148;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
  const int nt = int(tiles.size());
  c->tc_ntiles = nt;
  c->tc_maxdim = 0;
  for (int d : c->basis.sector_dim) c->tc_maxdim = std::max(c->tc_maxdim, d);
  // one CTA per SM: the split that fills whole waves (unless the autotuner
  // chose one)
  c->tc_splits = force_splits > 0 ? std::min(force_splits, std::max(1, c->Wpad / 128))
                                  : wave_split(nt, sm, std::max(1, c->Wpad / 128), c->Wpad);
  c->tc_tiles.clear();
  for (int sp = 0; sp < c->tc_splits; ++sp)
    for (int t = 0; t < nt; ++t)
      c->tc_tiles.push_back({tiles[t].first, tiles[t].second, sp, sp * nt + t});
  LEMC_TRY(c->d_tc_tiles.alloc(c->tc_tiles.size()));
  LEMC_CUDA(cudaMemcpy(c->d_tc_tiles.p, c->tc_tiles.data(), sizeof(TcTile) * c->tc_tiles.size(),
                       cudaMemcpyHostToDevice));
  LEMC_TRY(c->d_tc_secs.alloc(ns));
  LEMC_CUDA(cudaMemcpy(c->d_tc_secs.p, secs.data(), sizeof(TcSector) * ns, cudaMemcpyHostToDevice));
  const size_t slot = size_t(kTcSlot);
  LEMC_TRY(c->tc_partials.alloc(slot * c->tc_tiles.size()));
  LEMC_CUDA(cudaMemsetAsync(c->tc_partials.p, 0, sizeof(double) * slot * c->tc_tiles.size(),
                            c->stream));
  return LEMC_OK;
}

// Fold the tcgen05 partial slots into the FP64 Gram planes (idempotent use:
// partials are zeroed afterwards).
int flush_tc(lemc_ctx* c) {
  if (c->tc_tiles.empty()) return LEMC_OK;
  LEMC_TRY(launch_gram_tc_reduce(c->tc_partials.p, c->d_tc_tiles.p, c->d_tc_secs.p,
                                 int(c->sec_row.size()), c->tc_ntiles, c->tc_splits, c->tc_maxdim,
                                 c->gram.p, c->gram_plane, c->stream));
  LEMC_CUDA(cudaMemsetAsync(c->tc_partials.p, 0, sizeof(double) * kTcSlot * c->tc_tiles.size(),
                            c->stream));
  return LEMC_OK;
}

}  // namespace

extern "C" {

int lemc_version(void) { return 10000; }

const char* lemc_status_string(int s) {
  switch (s) {
    case LEMC_OK: return "ok";
    case LEMC_ERR_ARG: return "invalid argument";
    case LEMC_ERR_CAPACITY: return "capacity exceeded";
    case LEMC_ERR_CUDA: return cudaGetErrorString(last_cuda_error());
    case LEMC_ERR_TIMEOUT: return "bounded device wait timed out";
    case LEMC_ERR_NUMERIC: return "numerical failure (metric not positive definite)";
    case LEMC_ERR_STATE: return "call out of order";
    case LEMC_ERR_NODEVICE: return "no CUDA device";
    case LEMC_ERR_IO: return "file i/o error";
    default: return "unknown status";
  }
}

int lemc_device_count(int* count) {
  if (!count) return LEMC_ERR_ARG;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    *count = 0;
    return LEMC_ERR_NODEVICE;
  }
  *count = n;
  return LEMC_OK;
}

int lemc_partitions(int particles, const int32_t* sectors, int n_sectors, lemc_partition_row* rows,
                    int max_rows, int32_t* pairs, int max_pair_ints, int* n_rows, int* n_pair_ints,
                    int* max_degree, int* longest) {
  if (particles <= 0 || n_sectors <= 0 || !sectors) return LEMC_ERR_ARG;
  std::vector<int> sec(sectors, sectors + n_sectors);
  for (int s : sec)
    if (s < 0 || s > 64) return LEMC_ERR_ARG;
  Basis B = build_basis(particles, sec);
  int total_pairs = 0;
  for (const auto& r : B.rows) total_pairs += 2 * int(r.pairs.size());
  if (n_rows) *n_rows = int(B.rows.size());
  if (n_pair_ints) *n_pair_ints = total_pairs;
  if (max_degree) *max_degree = B.max_degree;
  if (longest) *longest = B.longest;
  if (!rows) return LEMC_OK;
  if (max_rows < int(B.rows.size()) || max_pair_ints < total_pairs || !pairs)
    return LEMC_ERR_CAPACITY;
  int off = 0;
  for (size_t i = 0; i < B.rows.size(); ++i) {
    rows[i].dL = B.rows[i].dL;
    rows[i].sector_size = B.rows[i].sector_size;
    rows[i].n_pairs = int(B.rows[i].pairs.size());
    rows[i].pairs_off = off;
    for (const auto& pp : B.rows[i].pairs) {
      pairs[off++] = pp.part;
      pairs[off++] = pp.mult;
    }
  }
  return LEMC_OK;
}

int lemc_create(const lemc_config* cfg, lemc_ctx** out) {
  if (!cfg || !out) return LEMC_ERR_ARG;
  *out = nullptr;
  if (cfg->particles < 2 || cfg->particles > LEMC_MAX_PARTICLES) return LEMC_ERR_ARG;
  if (cfg->inverse_filling < 1 || cfg->n_walkers < 1 || !(cfg->step_sigma > 0.f))
    return LEMC_ERR_ARG;
  if (cfg->guide != LEMC_GUIDE_LAUGHLIN && cfg->guide != LEMC_GUIDE_ROW) return LEMC_ERR_ARG;
  if (cfg->gram_mode < LEMC_GRAM_FP64 || cfg->gram_mode > LEMC_GRAM_TF32X3) return LEMC_ERR_ARG;
  if (cfg->graph_batch < 0 || cfg->graph_batch > 4096) return LEMC_ERR_ARG;
  int ndev = 0;
  if (lemc_device_count(&ndev) != LEMC_OK) return LEMC_ERR_NODEVICE;
  lemc_ctx* c = new lemc_ctx();
  c->cfg = *cfg;
  c->N = cfg->particles;
  c->m = cfg->inverse_filling;
  c->W = cfg->n_walkers;
  c->Wpad = (c->W + 63) / 64 * 64;
  const double rcl = std::sqrt(2.0 * c->m * c->N);
  c->R = float(cfg->radius_scale > 0 ? cfg->radius_scale : rcl);
  c->profile = cfg->profile != 0;
  c->G = cfg->lanes_per_walker > 0 ? cfg->lanes_per_walker : pick_lanes(c->N);
  if (!sweep_config_ok(c->G, c->N)) {
    delete c;
    return LEMC_ERR_CAPACITY;
  }
  int st = LEMC_OK;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) st = LEMC_ERR_CUDA;
  for (auto& e : c->ev)
    if (st == LEMC_OK && cudaEventCreate(&e) != cudaSuccess) st = LEMC_ERR_CUDA;
  if (st == LEMC_OK) st = c->pos.alloc(size_t(c->W) * c->N);
  if (st == LEMC_OK) st = c->accepted.alloc(2 * size_t(c->W));  // accepted | reverse evaluations
  if (st == LEMC_OK) st = c->err.alloc(1);
  if (st == LEMC_OK && cudaMemset(c->accepted.p, 0, 8 * c->W) != cudaSuccess) st = LEMC_ERR_CUDA;
  if (st == LEMC_OK && cudaMemset(c->err.p, 0, sizeof(int)) != cudaSuccess) st = LEMC_ERR_CUDA;
  if (st != LEMC_OK) {
    lemc_destroy(c);
    return st;
  }
  *out = c;
  return LEMC_OK;
}

int lemc_destroy(lemc_ctx* c) {
  if (!c) return LEMC_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->pos.release();
  c->rec_p.release();
  c->rec_w.release();
  c->V.release();
  c->accepted.release();
  c->prog.release();
  c->prog_seg.release();
  c->jobs.release();
  c->gram.release();
  c->cross.release();
  c->series.release();
  c->d_walker_row.release();
  c->d_guide_pairs.release();
  c->d_guide_npairs.release();
  c->d_row_first.release();
  c->d_row_re.release();
  c->d_row_im.release();
  c->rowacc.release();
  c->err.release();
  c->d_tc_tiles.release();
  c->d_tc_secs.release();
  c->tc_partials.release();
  c->d_node_scale.release();
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : c->pev) cudaEventDestroy(e);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  c->d_ctr.release();
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return LEMC_OK;
}

int lemc_set_sectors(lemc_ctx* c, const int32_t* sectors, int n) {
  if (!c || !sectors || n <= 0) return LEMC_ERR_ARG;
  ++c->version;
  std::vector<int> sec(sectors, sectors + n);
  for (size_t i = 0; i < sec.size(); ++i) {
    if (sec[i] < 0 || sec[i] > kMaxDegree) return LEMC_ERR_CAPACITY;
    for (size_t j = 0; j < i; ++j)
      if (sec[j] == sec[i]) return LEMC_ERR_ARG;
  }
  c->basis = build_basis(c->N, sec);
  c->has_basis = true;
  c->D = int(c->basis.rows.size());
  c->K = std::max(4, c->basis.max_degree);
  if (c->K > kMaxDegree) return LEMC_ERR_CAPACITY;
  // V rows: sector s occupies [2*first_s, 2*first_s + 2*D_s): Re rows then Im rows
  c->sec_row.clear();
  c->sec_goff.clear();
  c->row_vre.assign(c->D, 0);
  c->row_vim.assign(c->D, 0);
  size_t goff = 0;
  for (size_t s = 0; s < sec.size(); ++s) {
    const int first = c->basis.sector_first[s], dim = c->basis.sector_dim[s];
    c->sec_row.push_back(2 * first);
    c->sec_goff.push_back(int(goff));
    goff += size_t(dim) * dim;
    for (int r = 0; r < dim; ++r) {
      c->row_vre[first + r] = 2 * first + r;
      c->row_vim[first + r] = 2 * first + dim + r;
    }
  }
  c->gram_plane = goff;
  LEMC_TRY(build_jobs(c));
  LEMC_TRY(c->gram.alloc(6 * c->gram_plane));
  LEMC_TRY(build_program(c));
  LEMC_TRY(alloc_records(c));
  c->row_scale.assign(c->D, 1.0);
  LEMC_TRY(c->d_node_scale.alloc(c->prog_host.size()));
  {
    std::vector<float> ones(c->prog_host.size(), 1.f);
    LEMC_CUDA(cudaMemcpy(c->d_node_scale.p, ones.data(), sizeof(float) * ones.size(),
                         cudaMemcpyHostToDevice));
  }
  c->bprog.node_scale = c->d_node_scale.p;
  c->scale_pending = c->cfg.guide == LEMC_GUIDE_LAUGHLIN;
  c->gram_tune_pending = c->cfg.lanes_per_walker < 0 && c->cfg.guide == LEMC_GUIDE_LAUGHLIN &&
                         c->cfg.gram_mode != LEMC_GRAM_FP64;
  c->gram_splits = 0;
  c->tc_tiles.clear();
  LEMC_TRY(upload_guide(c));
  return lemc_reset_accumulators(c);
}

int lemc_set_guide_rows(lemc_ctx* c, const int32_t* rows, int n_rows) {
  if (!c) return LEMC_ERR_ARG;
  ++c->version;
  if (!c->has_basis) return LEMC_ERR_STATE;
  c->walker_row.clear();
  if (rows && n_rows > 0) {
    const int R = int(c->basis.rows.size());
    c->walker_row.resize(c->W);
    for (int q = 0; q < n_rows; ++q)
      if (rows[q] < 0 || rows[q] >= R) return LEMC_ERR_ARG;
    // contiguous blocks: walker w -> rows[(w * n_rows) / W]
    for (int w = 0; w < c->W; ++w) c->walker_row[w] = rows[(int64_t(w) * n_rows) / c->W];
    for (int w = 1; w < c->W; ++w)
      if (c->walker_row[w] < c->walker_row[w - 1]) return LEMC_ERR_ARG;
  }
  return upload_guide(c);
}

// Walker-width autotuner: times single sweeps per feasible G on a copy of the
// current walkers (restored afterwards, sweep counter unchanged), measured
// ones when the context has a basis, as a sampling step runs them, and keeps
// the fastest (best of two rounds of three).  Used when lanes_per_walker < 0.
static int autotune_lanes(lemc_ctx* c) {
  DevBuf<float2> save;
  LEMC_TRY(save.alloc(size_t(c->W) * c->N));
  LEMC_CUDA(cudaMemcpyAsync(save.p, c->pos.p, sizeof(float2) * c->W * c->N,
                            cudaMemcpyDeviceToDevice, c->stream));
  const int keep_G = c->G;
  float best = 1e30f;
  int bestG = keep_G;
  const int meas = (c->has_basis && c->rec_p.p && c->rec_w.p) ? 1 : 0;
  for (int G = 1; G <= 32; G *= 2) {
    if (!sweep_config_ok(G, c->N)) continue;
    c->G = G;
    LEMC_TRY(sweep_once(c, 1, meas));  // warm the instruction cache / attributes
    float ms = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {
      LEMC_CUDA(cudaEventRecord(c->ev[0], c->stream));
      for (int k = 0; k < 3; ++k) LEMC_TRY(sweep_once(c, 1, meas));
      LEMC_CUDA(cudaEventRecord(c->ev[1], c->stream));
      LEMC_CUDA(cudaEventSynchronize(c->ev[1]));
      float t = 0;
      cudaEventElapsedTime(&t, c->ev[0], c->ev[1]);
      ms = std::min(ms, t);
    }
    if (ms < best) {
      best = ms;
      bestG = G;
    }
    LEMC_CUDA(cudaMemcpyAsync(c->pos.p, save.p, sizeof(float2) * c->W * c->N,
                              cudaMemcpyDeviceToDevice, c->stream));
  }
  c->G = bestG;
  ++c->version;
  if (c->accepted.p) LEMC_CUDA(cudaMemsetAsync(c->accepted.p, 0, 8 * c->W, c->stream));
  LEMC_CUDA(cudaStreamSynchronize(c->stream));
  save.release();
  return LEMC_OK;
}

int lemc_gram_splits(const lemc_ctx* c, int* splits) {
  if (!c || !splits) return LEMC_ERR_ARG;
  *splits = c->tc_tiles.empty() ? c->gram_splits : c->tc_splits;
  return LEMC_OK;
}

int lemc_lanes_per_walker(const lemc_ctx* c, int* G) {
  if (!c || !G) return LEMC_ERR_ARG;
  *G = c->G;
  return LEMC_OK;
}

int lemc_init_walkers(lemc_ctx* c, const float* host_xy) {
  if (!c) return LEMC_ERR_ARG;
  if (host_xy) {
    LEMC_CUDA(cudaMemcpyAsync(c->pos.p, host_xy, sizeof(float2) * c->W * c->N,
                              cudaMemcpyHostToDevice, c->stream));
  } else {
    const double r0 = c->cfg.init_radius > 0 ? c->cfg.init_radius : std::sqrt(2.0 * c->m * c->N);
    LEMC_TRY(launch_init_walkers(c->pos.p, c->W, c->N, float(r0), uint32_t(c->cfg.seed),
                                 uint32_t(c->cfg.seed >> 32), c->stream));
  }
  c->walkers_ready = true;
  if (c->cfg.lanes_per_walker < 0) LEMC_TRY(autotune_lanes(c));
  return LEMC_OK;
}

int lemc_reset_accumulators(lemc_ctx* c) {
  if (!c) return LEMC_ERR_ARG;
  if (c->gram.p) LEMC_CUDA(cudaMemsetAsync(c->gram.p, 0, sizeof(double) * c->gram.n, c->stream));
  if (c->cross.p) LEMC_CUDA(cudaMemsetAsync(c->cross.p, 0, sizeof(double) * c->cross.n, c->stream));
  if (c->rowacc.p) LEMC_CUDA(cudaMemsetAsync(c->rowacc.p, 0, sizeof(double) * c->rowacc.n, c->stream));
  if (c->tc_partials.p)
    LEMC_CUDA(cudaMemsetAsync(c->tc_partials.p, 0, sizeof(double) * c->tc_partials.n, c->stream));
  if (c->accepted.p) LEMC_CUDA(cudaMemsetAsync(c->accepted.p, 0, 8 * c->W, c->stream));
  if (c->err.p) LEMC_CUDA(cudaMemsetAsync(c->err.p, 0, sizeof(int), c->stream));
  c->meas = 0;
  c->bins.clear();
  c->bin_samples.clear();
  c->bin_last.clear();
  c->bin_last_meas = 0;
  c->host_series.clear();
  c->ms_sweep = c->ms_basis = c->ms_gram = 0;
  c->sweeps_at_reset = c->sweeps;
  return LEMC_OK;
}

int lemc_synchronize(lemc_ctx* c) {
  if (!c) return LEMC_ERR_ARG;
  LEMC_CUDA(cudaStreamSynchronize(c->stream));
  int herr = 0;
  LEMC_CUDA(cudaMemcpy(&herr, c->err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (herr != 0) return LEMC_ERR_TIMEOUT;
  return LEMC_OK;
}

int lemc_set_step(lemc_ctx* c, float sigma) {
  if (!c || !(sigma > 0.f)) return LEMC_ERR_ARG;
  c->cfg.step_sigma = sigma;
  ++c->version;
  return LEMC_OK;
}

int lemc_set_proposal(lemc_ctx* c, const lemc_proposal* p) {
  if (!c) return LEMC_ERR_ARG;
  if (p) {
    if (lemc_proposal_particles(p) != c->N || lemc_proposal_filling(p) != c->m) return LEMC_ERR_ARG;
    if (c->cfg.guide != LEMC_GUIDE_LAUGHLIN) return LEMC_ERR_ARG;
  }
  c->prop = p;
  ++c->version;
  return LEMC_OK;
}

int lemc_copy_positions_device(lemc_ctx* c, void* dst) {
  if (!c || !dst) return LEMC_ERR_ARG;
  LEMC_CUDA(cudaMemcpyAsync(dst, c->pos.p, sizeof(float2) * size_t(c->W) * c->N,
                            cudaMemcpyDeviceToDevice, c->stream));
  return LEMC_OK;
}

int lemc_stream(lemc_ctx* c, void** stream) {
  if (!c || !stream) return LEMC_ERR_ARG;
  *stream = static_cast<void*>(c->stream);
  return LEMC_OK;
}

static int run_impl(lemc_ctx* c, int n_sweeps, int measure, lemc_step_hook hook, void* user);

int lemc_run(lemc_ctx* c, int n_sweeps, int measure) {
  return run_impl(c, n_sweeps, measure, nullptr, nullptr);
}

int lemc_run_hooked(lemc_ctx* c, int n_sweeps, lemc_step_hook hook, void* user) {
  if (!hook) return LEMC_ERR_ARG;
  return run_impl(c, n_sweeps, 1, hook, user);
}

int lemc_set_multipole_potential(lemc_ctx* c, int k, double amplitude) {
  if (!c || k < 0) return LEMC_ERR_ARG;
  if (k > 0 && !c->has_basis) return LEMC_ERR_STATE;
  if (k > c->K) return LEMC_ERR_CAPACITY;
  c->multipole_k = k;
  c->multipole_amp = amplitude;
  ++c->version;
  return LEMC_OK;
}

int lemc_set_probes(lemc_ctx* c, const int32_t* l, int n) {
  if (!c || n < 0 || n > LEMC_MAX_PROBES || (n > 0 && !l)) return LEMC_ERR_ARG;
  ++c->version;
  c->probes.assign(l, l + n);
  for (int q : c->probes)
    if (q < 0 || q > 1024) return LEMC_ERR_ARG;
  if (c->has_basis) LEMC_TRY(build_jobs(c));
  return LEMC_OK;
}

static int multipole_step(lemc_ctx* c) {
  if (c->multipole_k <= 0) return LEMC_OK;
  return launch_multipole_plane(c->rec_p.p, c->W, c->K, c->multipole_k,
                                c->multipole_amp * std::pow(double(c->R), c->multipole_k),
                                c->rec_w.p + size_t(LEMC_W_USER) * c->Wpad, c->stream);
}

// One measured sweep with every per-step value taken from the device counters
// (sweep index ctr[0], measurement index ctr[1]), then the counters advance:
// G of these are captured once into a CUDA graph and replayed.
static int graph_step(lemc_ctx* c) {
  SweepArgs a = sweep_args(c, 1, 1);
  a.sweep0 = 0;
  a.sweep_ctr = c->d_ctr.p;
  LEMC_TRY(launch_sweep_for(c, a));
  LEMC_TRY(launch_basis(c->rec_p.p, c->W, c->K, c->N, c->bprog, c->V.p, c->Wpad,
                        c->series.p, c->d_ctr.p + 1, c->stream));
  LEMC_TRY(multipole_step(c));
  LEMC_TRY(gram_step(c, c->V.p, c->rec_w.p, c->Wpad, c->W, c->cfg.gram_mode));
  return launch_advance_counters(c->d_ctr.p, c->stream);
}

// Instantiate (or reuse) the graph of G measured sweeps for the current state.
static int ensure_graph(lemc_ctx* c, int G) {
  if (c->gexec && c->graph_version == c->version && c->graph_steps == G &&
      c->graph_series == c->series.p)
    return LEMC_OK;
  if (c->gexec) {
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  // everything the captured launches point at must exist before capture
  LEMC_TRY(c->d_ctr.alloc(2));
  if (c->cfg.guide != LEMC_GUIDE_ROW && c->cfg.gram_mode != LEMC_GRAM_FP64 && c->tc_tiles.empty())
    LEMC_TRY(setup_tc(c, c->gram_splits));
  cudaGraph_t g = nullptr;
  LEMC_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
  int st = LEMC_OK;
  for (int i = 0; i < G && st == LEMC_OK; ++i) st = graph_step(c);
  const cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
  if (st != LEMC_OK || ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return st != LEMC_OK ? st : LEMC_ERR_CUDA;
  }
  const cudaError_t ie = cudaGraphInstantiate(&c->gexec, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) {
    c->gexec = nullptr;
    cudaGetLastError();
    return LEMC_ERR_CUDA;
  }
  c->graph_version = c->version;
  c->graph_steps = G;
  c->graph_series = c->series.p;
  return LEMC_OK;
}

// Range factors c_r = exp(-<ln|v_r|>), the inverse geometric mean of |v_r| over
// up to 2048 of the current walkers (p_k from their positions in FP64, p_0 = N,
// ln|p| floored at -80), clamped to [1e-30, 1e30].  Called once per basis
// before its first measured sweep, with the accumulators empty.
static int compute_row_scales(lemc_ctx* c) {
  const int Ws = std::min(c->W, 2048), N = c->N, K = c->K, D = c->D;
  std::vector<float2> xy(size_t(Ws) * N);
  LEMC_CUDA(cudaMemcpyAsync(xy.data(), c->pos.p, sizeof(float2) * xy.size(), cudaMemcpyDeviceToHost,
                            c->stream));
  LEMC_CUDA(cudaStreamSynchronize(c->stream));
  std::vector<double> lp(size_t(K + 1) * Ws);  // ln|p_k| per walker
  const double invR = 1.0 / c->R;
  for (int w = 0; w < Ws; ++w) {
    std::vector<double> re(K + 1, 0.0), im(K + 1, 0.0);
    for (int i = 0; i < N; ++i) {
      const double x = xy[size_t(w) * N + i].x * invR, y = xy[size_t(w) * N + i].y * invR;
      double zr = 1, zi = 0;
      for (int k = 1; k <= K; ++k) {
        const double t = zr * x - zi * y;
        zi = zr * y + zi * x;
        zr = t;
        re[k] += zr;
        im[k] += zi;
      }
    }
    lp[w] = std::log(double(N));
    for (int k = 1; k <= K; ++k)
      lp[size_t(k) * Ws + w] = std::max(-80.0, 0.5 * std::log(re[k] * re[k] + im[k] * im[k]));
  }
  std::vector<float> vrow(2 * size_t(D), 1.f);  // per V row
  for (int r = 0; r < D; ++r) {
    double mean = 0;
    for (const auto& pp : c->basis.rows[r].pairs) {
      double sk = 0;
      for (int w = 0; w < Ws; ++w) sk += lp[size_t(pp.part) * Ws + w];
      mean += pp.mult * sk / Ws;
    }
    const double sc = std::min(1e30, std::max(1e-30, std::exp(-mean)));
    const float scf = float(sc);
    c->row_scale[r] = double(scf);  // the factor the kernel applies, exactly
    vrow[c->row_vre[r]] = scf;
    vrow[c->row_vim[r]] = scf;
  }
  std::vector<float> dev(c->prog_host.size(), 1.f);  // per program node
  for (size_t t = 0; t < dev.size(); ++t)
    if (c->prog_host[t].row_re >= 0) dev[t] = vrow[c->prog_host[t].row_re];
  LEMC_CUDA(cudaMemcpyAsync(c->d_node_scale.p, dev.data(), sizeof(float) * dev.size(),
                            cudaMemcpyHostToDevice, c->stream));
  LEMC_CUDA(cudaStreamSynchronize(c->stream));
  return LEMC_OK;
}

// Contraction autotuner (lanes_per_walker < 0, tensor-core modes): the walker
// split of the tcgen05 jobs decides how many CTAs a launch has (tiles x split)
// and how full its last wave is.  On a copy of the walkers, one sweep and one
// basis build fill V; each candidate split (the wave-filling rule, the splits
// that give 1, 2, 3 or 4 full waves of jobs, and 1, 2, 4, 8) is timed over three launches
// (best of two), the fastest kept.  The walkers are restored and the
// accumulators zeroed, so the chain and its sums are those of an untuned run.
static int autotune_gram_splits(lemc_ctx* c) {
  int sm = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
  LEMC_TRY(setup_tc(c, 0));
  const int nt = c->tc_ntiles, smax = std::max(1, c->Wpad / 128);
  std::vector<int> cand{c->tc_splits};
  for (int waves = 1; waves <= 4; ++waves) {
    const int sp = std::min(smax, std::max(1, (waves * sm) / std::max(1, nt)));
    if (std::find(cand.begin(), cand.end(), sp) == cand.end()) cand.push_back(sp);
  }
  for (int sp : {1, 2, 4, 8})
    if (sp <= smax && std::find(cand.begin(), cand.end(), sp) == cand.end()) cand.push_back(sp);
  DevBuf<float2> save;
  LEMC_TRY(save.alloc(size_t(c->W) * c->N));
  LEMC_CUDA(cudaMemcpyAsync(save.p, c->pos.p, sizeof(float2) * c->W * c->N,
                            cudaMemcpyDeviceToDevice, c->stream));
  LEMC_TRY(sweep_once(c, 1, 1));
  LEMC_TRY(launch_basis(c->rec_p.p, c->W, c->K, c->N, c->bprog, c->V.p, c->Wpad, nullptr,
                        nullptr, c->stream));
  float best = 1e30f;
  int best_sp = cand[0];
  for (int sp : cand) {
    LEMC_TRY(setup_tc(c, sp));
    auto launch = [&]() {
      return launch_gram_tc_rows(c->V.p, c->Wpad, 2 * c->D, c->rec_w.p, c->Wpad, c->Wpad,
                                 c->d_tc_tiles.p, int(c->tc_tiles.size()), c->tc_splits,
                                 c->tc_partials.p, c->cfg.gram_mode, c->cfg.flush_every, c->err.p,
                                 c->stream);
    };
    LEMC_TRY(launch());  // warm
    float ms = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {
      LEMC_CUDA(cudaEventRecord(c->ev[0], c->stream));
      for (int k = 0; k < 3; ++k) LEMC_TRY(launch());
      LEMC_CUDA(cudaEventRecord(c->ev[1], c->stream));
      LEMC_CUDA(cudaEventSynchronize(c->ev[1]));
      float t = 0;
      cudaEventElapsedTime(&t, c->ev[0], c->ev[1]);
      ms = std::min(ms, t);
    }
    if (ms < best) {
      best = ms;
      best_sp = sp;
    }
  }
  c->gram_splits = best_sp;
  LEMC_TRY(setup_tc(c, best_sp));
  LEMC_CUDA(cudaMemcpyAsync(c->pos.p, save.p, sizeof(float2) * c->W * c->N,
                            cudaMemcpyDeviceToDevice, c->stream));
  if (c->accepted.p) LEMC_CUDA(cudaMemsetAsync(c->accepted.p, 0, 8 * c->W, c->stream));
  LEMC_CUDA(cudaMemsetAsync(c->tc_partials.p, 0, sizeof(double) * c->tc_partials.n, c->stream));
  LEMC_CUDA(cudaMemsetAsync(c->gram.p, 0, sizeof(double) * c->gram.n, c->stream));
  LEMC_CUDA(cudaStreamSynchronize(c->stream));
  ++c->version;
  save.release();
  return lemc_synchronize(c);
}

static int run_impl(lemc_ctx* c, int n_sweeps, int measure, lemc_step_hook hook, void* user) {
  if (!c || n_sweeps < 0) return LEMC_ERR_ARG;
  if (!c->walkers_ready) return LEMC_ERR_STATE;
  if (measure && !c->has_basis) return LEMC_ERR_STATE;
  if (n_sweeps == 0) return LEMC_OK;
  if (!measure) {
    // burn-in: chunks of sweeps per launch, no records
    for (int done = 0; done < n_sweeps;) {
      const int chunk = std::min(64, n_sweeps - done);
      LEMC_TRY(sweep_once(c, chunk, 0));
      c->sweeps += chunk;
      done += chunk;
    }
    return LEMC_OK;
  }
  if (c->scale_pending && c->meas == 0) {
    LEMC_TRY(compute_row_scales(c));
    c->scale_pending = false;
  }
  if (c->gram_tune_pending && c->meas == 0) {
    LEMC_TRY(autotune_gram_splits(c));
    c->gram_tune_pending = false;
  }
  LEMC_TRY(c->series.alloc(size_t(8) * n_sweeps));
  LEMC_CUDA(cudaMemsetAsync(c->series.p, 0, sizeof(double) * 8 * n_sweeps, c->stream));
  // profile mode: four events per step, read after the loop (no per-step sync)
  if (c->profile) {
    while (c->pev.size() < size_t(4) * n_sweeps) {
      cudaEvent_t e;
      LEMC_CUDA(cudaEventCreate(&e));
      c->pev.push_back(e);
    }
  }
  int s0 = 0;
  const int G = c->cfg.graph_batch;
  if (G > 0 && !hook && !c->profile && n_sweeps >= G) {
    // whole batches of G measured sweeps as one graph launch each
    LEMC_TRY(ensure_graph(c, G));
    const uint32_t h_ctr[2] = {uint32_t(c->sweeps), 0u};
    LEMC_CUDA(cudaMemcpyAsync(c->d_ctr.p, h_ctr, sizeof(h_ctr), cudaMemcpyHostToDevice, c->stream));
    const int reps = n_sweeps / G;
    for (int r = 0; r < reps; ++r) LEMC_CUDA(cudaGraphLaunch(c->gexec, c->stream));
    s0 = reps * G;
    c->sweeps += uint64_t(s0);
    c->meas += uint64_t(s0);
  }
  for (int s = s0; s < n_sweeps; ++s) {
    if (c->profile) LEMC_CUDA(cudaEventRecord(c->pev[4 * s], c->stream));
    LEMC_TRY(sweep_once(c, 1, 1));
    c->sweeps += 1;
    if (c->profile) LEMC_CUDA(cudaEventRecord(c->pev[4 * s + 1], c->stream));
    LEMC_TRY(launch_basis(c->rec_p.p, c->W, c->K, c->N, c->bprog, c->V.p, c->Wpad,
                          c->series.p + 8 * size_t(s), nullptr, c->stream));
    LEMC_TRY(multipole_step(c));
    if (hook) {
      if (!c->hooked) ++c->version;
      c->hooked = true;
      const int hs = hook(user, reinterpret_cast<const float*>(c->pos.p),
                          c->rec_w.p + size_t(LEMC_W_USER) * c->Wpad, c->W, c->N,
                          static_cast<void*>(c->stream));
      if (hs != LEMC_OK) return hs;
    }
    if (c->profile) LEMC_CUDA(cudaEventRecord(c->pev[4 * s + 2], c->stream));
    LEMC_TRY(gram_step(c, c->V.p, c->rec_w.p, c->Wpad, c->W, c->cfg.gram_mode));
    if (c->profile) LEMC_CUDA(cudaEventRecord(c->pev[4 * s + 3], c->stream));
    c->meas += 1;
  }
  std::vector<double> ser(size_t(8) * n_sweeps);
  LEMC_CUDA(cudaMemcpyAsync(ser.data(), c->series.p, sizeof(double) * ser.size(),
                            cudaMemcpyDeviceToHost, c->stream));
  LEMC_TRY(lemc_synchronize(c));
  if (c->profile) {
    for (int s = 0; s < n_sweeps; ++s) {
      float t = 0;
      cudaEventElapsedTime(&t, c->pev[4 * s], c->pev[4 * s + 1]);
      c->ms_sweep += t;
      cudaEventElapsedTime(&t, c->pev[4 * s + 1], c->pev[4 * s + 2]);
      c->ms_basis += t;
      cudaEventElapsedTime(&t, c->pev[4 * s + 2], c->pev[4 * s + 3]);
      c->ms_gram += t;
    }
  }
  for (double& v : ser) v /= c->W;
  c->host_series.insert(c->host_series.end(), ser.begin(), ser.end());
  return LEMC_OK;
}

int lemc_sector_dim(const lemc_ctx* c, int s, int* dim) {
  if (!c || !dim) return LEMC_ERR_ARG;
  if (!c->has_basis) return LEMC_ERR_STATE;
  if (s < 0 || s >= int(c->basis.sector_dim.size())) return LEMC_ERR_ARG;
  *dim = c->basis.sector_dim[s];
  return LEMC_OK;
}

int lemc_total_dim(const lemc_ctx* c, int* dim) {
  if (!c || !dim) return LEMC_ERR_ARG;
  if (!c->has_basis) return LEMC_ERR_STATE;
  *dim = c->D;
  return LEMC_OK;
}

int lemc_read_gram(lemc_ctx* c, int s, double* S, double* H2, double* H4, double* n_samples) {
  if (!c) return LEMC_ERR_ARG;
  if (!c->has_basis) return LEMC_ERR_STATE;
  if (s < 0 || s >= int(c->sec_row.size())) return LEMC_ERR_ARG;
  LEMC_TRY(flush_tc(c));
  const int dim = c->basis.sector_dim[s];
  const size_t off = 2 * size_t(c->sec_goff[s]);
  const size_t bytes = sizeof(double) * 2 * dim * dim;
  double* outs[3] = {S, H2, H4};
  for (int h = 0; h < 3; ++h)
    if (outs[h])
      LEMC_CUDA(cudaMemcpyAsync(outs[h], c->gram.p + 2 * c->gram_plane * h + off, bytes,
                                cudaMemcpyDeviceToHost, c->stream));
  LEMC_TRY(lemc_synchronize(c));
  if (n_samples) *n_samples = double(c->meas) * c->W;
  // undo the range factors; a non-finite sum (an FP32 overflow of the basis
  // values or of the accumulation) is reported, never returned silently
  const double* sc = c->row_scale.data() + c->basis.sector_first[s];
  bool finite = true;
  for (int h = 0; h < 3; ++h) {
    if (!outs[h]) continue;
    for (int a = 0; a < dim; ++a)
      for (int b = 0; b < dim; ++b) {
        const double f = 1.0 / (sc[a] * sc[b]);
        double* e = outs[h] + 2 * (size_t(a) * dim + b);
        e[0] *= f;
        e[1] *= f;
        finite = finite && std::isfinite(e[0]) && std::isfinite(e[1]);
      }
  }
  return finite ? LEMC_OK : LEMC_ERR_NUMERIC;
}

int lemc_read_cross(lemc_ctx* c, int sa, int sb, double* Cuser, double* Ccos, double* Csin) {
  if (!c) return LEMC_ERR_ARG;
  if (!c->has_basis) return LEMC_ERR_STATE;
  for (size_t q = 0; q < c->cross_pairs.size(); ++q) {
    if (c->cross_pairs[q].first != sa || c->cross_pairs[q].second != sb) continue;
    const int da = c->basis.sector_dim[sa], db = c->basis.sector_dim[sb];
    const size_t n = size_t(da) * db;
    double* outs[3] = {Cuser, Ccos, Csin};
    for (int h = 0; h < 3; ++h)
      if (outs[h])
        LEMC_CUDA(cudaMemcpyAsync(outs[h], c->cross.p + 2 * c->cross_plane * h + 2 * c->cross_off[q],
                                  sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, c->stream));
    LEMC_TRY(lemc_synchronize(c));
    const double* ca = c->row_scale.data() + c->basis.sector_first[sa];
    const double* cb = c->row_scale.data() + c->basis.sector_first[sb];
    bool finite = true;
    for (int h = 0; h < 3; ++h) {
      if (!outs[h]) continue;
      for (int a = 0; a < da; ++a)
        for (int b = 0; b < db; ++b) {
          const double f = 1.0 / (ca[a] * cb[b]);
          double* e = outs[h] + 2 * (size_t(a) * db + b);
          e[0] *= f;
          e[1] *= f;
          finite = finite && std::isfinite(e[0]) && std::isfinite(e[1]);
        }
    }
    return finite ? LEMC_OK : LEMC_ERR_NUMERIC;
  }
  return LEMC_ERR_ARG;
}

int lemc_read_rows(lemc_ctx* c, double omega, double kappa, double* fg, double* gg, double* fh,
                   double* fcos, double* fsin, double* fuser, double* n_per_row) {
  if (!c) return LEMC_ERR_ARG;
  if (!c->has_basis || c->cfg.guide != LEMC_GUIDE_ROW) return LEMC_ERR_STATE;
  const int D = c->D;
  std::vector<double> acc(size_t(D) * D * kRowAcc);
  LEMC_CUDA(cudaMemcpyAsync(acc.data(), c->rowacc.p, sizeof(double) * acc.size(),
                            cudaMemcpyDeviceToHost, c->stream));
  LEMC_TRY(lemc_synchronize(c));
  for (int a = 0; a < D; ++a) {
    const double n = double(c->meas) * (c->row_first[a + 1] - c->row_first[a]);
    const double inv = n > 0 ? 1.0 / n : 0.0;
    for (int b = 0; b < D; ++b) {
      const double* q = &acc[(size_t(a) * D + b) * kRowAcc];
      const size_t o = size_t(a) * D + b;
      if (fg) { fg[2 * o] = q[0] * inv; fg[2 * o + 1] = q[1] * inv; }
      if (gg) gg[o] = q[2] * inv;
      if (fh) {
        fh[2 * o] = (omega * q[3] + kappa * q[5]) * inv;
        fh[2 * o + 1] = (omega * q[4] + kappa * q[6]) * inv;
      }
      if (fcos) { fcos[2 * o] = q[7] * inv; fcos[2 * o + 1] = q[8] * inv; }
      if (fsin) { fsin[2 * o] = q[9] * inv; fsin[2 * o + 1] = q[10] * inv; }
      if (fuser) { fuser[2 * o] = q[11] * inv; fuser[2 * o + 1] = q[12] * inv; }
    }
    if (n_per_row) n_per_row[a] = n;
  }
  return LEMC_OK;
}

int lemc_read_stats(lemc_ctx* c, lemc_stats* st) {
  if (!c || !st) return LEMC_ERR_ARG;
  std::memset(st, 0, sizeof(*st));
  std::vector<uint32_t> acc(2 * size_t(c->W));
  LEMC_CUDA(cudaMemcpyAsync(acc.data(), c->accepted.p, 8 * c->W, cudaMemcpyDeviceToHost, c->stream));
  LEMC_TRY(lemc_synchronize(c));
  double tot = 0, rev = 0;
  for (int w = 0; w < c->W; ++w) {
    tot += acc[w];
    rev += acc[c->W + w];
  }
  const double swept = double(c->sweeps - c->sweeps_at_reset);
  const double moves = swept * c->W * c->N;
  st->sweeps = c->sweeps;
  st->measurements = c->meas;
  st->acceptance = swept > 0 ? tot / moves : 0.0;
  st->reverse_fraction = swept > 0 ? rev / moves : 0.0;
  // tau_int: Sokal windowing on the walker-mean series of Re and Im p_k; NaN
  // (for that k, and then for the maximum) when the series is too short for a
  // self-consistent window.
  const size_t M = c->host_series.size() / 8;
  double tmax = 0;
  for (int k = 0; k < 4; ++k) {
    double tk = 0;
    for (int comp = 0; comp < 2; ++comp) {
      std::vector<double> x(M);
      for (size_t i = 0; i < M; ++i) x[i] = c->host_series[8 * i + 2 * k + comp];
      tk += 0.5 * tau_int_sokal(x.data(), x.size());
    }
    st->tau_int_each[k] = tk;
    tmax = (std::isnan(tk) || std::isnan(tmax)) ? NAN : std::max(tmax, tk);
  }
  st->tau_int = M > 0 ? tmax : NAN;
  st->ms_sweep = c->ms_sweep;
  st->ms_basis = c->ms_basis;
  st->ms_gram = c->ms_gram;
  return LEMC_OK;
}

int lemc_read_positions(lemc_ctx* c, float* xy) {
  if (!c || !xy) return LEMC_ERR_ARG;
  LEMC_CUDA(cudaMemcpyAsync(xy, c->pos.p, sizeof(float2) * c->W * c->N, cudaMemcpyDeviceToHost,
                            c->stream));
  return lemc_synchronize(c);
}

int lemc_read_series(lemc_ctx* c, double* series, int max_meas, int* n_meas) {
  if (!c) return LEMC_ERR_ARG;
  const int M = int(c->host_series.size() / 8);
  if (n_meas) *n_meas = M;
  if (series) std::memcpy(series, c->host_series.data(), sizeof(double) * 8 * std::min(M, max_meas));
  return LEMC_OK;
}

int lemc_sweep_device(void* pos, int W, int N, int m, float sigma, uint64_t seed, uint32_t sweep0,
                      int n_sweeps, int K, double radius_scale, int G, int measure,
                      const int32_t* probes, int n_probes, void* rec_p, void* rec_w,
                      void* accepted, void* stream) {
  if (!pos || W <= 0 || N < 2 || m < 1 || K < 1 || K > kMaxDegree) return LEMC_ERR_ARG;
  if (n_probes < 0 || n_probes > LEMC_MAX_PROBES || (n_probes > 0 && !probes)) return LEMC_ERR_ARG;
  if (measure && (!rec_p || !rec_w)) return LEMC_ERR_ARG;
  if (G <= 0) G = pick_lanes(N);
  if (!sweep_config_ok(G, N)) return LEMC_ERR_CAPACITY;
  SweepArgs a{};
  a.pos = static_cast<float2*>(pos);
  a.rec_p = static_cast<float2*>(rec_p);
  a.rec_w = static_cast<float*>(rec_w);
  a.accepted = static_cast<uint32_t*>(accepted);
  a.W = W;
  a.ldw = W;
  a.N = N;
  a.Npad = N;
  a.m = m;
  a.K = K;
  a.sigma = sigma;
  a.invR = float(1.0 / (radius_scale > 0 ? radius_scale : std::sqrt(2.0 * m * N)));
  a.seed_lo = uint32_t(seed);
  a.seed_hi = uint32_t(seed >> 32);
  a.sweep0 = sweep0;
  a.n_sweeps = n_sweeps;
  a.measure = measure;
  a.guide = LEMC_GUIDE_LAUGHLIN;
  a.n_probes = n_probes;
  for (int q = 0; q < n_probes; ++q) a.probes[q] = probes[q];
  return launch_sweep(a, G, static_cast<cudaStream_t>(stream));
}

// Work launched on a caller's stream is ordered before everything the context
// issues afterwards on its own (non-blocking) stream.
static int order_after(lemc_ctx* c, cudaStream_t user) {
  if (user == c->stream) return LEMC_OK;
  LEMC_CUDA(cudaEventRecord(c->ev[3], user));
  LEMC_CUDA(cudaStreamWaitEvent(c->stream, c->ev[3], 0));
  return LEMC_OK;
}

int lemc_basis_device(lemc_ctx* c, const void* rec_p, int W, void* V, int ldv, void* stream) {
  if (!c || !rec_p || !V || W <= 0 || ldv < W) return LEMC_ERR_ARG;
  if (!c->has_basis) return LEMC_ERR_STATE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  LEMC_TRY(launch_basis(static_cast<const float2*>(rec_p), W, c->K, c->N, c->bprog,
                        static_cast<float*>(V), ldv, nullptr, nullptr, st));
  return order_after(c, st);
}

int lemc_gram_device(lemc_ctx* c, const void* V, const void* rec_w, int W, int ldv, int mode,
                     void* stream) {
  if (!c || !V || !rec_w || W <= 0) return LEMC_ERR_ARG;
  if (!c->has_basis) return LEMC_ERR_STATE;
  if (ldv != c->Wpad || W != c->W) return LEMC_ERR_ARG;
  // the context's accumulators are only touched on its own stream: wait for the
  // caller's stream, run there, and hand the ordering back
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  LEMC_CUDA(cudaEventRecord(c->ev[2], user));
  LEMC_CUDA(cudaStreamWaitEvent(c->stream, c->ev[2], 0));
  LEMC_TRY(gram_step(c, static_cast<const float*>(V), static_cast<const float*>(rec_w), ldv, W,
                     mode));
  LEMC_CUDA(cudaEventRecord(c->ev[3], c->stream));
  LEMC_CUDA(cudaStreamWaitEvent(user, c->ev[3], 0));
  return LEMC_OK;
}

// Acceptance of the current step over `moves` unmeasured sweeps of the live
// chain (the walkers advance; the accumulators are reset).
static int acceptance_at(lemc_ctx* c, float sigma, int moves, double* acc) {
  LEMC_TRY(lemc_set_step(c, sigma));
  LEMC_TRY(lemc_reset_accumulators(c));
  LEMC_TRY(lemc_run(c, moves, 0));
  lemc_stats st;
  LEMC_TRY(lemc_read_stats(c, &st));
  *acc = st.acceptance;
  return LEMC_OK;
}

int lemc_tune_step(lemc_ctx* c, double target, double tol, int moves, float* sigma,
                   double* acceptance) {
  if (!c || !(target > 0 && target < 1) || !(tol > 0) || moves <= 0) return LEMC_ERR_ARG;
  if (!c->walkers_ready) return LEMC_ERR_STATE;
  float s2 = c->cfg.step_sigma;
  double a2 = 0;
  LEMC_TRY(acceptance_at(c, s2, moves, &a2));
  auto done = [&](float s, double a) {
    if (sigma) *sigma = s;
    if (acceptance) *acceptance = a;
    return lemc_set_step(c, s);
  };
  if (std::fabs(a2 - target) < tol) return done(s2, a2);
  // bracket: double (acceptance too high) or halve the step until it crosses
  float s1 = s2;
  double a1 = a2;
  for (int it = 0; it < 40 && (a2 - target) * (a1 - target) > 0; ++it) {
    s1 *= (a2 > target) ? 2.0f : 0.5f;
    LEMC_TRY(acceptance_at(c, s1, moves, &a1));
  }
  if (std::fabs(a1 - target) < tol) return done(s1, a1);
  if ((a2 - target) * (a1 - target) > 0) return LEMC_ERR_NUMERIC;
  if (s2 < s1) {
    std::swap(s1, s2);
    std::swap(a1, a2);
  }
  // regula falsi on the bracket [s1, s2]
  for (int it = 0; it < 60; ++it) {
    const float g = float(((target - a1) * s2 + (a2 - target) * s1) / (a2 - a1));
    double ag = 0;
    LEMC_TRY(acceptance_at(c, g, moves, &ag));
    if (std::fabs(ag - target) < tol) return done(g, ag);
    if ((ag - target) * (a1 - target) < 0) {
      a2 = ag;
      s2 = g;
    } else if ((ag - target) * (a2 - target) < 0) {
      a1 = ag;
      s1 = g;
    } else {
      break;
    }
  }
  return LEMC_ERR_NUMERIC;
}

int lemc_debug_gram_wait(long long cycles, int hold_loads) {
  return set_gram_wait(cycles, hold_loads);
}

int lemc_close_bin(lemc_ctx* c) {
  if (!c) return LEMC_ERR_ARG;
  if (!c->has_basis || c->cfg.guide != LEMC_GUIDE_LAUGHLIN) return LEMC_ERR_STATE;
  if (c->meas == c->bin_last_meas) return LEMC_ERR_STATE;  // empty bin
  LEMC_TRY(flush_tc(c));
  std::vector<double> cur(6 * c->gram_plane);
  LEMC_CUDA(cudaMemcpyAsync(cur.data(), c->gram.p, sizeof(double) * cur.size(),
                            cudaMemcpyDeviceToHost, c->stream));
  LEMC_TRY(lemc_synchronize(c));
  std::vector<double> bin(cur);
  if (!c->bin_last.empty())
    for (size_t i = 0; i < bin.size(); ++i) bin[i] -= c->bin_last[i];
  c->bins.push_back(std::move(bin));
  c->bin_samples.push_back(double(c->meas - c->bin_last_meas) * c->W);
  c->bin_last = std::move(cur);
  c->bin_last_meas = c->meas;
  return LEMC_OK;
}

int lemc_n_bins(const lemc_ctx* c, int* n) {
  if (!c || !n) return LEMC_ERR_ARG;
  *n = int(c->bins.size());
  return LEMC_OK;
}

int lemc_read_gram_bin(lemc_ctx* c, int bin, int s, double* S, double* H2, double* H4,
                       double* n_samples) {
  if (!c) return LEMC_ERR_ARG;
  if (bin < 0 || bin >= int(c->bins.size()) || s < 0 || s >= int(c->sec_row.size()))
    return LEMC_ERR_ARG;
  const int dim = c->basis.sector_dim[s];
  const size_t off = 2 * size_t(c->sec_goff[s]);
  const double* sc = c->row_scale.data() + c->basis.sector_first[s];
  double* outs[3] = {S, H2, H4};
  bool finite = true;
  for (int h = 0; h < 3; ++h) {
    if (!outs[h]) continue;
    const double* src = c->bins[bin].data() + 2 * c->gram_plane * h + off;
    for (int a = 0; a < dim; ++a)
      for (int b = 0; b < dim; ++b) {
        const double f = 1.0 / (sc[a] * sc[b]);
        const size_t o = 2 * (size_t(a) * dim + b);
        outs[h][o] = src[o] * f;
        outs[h][o + 1] = src[o + 1] * f;
        finite = finite && std::isfinite(outs[h][o]) && std::isfinite(outs[h][o + 1]);
      }
  }
  if (n_samples) *n_samples = c->bin_samples[bin];
  return finite ? LEMC_OK : LEMC_ERR_NUMERIC;
}

int lemc_tau_sokal(const double* x, int T, double c, double* tau) {
  if (!x || T < 0 || !tau) return LEMC_ERR_ARG;
  *tau = tau_int_sokal(x, size_t(T), c > 0 ? c : 5.0);
  return LEMC_OK;
}

int lemc_tau_binning(const double* x, int T, int min_bins, double* tau, double* tau_err,
                     double* err_of_mean, int* converged) {
  if (!x || T < 0) return LEMC_ERR_ARG;
  return binning(x, size_t(T), min_bins > 0 ? min_bins : 16, tau, tau_err, err_of_mean, converged);
}

}  // extern "C"
