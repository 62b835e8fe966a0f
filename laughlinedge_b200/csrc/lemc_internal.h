// Internal declarations shared by the CUDA translation units of liblemc.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lemc.h"

namespace lemc {

constexpr int kMaxDegree = LEMC_MAX_DEGREE;
constexpr int kMaxGuideParts = LEMC_MAX_GUIDE_PARTS;
constexpr int kSweepThreads = 256;  // 8 warps per sweep block

// Arguments of one sweep-kernel launch (device pointers).
struct SweepArgs {
  float2* pos;              // [W][N]
  float2* rec_p;            // [K][W] power sums p_1..p_K (measure != 0)
  float* rec_w;             // [LEMC_N_WEIGHTS][W] weight planes (measure != 0)
  uint32_t* accepted;       // [W] accumulated accepted moves (may be null)
  uint32_t* reverse_evals;  // [W] moves whose reverse density was evaluated (learned; may be null)
  const int32_t* walker_row;   // [W] guide row (row guide only)
  const int32_t* guide_pairs;  // [rows][2*kMaxGuideParts] (part, mult)
  const int32_t* guide_npairs; // [rows]
  int* err;                 // device error word (may be null)
  int W, ldw, N, Npad, T2, m, K;  // rec_w row stride ldw; Npad >= T2 * G (sweep_layout)
  float sigma, invR;
  uint32_t seed_lo, seed_hi;
  uint32_t sweep0;
  const uint32_t* sweep_ctr;  // if set, *sweep_ctr is added to sweep0 (graph replay)
  int n_sweeps;
  int measure;
  int guide;
  int n_probes;                  // angular probes l_q recorded as cos/sin planes
  int probes[LEMC_MAX_PROBES];
};

// Node of the depth-first basis program: value[depth] = value[depth-1] * p_part
// (part 0 stands for p_0 = N); rows < 0 mean "not an output".
struct alignas(16) BasisNode {
  int depth;
  int part;
  int row_re;
  int row_im;
};

// The program on the device, cut at depth-1 nodes into segments that need
// only value[0] = 1 and so run as independent thread blocks.  The device
// array holds n_nodes nodes followed by two sentinels {0, 0, -1, -1}.
constexpr int kMaxBasisSegments = 8;
struct BasisProgram {
  const BasisNode* nodes = nullptr;
  int n_nodes = 0;
  int max_depth = 0;
  int max_part = 0;
  int n_seg = 0;
  int max_seg = 0;  // longest segment, in nodes
  const int* seg_dev = nullptr;  // n_seg + 1 segment starts (node indices), on the device
  // per-node factor applied when a node's value is stored (its state's range
  // factor; n_nodes + 2 entries with the sentinels); nullptr stores the plain
  // products
  const float* node_scale = nullptr;
};

// One tile of the SIMT FP64 Gram accumulation: three weighted sums
//   out_h[a][b] += sum_w ONE(w) * P_h(w) * conj(v_a(w)) v_b(w),
// P_h = rec_w plane plane[h] (plane[h] == LEMC_W_ONE: no extra factor,
// plane[h] < 0: the sum is skipped).
struct GramJob {
  int row_a;   // first V row of the Re part of sector a (Im rows follow at +Da)
  int Da;
  int row_b;
  int Db;
  int a0, b0;  // tile origin inside the (Da x Db) block
  int plane[3];
  int buf;     // 0: Gram planes, 1: cross planes
  int out;     // offset (in complex entries) of the (Da x Db) block in the output
};

int launch_sweep(const SweepArgs& a, int lanes_per_walker, cudaStream_t st);
size_t sweep_smem_bytes(int lanes_per_walker, int Npad);
// Shared-memory layout of a walker: T2 slots per lane (ceil(N/G) rounded up
// to even), stored as 16-byte slot-pair records, and an even per-walker stride
// Npad >= T2*G (float2 units) chosen so that the walker groups of a
// quarter-warp hit disjoint banks (Npad = 2G mod 16 for G < 8).
void sweep_layout(int lanes_per_walker, int N, int* T2, int* Npad);
bool sweep_config_ok(int lanes_per_walker, int N);

int launch_init_walkers(float2* pos, int W, int N, float radius, uint32_t seed_lo,
                        uint32_t seed_hi, cudaStream_t st);

// series_idx (may be null): the walker-mean series goes to series + 8 * *series_idx
int launch_basis(const float2* rec_p, int W, int K, int N, const BasisProgram& prog, float* V,
                 int ldv, double* series, const uint32_t* series_idx, cudaStream_t st);
// Bound (cycles, 0 = default) of the contraction's mbarrier waits, and the test
// hook that keeps its loader from issuing (so that every wait expires).
int set_gram_wait(long long cycles, int hold_loads);
// plane[w] = scale * Re p_k[w] (the multipole potential's USER plane)
int launch_multipole_plane(const float2* rec_p, int W, int K, int k, double scale, float* plane,
                           cudaStream_t st);
// Learned-proposal sweep (one walker per warp) with BF16 network weights wts;
// same arguments, records and error conventions as launch_sweep (Laughlin guide).
int launch_learned_sweep(const SweepArgs& a, const void* wts, cudaStream_t st);
// ctr[0] += 1, ctr[1] += 1: sweep and measurement counters of a replayed graph
int launch_advance_counters(uint32_t* ctr, cudaStream_t st);

int launch_gram_simt(const float* V, int ldv, const float* rec_w, int ldw, int W,
                     const GramJob* jobs, int n_jobs, int n_splits, double* out_set0,
                     size_t plane0, double* out_set1, size_t plane1, cudaStream_t st);

int launch_row_accumulate(const float* V, int ldv, const float* rec_w, int ldw, int W,
                          const int32_t* row_first, int n_rows, int D,
                          const int32_t* row_re, const int32_t* row_im, double* acc,
                          cudaStream_t st);

// tcgen05 split-precision Gram (gram_tc.cu).
struct TcTile {
  int row0;   // first V row of the 128-row A panel
  int col0;   // first V row of the 32-row B panel
  int ksplit; // walker split index
  int slot;   // FP64 partial slot index (ksplit * n_tiles + tile)
};
// Where a sector's Gram block lives in the tile list.  A slice x = (r1 -
// a_base) / 128 keeps B panels y = (r2 - b_base) / 32 >= 4 x only (the rest
// are transposes of kept tiles), so the tile of rows (r1, r2) with y >= 4 x is
// tile0 + x * n_bpanels - 2 x (x - 1) + (y - 4 x).
struct TcSector {
  int row;        // first V row (Re rows; Im rows follow at +dim)
  int dim;
  int goff;       // complex offset of the sector's dim x dim block in a Gram plane
  int tile0;
  int a_base, b_base, n_bpanels;
};
int launch_gram_tc_rows(const float* V, int ldv, int total_rows, const float* rec_w, int ldw,
                        int Wpad, const TcTile* tiles, int n_jobs, int n_splits, double* partials,
                        int mode, int flush_every, int* err, cudaStream_t st);
int launch_gram_tc_reduce(const double* partials, const TcTile* tiles, const TcSector* secs,
                          int n_sec, int n_tiles, int n_splits, int max_dim, double* gram,
                          size_t plane, cudaStream_t st);
size_t gram_tc_smem_bytes(int mode);
constexpr int kTcSlot = 128 * 96;  // doubles per partial slot

}  // namespace lemc

// Internal accessors of a learned proposal (csrc/learned.cu).
const void* lemc_proposal_weights(const lemc_proposal* p);
int lemc_proposal_particles(const lemc_proposal* p);
int lemc_proposal_filling(const lemc_proposal* p);

