/*
 * lemc_oracle.c -- CPU restatement of the LaughlinEdge edge-state estimator.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
 * path: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * may load it.  It is never the thing measured as the product and never a
 * fallback of the product path.
 *
 * It restates, in plain C with FP64 arithmetic, the algorithm of the
 * reference project (paths relative to the LaughlinEdge project):
 *  - partitions: accelerated ascending generation, <= N parts, compression to
 *    (part, multiplicity) pairs stably ordered by multiplicity
 *    (modules/partitions/integer_partitions.cu:10-47, :64-77, :79-140);
 *  - the Metropolis sweep over |P_a Psi_m|^2 with single-particle Gaussian
 *    moves and the acceptance |P_a'/P_a|^2 |J'/J|^{2m} exp((|z|^2-|z'|^2)/2)
 *    (modules/edge_mc/em_markovchain.cu:266-334);
 *  - power sums p_k = sum_i (z_i/R)^k and v_lambda = prod_j p_{lambda_j}
 *    (em_markovchain.cu:120-183);
 *  - the per-row estimator sums fg += v_b/v_a, gg += |v_b/v_a|^2,
 *    fHg += V v_b/v_a (modules/edge_mc/em_spectrum.cu:99-115) and the
 *    reference normalisation (em_spectrum.cu:331-335);
 *  - the shared-guide Gram sums S = sum conj(v_a) v_b, H_e = sum r^e conj(v_a) v_b.
 * The random stream is the library's Philox-4x32-10 layout
 * (counter {i, sweep, walker, tag}, key {seed_lo, seed_hi}; Salmon et al.,
 * SC'11), so small cases can be compared move by move with the GPU.
 * Differences from the reference that are deliberate: the RNG (the reference
 * seeds XORWOW from wall-clock time) and positions kept in FP32 exactly as the
 * GPU keeps them, with all ratios evaluated in FP64.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAXK 24
#define ORC_MAXGP 8

/* ---------------- Philox-4x32-10 ---------------- */
void orc_philox(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static double u01(uint32_t x) { return ((double)(x >> 9) + 0.5) * (1.0 / 8388608.0); }

/* ---------------- partitions ---------------- */
/* Writes the basis rows of the given sectors: rows_dL[r], rows_np[r] and
 * pairs[r*2*ORC_MAXK + 2q + {0,1}] = (part, mult).  Returns the row count or
 * -1 if max_rows is too small. */
int orc_partitions(int N, const int* sectors, int ns, int* rows_dL, int* rows_np, int* pairs,
                   int max_rows) {
  int nrows = 0;
  for (int s = 0; s < ns; ++s) {
    const int n = sectors[s];
    int a[64 + 2];
    memset(a, 0, sizeof(a));
    int k = 1, y = n - 1;
    while (k != 0) {
      int x = a[k - 1] + 1;
      k -= 1;
      while (2 * x <= y) { a[k] = x; y -= x; k += 1; }
      int l = k + 1;
      for (int pass = 0;; ++pass) {
        int len;
        int seq[66];
        if (x <= y) {
          a[k] = x; a[l] = y;
          len = k + 2;
          memcpy(seq, a, sizeof(int) * len);
          x += 1; y -= 1;
        } else {
          a[k] = x + y;
          y = x + y - 1;
          len = k + 1;
          memcpy(seq, a, sizeof(int) * len);
        }
        if (len <= N) {
          if (nrows >= max_rows) return -1;
          /* compress ascending sequence */
          int np = 0, pp[ORC_MAXK][2];
          for (int i = 0; i < len;) {
            int j = i;
            while (j < len && seq[j] == seq[i]) ++j;
            pp[np][0] = seq[i]; pp[np][1] = j - i; ++np;
            i = j;
          }
          /* stable bubble sort by multiplicity */
          for (int i = 0; i < np; ++i)
            for (int j = 0; j < np - i - 1; ++j)
              if (pp[j][1] > pp[j + 1][1]) {
                int t0 = pp[j][0], t1 = pp[j][1];
                pp[j][0] = pp[j + 1][0]; pp[j][1] = pp[j + 1][1];
                pp[j + 1][0] = t0; pp[j + 1][1] = t1;
              }
          rows_dL[nrows] = n;
          rows_np[nrows] = np;
          for (int q = 0; q < np; ++q) {
            pairs[nrows * 2 * ORC_MAXK + 2 * q] = pp[q][0];
            pairs[nrows * 2 * ORC_MAXK + 2 * q + 1] = pp[q][1];
          }
          ++nrows;
        }
        if (len == k + 1) break; /* the closing partition of this outer step */
      }
    }
  }
  return nrows;
}

/* ---------------- complex helpers ---------------- */
typedef struct { double re, im; } cx;
static cx cmul(cx a, cx b) { cx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static cx cpowi(cx z, int k) {
  cx r = {1.0, 0.0};
  for (int i = 0; i < k; ++i) r = cmul(r, z);
  return r;
}

/* guide polynomial value |P|^2 from the guide's power sums */
static double guide_log_norm(const cx* gp, const int* gk, const int* gr, int np) {
  double s = 0.0;
  for (int q = 0; q < np; ++q) {
    if (gk[q] == 0) continue;
    s += gr[q] * log(gp[q].re * gp[q].re + gp[q].im * gp[q].im);
  }
  return s;
}

/* One walker, n_sweeps sweeps.  pos: N float pairs.  guide parts (gk, gr, np)
 * with np = 0 for the Laughlin guide.  Returns accepted moves. */
static uint32_t walker_sweeps(float* pos, int N, int m, double sigma, uint32_t k0, uint32_t k1,
                              uint32_t w, uint32_t sweep0, int n_sweeps, double invR,
                              const int* gk, const int* gr, int np, double* margin) {
  uint32_t acc = 0;
  if (margin) *margin = INFINITY;
  cx gp[ORC_MAXGP];
  for (int s = 0; s < n_sweeps; ++s) {
    const uint32_t sweep = sweep0 + (uint32_t)s;
    for (int q = 0; q < np; ++q) {
      gp[q].re = gp[q].im = 0.0;
      if (gk[q] == 0) continue;
      for (int j = 0; j < N; ++j) {
        cx z = {pos[2 * j] * invR, pos[2 * j + 1] * invR};
        cx v = cpowi(z, gk[q]);
        gp[q].re += v.re; gp[q].im += v.im;
      }
    }
    for (int i = 0; i < N; ++i) {
      uint32_t ctr[4] = {(uint32_t)i, sweep, w, 0u}, key[2] = {k0, k1}, r[4];
      orc_philox(ctr, key, r);
      const double u1 = u01(r[0]), u2 = u01(r[1]), u3 = u01(r[2]);
      const double rad = sqrt(-2.0 * log(u1));
      const double ang = 2.0 * M_PI * u2;
      const float zx = pos[2 * i], zy = pos[2 * i + 1];
      const float nx = (float)(zx + sigma * rad * cos(ang));
      const float ny = (float)(zy + sigma * rad * sin(ang));
      double lj = 0.0;
      for (int j = 0; j < N; ++j) {
        if (j == i) continue;
        const double dx = (double)nx - pos[2 * j], dy = (double)ny - pos[2 * j + 1];
        const double ex = (double)zx - pos[2 * j], ey = (double)zy - pos[2 * j + 1];
        lj += log(dx * dx + dy * dy) - log(ex * ex + ey * ey);
      }
      double delta = m * lj + 0.5 * (((double)zx * zx + (double)zy * zy) - ((double)nx * nx + (double)ny * ny));
      cx gnew[ORC_MAXGP];
      if (np > 0) {
        const cx wo = {zx * invR, zy * invR}, wn = {nx * invR, ny * invR};
        const double before = guide_log_norm(gp, gk, gr, np);
        for (int q = 0; q < np; ++q) {
          gnew[q] = gp[q];
          if (gk[q] == 0) continue;
          const cx po = cpowi(wo, gk[q]), pn = cpowi(wn, gk[q]);
          gnew[q].re += pn.re - po.re;
          gnew[q].im += pn.im - po.im;
        }
        delta += guide_log_norm(gnew, gk, gr, np) - before;
      }
      if (margin && fabs(delta - log(u3)) < *margin) *margin = fabs(delta - log(u3));
      if (delta >= log(u3)) {
        pos[2 * i] = nx;
        pos[2 * i + 1] = ny;
        ++acc;
        for (int q = 0; q < np; ++q) gp[q] = gnew[q];
      }
    }
  }
  return acc;
}

/* Advance W walkers.  guide_pairs: [rows][2*ORC_MAXGP] (part, mult) and
 * guide_np[rows]; walker_row == NULL selects the Laughlin guide. */
/* As orc_sweep; min_margin[w] (may be NULL) receives the smallest
 * |ln A - ln u| of walker w's moves: the closest its accept decisions came to a
 * tie, which is where a GPU path that forms ln A in FP32 may decide otherwise. */
void orc_sweep_margin(float* pos, int W, int N, int m, double sigma, uint64_t seed,
                      uint32_t sweep0, int n_sweeps, double invR, const int* walker_row,
                      const int* guide_pairs, const int* guide_np, uint32_t* accepted,
                      double* min_margin, int nthreads);

void orc_sweep(float* pos, int W, int N, int m, double sigma, uint64_t seed, uint32_t sweep0,
               int n_sweeps, double invR, const int* walker_row, const int* guide_pairs,
               const int* guide_np, uint32_t* accepted, int nthreads) {
  orc_sweep_margin(pos, W, N, m, sigma, seed, sweep0, n_sweeps, invR, walker_row, guide_pairs,
                   guide_np, accepted, NULL, nthreads);
}

void orc_sweep_margin(float* pos, int W, int N, int m, double sigma, uint64_t seed,
                      uint32_t sweep0, int n_sweeps, double invR, const int* walker_row,
                      const int* guide_pairs, const int* guide_np, uint32_t* accepted,
                      double* min_margin, int nthreads) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
#endif
  for (int w = 0; w < W; ++w) {
    int gk[ORC_MAXGP] = {0}, gr[ORC_MAXGP] = {0}, np = 0;
    if (walker_row) {
      const int row = walker_row[w];
      np = guide_np[row];
      for (int q = 0; q < np; ++q) {
        gk[q] = guide_pairs[row * 2 * ORC_MAXGP + 2 * q];
        gr[q] = gk[q] > 0 ? guide_pairs[row * 2 * ORC_MAXGP + 2 * q + 1] : 0;
      }
    }
    const uint32_t a = walker_sweeps(pos + (size_t)w * N * 2, N, m, sigma, k0, k1, (uint32_t)w,
                                     sweep0, n_sweeps, invR, gk, gr, np,
                                     min_margin ? min_margin + w : NULL);
    if (accepted) accepted[w] += a;
  }
}

/* Uniform initial positions in a disk (counter {i, 0, w, 1}). */
void orc_init(float* pos, int W, int N, double radius, uint64_t seed) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int w = 0; w < W; ++w)
    for (int i = 0; i < N; ++i) {
      uint32_t ctr[4] = {(uint32_t)i, 0u, (uint32_t)w, 1u}, r[4];
      orc_philox(ctr, key, r);
      const double rho = radius * sqrt(u01(r[0]));
      const double ang = 2.0 * M_PI * u01(r[1]);
      pos[((size_t)w * N + i) * 2] = (float)(rho * cos(ang));
      pos[((size_t)w * N + i) * 2 + 1] = (float)(rho * sin(ang));
    }
}

/* Measurement record of W walkers: rec_p[w][k] = p_{k+1} (complex), k < K;
 * rec_w[w][0..5] = {1, sum r^2, sum r^4, sum cos l theta, sum sin l theta, 0}. */
void orc_measure(const float* pos, int W, int N, int K, double invR, int lprobe, double* rec_p,
                 double* rec_w) {
  for (int w = 0; w < W; ++w) {
    const float* z = pos + (size_t)w * N * 2;
    double h2 = 0, h4 = 0, hc = 0, hs = 0;
    for (int k = 0; k < K; ++k) rec_p[((size_t)w * K + k) * 2] = rec_p[((size_t)w * K + k) * 2 + 1] = 0.0;
    for (int i = 0; i < N; ++i) {
      const cx wv = {z[2 * i] * invR, z[2 * i + 1] * invR};
      cx pw = wv;
      for (int k = 0; k < K; ++k) {
        rec_p[((size_t)w * K + k) * 2] += pw.re;
        rec_p[((size_t)w * K + k) * 2 + 1] += pw.im;
        pw = cmul(pw, wv);
      }
      const double r2 = (double)z[2 * i] * z[2 * i] + (double)z[2 * i + 1] * z[2 * i + 1];
      h2 += r2;
      h4 += r2 * r2;
      if (lprobe > 0) {
        const double th = atan2((double)z[2 * i + 1], (double)z[2 * i]);
        hc += cos(lprobe * th);
        hs += sin(lprobe * th);
      }
    }
    double* o = rec_w + (size_t)w * 6;
    o[0] = 1.0; o[1] = h2; o[2] = h4; o[3] = hc; o[4] = hs; o[5] = 0.0;
  }
}

/* v_lambda = prod_q p_{part_q}^{mult_q}; part 0 means p_0 = N. */
static cx basis_value(const cx* p, int N, const int* pairs, int np) {
  cx v = {1.0, 0.0};
  for (int q = 0; q < np; ++q) {
    const int k = pairs[2 * q], r = pairs[2 * q + 1];
    cx base;
    if (k == 0) { base.re = N; base.im = 0.0; } else base = p[k - 1];
    for (int t = 0; t < r; ++t) v = cmul(v, base);
  }
  return v;
}

/*
 * Full estimator runs (burn-in + n_meas sweeps with a measurement after each),
 * all rows of one basis, OpenMP over walkers.
 *
 * orc_run_rows: the reference estimator.  Walkers are split into contiguous
 * equal blocks per row a (walker w -> row (w * D) / W) and guided by
 * |P_a Psi|^2.  Outputs (D x D): fg (complex), gg (real), fh2, fh4 (complex)
 * raw sums, and n_row[a] samples per row.
 *
 * orc_run_gram: the shared Laughlin guide.  Outputs S, H2, H4 (complex D x D,
 * one block per sector in row order; only same-sector entries are filled).
 */
static void run_common(int mode, int N, int m, int W, double sigma, uint64_t seed, int n_burn,
                       int n_meas, double invR, double init_radius, int D, const int* rows_np,
                       const int* pairs, const int* rows_dL, int K, double* o1, double* o2,
                       double* o3, double* o4, double* n_row, double* series, int nthreads) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  const size_t DD = (size_t)D * D;
  memset(o1, 0, sizeof(double) * 2 * DD);
  if (mode == 0) memset(o2, 0, sizeof(double) * DD); else memset(o2, 0, sizeof(double) * 2 * DD);
  memset(o3, 0, sizeof(double) * 2 * DD);
  if (mode == 0) memset(o4, 0, sizeof(double) * 2 * DD);
  if (n_row) memset(n_row, 0, sizeof(double) * D);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const int nth =
#ifdef _OPENMP
      omp_get_max_threads();
#else
      1;
#endif
  double* priv = (double*)calloc((size_t)nth * 7 * DD + 1, sizeof(double));
  double* pser = series ? (double*)calloc((size_t)nth * n_meas * 8 + 1, sizeof(double)) : NULL;
  float* pos = (float*)malloc(sizeof(float) * 2 * (size_t)W * N);
  orc_init(pos, W, N, init_radius, seed);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int w = 0; w < W; ++w) {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* acc = priv + (size_t)tid * 7 * DD;
    int gk[ORC_MAXGP] = {0}, gr[ORC_MAXGP] = {0}, np = 0, row = -1;
    if (mode == 0) {
      row = (int)(((int64_t)w * D) / W);
      np = rows_np[row];
      for (int q = 0; q < np; ++q) {
        gk[q] = pairs[row * 2 * ORC_MAXK + 2 * q];
        gr[q] = gk[q] > 0 ? pairs[row * 2 * ORC_MAXK + 2 * q + 1] : 0;
      }
    }
    float* z = pos + (size_t)w * N * 2;
    walker_sweeps(z, N, m, sigma, k0, k1, (uint32_t)w, 0u, n_burn, invR, gk, gr, np, NULL);
    double rp[2 * ORC_MAXK], rw[6];
    cx v[4096];
    for (int s = 0; s < n_meas; ++s) {
      walker_sweeps(z, N, m, sigma, k0, k1, (uint32_t)w, (uint32_t)(n_burn + s), 1, invR, gk, gr, np, NULL);
      orc_measure(z, 1, N, K, invR, 0, rp, rw);
      if (pser)
        for (int q = 0; q < 8 && q < 2 * K; ++q) pser[((size_t)tid * n_meas + s) * 8 + q] += rp[q];
      for (int b = 0; b < D; ++b) v[b] = basis_value((const cx*)rp, N, pairs + b * 2 * ORC_MAXK, rows_np[b]);
      if (mode == 0) {
        const cx va = v[row];
        const double den = va.re * va.re + va.im * va.im;
        for (int b = 0; b < D; ++b) {
          const cx r = {(v[b].re * va.re + v[b].im * va.im) / den, (v[b].im * va.re - v[b].re * va.im) / den};
          const size_t o = (size_t)row * D + b;
          acc[2 * o] += r.re; acc[2 * o + 1] += r.im;
          acc[2 * DD + o] += r.re * r.re + r.im * r.im;
          acc[3 * DD + 2 * o] += rw[1] * r.re; acc[3 * DD + 2 * o + 1] += rw[1] * r.im;
          acc[5 * DD + 2 * o] += rw[2] * r.re; acc[5 * DD + 2 * o + 1] += rw[2] * r.im;
        }
      } else {
        for (int a = 0; a < D; ++a)
          for (int b = 0; b < D; ++b) {
            if (rows_dL[a] != rows_dL[b]) continue;
            const double pr = v[a].re * v[b].re + v[a].im * v[b].im;
            const double pi = v[a].re * v[b].im - v[a].im * v[b].re;
            const size_t o = (size_t)a * D + b;
            acc[2 * o] += pr; acc[2 * o + 1] += pi;
            acc[2 * DD + 2 * o] += rw[1] * pr; acc[2 * DD + 2 * o + 1] += rw[1] * pi;
            acc[4 * DD + 2 * o] += rw[2] * pr; acc[4 * DD + 2 * o + 1] += rw[2] * pi;
          }
      }
    }
    if (mode == 0 && n_row) {
#ifdef _OPENMP
#pragma omp atomic
#endif
      n_row[row] += n_meas;
    }
  }
  for (int t = 0; t < nth; ++t) {
    const double* acc = priv + (size_t)t * 7 * DD;
    if (mode == 0) {
      for (size_t o = 0; o < 2 * DD; ++o) { o1[o] += acc[o]; o3[o] += acc[3 * DD + o]; o4[o] += acc[5 * DD + o]; }
      for (size_t o = 0; o < DD; ++o) o2[o] += acc[2 * DD + o];
    } else {
      for (size_t o = 0; o < 2 * DD; ++o) { o1[o] += acc[o]; o2[o] += acc[2 * DD + o]; o3[o] += acc[4 * DD + o]; }
    }
  }
  if (pser) {
    for (int s = 0; s < n_meas; ++s)
      for (int q = 0; q < 8; ++q) {
        double v = 0.0;
        for (int t = 0; t < nth; ++t) v += pser[((size_t)t * n_meas + s) * 8 + q];
        series[(size_t)s * 8 + q] = v / W;
      }
    free(pser);
  }
  free(priv);
  free(pos);
  (void)o4;
}

void orc_run_rows(int N, int m, int W, double sigma, uint64_t seed, int n_burn, int n_meas,
                  double invR, double init_radius, int D, const int* rows_np, const int* pairs,
                  const int* rows_dL, int K, double* fg, double* gg, double* fh2, double* fh4,
                  double* n_row, double* series, int nthreads) {
  run_common(0, N, m, W, sigma, seed, n_burn, n_meas, invR, init_radius, D, rows_np, pairs, rows_dL,
             K, fg, gg, fh2, fh4, n_row, series, nthreads);
}

void orc_run_gram(int N, int m, int W, double sigma, uint64_t seed, int n_burn, int n_meas,
                  double invR, double init_radius, int D, const int* rows_np, const int* pairs,
                  const int* rows_dL, int K, double* S, double* H2, double* H4, double* series,
                  int nthreads) {
  double dummy[2];
  run_common(1, N, m, W, sigma, seed, n_burn, n_meas, invR, init_radius, D, rows_np, pairs, rows_dL,
             K, S, H2, H4, dummy, NULL, series, nthreads);
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------
 * Occupation numbers with the two-state walker (reference
 * modules/green_function/green_function.cu:199-373 and
 * gf_occupation_numbers.cu:16-239): N+1 particles, |f_L(z_0..z_{N-1})| |f_R(z_1..z_N)|,
 * three move types, estimator sum_l exp(-ln(2 pi l!) + l ln(z_0 conj z_N / 2)
 * - (|z_0|^2+|z_N|^2)/4 + i phase).  Pair (L, R) = rows L, R of one sector;
 * out[l] receives the average over W walkers x n_meas sweeps (complex).
 * Philox counter {particle, sweep, walker, 2}, init {particle, 0, walker, 3}.
 */
static double gl_lognorm(const cx* p, const int* k, const int* r, int n) {
  double s = 0;
  for (int q = 0; q < n; ++q)
    if (k[q] > 0) s += 0.5 * r[q] * log(p[q].re * p[q].re + p[q].im * p[q].im);
  return s;
}

void orc_occupation(int N, int m, int W, double sigma, uint64_t seed, int n_burn, int n_meas,
                    const int* gkL, const int* grL, int nL, const int* gkR, const int* grR, int nR,
                    int Lc, double* out, int nthreads) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  const double invR = 1.0 / sqrt(2.0 * m * N);
  const int NP = N + 1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const int nth =
#ifdef _OPENMP
      omp_get_max_threads();
#else
      1;
#endif
  double* priv = (double*)calloc((size_t)nth * 2 * Lc, sizeof(double));
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int w = 0; w < W; ++w) {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* acc = priv + (size_t)tid * 2 * Lc;
    float z[2 * 1025];
    const double r0 = sqrt(2.0 * m * N);
    for (int j = 0; j < NP; ++j) {
      uint32_t ctr[4] = {(uint32_t)j, 0u, (uint32_t)w, 3u}, key[2] = {k0, k1}, rr[4];
      orc_philox(ctr, key, rr);
      const float rho = (float)(r0 * sqrt(u01(rr[0])));
      const double ang = 2.0 * M_PI * u01(rr[1]);
      z[2 * j] = (float)(rho * cos(ang));
      z[2 * j + 1] = (float)(rho * sin(ang));
    }
    cx pL[ORC_MAXGP], pR[ORC_MAXGP], nLp[ORC_MAXGP], nRp[ORC_MAXGP];
    for (int s = 0; s < n_burn + n_meas; ++s) {
      for (int q = 0; q < nL; ++q) {
        pL[q].re = pL[q].im = 0;
        if (gkL[q] == 0) continue;
        for (int j = 0; j < N; ++j) {
          cx v = cpowi((cx){z[2 * j] * invR, z[2 * j + 1] * invR}, gkL[q]);
          pL[q].re += v.re; pL[q].im += v.im;
        }
      }
      for (int q = 0; q < nR; ++q) {
        pR[q].re = pR[q].im = 0;
        if (gkR[q] == 0) continue;
        for (int j = 1; j <= N; ++j) {
          cx v = cpowi((cx){z[2 * j] * invR, z[2 * j + 1] * invR}, gkR[q]);
          pR[q].re += v.re; pR[q].im += v.im;
        }
      }
      for (int i = 0; i < NP; ++i) {
        uint32_t ctr[4] = {(uint32_t)i, (uint32_t)s, (uint32_t)w, 2u}, key[2] = {k0, k1}, rr[4];
        orc_philox(ctr, key, rr);
        const double rad = sqrt(-2.0 * log(u01(rr[0]))), ang = 2.0 * M_PI * u01(rr[1]);
        const float ox = z[2 * i], oy = z[2 * i + 1];
        const float nx = (float)(ox + sigma * rad * cos(ang)), ny = (float)(oy + sigma * rad * sin(ang));
        double lj = 0;
        for (int j = 1; j < N; ++j) {
          if (j == i) continue;
          const double dx = (double)nx - z[2 * j], dy = (double)ny - z[2 * j + 1];
          const double ex = (double)ox - z[2 * j], ey = (double)oy - z[2 * j + 1];
          lj += 0.5 * (log(dx * dx + dy * dy) - log(ex * ex + ey * ey));
        }
        const double gz = ((double)ox * ox + (double)oy * oy) - ((double)nx * nx + (double)ny * ny);
        const cx wo = {ox * invR, oy * invR}, wn = {nx * invR, ny * invR};
        double dlL = 0, dlR = 0;
        if (i < N) {
          for (int q = 0; q < nL; ++q) {
            nLp[q] = pL[q];
            if (gkL[q] == 0) continue;
            cx a = cpowi(wo, gkL[q]), b = cpowi(wn, gkL[q]);
            nLp[q].re += b.re - a.re; nLp[q].im += b.im - a.im;
          }
          dlL = gl_lognorm(nLp, gkL, grL, nL) - gl_lognorm(pL, gkL, grL, nL);
        }
        if (i > 0) {
          for (int q = 0; q < nR; ++q) {
            nRp[q] = pR[q];
            if (gkR[q] == 0) continue;
            cx a = cpowi(wo, gkR[q]), b = cpowi(wn, gkR[q]);
            nRp[q].re += b.re - a.re; nRp[q].im += b.im - a.im;
          }
          dlR = gl_lognorm(nRp, gkR, grR, nR) - gl_lognorm(pR, gkR, grR, nR);
        }
        double delta;
        if (i == 0 || i == N) {
          delta = m * lj + dlL + dlR + 0.25 * gz;
        } else {
          const double z0x = z[0], z0y = z[1], zNx = z[2 * N], zNy = z[2 * N + 1];
          const double c0 = 0.5 * (log((nx - z0x) * (nx - z0x) + (ny - z0y) * (ny - z0y)) -
                                   log((ox - z0x) * (ox - z0x) + (oy - z0y) * (oy - z0y)));
          const double cN = 0.5 * (log((nx - zNx) * (nx - zNx) + (ny - zNy) * (ny - zNy)) -
                                   log((ox - zNx) * (ox - zNx) + (oy - zNy) * (oy - zNy)));
          delta = m * (c0 + cN) + dlL + dlR + 2.0 * m * lj + 0.5 * gz;
        }
        if (delta >= log(u01(rr[2]))) {
          z[2 * i] = nx; z[2 * i + 1] = ny;
          if (i < N) for (int q = 0; q < nL; ++q) pL[q] = nLp[q];
          if (i > 0) for (int q = 0; q < nR; ++q) pR[q] = nRp[q];
        }
      }
      if (s < n_burn) continue;
      const double z0x = z[0], z0y = z[1], zNx = z[2 * N], zNy = z[2 * N + 1];
      double ph = 0;
      for (int q = 0; q < nR; ++q) if (gkR[q] > 0) ph += grR[q] * atan2(pR[q].im, pR[q].re);
      for (int q = 0; q < nL; ++q) if (gkL[q] > 0) ph -= grL[q] * atan2(pL[q].im, pL[q].re);
      double jarg = 0;
      for (int i = 1; i < N; ++i) {
        jarg += atan2(z[2 * i + 1] - zNy, z[2 * i] - zNx) - atan2(z0y - z[2 * i + 1], z0x - z[2 * i]);
      }
      ph += m * jarg;
      const double qx = 0.5 * (z0x * zNx + z0y * zNy), qy = 0.5 * (z0y * zNx - z0x * zNy);
      const double lx = 0.5 * log(qx * qx + qy * qy), phi = atan2(qy, qx);
      double la = -0.25 * (z0x * z0x + z0y * z0y + zNx * zNx + zNy * zNy) - log(2.0 * M_PI);
      for (int l = 0; l < Lc; ++l) {
        if (l > 0) la += lx - log((double)l);
        const double mag = exp(la);
        acc[2 * l] += mag * cos(l * phi + ph);
        acc[2 * l + 1] += mag * sin(l * phi + ph);
      }
    }
  }
  for (int l = 0; l < 2 * Lc; ++l) {
    double v = 0;
    for (int t = 0; t < nth; ++t) v += priv[(size_t)t * 2 * Lc + l];
    out[l] = v / ((double)W * n_meas);
  }
  free(priv);
}
