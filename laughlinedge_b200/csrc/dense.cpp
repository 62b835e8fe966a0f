// FP64 dense tail: generalized Hermitian eigenproblem, the reference's
// normalisation of sampled matrices, and the edge-basis time evolution.
//
// Generalized eigenproblem H c = E M c (reference: Eigen's
// GeneralizedSelfAdjointEigenSolver, modules/eigensolver/generalized_eigenproblem.cpp:45-95):
//   1. M = L L^H by Cholesky; if M is not positive definite, M = U diag(mu) U^H
//      and the directions with mu <= eps * max(mu) are dropped (X = U_k mu_k^-1/2).
//   2. C = X^H H X with X = L^-H (or the truncated X above), Hermitian.
//   3. C is diagonalised through its real symmetric embedding
//      [[Re C, -Im C], [Im C, Re C]] by Householder tridiagonalisation followed
//      by the implicit QL algorithm with Wilkinson-type shifts (Golub & Van
//      Loan, "Matrix Computations", 4th ed., sections 8.3.1 and 8.3.5).  Each
//      eigenvalue of C appears twice; complex eigenvectors are recovered as
//      x + i y from the embedded [x; y] and orthonormalised inside clusters.
//   4. c = X y, so that c^H M c = 1.
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "../../include/lemc.h"

namespace {

using cd = std::complex<double>;

// Householder reduction of a real symmetric matrix a (n x n, row-major) to
// tridiagonal form: diag d, off-diagonal e (e[i] couples i-1 and i, e[0] = 0).
// With want_q, a is overwritten by the orthogonal Q with A = Q T Q^T.
void tridiagonalize(int n, std::vector<double>& a, std::vector<double>& d, std::vector<double>& e,
                    bool want_q) {
  d.assign(n, 0.0);
  e.assign(n, 0.0);
  auto A = [&](int i, int j) -> double& { return a[size_t(i) * n + j]; };
  for (int i = n - 1; i > 0; --i) {
    const int l = i - 1;
    double h = 0.0;
    if (l > 0) {
      double scale = 0.0;
      for (int k = 0; k <= l; ++k) scale += std::fabs(A(i, k));
      if (scale == 0.0) {
        e[i] = A(i, l);
      } else {
        for (int k = 0; k <= l; ++k) {
          A(i, k) /= scale;
          h += A(i, k) * A(i, k);
        }
        double f = A(i, l);
        double g = (f >= 0.0) ? -std::sqrt(h) : std::sqrt(h);
        e[i] = scale * g;
        h -= f * g;
        A(i, l) = f - g;
        f = 0.0;
        for (int j = 0; j <= l; ++j) {
          if (want_q) A(j, i) = A(i, j) / h;
          g = 0.0;
          for (int k = 0; k <= j; ++k) g += A(j, k) * A(i, k);
          for (int k = j + 1; k <= l; ++k) g += A(k, j) * A(i, k);
          e[j] = g / h;
          f += e[j] * A(i, j);
        }
        const double hh = f / (h + h);
        for (int j = 0; j <= l; ++j) {
          f = A(i, j);
          e[j] = g = e[j] - hh * f;
          for (int k = 0; k <= j; ++k) A(j, k) -= (f * e[k] + g * A(i, k));
        }
      }
    } else {
      e[i] = A(i, l);
    }
    d[i] = h;
  }
  d[0] = 0.0;
  e[0] = 0.0;
  for (int i = 0; i < n; ++i) {
    if (want_q) {
      const int l = i - 1;
      if (d[i] != 0.0) {
        for (int j = 0; j <= l; ++j) {
          double g = 0.0;
          for (int k = 0; k <= l; ++k) g += A(i, k) * A(k, j);
          for (int k = 0; k <= l; ++k) A(k, j) -= g * A(k, i);
        }
      }
      d[i] = A(i, i);
      A(i, i) = 1.0;
      for (int j = 0; j <= l; ++j) A(j, i) = A(i, j) = 0.0;
    } else {
      d[i] = A(i, i);
    }
  }
}

// Implicit QL on the tridiagonal (d, e); with z (n x n) the rotations are
// accumulated into its columns.  Returns false if an eigenvalue fails to
// converge in 60 iterations.
bool tridiagonal_ql(int n, std::vector<double>& d, std::vector<double>& e, double* z) {
  for (int i = 1; i < n; ++i) e[i - 1] = e[i];
  if (n > 0) e[n - 1] = 0.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    int mm;
    do {
      for (mm = l; mm < n - 1; ++mm) {
        const double dd = std::fabs(d[mm]) + std::fabs(d[mm + 1]);
        if (std::fabs(e[mm]) <= 1e-15 * dd) break;
      }
      if (mm != l) {
        if (iter++ == 60) return false;
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = std::hypot(g, 1.0);
        g = d[mm] - d[l] + e[l] / (g + (g >= 0 ? std::fabs(r) : -std::fabs(r)));
        double s = 1.0, c = 1.0, p = 0.0;
        int i;
        for (i = mm - 1; i >= l; --i) {
          double f = s * e[i];
          const double b = c * e[i];
          r = std::hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) {
            d[i + 1] -= p;
            e[mm] = 0.0;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * b;
          p = s * r;
          d[i + 1] = g + p;
          g = c * r - b;
          if (z) {
            for (int k = 0; k < n; ++k) {
              f = z[size_t(k) * n + i + 1];
              z[size_t(k) * n + i + 1] = s * z[size_t(k) * n + i] + c * f;
              z[size_t(k) * n + i] = c * z[size_t(k) * n + i] - s * f;
            }
          }
        }
        if (r == 0.0 && i >= l) continue;
        d[l] -= p;
        e[l] = g;
        e[mm] = 0.0;
      }
    } while (mm != l);
  }
  return true;
}

// Hermitian eigen-decomposition of C (n x n, complex row-major).
// evals ascending; vecs (optional) column j = eigenvector j.
bool hermitian_eig(int n, const std::vector<cd>& C, std::vector<double>& evals,
                   std::vector<cd>* vecs) {
  const int n2 = 2 * n;
  std::vector<double> a(size_t(n2) * n2);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const cd v = C[size_t(i) * n + j];
      a[size_t(i) * n2 + j] = v.real();
      a[size_t(i) * n2 + j + n] = -v.imag();
      a[size_t(i + n) * n2 + j] = v.imag();
      a[size_t(i + n) * n2 + j + n] = v.real();
    }
  std::vector<double> d, e;
  const bool want = vecs != nullptr;
  tridiagonalize(n2, a, d, e, want);
  if (!tridiagonal_ql(n2, d, e, want ? a.data() : nullptr)) return false;
  std::vector<int> idx(n2);
  for (int i = 0; i < n2; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int x, int y) { return d[x] < d[y]; });
  evals.clear();
  if (!want) {
    for (int k = 0; k < n2; k += 2) evals.push_back(0.5 * (d[idx[k]] + d[idx[k + 1]]));
    return true;
  }
  // recover complex vectors: z = x + i y from [x; y]; orthonormalise inside
  // eigenvalue clusters and drop the dependent partner of each pair.
  double scale = 0;
  for (double v : d) scale = std::max(scale, std::fabs(v));
  const double tol = 1e-9 * std::max(scale, 1e-300);
  std::vector<std::vector<cd>> acc;
  std::vector<double> acc_e;
  for (int q = 0; q < n2 && int(acc.size()) < n; ++q) {
    const int col = idx[q];
    std::vector<cd> z(n);
    for (int i = 0; i < n; ++i) z[i] = cd(a[size_t(i) * n2 + col], a[size_t(i + n) * n2 + col]);
    for (size_t p = 0; p < acc.size(); ++p) {
      if (std::fabs(acc_e[p] - d[col]) > 1e3 * tol) continue;
      cd dot = 0;
      for (int i = 0; i < n; ++i) dot += std::conj(acc[p][i]) * z[i];
      for (int i = 0; i < n; ++i) z[i] -= dot * acc[p][i];
    }
    double nrm = 0;
    for (int i = 0; i < n; ++i) nrm += std::norm(z[i]);
    nrm = std::sqrt(nrm);
    if (nrm < 0.5) continue;
    for (int i = 0; i < n; ++i) z[i] /= nrm;
    acc.push_back(std::move(z));
    acc_e.push_back(d[col]);
  }
  if (int(acc.size()) != n) return false;
  vecs->assign(size_t(n) * n, 0.0);
  for (int j = 0; j < n; ++j) {
    evals.push_back(acc_e[j]);
    for (int i = 0; i < n; ++i) (*vecs)[size_t(i) * n + j] = acc[j][i];
  }
  return true;
}

// In-place complex Cholesky M = L L^H (lower). Returns false if not PD.
bool cholesky(int n, std::vector<cd>& L) {
  for (int j = 0; j < n; ++j) {
    double s = L[size_t(j) * n + j].real();
    for (int k = 0; k < j; ++k) s -= std::norm(L[size_t(j) * n + k]);
    if (!(s > 0.0)) return false;
    const double ljj = std::sqrt(s);
    L[size_t(j) * n + j] = ljj;
    for (int i = j + 1; i < n; ++i) {
      cd t = L[size_t(i) * n + j];
      for (int k = 0; k < j; ++k) t -= L[size_t(i) * n + k] * std::conj(L[size_t(j) * n + k]);
      L[size_t(i) * n + j] = t / ljj;
    }
    for (int k = j + 1; k < n; ++k) L[size_t(j) * n + k] = 0.0;
  }
  return true;
}

std::vector<cd> to_complex(int D, const double* x) {
  std::vector<cd> v(size_t(D) * D);
  for (size_t i = 0; i < v.size(); ++i) v[i] = cd(x[2 * i], x[2 * i + 1]);
  return v;
}

}  // namespace

extern "C" int lemc_geneig(int D, const double* H, const double* M, double eps, double* evals,
                           double* evecs, int* rank) {
  if (D <= 0 || !H || !M || !evals) return LEMC_ERR_ARG;
  std::vector<cd> h = to_complex(D, H), m = to_complex(D, M);
  // Hermitise defensively
  for (int i = 0; i < D; ++i)
    for (int j = i; j < D; ++j) {
      const cd a = 0.5 * (h[size_t(i) * D + j] + std::conj(h[size_t(j) * D + i]));
      h[size_t(i) * D + j] = a;
      h[size_t(j) * D + i] = std::conj(a);
      const cd b = 0.5 * (m[size_t(i) * D + j] + std::conj(m[size_t(j) * D + i]));
      m[size_t(i) * D + j] = b;
      m[size_t(j) * D + i] = std::conj(b);
    }
  if (eps <= 0) eps = 1e-12;
  // X: D x k transformation with X^H M X = I
  int k = D;
  std::vector<cd> X;
  std::vector<cd> L = m;
  int status = LEMC_OK;
  if (cholesky(D, L)) {
    // X = L^-H : solve L^H X = I column by column (upper-triangular back substitution)
    X.assign(size_t(D) * D, 0.0);
    for (int c = 0; c < D; ++c) {
      for (int i = D - 1; i >= 0; --i) {
        cd t = (i == c) ? 1.0 : 0.0;
        for (int j = i + 1; j < D; ++j) t -= std::conj(L[size_t(j) * D + i]) * X[size_t(j) * D + c];
        X[size_t(i) * D + c] = t / L[size_t(i) * D + i].real();
      }
    }
  } else {
    std::vector<double> mu;
    std::vector<cd> U;
    if (!hermitian_eig(D, m, mu, &U)) return LEMC_ERR_NUMERIC;
    const double mmax = mu.empty() ? 0.0 : mu.back();
    if (!(mmax > 0)) return LEMC_ERR_NUMERIC;
    std::vector<int> keep;
    for (int j = 0; j < D; ++j)
      if (mu[j] > eps * mmax) keep.push_back(j);
    k = int(keep.size());
    X.assign(size_t(D) * k, 0.0);
    for (int c = 0; c < k; ++c) {
      const double s = 1.0 / std::sqrt(mu[keep[c]]);
      for (int i = 0; i < D; ++i) X[size_t(i) * k + c] = U[size_t(i) * D + keep[c]] * s;
    }
    status = LEMC_OK;
  }
  // C = X^H H X  (k x k)
  std::vector<cd> HX(size_t(D) * k, 0.0), Cm(size_t(k) * k, 0.0);
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j) {
      const cd hij = h[size_t(i) * D + j];
      if (hij == cd(0.0)) continue;
      for (int c = 0; c < k; ++c) HX[size_t(i) * k + c] += hij * X[size_t(j) * k + c];
    }
  for (int a = 0; a < k; ++a)
    for (int i = 0; i < D; ++i) {
      const cd xa = std::conj(X[size_t(i) * k + a]);
      for (int b = 0; b < k; ++b) Cm[size_t(a) * k + b] += xa * HX[size_t(i) * k + b];
    }
  for (int a = 0; a < k; ++a)
    for (int b = a; b < k; ++b) {
      const cd v = 0.5 * (Cm[size_t(a) * k + b] + std::conj(Cm[size_t(b) * k + a]));
      Cm[size_t(a) * k + b] = v;
      Cm[size_t(b) * k + a] = std::conj(v);
    }
  std::vector<double> ev;
  std::vector<cd> Y;
  if (!hermitian_eig(k, Cm, ev, evecs ? &Y : nullptr)) return LEMC_ERR_NUMERIC;
  for (int j = 0; j < D; ++j) evals[j] = (j < k) ? ev[j] : NAN;
  if (evecs) {
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) {
        cd v = 0.0;
        if (j < k)
          for (int c = 0; c < k; ++c) v += X[size_t(i) * k + c] * Y[size_t(c) * k + j];
        evecs[2 * (size_t(i) * D + j)] = (j < k) ? v.real() : NAN;
        evecs[2 * (size_t(i) * D + j) + 1] = (j < k) ? v.imag() : NAN;
      }
  }
  if (rank) *rank = k;
  return status;
}

// Edge dynamic structure factor of one (dL = 0) + (dL) problem, reference
// generalized_eigenproblem.cpp:54-95: drop row/column 0 (the Laughlin state),
// solve h c = E m c with c^H m c = 1, and weight mode j by |(Vc - i Vs)[0, 1:] c_j|^2.
extern "C" int lemc_dsf_weights(int D, const double* H, const double* M, const double* Vc,
                                const double* Vs, double eps, double* energies, double* weights,
                                int* n_modes) {
  if (D < 2 || !H || !M || !Vc || !Vs || !energies || !weights) return LEMC_ERR_ARG;
  const int n = D - 1;
  std::vector<double> h(2 * size_t(n) * n), m(2 * size_t(n) * n), ev(n), vec(2 * size_t(n) * n);
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      const size_t o = 2 * (size_t(a) * n + b), q = 2 * (size_t(a + 1) * D + (b + 1));
      h[o] = H[q];
      h[o + 1] = H[q + 1];
      m[o] = M[q];
      m[o + 1] = M[q + 1];
    }
  int rank = 0;
  const int st = lemc_geneig(n, h.data(), m.data(), eps, ev.data(), vec.data(), &rank);
  if (st != LEMC_OK) return st;
  for (int j = 0; j < n; ++j) {
    double re = 0, im = 0;
    for (int a = 0; a < n; ++a) {
      // v = Vc[0][a+1] - i Vs[0][a+1]
      const double vr = Vc[2 * (a + 1)] + Vs[2 * (a + 1) + 1];
      const double vi = Vc[2 * (a + 1) + 1] - Vs[2 * (a + 1)];
      const double cr = vec[2 * (size_t(a) * n + j)], ci = vec[2 * (size_t(a) * n + j) + 1];
      re += vr * cr - vi * ci;
      im += vr * ci + vi * cr;
    }
    energies[j] = ev[j];
    weights[j] = j < rank ? re * re + im * im : NAN;
  }
  if (n_modes) *n_modes = rank;
  return LEMC_OK;
}

// Jackknife over bins of raw Gram sums (leave one bin out): the normalised
// M, H (lemc_normalise) and the generalized eigenvalues (lemc_geneig) of the
// full sums, with their jackknife standard errors
// err^2 = (B-1)/B sum_b |x_(-b) - mean_(-b)|^2.
extern "C" int lemc_jackknife_spectrum(int D, int n_bins, const double* S, const double* H2,
                                       const double* H4, double omega, double kappa, double eps,
                                       double* evals, double* evals_err, double* M_err,
                                       double* H_err) {
  if (D <= 0 || n_bins < 2 || !S || !H2 || !H4 || !evals || !evals_err) return LEMC_ERR_ARG;
  const size_t P = 2 * size_t(D) * D;
  std::vector<double> tot[3];
  const double* in[3] = {S, H2, H4};
  for (int h = 0; h < 3; ++h) {
    tot[h].assign(P, 0.0);
    for (int b = 0; b < n_bins; ++b)
      for (size_t i = 0; i < P; ++i) tot[h][i] += in[h][size_t(b) * P + i];
  }
  std::vector<double> M(P), H(P);
  int rank = 0;
  int st = lemc_normalise(D, tot[0].data(), tot[1].data(), tot[2].data(), omega, kappa, M.data(),
                          H.data());
  if (st != LEMC_OK) return st;
  st = lemc_geneig(D, H.data(), M.data(), eps, evals, nullptr, &rank);
  if (st != LEMC_OK) return st;
  std::vector<double> ev_b(size_t(n_bins) * D), M_b(size_t(n_bins) * P), H_b(size_t(n_bins) * P);
  std::vector<double> part[3];
  for (int h = 0; h < 3; ++h) part[h].resize(P);
  for (int b = 0; b < n_bins; ++b) {
    for (int h = 0; h < 3; ++h)
      for (size_t i = 0; i < P; ++i) part[h][i] = tot[h][i] - in[h][size_t(b) * P + i];
    st = lemc_normalise(D, part[0].data(), part[1].data(), part[2].data(), omega, kappa,
                        M_b.data() + size_t(b) * P, H_b.data() + size_t(b) * P);
    if (st != LEMC_OK) return st;
    int rk = 0;
    st = lemc_geneig(D, H_b.data() + size_t(b) * P, M_b.data() + size_t(b) * P, eps,
                     ev_b.data() + size_t(b) * D, nullptr, &rk);
    if (st != LEMC_OK) return st;
  }
  const double f = double(n_bins - 1) / n_bins;
  for (int j = 0; j < D; ++j) {
    double mean = 0;
    for (int b = 0; b < n_bins; ++b) mean += ev_b[size_t(b) * D + j];
    mean /= n_bins;
    double var = 0;
    for (int b = 0; b < n_bins; ++b) {
      const double d = ev_b[size_t(b) * D + j] - mean;
      var += d * d;
    }
    evals_err[j] = std::sqrt(f * var);
  }
  double* errs[2] = {M_err, H_err};
  const std::vector<double>* samples[2] = {&M_b, &H_b};
  for (int q = 0; q < 2; ++q) {
    if (!errs[q]) continue;
    for (size_t e = 0; e < P / 2; ++e) {
      double mr = 0, mi = 0;
      for (int b = 0; b < n_bins; ++b) {
        mr += (*samples[q])[size_t(b) * P + 2 * e];
        mi += (*samples[q])[size_t(b) * P + 2 * e + 1];
      }
      mr /= n_bins;
      mi /= n_bins;
      double var = 0;
      for (int b = 0; b < n_bins; ++b) {
        const double dr = (*samples[q])[size_t(b) * P + 2 * e] - mr;
        const double di = (*samples[q])[size_t(b) * P + 2 * e + 1] - mi;
        var += dr * dr + di * di;
      }
      errs[q][e] = std::sqrt(f * var);
    }
  }
  return LEMC_OK;
}

// Energy-resolved edge occupations: the occupation matrices of one sector,
// normalised as the reference does with the metric (gf_occupation_numbers.cu:
// 432-445: n_l(L,R) = occ_l(L,R) / sum_l occ_l(L,R) * N * M(L,R), then made
// Hermitian per l), rotated onto the generalized eigenvectors of H c = E M c
// (c^H M c = 1): w_j(l) = Re c_j^H n_l c_j, so that sum_l w_j(l) = N.
extern "C" int lemc_spectral_weights(int D, int Lc, const double* occ, const double* H,
                                     const double* M, int N, double eps, double* energies,
                                     double* weights, int* n_modes) {
  if (D <= 0 || Lc <= 0 || !occ || !H || !M || N <= 0 || !energies || !weights) return LEMC_ERR_ARG;
  using cd = std::complex<double>;
  std::vector<cd> n(size_t(D) * D * Lc);
  for (int a = 0; a < D; ++a)
    for (int b = 0; b < D; ++b) {
      cd sum = 0;
      for (int l = 0; l < Lc; ++l) {
        const size_t o = 2 * ((size_t(a) * D + b) * Lc + l);
        sum += cd(occ[o], occ[o + 1]);
      }
      if (std::abs(sum) == 0) return LEMC_ERR_NUMERIC;
      const cd mab(M[2 * (size_t(a) * D + b)], M[2 * (size_t(a) * D + b) + 1]);
      for (int l = 0; l < Lc; ++l) {
        const size_t o = (size_t(a) * D + b) * Lc + l;
        n[o] = cd(occ[2 * o], occ[2 * o + 1]) / sum * double(N) * mab;
      }
    }
  for (int l = 0; l < Lc; ++l)
    for (int a = 0; a < D; ++a)
      for (int b = a; b < D; ++b) {
        const size_t ab = (size_t(a) * D + b) * Lc + l, ba = (size_t(b) * D + a) * Lc + l;
        const cd v = 0.5 * (n[ab] + std::conj(n[ba]));
        n[ab] = v;
        n[ba] = std::conj(v);
      }
  std::vector<double> vec(2 * size_t(D) * D);
  int rank = 0;
  const int st = lemc_geneig(D, H, M, eps, energies, vec.data(), &rank);
  if (st != LEMC_OK) return st;
  for (int j = 0; j < D; ++j)
    for (int l = 0; l < Lc; ++l) {
      if (j >= rank) {
        weights[size_t(j) * Lc + l] = NAN;
        continue;
      }
      cd acc = 0;
      for (int a = 0; a < D; ++a) {
        const cd ca(vec[2 * (size_t(a) * D + j)], vec[2 * (size_t(a) * D + j) + 1]);
        cd row = 0;
        for (int b = 0; b < D; ++b) {
          const cd cb(vec[2 * (size_t(b) * D + j)], vec[2 * (size_t(b) * D + j) + 1]);
          row += n[(size_t(a) * D + b) * Lc + l] * cb;
        }
        acc += std::conj(ca) * row;
      }
      weights[size_t(j) * Lc + l] = acc.real();
    }
  if (n_modes) *n_modes = rank;
  return LEMC_OK;
}

extern "C" int lemc_normalise(int D, const double* S, const double* H2, const double* H4,
                              double omega, double kappa, double* Mout, double* Hout) {
  if (D <= 0 || !S) return LEMC_ERR_ARG;
  std::vector<double> nrm(D);
  for (int a = 0; a < D; ++a) {
    const double saa = S[2 * (size_t(a) * D + a)];
    if (!(saa > 0)) return LEMC_ERR_NUMERIC;
    nrm[a] = std::sqrt(saa);
  }
  auto fill = [&](double* out, auto getter) {
    for (int a = 0; a < D; ++a)
      for (int b = 0; b < D; ++b) {
        const cd x = getter(a, b), y = std::conj(getter(b, a));
        const cd v = 0.5 * (x + y) / (nrm[a] * nrm[b]);
        out[2 * (size_t(a) * D + b)] = v.real();
        out[2 * (size_t(a) * D + b) + 1] = v.imag();
      }
  };
  if (Mout)
    fill(Mout, [&](int a, int b) { return cd(S[2 * (size_t(a) * D + b)], S[2 * (size_t(a) * D + b) + 1]); });
  if (Hout) {
    fill(Hout, [&](int a, int b) {
      cd v = 0.0;
      const size_t o = 2 * (size_t(a) * D + b);
      if (H2) v += omega * cd(H2[o], H2[o + 1]);
      if (H4) v += kappa * cd(H4[o], H4[o + 1]);
      return v;
    });
  }
  return LEMC_OK;
}

// ---------------------------------------------------------------------------
// Time evolution: dC/dt = -i (A + f(t) B) C with A = M^-1 H, B = M^-1 U,
// embedded Cash-Karp RK5(4) (J. R. Cash and A. H. Karp, ACM TOMS 16 (1990)
// 201-222) with per-component error control
//   err_i = |delta_i| / (eps_abs + eps_rel (|C_i| + dt |dC/dt_i|)),
// step accepted when max_i err_i <= 1, step-size factor 0.9 err^-1/5 clipped
// to [0.2, 5] (reference: odeint's controlled runge_kutta_cash_karp54 with
// abs 1e-10, rel 1e-8 and integrate_times, dynamics.cpp:280-290).
namespace {

struct Rhs {
  int D;
  std::vector<cd> A, B;
  lemc_profile_fn f;
  void* user;
  void operator()(double t, const std::vector<cd>& c, std::vector<cd>& out) const {
    const double ft = f ? f(t, user) : 0.0;
    for (int i = 0; i < D; ++i) {
      cd s = 0.0;
      const cd* ai = &A[size_t(i) * D];
      const cd* bi = &B[size_t(i) * D];
      for (int j = 0; j < D; ++j) s += (ai[j] + ft * bi[j]) * c[j];
      out[i] = cd(s.imag(), -s.real());  // -i * s
    }
  }
};

// solve M X = R for X (complex, D x D) by Gaussian elimination with partial pivoting
bool solve_left(int D, std::vector<cd> M, std::vector<cd>& R) {
  for (int k = 0; k < D; ++k) {
    int p = k;
    double best = std::abs(M[size_t(k) * D + k]);
    for (int i = k + 1; i < D; ++i)
      if (std::abs(M[size_t(i) * D + k]) > best) {
        best = std::abs(M[size_t(i) * D + k]);
        p = i;
      }
    if (!(best > 0)) return false;
    if (p != k)
      for (int j = 0; j < D; ++j) {
        std::swap(M[size_t(k) * D + j], M[size_t(p) * D + j]);
        std::swap(R[size_t(k) * D + j], R[size_t(p) * D + j]);
      }
    const cd piv = M[size_t(k) * D + k];
    for (int i = k + 1; i < D; ++i) {
      const cd fct = M[size_t(i) * D + k] / piv;
      if (fct == cd(0.0)) continue;
      for (int j = k; j < D; ++j) M[size_t(i) * D + j] -= fct * M[size_t(k) * D + j];
      for (int j = 0; j < D; ++j) R[size_t(i) * D + j] -= fct * R[size_t(k) * D + j];
    }
  }
  for (int k = D - 1; k >= 0; --k) {
    const cd piv = M[size_t(k) * D + k];
    for (int j = 0; j < D; ++j) {
      cd s = R[size_t(k) * D + j];
      for (int i = k + 1; i < D; ++i) s -= M[size_t(k) * D + i] * R[size_t(i) * D + j];
      R[size_t(k) * D + j] = s / piv;
    }
  }
  return true;
}

}  // namespace

extern "C" int lemc_evolve(int D, const double* M, const double* H, const double* U, int L,
                           const double* rho, lemc_profile_fn f, void* user, double end_time,
                           double save_step, double* out, double* norms, int* n_save) {
  if (D <= 0 || !M || !H || !U || L < 0 || !(save_step > 0) || !(end_time > 0)) return LEMC_ERR_ARG;
  Rhs rhs;
  rhs.D = D;
  rhs.f = f;
  rhs.user = user;
  const std::vector<cd> Mc = to_complex(D, M);
  rhs.A = to_complex(D, H);
  rhs.B = to_complex(D, U);
  if (!solve_left(D, Mc, rhs.A) || !solve_left(D, Mc, rhs.B)) return LEMC_ERR_NUMERIC;
  std::vector<std::vector<cd>> rh(L);
  for (int l = 0; l < L; ++l) rh[l] = to_complex(D, rho + size_t(2) * D * D * l);
  const int ns = int(std::ceil(end_time / save_step));
  if (n_save) *n_save = ns;
  std::vector<cd> c(D, 0.0), k1(D), k2(D), k3(D), k4(D), k5(D), k6(D), tmp(D), c5(D);
  c[0] = 1.0;
  auto observe = [&](int s) {
    if (norms) {
      cd nm = 0.0;
      for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) nm += std::conj(c[i]) * Mc[size_t(i) * D + j] * c[j];
      norms[s] = nm.real();
    }
    if (out)
      for (int l = 0; l < L; ++l) {
        cd v = 0.0;
        for (int i = 0; i < D; ++i)
          for (int j = 0; j < D; ++j) v += std::conj(c[i]) * rh[l][size_t(i) * D + j] * c[j];
        out[2 * (size_t(s) * L + l)] = v.real();
        out[2 * (size_t(s) * L + l) + 1] = v.imag();
      }
  };
  // Cash-Karp tableau
  const double a2 = 0.2, a3 = 0.3, a4 = 0.6, a5 = 1.0, a6 = 0.875;
  const double b21 = 0.2, b31 = 3.0 / 40, b32 = 9.0 / 40, b41 = 0.3, b42 = -0.9, b43 = 1.2,
               b51 = -11.0 / 54, b52 = 2.5, b53 = -70.0 / 27, b54 = 35.0 / 27,
               b61 = 1631.0 / 55296, b62 = 175.0 / 512, b63 = 575.0 / 13824,
               b64 = 44275.0 / 110592, b65 = 253.0 / 4096;
  const double c1 = 37.0 / 378, c3 = 250.0 / 621, c4 = 125.0 / 594, c6 = 512.0 / 1771;
  const double d1 = c1 - 2825.0 / 27648, d3 = c3 - 18575.0 / 48384, d4 = c4 - 13525.0 / 55296,
               d5 = -277.0 / 14336, d6 = c6 - 0.25;
  const double eabs = 1e-10, erel = 1e-8;
  double t = 0.0, dt = save_step;
  observe(0);
  for (int s = 1; s < ns; ++s) {
    const double target = s * save_step;
    int guard = 0;
    while (t < target) {
      if (++guard > 10000000) return LEMC_ERR_NUMERIC;
      double h = std::min(dt, target - t);
      rhs(t, c, k1);
      for (int i = 0; i < D; ++i) tmp[i] = c[i] + h * b21 * k1[i];
      rhs(t + a2 * h, tmp, k2);
      for (int i = 0; i < D; ++i) tmp[i] = c[i] + h * (b31 * k1[i] + b32 * k2[i]);
      rhs(t + a3 * h, tmp, k3);
      for (int i = 0; i < D; ++i) tmp[i] = c[i] + h * (b41 * k1[i] + b42 * k2[i] + b43 * k3[i]);
      rhs(t + a4 * h, tmp, k4);
      for (int i = 0; i < D; ++i)
        tmp[i] = c[i] + h * (b51 * k1[i] + b52 * k2[i] + b53 * k3[i] + b54 * k4[i]);
      rhs(t + a5 * h, tmp, k5);
      for (int i = 0; i < D; ++i)
        tmp[i] = c[i] + h * (b61 * k1[i] + b62 * k2[i] + b63 * k3[i] + b64 * k4[i] + b65 * k5[i]);
      rhs(t + a6 * h, tmp, k6);
      double emax = 0.0;
      for (int i = 0; i < D; ++i) {
        c5[i] = c[i] + h * (c1 * k1[i] + c3 * k3[i] + c4 * k4[i] + c6 * k6[i]);
        const cd de = h * (d1 * k1[i] + d3 * k3[i] + d4 * k4[i] + d5 * k5[i] + d6 * k6[i]);
        const double sc = eabs + erel * (std::abs(c[i]) + h * std::abs(k1[i]));
        emax = std::max(emax, std::abs(de) / sc);
      }
      if (emax <= 1.0) {
        t += h;
        c.swap(c5);
        const double fac = emax > 0 ? 0.9 * std::pow(emax, -0.2) : 5.0;
        if (h == dt) dt = h * std::min(5.0, std::max(1.0, fac));
      } else {
        dt = h * std::max(0.2, 0.9 * std::pow(emax, -0.25));
      }
    }
    observe(s);
  }
  return LEMC_OK;
}
