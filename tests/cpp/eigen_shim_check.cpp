// Reads n, then A and B (n x n complex, row-major "re im" pairs) from stdin and
// prints the generalized eigenvalues and eigenvectors (column k = vector k) of
// the Eigen stand-in under oracle/eigen_shim, for tests/test_eigen_shim.py.
#include <cstdio>
#include <iostream>

#include <Eigen/Dense>
#include <Eigen/Eigenvalues>

int main() {
  int n = 0;
  std::cin >> n;
  Eigen::MatrixXcd A(n, n), B(n, n);
  for (Eigen::MatrixXcd* M : {&A, &B})
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double re, im;
        std::cin >> re >> im;
        (*M)(i, j) = std::complex<double>(re, im);
      }
  Eigen::GeneralizedSelfAdjointEigenSolver<Eigen::MatrixXcd> es(A, B);
  for (int k = 0; k < n; ++k) std::printf("%.17g\n", es.eigenvalues()[k]);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k)
      std::printf("%.17g %.17g\n", es.eigenvectors()(i, k).real(), es.eigenvectors()(i, k).imag());
  Eigen::GeneralizedSelfAdjointEigenSolver<Eigen::MatrixXcd> ev(A, B, Eigen::EigenvaluesOnly);
  std::printf("%zu\n", lemc_eigen_shim::captured().size());
  return 0;
}
