// Test infrastructure only: the reference's own eigensolver path
// (src/model_lmm.cpp:106-113: Eigen::SelfAdjointEigenSolver on the GRM,
// eigenvalues clipped at 0) as a tiny filter program, so the oracle can use
// exactly the eigenvectors - including their signs - that the reference
// binary uses. LMM permutations (include/eqtl/scan_cis.hpp:77-87,135-147)
// shuffle residuals in eigen-coordinates, so their result depends on those
// signs. Usage: eigsolve in.bin out.bin; in = int64 n + n*n float64
// (row-major K); out = n float64 lambda + n*n float64 Q (column-major).
#include <Eigen/Dense>
#include <cstdint>
#include <cstdio>
#include <vector>

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  int64_t n = 0;
  if (std::fread(&n, sizeof(n), 1, f) != 1 || n <= 0) return 4;
  Eigen::MatrixXd K(n, n);
  std::vector<double> buf(static_cast<size_t>(n * n));
  if (std::fread(buf.data(), sizeof(double), buf.size(), f) != buf.size()) return 5;
  std::fclose(f);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = 0; j < n; ++j) K(i, j) = buf[static_cast<size_t>(i * n + j)];
  Eigen::SelfAdjointEigenSolver<Eigen::MatrixXd> es(K);
  if (es.info() != Eigen::Success) return 6;
  Eigen::VectorXd lam = es.eigenvalues().cwiseMax(0.0);
  Eigen::MatrixXd Q = es.eigenvectors();
  FILE* o = std::fopen(argv[2], "wb");
  if (!o) return 7;
  std::fwrite(lam.data(), sizeof(double), static_cast<size_t>(n), o);
  std::fwrite(Q.data(), sizeof(double), static_cast<size_t>(n * n), o);
  std::fclose(o);
  return 0;
}
