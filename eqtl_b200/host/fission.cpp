// eqtl fission (run_fission, src/fission.cpp:277-393): data thinning of the
// phenotype table into Y1 + Y2, optional residualisation of Y1 on the
// covariates, and PEER factors of Y1 on the device (eqtl_peer).
//
// The thinning and PEER's starting values come from the C++ standard
// library's own distributions on std::mt19937, drawn in the reference's
// order, so Y1, Y2 and the starting point are the reference's:
//   counts (every value a non-negative integer within 1e-9, NaN skipped)
//       Y1 ~ Binomial(y, eps) per entry, genes outer, samples inner; Y2 = y - Y1
//   otherwise
//       per gene, one normal_distribution(0, sqrt(var * eps * (1 - eps)))
//       (var: sample variance of the gene's non-NaN values, 0 below two;
//       the sd floored at 1e-15); Y1 = eps y + z, Y2 = (1 - eps) y - z
//   start (seed + 1): X [n, K] then W [G, K], each column by column, from one
//       normal_distribution(0, 1).
// The three matrices are written as the reference writes them (std::ostream
// defaults: six significant digits).
#include <cmath>
#include <fstream>
#include <iostream>
#include <random>
#include <unordered_map>

#include "scan.hpp"

namespace eqtl_host {

namespace {

std::string trim_ws(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
  while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
  return s.substr(a, b - a);
}

std::vector<std::string> tokens(const std::string& s) {
  std::vector<std::string> out;
  size_t i = 0;
  while (i < s.size()) {
    while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i;
    size_t j = i;
    while (j < s.size() && !std::isspace(static_cast<unsigned char>(s[j]))) ++j;
    if (j > i) out.push_back(s.substr(i, j - i));
    i = j;
  }
  return out;
}

// Y [n][G] row-major (as the table is read)
bool integer_counts(const std::vector<double>& Y) {
  for (double v : Y) {
    if (std::isnan(v)) continue;
    if (v < 0.0 || std::abs(v - std::round(v)) > 1e-9) return false;
  }
  return true;
}

void write_matrix(const std::string& path, const std::vector<double>& M, size_t rows, size_t cols, bool col_major,
                  const std::vector<std::string>& row_ids, const std::vector<std::string>& col_ids) {
  std::ofstream f(path);
  if (!f) die("cannot write: " + path);
  f << "sample_id";
  for (const auto& c : col_ids) f << '\t' << c;
  f << '\n';
  for (size_t i = 0; i < rows; ++i) {
    f << row_ids[i];
    for (size_t j = 0; j < cols; ++j) f << '\t' << (col_major ? M[j * rows + i] : M[i * cols + j]);
    f << '\n';
  }
}

// sample ids of a covariate file, skipping a header line (src/fission.cpp:301-320)
std::vector<std::string> covar_ids(const std::string& path) {
  std::ifstream in(path);
  if (!in) die("cannot open covar: " + path);
  std::vector<std::string> ids;
  std::string line;
  bool first = true;
  while (std::getline(in, line)) {
    line = trim_ws(line);
    if (line.empty() || line[0] == '#') continue;
    const auto tok = tokens(line);
    if (tok.size() < 2) continue;
    if (first) {
      first = false;
      char* end = nullptr;
      std::strtod(tok[1].c_str(), &end);
      if (!(end && *end == '\0')) continue;  // header
    }
    ids.push_back(tok[0]);
  }
  return ids;
}

}  // namespace

int run_fission(const Options& opt) {
  Pheno P = load_pheno(opt.pheno);
  int n = static_cast<int>(P.samples.size());
  const int G = static_cast<int>(P.genes.size());
  if (opt.peer_factors >= n || opt.peer_factors >= G)
    die("--peer-factors must be < min(n_samples, n_genes)  [got " + std::to_string(opt.peer_factors) +
        ", n=" + std::to_string(n) + ", G=" + std::to_string(G) + "]");
  const unsigned seed = static_cast<unsigned>(opt.seed >= 0 ? opt.seed : 42);
  const double eps = opt.fission_epsilon;
  // Y1, Y2 row-major [n][G] like the table
  std::vector<double> Y1(P.Y.size()), Y2(P.Y.size());
  auto at = [&](int i, int j) { return static_cast<size_t>(i) * G + j; };
  if (integer_counts(P.Y)) {
    info("fission: integer counts detected → Binomial thinning");
    std::mt19937 rng(seed);
    for (int j = 0; j < G; ++j)
      for (int i = 0; i < n; ++i) {
        const double v = P.Y[at(i, j)];
        if (std::isnan(v)) {
          Y1[at(i, j)] = Y2[at(i, j)] = v;
          continue;
        }
        const int cnt = static_cast<int>(std::round(v));
        const int y1 = std::binomial_distribution<int>{cnt, eps}(rng);
        Y1[at(i, j)] = static_cast<double>(y1);
        Y2[at(i, j)] = static_cast<double>(cnt - y1);
      }
  } else {
    info("fission: continuous data detected → Gaussian fission");
    std::vector<double> var(static_cast<size_t>(G), 0.0);
    for (int j = 0; j < G; ++j) {
      double mean = 0.0;
      int cnt = 0;
      for (int i = 0; i < n; ++i)
        if (!std::isnan(P.Y[at(i, j)])) {
          mean += P.Y[at(i, j)];
          ++cnt;
        }
      if (cnt < 2) continue;
      mean /= cnt;
      double v = 0.0;
      for (int i = 0; i < n; ++i)
        if (!std::isnan(P.Y[at(i, j)])) v += (P.Y[at(i, j)] - mean) * (P.Y[at(i, j)] - mean);
      var[static_cast<size_t>(j)] = v / (cnt - 1);
    }
    std::mt19937 rng(seed);
    for (int j = 0; j < G; ++j) {
      const double sigma = std::sqrt(var[static_cast<size_t>(j)] * eps * (1.0 - eps));
      std::normal_distribution<double> nd(0.0, sigma > 1e-15 ? sigma : 1e-15);
      for (int i = 0; i < n; ++i) {
        const double v = P.Y[at(i, j)];
        if (std::isnan(v)) {
          Y1[at(i, j)] = Y2[at(i, j)] = v;
          continue;
        }
        const double z = nd(rng);
        Y1[at(i, j)] = eps * v + z;
        Y2[at(i, j)] = (1.0 - eps) * v - z;
      }
    }
  }

  // PEER input, column-major [n, G]: Y1, or Y1 residualised on the covariates
  std::vector<std::string> samples = P.samples;
  std::vector<double> Y_peer;
  if (!opt.covar.empty()) {
    const std::vector<std::string> cov = covar_ids(opt.covar);
    std::unordered_map<std::string, int> in_cov;
    for (const auto& id : cov) in_cov.emplace(id, 0);
    std::vector<int> rows;
    for (int i = 0; i < n; ++i)
      if (in_cov.count(P.samples[i])) rows.push_back(i);
    if (rows.empty()) die("fission: no overlapping samples between pheno and covar");
    if (static_cast<int>(rows.size()) < n)
      info("fission: using " + std::to_string(rows.size()) + " samples (dropped " +
           std::to_string(n - static_cast<int>(rows.size())) + " not in covar)");
    std::vector<double> A1, A2;
    samples.clear();
    for (int r : rows) {
      samples.push_back(P.samples[r]);
      A1.insert(A1.end(), Y1.begin() + static_cast<size_t>(r) * G, Y1.begin() + static_cast<size_t>(r + 1) * G);
      A2.insert(A2.end(), Y2.begin() + static_cast<size_t>(r) * G, Y2.begin() + static_cast<size_t>(r + 1) * G);
    }
    Y1.swap(A1);
    Y2.swap(A2);
    n = static_cast<int>(rows.size());
    int p = 0;
    const std::vector<double> X = load_covar(opt.covar, samples, p);  // [n, p] column-major
    // X'X by Cholesky; the fit of each gene removed
    std::vector<double> L(static_cast<size_t>(p) * p, 0.0);
    for (int a = 0; a < p; ++a)
      for (int b = 0; b <= a; ++b) {
        double s = 0;
        for (int i = 0; i < n; ++i) s += X[static_cast<size_t>(a) * n + i] * X[static_cast<size_t>(b) * n + i];
        L[static_cast<size_t>(a) * p + b] = s;
      }
    for (int j = 0; j < p; ++j) {
      double d = L[static_cast<size_t>(j) * p + j];
      for (int k = 0; k < j; ++k) d -= L[static_cast<size_t>(j) * p + k] * L[static_cast<size_t>(j) * p + k];
      if (!(d > 0)) die("fission: covariate XtX not invertible");
      d = std::sqrt(d);
      L[static_cast<size_t>(j) * p + j] = d;
      for (int i = j + 1; i < p; ++i) {
        double v = L[static_cast<size_t>(i) * p + j];
        for (int k = 0; k < j; ++k) v -= L[static_cast<size_t>(i) * p + k] * L[static_cast<size_t>(j) * p + k];
        L[static_cast<size_t>(i) * p + j] = v / d;
      }
    }
    Y_peer.resize(static_cast<size_t>(n) * G);
    std::vector<double> yy(n), rhs(p), b(p);
    for (int j = 0; j < G; ++j) {
      double mean = 0;
      int cnt = 0;
      for (int i = 0; i < n; ++i) {
        yy[i] = Y1[at(i, j)];
        if (std::isfinite(yy[i])) {
          mean += yy[i];
          ++cnt;
        }
      }
      if (cnt > 0) mean /= cnt;
      for (int i = 0; i < n; ++i)
        if (!std::isfinite(yy[i])) yy[i] = mean;
      for (int a = 0; a < p; ++a) {
        double s = 0;
        for (int i = 0; i < n; ++i) s += X[static_cast<size_t>(a) * n + i] * yy[i];
        rhs[a] = s;
      }
      for (int a = 0; a < p; ++a) {
        double t = rhs[a];
        for (int k = 0; k < a; ++k) t -= L[static_cast<size_t>(a) * p + k] * b[k];
        b[a] = t / L[static_cast<size_t>(a) * p + a];
      }
      for (int a = p - 1; a >= 0; --a) {
        double t = b[a];
        for (int k = a + 1; k < p; ++k) t -= L[static_cast<size_t>(k) * p + a] * b[k];
        b[a] = t / L[static_cast<size_t>(a) * p + a];
      }
      for (int i = 0; i < n; ++i) {
        double fit = 0;
        for (int a = 0; a < p; ++a) fit += X[static_cast<size_t>(a) * n + i] * b[a];
        Y_peer[static_cast<size_t>(j) * n + i] = yy[i] - fit;
      }
    }
    info("fission: residualized " + std::to_string(p) + " covar columns from Y1 before PEER");
  } else {
    Y_peer.resize(static_cast<size_t>(n) * G);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < G; ++j) Y_peer[static_cast<size_t>(j) * n + i] = Y1[at(i, j)];
  }
  const int K = opt.peer_factors;
  if (K >= n || K >= G) die("--peer-factors must be < min(n_samples, n_genes) after sample filter");
  info("fission: estimating " + std::to_string(K) + " PEER factors from Y1 (n=" + std::to_string(n) +
       " samples, G=" + std::to_string(G) + " genes)");

  // the reference's starting values (peer_factors' seed is the run's + 1)
  std::vector<double> X0(static_cast<size_t>(n) * K), W0(static_cast<size_t>(G) * K);
  {
    std::mt19937 rng(seed + 1u);
    std::normal_distribution<double> nd;
    for (double& v : X0) v = nd(rng);  // column by column
    for (double& v : W0) v = nd(rng);
  }
  // the thinned tables first (they do not depend on the factors)
  const std::string y2 = opt.out + ".Y2.tsv", y1 = opt.out + ".Y1.tsv", fp = opt.out + ".factors.tsv";
  write_matrix(y2, Y2, static_cast<size_t>(n), static_cast<size_t>(G), false, samples, P.genes);
  info("fission: wrote " + y2);
  write_matrix(y1, Y1, static_cast<size_t>(n), static_cast<size_t>(G), false, samples, P.genes);
  info("fission: wrote " + y1);
  std::vector<double> F(static_cast<size_t>(n) * K);
  int32_t iters = 0;
  {
    Device dev;
    dev.check(eqtl_peer(dev.ctx, Y_peer.data(), n, G, K, opt.fission_max_iter, opt.fission_tol, X0.data(), W0.data(),
                        F.data(), &iters),
              "PEER");
  }
  info("fission: PEER stopped after " + std::to_string(iters) + " iterations");
  std::vector<std::string> names;
  for (int k = 0; k < K; ++k) names.push_back("factor" + std::to_string(k + 1));
  write_matrix(fp, F, static_cast<size_t>(n), static_cast<size_t>(K), true, samples, names);
  info("fission: wrote " + fp);
  return 0;
}

}  // namespace eqtl_host
