// Gene-level permutations.
//   LM    the permuted phenotype is the null residual y_s = y - X (X'X)^-1 X'y
//         with its entries shuffled (include/eqtl/scan_cis.hpp:68-176).
//   LMM   the whitened spectral residual w = (y~ - X~ b0) * sqrt(dinv) is
//         shuffled, un-whitened and mapped back to samples:
//         y_b = Q (X~ b0 + w_perm / sqrt(max(dinv, 1e-12)))
//         (src/scan_perm.cpp:48-120), with the gene's REML delta from the scan.
// Each permutation b of a gene draws its shuffle from std::mt19937 seeded
// with (seed or 1) + 9973 b + fnv1a(gene) through std::shuffle, so the index
// sequences are the reference's. Every permuted column gets a fresh null fit
// and the FP64 tests of the gene's cached SNPs on the device
// (eqtl_test_pairs); min p over finite p gives T_b = -log10 min p, then
// p_emp and the beta approximation per gene.
#include <algorithm>
#include <numeric>
#include <random>

#include "perm.hpp"

namespace eqtl_host {

namespace {

// Solves A x = b for a small SPD A (p x p, row-major) by Cholesky.
std::vector<double> spd_solve(std::vector<double> A, std::vector<double> b, int p) {
  for (int j = 0; j < p; ++j) {
    double d = A[j * p + j];
    for (int k = 0; k < j; ++k) d -= A[j * p + k] * A[j * p + k];
    if (!(d > 0)) die("covariate matrix is not positive definite");
    d = std::sqrt(d);
    A[j * p + j] = d;
    for (int i = j + 1; i < p; ++i) {
      double s = A[i * p + j];
      for (int k = 0; k < j; ++k) s -= A[i * p + k] * A[j * p + k];
      A[i * p + j] = s / d;
    }
  }
  for (int i = 0; i < p; ++i) {
    double s = b[i];
    for (int k = 0; k < i; ++k) s -= A[i * p + k] * b[k];
    b[i] = s / A[i * p + i];
  }
  for (int i = p - 1; i >= 0; --i) {
    double s = b[i];
    for (int k = i + 1; k < p; ++k) s -= A[k * p + i] * b[k];
    b[i] = s / A[i * p + i];
  }
  return b;
}

// What a gene's permutations shuffle, and how a shuffled vector becomes a
// phenotype column.
struct PermBase {
  std::vector<double> base;  // shuffled entries
  std::vector<double> xb0;   // LMM: X~ b0
  std::vector<double> dinv;  // LMM
};

PermBase lm_base(const Study& st, const std::vector<double>& y) {
  const size_t n = st.samples.size();
  const int p = st.p;
  std::vector<double> XtX(static_cast<size_t>(p) * p), Xty(p);
  for (int a = 0; a < p; ++a) {
    const double* xa = &st.X[static_cast<size_t>(a) * n];
    for (int b = 0; b <= a; ++b) {
      const double* xb = &st.X[static_cast<size_t>(b) * n];
      double s = 0;
      for (size_t i = 0; i < n; ++i) s += xa[i] * xb[i];
      XtX[a * p + b] = XtX[b * p + a] = s;
    }
    double s = 0;
    for (size_t i = 0; i < n; ++i) s += xa[i] * y[i];
    Xty[a] = s;
  }
  const std::vector<double> beta = spd_solve(XtX, Xty, p);
  PermBase B;
  B.base = y;
  for (int a = 0; a < p; ++a)
    for (size_t i = 0; i < n; ++i) B.base[i] -= st.X[static_cast<size_t>(a) * n + i] * beta[a];
  return B;
}

PermBase lmm_base(const Study& st, const std::vector<double>& y, double delta) {
  const size_t n = st.samples.size();
  const int p = st.p;
  const std::vector<double>& Q = st.basis_Q;  // column-major, column j = eigenvector j
  std::vector<double> yt(n), Xt(static_cast<size_t>(p) * n), dinv(n);
  for (size_t j = 0; j < n; ++j) {
    const double* q = &Q[j * n];
    double s = 0;
    for (size_t i = 0; i < n; ++i) s += q[i] * y[i];
    yt[j] = s;
    for (int a = 0; a < p; ++a) {
      double sa = 0;
      const double* xa = &st.X[static_cast<size_t>(a) * n];
      for (size_t i = 0; i < n; ++i) sa += q[i] * xa[i];
      Xt[static_cast<size_t>(a) * n + j] = sa;
    }
    dinv[j] = 1.0 / std::max(delta * st.basis_lambda[j] + 1.0, 1e-12);
  }
  std::vector<double> A(static_cast<size_t>(p) * p), r(p);
  for (int a = 0; a < p; ++a) {
    for (int b = 0; b <= a; ++b) {
      double s = 0;
      for (size_t j = 0; j < n; ++j) s += Xt[a * n + j] * dinv[j] * Xt[b * n + j];
      A[a * p + b] = A[b * p + a] = s;
    }
    double s = 0;
    for (size_t j = 0; j < n; ++j) s += Xt[a * n + j] * dinv[j] * yt[j];
    r[a] = s;
  }
  const std::vector<double> b0 = spd_solve(A, r, p);
  PermBase B;
  B.xb0.assign(n, 0.0);
  for (int a = 0; a < p; ++a)
    for (size_t j = 0; j < n; ++j) B.xb0[j] += Xt[a * n + j] * b0[a];
  B.base.resize(n);
  for (size_t j = 0; j < n; ++j) B.base[j] = (yt[j] - B.xb0[j]) * std::sqrt(dinv[j]);
  B.dinv = std::move(dinv);
  return B;
}

// Phenotype column of permutation b of `gene`.
void permuted_column(const Study& st, const std::string& model, const PermBase& B, const std::string& gene, int b,
                     double* col) {
  const size_t n = B.base.size();
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::mt19937 rng(perm_seed(st.opt->seed, b, gene));
  std::shuffle(idx.begin(), idx.end(), rng);
  if (model == "lm") {
    for (size_t i = 0; i < n; ++i) col[i] = B.base[idx[i]];
    return;
  }
  std::vector<double> v(n);
  for (size_t j = 0; j < n; ++j) v[j] = B.xb0[j] + B.base[idx[j]] / std::sqrt(std::max(B.dinv[j], 1e-12));
  const std::vector<double>& Q = st.basis_Q;
  std::fill(col, col + n, 0.0);
  for (size_t j = 0; j < n; ++j) {
    const double* q = &Q[j * n];
    const double vj = v[j];
    for (size_t i = 0; i < n; ++i) col[i] += q[i] * vj;
  }
}

}  // namespace

std::vector<PermOut> run_permutations(const Study& st, const std::string& model, const std::vector<PermGene>& genes,
                                      const std::vector<double>& delta) {
  const Options& opt = *st.opt;
  const size_t n = st.samples.size();
  const int B = opt.perm;
  std::vector<PermOut> out(genes.size());
  std::vector<size_t> active;
  for (size_t j = 0; j < genes.size(); ++j)
    if (genes[j].active && !genes[j].snps.empty()) active.push_back(j);
  if (active.empty() || B <= 0) return out;
  if (model == "lmm" && st.basis_Q.size() != n * n) die("internal: LMM permutations need the eigenbasis on the host");
  // genes per device batch: keep the permuted phenotype block near 2^26 doubles
  const size_t cols_budget = std::max<size_t>(static_cast<size_t>(B), (size_t(1) << 26) / std::max<size_t>(n, 1));
  const size_t genes_per_batch = std::max<size_t>(1, cols_budget / static_cast<size_t>(B));
  eqtl_scan_params prm{};
  prm.n = static_cast<int32_t>(n);
  prm.p = st.p;
  for (size_t a = 0; a < active.size(); a += genes_per_batch) {
    const size_t nb = std::min(genes_per_batch, active.size() - a);
    const size_t cols = nb * static_cast<size_t>(B);
    std::vector<double> Y(cols * n);
    std::vector<int32_t> pc;
    std::vector<int64_t> ps;
    for (size_t gi = 0; gi < nb; ++gi) {
      const PermGene& g = genes[active[a + gi]];
      const PermBase base = model == "lm" ? lm_base(st, g.y) : lmm_base(st, g.y, delta[active[a + gi]]);
      for (int b = 0; b < B; ++b) {
        const size_t c = gi * B + b;
        permuted_column(st, model, base, g.name, b, &Y[c * n]);
        for (int64_t s : g.snps) {
          pc.push_back(static_cast<int32_t>(c));
          ps.push_back(s);
        }
      }
    }
    prm.n_genes = static_cast<int32_t>(cols);
    std::vector<eqtl_pair> res(pc.size());
    st.dev->check(eqtl_test_pairs(st.dev->ctx, model == "lm" ? EQTL_MODEL_LM : EQTL_MODEL_LMM, &prm, Y.data(),
                                  st.X.data(), pc.data(), ps.data(), static_cast<int64_t>(pc.size()), res.data(),
                                  nullptr),
                  "permutation tests");
    std::vector<double> minp(cols, 1.0);
    for (size_t i = 0; i < res.size(); ++i)
      if (std::isfinite(res[i].p) && res[i].p < minp[pc[i]]) minp[pc[i]] = res[i].p;
    for (size_t gi = 0; gi < nb; ++gi) {
      const PermGene& g = genes[active[a + gi]];
      PermOut& o = out[active[a + gi]];
      std::vector<double> T(B), mp(B);
      for (int b = 0; b < B; ++b) {
        mp[b] = minp[gi * B + b];
        T[b] = -std::log10(std::max(mp[b], 1e-300));
      }
      o.done = true;
      o.p_emp = p_emp(-std::log10(std::max(g.obs_min_p, 1e-300)), T);
      if (!opt.disable_beta_approx) {
        o.beta = beta_approx(mp, g.obs_min_p);
      } else {
        o.beta.p = NAN;
        o.beta.s1 = o.beta.s2 = 0.0;
      }
    }
  }
  return out;
}

}  // namespace eqtl_host
