// Gene-level permutations.
//   LM    the permuted phenotype is the null residual y_s = y - X (X'X)^-1 X'y
//         with its entries shuffled (include/eqtl/scan_cis.hpp:68-176).
//   LMM   the whitened spectral residual w = (y~ - X~ b0) * sqrt(dinv) is
//         shuffled and un-whitened, y~_b = X~ b0 + w_perm / sqrt(max(dinv, 1e-12))
//         (src/scan_perm.cpp:48-120), with the gene's REML delta from the scan.
//         The reference maps y~_b back to samples through Q and its null fit
//         rotates it again; the device takes y~_b as it is (y_rotated).
// Each permutation b of a gene draws its shuffle from std::mt19937 seeded
// with (seed or 1) + 9973 b + fnv1a(gene) through std::shuffle, so the index
// sequences are the reference's; columns are built on all host threads,
// one batch ahead of the device. With --perm-rng device the LM and LMM
// shuffles are drawn on the device instead (eqtl_pheno_permute: Philox keyed
// by (seed or 1) and the 64-bit fnv1a of the gene): independent uniform
// permutations, not the reference's sequences, and only the per-gene base
// vectors cross to the device.
//   GLM   parametric: after the same shuffle draws, y_i ~ Poisson(Gamma(1/phi,
//         phi mu_i)) from the observed null fit (Poisson(mu_i) when phi <= 1e-9,
//         0 when mu_i <= 1e-12), with the standard library's distributions
//         on the same generator (include/eqtl/scan_cis.hpp:115-127); every
//         SNP of the gene's scope is tested.
// Every permuted column gets a fresh null fit on the device. Cis: the banded
// cis scan of all columns, each with its gene's window; min p = the column's
// FP64-refined best SNP. Trans/gw stage 2: FP64 tests of the gene's top-K
// SNPs (eqtl_test_pairs). Then p_emp and the beta approximation per gene.
#include <algorithm>
#include <future>
#include <numeric>
#include <random>
#include <thread>

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

// y~ = Q'y, X~ = Q'X and the gene's GLS fit at its REML delta: the base of
// the LMM permutations, in the eigenbasis.
PermBase lmm_base(const Study& st, const std::vector<double>& y, double delta, const std::vector<double>& Xt) {
  const size_t n = st.samples.size();
  const int p = st.p;
  const std::vector<double>& Q = st.basis_Q;  // column-major, column j = eigenvector j
  std::vector<double> yt(n), dinv(n);
  for (size_t j = 0; j < n; ++j) {
    const double* q = &Q[j * n];
    double s = 0;
    for (size_t i = 0; i < n; ++i) s += q[i] * y[i];
    yt[j] = s;
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

// Column of permutation b of `gene`: LM in sample space, LMM rotated.
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
  for (size_t j = 0; j < n; ++j) col[j] = B.xb0[j] + B.base[idx[j]] / std::sqrt(std::max(B.dinv[j], 1e-12));
}

// Column of permutation b of a GLM gene: NB resampling of its null means.
void glm_column(const Options& opt, const PermGene& g, int b, double* col) {
  const size_t n = g.mu.size();
  std::vector<int> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::mt19937 rng(perm_seed(opt.seed, b, g.name));
  std::shuffle(idx.begin(), idx.end(), rng);  // drawn as the reference draws it, then unused
  for (size_t i = 0; i < n; ++i) {
    const double mu = g.mu[i];
    if (mu <= 1e-12) {
      col[i] = 0.0;
      continue;
    }
    if (g.phi > 1e-9) {
      std::gamma_distribution<double> gam(1.0 / g.phi, g.phi * mu);
      std::poisson_distribution<long> pois(gam(rng));
      col[i] = static_cast<double>(pois(rng));
    } else {
      std::poisson_distribution<long> pois(mu);
      col[i] = static_cast<double>(pois(rng));
    }
  }
}

template <class F>
void parallel_for(size_t n, F&& f) {
  const size_t nt = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), std::max<size_t>(n, 1));
  if (nt <= 1) {
    for (size_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> th;
  for (size_t t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      for (size_t i = t; i < n; i += nt) f(i);
    });
  for (auto& x : th) x.join();
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
    if (genes[j].active && (genes[j].window || !genes[j].snps.empty() || genes[j].scan_mode >= 0))
      active.push_back(j);
  if (active.empty() || B <= 0) return out;
  const bool lmm = model == "lmm";
  if (lmm && st.basis_Q.size() != n * n) die("internal: LMM permutations need the eigenbasis on the host");
  std::vector<double> Xt;  // LMM: X~ = Q'X, shared by every gene
  if (lmm) {
    Xt.assign(static_cast<size_t>(st.p) * n, 0.0);
    for (int a = 0; a < st.p; ++a)
      for (size_t j = 0; j < n; ++j) {
        const double* q = &st.basis_Q[j * n];
        double s = 0;
        for (size_t i = 0; i < n; ++i) s += q[i] * st.X[static_cast<size_t>(a) * n + i];
        Xt[a * n + j] = s;
      }
  }
  // genes per device batch: keep the permuted phenotype block near 2^26 doubles
  const size_t cols_budget = std::max<size_t>(static_cast<size_t>(B), (size_t(1) << 26) / std::max<size_t>(n, 1));
  const size_t genes_per_batch = std::max<size_t>(1, cols_budget / static_cast<size_t>(B));
  // --perm-rng device (LM and LMM): the host prepares each gene's base
  // vectors only; eqtl_pheno_permute draws and builds the columns on the
  // device, where they stay for the scan
  const bool on_device = opt.perm_device && model != "glm";
  const uint64_t dev_seed = opt.seed >= 0 ? static_cast<uint64_t>(opt.seed) : 1u;
  Trace tr;
  tr.mark(std::string("permutations: setup (") + (on_device ? "device" : "host") + " draws)");
  struct Batch {
    std::vector<double> Y;                 // host draws: the columns [cols][n]
    std::vector<double> base, xb0, dinv;   // device draws: per gene [nb][n]
    std::vector<uint64_t> keys;
  };
  // batch k + 1 is prepared on the host while batch k runs on the device
  auto build = [&](size_t a) {
    const size_t nb = std::min(genes_per_batch, active.size() - a);
    const size_t cols = nb * static_cast<size_t>(B);
    Batch bt;
    if (model == "glm") {
      bt.Y.resize(cols * n);
      parallel_for(cols, [&](size_t c) { glm_column(opt, genes[active[a + c / B]], static_cast<int>(c % B), &bt.Y[c * n]); });
      return bt;
    }
    std::vector<PermBase> bases(nb);
    parallel_for(nb, [&](size_t gi) {
      const PermGene& g = genes[active[a + gi]];
      bases[gi] = lmm ? lmm_base(st, g.y, delta[active[a + gi]], Xt) : lm_base(st, g.y);
    });
    if (on_device) {
      bt.base.resize(nb * n);
      if (lmm) {
        bt.xb0.resize(nb * n);
        bt.dinv.resize(nb * n);
      }
      bt.keys.resize(nb);
      for (size_t gi = 0; gi < nb; ++gi) {
        std::copy(bases[gi].base.begin(), bases[gi].base.end(), bt.base.begin() + gi * n);
        if (lmm) {
          std::copy(bases[gi].xb0.begin(), bases[gi].xb0.end(), bt.xb0.begin() + gi * n);
          std::copy(bases[gi].dinv.begin(), bases[gi].dinv.end(), bt.dinv.begin() + gi * n);
        }
        bt.keys[gi] = fnv1a64(genes[active[a + gi]].name);
      }
      return bt;
    }
    bt.Y.resize(cols * n);
    parallel_for(cols, [&](size_t c) {
      const size_t gi = c / B;
      permuted_column(st, model, bases[gi], genes[active[a + gi]].name, static_cast<int>(c % B), &bt.Y[c * n]);
    });
    return bt;
  };
  std::future<Batch> next = std::async(std::launch::async, build, size_t(0));
  for (size_t a = 0; a < active.size(); a += genes_per_batch) {
    const size_t nb = std::min(genes_per_batch, active.size() - a);
    const size_t cols = nb * static_cast<size_t>(B);
    const Batch bt = next.get();
    const std::vector<double>& Y = bt.Y;  // empty with device draws: the scans read the resident columns
    if (a + genes_per_batch < active.size()) next = std::async(std::launch::async, build, a + genes_per_batch);
    if (on_device) {
      st.dev->check(eqtl_pheno_permute(st.dev->ctx, bt.base.data(), lmm ? bt.xb0.data() : nullptr,
                                       lmm ? bt.dinv.data() : nullptr, bt.keys.data(), static_cast<int32_t>(n),
                                       static_cast<int32_t>(nb), B, dev_seed, st.X.data(), st.p, nullptr),
                    "device permutation draws");
      tr.mark("permutations: " + std::to_string(cols) + " columns drawn on the device");
    } else {
      tr.mark("permutations: " + std::to_string(cols) + " columns ready (host build overlapped)");
    }
    std::vector<double> minp(cols, 1.0);
    if (model == "glm") {
      // every SNP of each gene's scope, with a fresh NB null fit per column
      std::vector<const GeneLoc*> win(cols);
      for (size_t c = 0; c < cols; ++c) win[c] = genes[active[a + c / B]].window;
      const ScanResult R = scan_columns(st, model, Y, cols, win, genes[active[a]].scan_mode, 0.0, 0.0, false);
      for (size_t c = 0; c < cols; ++c)
        if (R.genes[c].n_tested > 0 && R.genes[c].best_snp >= 0 && std::isfinite(R.genes[c].best_p))
          minp[c] = std::min(1.0, R.genes[c].best_p);
    } else if (genes[active[a]].window) {
      // cis: one banded cis scan of every column with its gene's window
      std::vector<const GeneLoc*> win(cols);
      for (size_t c = 0; c < cols; ++c) win[c] = genes[active[a + c / B]].window;
      const ScanResult R = scan_columns(st, model, Y, cols, win, 2, 0.0, 0.0, lmm);
      for (size_t c = 0; c < cols; ++c)
        if (R.genes[c].n_tested > 0 && R.genes[c].best_snp >= 0 && std::isfinite(R.genes[c].best_p))
          minp[c] = std::min(1.0, R.genes[c].best_p);
    } else {
      // stage 2: FP64 tests of each gene's top-K SNPs
      std::vector<int32_t> pc;
      std::vector<int64_t> ps;
      for (size_t c = 0; c < cols; ++c)
        for (int64_t s : genes[active[a + c / B]].snps) {
          pc.push_back(static_cast<int32_t>(c));
          ps.push_back(s);
        }
      eqtl_scan_params prm{};
      prm.n = static_cast<int32_t>(n);
      prm.p = st.p;
      prm.n_genes = static_cast<int32_t>(cols);
      prm.y_rotated = lmm ? 1 : 0;
      std::vector<eqtl_pair> res(pc.size());
      st.dev->check(eqtl_test_pairs(st.dev->ctx, lmm ? EQTL_MODEL_LMM : EQTL_MODEL_LM, &prm,
                                    on_device ? nullptr : Y.data(), on_device ? nullptr : st.X.data(),
                                    pc.data(), ps.data(), static_cast<int64_t>(pc.size()), res.data(), nullptr),
                    "permutation tests");
      for (size_t i = 0; i < res.size(); ++i)
        if (std::isfinite(res[i].p) && res[i].p < minp[pc[i]]) minp[pc[i]] = res[i].p;
    }
    tr.mark("permutations: device scan of " + std::to_string(cols) + " columns");
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
    tr.mark("permutations: p_emp and beta fits of " + std::to_string(nb) + " genes");
  }
  return out;
}

}  // namespace eqtl_host
