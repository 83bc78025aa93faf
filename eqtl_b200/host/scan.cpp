// Per-(model, scope) drivers. Both scopes run one device scan over all the
// scope's genes:
//   trans/gw   scan_lm_snp_outer / scan_lmm_snp_outer (src/scan_trans_lm.cpp:41-163,
//              src/scan_trans_lmm.cpp:82-251): genes with a GFF location
//              (trans; gw also takes genes without one), trans skipping each
//              gene's cis window; pairs sorted by (SNP, gene).
//   cis        the gene-outer cis scan (include/eqtl/scan_cis.hpp:15-185,
//              src/scan_cis.cpp:18-163): only the SNPs inside each gene's
//              window [max(start - w, 1), end + w]; pairs per gene in gene
//              order (GFF position order when -t > 1, as the reference's
//              per-thread scan writes them), SNPs in .bim order.
//   glm        NB-GLM, gene-outer in every scope (src/scan.cpp:227-300): one
//              device scan of the scope's count genes, pairs per gene in
//              gene order, SNPs in .bim order, phi and glm_converged columns.
// Per gene: n_tested, n_sig, ACAT and the best SNP (strict <, first index
// on ties) come from the device; the printed statistics of every pair are
// the device's FP64 refinement.
#include <algorithm>
#include <map>
#include <numeric>

#include "perm.hpp"

namespace eqtl_host {

Genotypes::Genotypes(const Device& d, const Plink& P, const std::vector<int32_t>& sample_col, const Options& opt)
    : dev(d), n(static_cast<int>(sample_col.size())) {
  const int64_t m = static_cast<int64_t>(P.chrom.size());
  std::vector<uint8_t> keep(m);
  std::vector<double> af(m);
  std::vector<int32_t> nm(m);
  int64_t n_kept = 0;
  const int miss_hand = opt.miss_filter ? EQTL_MISS_FILTER : EQTL_MISS_IMPUTE;
  if (P.dense)
    dev.check(eqtl_geno_load_dosage(dev.ctx, P.ds.data(), m, P.n_file, sample_col.data(), n, miss_hand,
                                    opt.max_miss, opt.maf, keep.data(), af.data(), nm.data(), &n_kept),
              "genotype decode");
  else
    dev.check(eqtl_geno_load_bed(dev.ctx, P.rows.data(), m, P.bytes_per_snp, P.n_file, sample_col.data(), n,
                                 miss_hand, opt.max_miss, opt.maf, keep.data(), af.data(), nm.data(), &n_kept),
              "genotype decode");
  for (int64_t s = 0; s < m; ++s)
    if (keep[s]) kept.push_back(s);
  info("genotypes: " + std::to_string(n_kept) + "/" + std::to_string(m) + " SNPs kept on " + std::to_string(n) +
       " samples");
}

std::unordered_map<int64_t, double> Genotypes::af(std::vector<int64_t> idx, int n_view) const {
  const int n = n_view > 0 ? n_view : this->n;
  std::sort(idx.begin(), idx.end());
  idx.erase(std::unique(idx.begin(), idx.end()), idx.end());
  std::unordered_map<int64_t, double> out;
  const size_t chunk = 4096;
  std::vector<double> d;
  for (size_t a = 0; a < idx.size(); a += chunk) {
    const size_t k = std::min(chunk, idx.size() - a);
    d.resize(k * n);
    dev.check(eqtl_geno_dosage_rows(dev.ctx, idx.data() + a, static_cast<int64_t>(k), d.data()), "dosage rows");
    for (size_t r = 0; r < k; ++r) {
      double sum = 0.0;
      for (int i = 0; i < n; ++i) sum += d[r * n + i];
      double f = (sum / static_cast<double>(n)) / 2.0;
      f = std::min(std::max(f, 0.0), 1.0);
      out.emplace(idx[a + r], f);
    }
  }
  return out;
}

namespace {

using AfMap = std::unordered_map<int64_t, double>;

struct Job {
  int gene = 0;                  // column of the phenotype matrix
  const GeneLoc* loc = nullptr;  // null in gw scope without a location
  int work = -1;                 // position in the per-thread cis driver's gene list
};

// The reference's per-thread cis driver (run_cis_parallel, src/scan_cis.cpp:
// 29-160; cis with -t > 1) gives thread t the genes [t c, (t + 1) c) of its
// (chromosome, TSS)-sorted list, c = ceil(genes / threads); each thread
// writes its pairs and tops to a temporary file, and the files are appended
// to the output in thread order with `dst << in.rdbuf()`. Appending a file
// that holds nothing sets the output stream's failbit, after which nothing
// more reaches that file. written[t] says whether thread t's rows appear.
std::vector<char> threads_written(const std::vector<char>& has_rows) {
  std::vector<char> written(has_rows.size(), 0);
  bool ok = true;
  for (size_t t = 0; t < has_rows.size(); ++t) {
    written[t] = ok && has_rows[t];
    if (!has_rows[t]) ok = false;
  }
  return written;
}

// Complete-case sample set of one gene (build_gene_ready, src/scan_common.cpp:
// 11-70): finite phenotype and covariates; fewer than 3 samples or an all-zero
// phenotype leave the gene out. keep (if given) receives the kept analysis
// samples; without it, a gene that does not keep every analysis sample stops
// the run (the scopes and models that take only the shared-keep case).
bool gene_ready(const Study& st, const std::vector<double>& y, bool checks,
                std::vector<int32_t>* keep = nullptr) {
  const size_t n = st.samples.size();
  size_t kept = 0;
  double mx = 0.0;
  if (keep) keep->clear();
  for (size_t i = 0; i < n; ++i) {
    bool ok = std::isfinite(y[i]);
    for (int j = 0; j < st.p && ok; ++j) ok = std::isfinite(st.X[static_cast<size_t>(j) * n + i]);
    if (ok) {
      ++kept;
      mx = std::max(mx, std::fabs(y[i]));
      if (keep) keep->push_back(static_cast<int32_t>(i));
    }
  }
  if (kept != n && !keep)
    die("phenotype or covariate values missing for some samples: the device scans take per-gene sample sets in "
        "the cis, trans and gw scopes of the LM and LMM without permutations; here every gene must keep every "
        "analysis sample");
  if (!checks) return true;
  return kept >= 3 && !(mx < 1e-15);
}

// The gene's phenotype after --pheno-norm (apply_pheno_norm,
// src/scan_common.cpp): the transformed copy when int is on.
std::vector<double> gene_y(const Study& st, int g) {
  const size_t n = st.samples.size();
  const std::vector<double>& src = st.opt->pheno_int ? st.Y_int : st.Y;
  return std::vector<double>(src.begin() + static_cast<size_t>(g) * n, src.begin() + static_cast<size_t>(g + 1) * n);
}

}  // namespace

ScanResult scan_columns(const Study& st, const std::string& model, const std::vector<double>& Y, size_t cols,
                        const std::vector<const GeneLoc*>& windows, int mode, double pthr, double perm_thr,
                        bool rotated, const std::vector<double>* X_view) {
  const Options& opt = *st.opt;
  const std::vector<double>& Xs = X_view ? *X_view : st.X;
  const size_t n = Xs.size() / static_cast<size_t>(st.p), J = cols;
  ScanResult R;
  R.n = static_cast<int>(n);
  // windows and the kept SNPs' positions, chromosomes by normalised name
  std::unordered_map<std::string, int32_t> cid;
  auto chrom_id = [&](const std::string& c) {
    return cid.emplace(chrom_key(c), static_cast<int32_t>(cid.size())).first->second;
  };
  const auto& kept = st.geno->kept;
  std::vector<int32_t> gchr(J, -1), schr;
  std::vector<int64_t> glo(J, 0), ghi(J, -1), spos;
  if (mode != 0) {
    schr.resize(kept.size());
    spos.resize(kept.size());
    for (size_t k = 0; k < kept.size(); ++k) {
      schr[k] = chrom_id(st.plink->chrom[kept[k]]);
      spos[k] = st.plink->pos[kept[k]];
    }
    for (size_t j = 0; j < J; ++j)
      if (windows[j]) {
        gchr[j] = chrom_id(windows[j]->chrom);
        glo[j] = std::max<int64_t>(windows[j]->start - opt.window, 1);
        ghi[j] = windows[j]->end + opt.window;
      }
  }
  eqtl_scan_params prm{};
  prm.n = static_cast<int32_t>(n);
  prm.n_genes = static_cast<int32_t>(J);
  prm.p = st.p;
  prm.exclude_cis = mode;
  prm.pthr = pthr;
  prm.perm_thr = perm_thr;
  prm.y_rotated = rotated ? 1 : 0;
  if (mode != 0) {
    prm.gene_chrom = gchr.data();
    prm.gene_lo = glo.data();
    prm.gene_hi = ghi.data();
    prm.snp_chrom = schr.data();
    prm.snp_pos = spos.data();
  }
  R.genes.resize(J);
  R.delta.assign(J, 0.0);
  if (model == "glm") {
    R.phi.assign(J, 0.0);
    R.conv.assign(J, 0);
  }
  int64_t cap = 1 << 18, ccap = perm_thr > 0 ? (1 << 18) : 1;
  // no host columns: scan the resident ones (eqtl_pheno_permute)
  const double* Yp = Y.empty() ? nullptr : Y.data();
  const double* Xp = Y.empty() ? nullptr : Xs.data();
  for (int attempt = 0; attempt < 3; ++attempt) {
    R.pairs.resize(static_cast<size_t>(cap));
    R.cands.resize(static_cast<size_t>(ccap));
    int64_t np = 0, nc = 0;
    const int rc = model == "lm"
                       ? eqtl_scan_trans_lm(st.dev->ctx, &prm, Yp, Xp, R.genes.data(), R.pairs.data(),
                                            cap, &np, R.cands.data(), ccap, &nc)
                   : model == "glm"
                       ? eqtl_scan_glm(st.dev->ctx, &prm, Yp, Xp, R.phi.data(), R.conv.data(),
                                       R.genes.data(), R.pairs.data(), cap, &np, R.cands.data(), ccap, &nc)
                       : eqtl_scan_trans_lmm(st.dev->ctx, &prm, Yp, Xp, R.delta.data(),
                                             R.genes.data(), R.pairs.data(), cap, &np, R.cands.data(), ccap, &nc);
    if (rc == EQTL_E_OVERFLOW) {
      cap = std::max(cap, np);
      ccap = std::max(ccap, nc);
      continue;
    }
    st.dev->check(rc, model + " scan");
    R.pairs.resize(static_cast<size_t>(np));
    R.cands.resize(static_cast<size_t>(nc));
    if (std::getenv("EQTL_TRACE")) {
      std::string line = "[eqtl trace] device stages of " + std::to_string(J) + " columns (ms):";
      const char* names[] = {"rotate", "prep", "scan", "refine"};
      const int stages[] = {EQTL_STAGE_ROTATE, EQTL_STAGE_PREP, EQTL_STAGE_SCAN, EQTL_STAGE_REFINE};
      for (int k = 0; k < 4; ++k) {
        double ms = 0;
        if (eqtl_stage_ms(st.dev->ctx, stages[k], &ms) == EQTL_OK) line += std::string(" ") + names[k] + " " + std::to_string(ms);
      }
      std::fprintf(stderr, "%s\n", line.c_str());
    }
    return R;
  }
  die("scan output did not fit after resizing");
}

namespace {

// One device scan over `jobs`; mode 0 gw, 1 trans (exclude windows), 2 cis.
ScanResult device_scan(const Study& st, const std::string& model, const std::vector<Job>& jobs, int mode,
                       double pthr, double perm_thr) {
  const size_t n = st.samples.size(), J = jobs.size();
  std::vector<double> Y(J * n);
  std::vector<const GeneLoc*> windows(J);
  for (size_t j = 0; j < J; ++j) {
    const std::vector<double> y = gene_y(st, jobs[j].gene);
    std::copy(y.begin(), y.end(), Y.begin() + j * n);
    windows[j] = jobs[j].loc;
  }
  return scan_columns(st, model, Y, J, windows, mode, pthr, perm_thr, false);
}

PairRow make_row(const Study& st, const std::string& gene, const GeneLoc* loc, int64_t kept_idx, double af,
                 double beta, double se, double t, double p, double r2, int n) {
  const int64_t s = st.geno->kept[kept_idx];
  const Plink& P = *st.plink;
  PairRow r;
  r.gene = gene;
  r.snp = !P.id[s].empty() ? P.id[s] : P.chrom[s] + ":" + std::to_string(P.pos[s]) + ":" + P.a2[s] + ":" + P.a1[s];
  r.chrom = P.chrom[s];
  r.pos = P.pos[s];
  r.ref = P.a2[s];
  r.alt = P.a1[s];
  r.af = af;
  r.beta = beta;
  r.se = se;
  r.t = t;
  r.p = p;
  r.r2 = r2;
  r.n = n;
  if (loc) {
    r.has_tss = true;
    r.tss_dist = static_cast<double>(P.pos[s] - loc->tss);
  }
  return r;
}

// Writes pairs (in `order`), tops and region rows of one device scan.
void emit(const Study& st, const std::vector<Job>& jobs, ScanResult& R, const std::string& scope, double pthr,
          const std::vector<size_t>& pair_order, ScopeFiles& out, std::vector<RegionRow>& regions,
          const std::vector<PermOut>* perms, size_t n_works_par = 0, const std::vector<int>* n_job = nullptr,
          const std::vector<const AfMap*>* af_job = nullptr) {
  AfMap af;
  if (!af_job) {
    std::vector<int64_t> need;
    for (const auto& q : R.pairs) need.push_back(q.snp);
    for (const auto& g : R.genes)
      if (g.best_snp >= 0 && g.best_p <= pthr) need.push_back(g.best_snp);
    af = st.geno->af(need);
  }
  // allele frequency and sample count of gene j's rows (its own sample set
  // when the genes keep different samples)
  auto af_of = [&](size_t j, int64_t snp) { return (af_job ? *(*af_job)[j] : af).at(snp); };
  auto n_of = [&](size_t j) { return n_job ? (*n_job)[j] : R.n; };
  std::vector<int> n_sig(jobs.size(), 0);
  const bool glm = !R.phi.empty();
  auto with_glm = [&](PairRow r, size_t j) {
    if (glm) {
      r.glm = true;
      r.phi = R.phi[j];
      r.converged = R.conv[j] ? 1 : 0;
    }
    return r;
  };
  // per-thread driver: which thread's pairs and tops reach the files
  const size_t T = n_works_par ? static_cast<size_t>(std::max(1, st.opt->threads)) : 0;
  const size_t chunk = T ? (n_works_par + T - 1) / T : 1;
  auto thread_of = [&](size_t j) { return static_cast<size_t>(jobs[j].work) / chunk; };
  std::vector<char> pairs_ok, tops_ok;
  if (T) {
    std::vector<char> hp(T, 0), ht(T, 0);
    for (const auto& q : R.pairs) hp[thread_of(q.gene)] = 1;
    for (size_t j = 0; j < jobs.size(); ++j)
      if (R.genes[j].best_snp >= 0 && R.genes[j].best_p <= pthr && R.genes[j].best_p <= 1.0) ht[thread_of(j)] = 1;
    pairs_ok = threads_written(hp);
    tops_ok = threads_written(ht);
  }
  for (size_t k : pair_order) {
    const eqtl_pair& q = R.pairs[k];
    const Job& jb = jobs[q.gene];
    ++n_sig[q.gene];
    if (T && !pairs_ok[thread_of(q.gene)]) continue;
    write_pair(out.pairs,
               with_glm(make_row(st, st.genes[jb.gene], jb.loc, q.snp, af_of(q.gene, q.snp), q.beta, q.se, q.t, q.p,
                                 q.r2, n_of(q.gene)),
                        q.gene),
               scope);
  }
  for (size_t j = 0; j < jobs.size(); ++j) {
    const eqtl_gene_result& g = R.genes[j];
    const Job& jb = jobs[j];
    RegionRow rr;
    rr.gene = st.genes[jb.gene];
    if (jb.loc) {
      rr.chrom = jb.loc->chrom;
      rr.tss = jb.loc->tss;
    }
    rr.n_tested = g.n_tested;
    rr.n_sig = n_sig[j];
    rr.acat = acat_p(g.acat_tan_sum, g.acat_used);
    if (perms && (*perms)[j].done) {
      rr.p_emp = (*perms)[j].p_emp;
      rr.p_beta = (*perms)[j].beta.p;
      rr.s1 = (*perms)[j].beta.s1;
      rr.s2 = (*perms)[j].beta.s2;
    }
    regions.push_back(rr);
    if (g.best_snp >= 0 && g.best_p <= pthr && g.best_p <= 1.0 && !(T && !tops_ok[thread_of(j)]))
      write_pair(out.top,
                 with_glm(make_row(st, rr.gene, jb.loc, g.best_snp, af_of(j, g.best_snp), g.best_beta, g.best_se,
                                   g.best_t, g.best_p, g.best_r2, n_of(j)),
                          j),
                 scope);
  }
}

// Trans/gw scans of genes whose sample sets differ (the reference's per-job
// paths for mixed keep sets, src/scan_trans_lm.cpp:121-151 and
// src/scan_trans_lmm.cpp:192-228): the genes are grouped by keep set, and
// each group is scanned over its own sample view (eqtl_geno_subset: the SNPs
// imputed and filtered over every analysis sample, then subset, as the
// reference's for_each_snp and g_buf do); the LMM takes the eigenbasis of the
// GRM sliced to the group's samples, as build_gene_ready slices it. The
// results come back in job order, pairs by (SNP, gene).
struct KeepScan {
  ScanResult R;
  std::vector<int> n_job;
  std::vector<AfMap> af_grp;
  std::vector<const AfMap*> af_job;
};

KeepScan scan_by_keep(const Study& st, const std::string& model, const std::vector<Job>& jobs,
                      const std::vector<std::vector<int32_t>>& keeps, int mode, double pthr) {
  const Device& dev = *st.dev;
  const size_t n = st.samples.size(), J = jobs.size();
  const size_t p = static_cast<size_t>(st.p);
  std::vector<std::vector<size_t>> groups;
  std::map<std::vector<int32_t>, size_t> gid;
  for (size_t j = 0; j < J; ++j) {
    auto it = gid.find(keeps[j]);
    if (it == gid.end()) {
      it = gid.emplace(keeps[j], groups.size()).first;
      groups.emplace_back();
    }
    groups[it->second].push_back(j);
  }
  const bool lmm = model == "lmm";
  if (lmm && (st.K_full.size() != n * n || st.basis_Q.size() != n * n))
    die("internal: per-gene sample sets of the LMM need the GRM and the eigenbasis on the host");
  KeepScan K;
  K.R.n = static_cast<int>(n);
  K.R.genes.resize(J);
  K.R.delta.assign(J, 0.0);
  K.n_job.assign(J, static_cast<int>(n));
  K.af_grp.resize(groups.size());
  K.af_job.assign(J, nullptr);
  Trace tr;
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    const std::vector<size_t>& grp = groups[gi];
    const std::vector<int32_t>& keep = keeps[grp[0]];
    const size_t ns = keep.size();
    const bool full = ns == n;
    dev.check(eqtl_geno_subset(dev.ctx, full ? nullptr : keep.data(), full ? 0 : static_cast<int32_t>(ns)),
              "sample view");
    if (lmm) {
      if (full) {
        dev.check(eqtl_lmm_set_basis(dev.ctx, st.basis_Q.data(), st.basis_lambda.data(), static_cast<int32_t>(n)),
                  "LMM basis");
      } else {
        std::vector<double> Ks(ns * ns);
        for (size_t b = 0; b < ns; ++b)
          for (size_t a = 0; a < ns; ++a) Ks[b * ns + a] = st.K_full[static_cast<size_t>(keep[b]) * n + keep[a]];
        int64_t zeroed = 0;
        dev.check(eqtl_lmm_basis_fast(dev.ctx, Ks.data(), static_cast<int32_t>(ns), st.opt->fast ? 1e-4 : 0.0, nullptr,
                                      nullptr, &zeroed),
                  "LMM basis of a gene sample set");
      }
    }
    const size_t Jg = grp.size();
    std::vector<double> Yg(Jg * ns), Xg(ns * p);
    std::vector<const GeneLoc*> win(Jg);
    for (size_t a = 0; a < p; ++a)
      for (size_t i = 0; i < ns; ++i) Xg[a * ns + i] = st.X[a * n + keep[i]];
    for (size_t k = 0; k < Jg; ++k) {
      const std::vector<double> y = gene_y(st, jobs[grp[k]].gene);
      for (size_t i = 0; i < ns; ++i) Yg[k * ns + i] = y[keep[i]];
      win[k] = jobs[grp[k]].loc;
    }
    ScanResult R = scan_columns(st, model, Yg, Jg, win, mode, pthr, 0.0, false, &Xg);
    // allele frequencies over the view, while it is active
    std::vector<int64_t> need;
    for (const auto& q : R.pairs) need.push_back(q.snp);
    for (const auto& g : R.genes)
      if (g.best_snp >= 0 && g.best_p <= pthr) need.push_back(g.best_snp);
    K.af_grp[gi] = st.geno->af(need, static_cast<int>(ns));
    for (size_t k = 0; k < Jg; ++k) {
      const size_t j = grp[k];
      K.R.genes[j] = R.genes[k];
      if (!R.delta.empty()) K.R.delta[j] = R.delta[k];
      K.n_job[j] = static_cast<int>(ns);
      K.af_job[j] = &K.af_grp[gi];
    }
    for (eqtl_pair q : R.pairs) {
      q.gene = static_cast<int32_t>(grp[q.gene]);
      K.R.pairs.push_back(q);
    }
    tr.mark("sample set " + std::to_string(gi + 1) + "/" + std::to_string(groups.size()) + ": " +
            std::to_string(Jg) + " genes on " + std::to_string(ns) + " samples");
  }
  // every analysis sample again, and the shared basis, for the scans after
  dev.check(eqtl_geno_subset(dev.ctx, nullptr, 0), "sample view");
  if (lmm)
    dev.check(eqtl_lmm_set_basis(dev.ctx, st.basis_Q.data(), st.basis_lambda.data(), static_cast<int32_t>(n)),
              "LMM basis");
  std::stable_sort(K.R.pairs.begin(), K.R.pairs.end(), [](const eqtl_pair& a, const eqtl_pair& b) {
    return a.snp != b.snp ? a.snp < b.snp : a.gene < b.gene;
  });
  return K;
}

}  // namespace

void run_trans(const Study& st, const std::string& model, const std::string& scope, ScopeFiles& out,
               std::vector<RegionRow>& regions) {
  const Options& opt = *st.opt;
  const bool have_gff = !opt.gff.empty();
  std::vector<Job> jobs;
  std::vector<std::vector<int32_t>> keeps;
  bool mixed = false;
  for (size_t g = 0; g < st.genes.size(); ++g) {
    Job jb;
    jb.gene = static_cast<int>(g);
    if (have_gff) {
      auto it = st.annot.find(st.genes[g]);
      if (it != st.annot.end()) jb.loc = &it->second;
      else if (scope != "gw") continue;
    }
    if (scope == "trans" && !jb.loc) continue;
    std::vector<int32_t> keep;
    if (!gene_ready(st, gene_y(st, jb.gene), true, &keep)) continue;
    mixed = mixed || keep.size() != st.samples.size();
    jobs.push_back(jb);
    keeps.push_back(std::move(keep));
  }
  info(std::string(scope) + " " + model + ": " + std::to_string(jobs.size()) + " genes");
  if (jobs.empty()) return;
  const double pthr = opt.pval_trans;
  const double perm_thr = opt.perm > 0 ? opt.perm_trans_thr : 0.0;
  Trace tr;
  if (mixed) {
    if (opt.perm > 0)
      die("phenotype or covariate values missing for some samples: gene-level permutations take the case where "
          "every gene keeps every analysis sample");
    KeepScan K = scan_by_keep(st, model, jobs, keeps, scope == "trans" ? 1 : 0, pthr);
    tr.mark(scope + " " + model + ": device scans of the gene sample sets");
    std::vector<size_t> order(K.R.pairs.size());
    std::iota(order.begin(), order.end(), 0);
    emit(st, jobs, K.R, scope, pthr, order, out, regions, nullptr, 0, &K.n_job, &K.af_job);
    return;
  }
  ScanResult R = device_scan(st, model, jobs, scope == "trans" ? 1 : 0, pthr, perm_thr);
  tr.mark(scope + " " + model + ": device scan");
  std::vector<PermOut> perms;
  if (opt.perm > 0) {
    std::vector<PermGene> pg(jobs.size());
    for (size_t j = 0; j < jobs.size(); ++j) {
      pg[j].name = st.genes[jobs[j].gene];
      pg[j].y = gene_y(st, jobs[j].gene);
      pg[j].obs_min_p = R.genes[j].best_p;
      pg[j].active = R.genes[j].n_tested > 0 && R.genes[j].best_snp >= 0 && R.genes[j].best_p < opt.perm_trans_thr;
    }
    // stage-2 SNPs: each gene's top-K candidates by nominal p (p < perm_trans_thr)
    for (const auto& q : R.cands)
      if (pg[q.gene].active && static_cast<int>(pg[q.gene].snps.size()) < opt.perm_trans_top &&
          std::isfinite(q.p))
        pg[q.gene].snps.push_back(q.snp);
    perms = run_permutations(st, model, pg, R.delta);
    tr.mark(scope + " " + model + ": stage-2 permutations");
  }
  std::vector<size_t> order(R.pairs.size());
  std::iota(order.begin(), order.end(), 0);  // already (SNP, gene)
  emit(st, jobs, R, scope, pthr, order, out, regions, opt.perm > 0 ? &perms : nullptr);
}

void run_cis(const Study& st, const std::string& model, ScopeFiles& out, std::vector<RegionRow>& regions) {
  const Options& opt = *st.opt;
  std::vector<Job> works, jobs;
  for (size_t g = 0; g < st.genes.size(); ++g) {
    auto it = st.annot.find(st.genes[g]);
    if (it == st.annot.end()) continue;
    Job jb;
    jb.gene = static_cast<int>(g);
    jb.loc = &it->second;
    works.push_back(jb);
  }
  if (opt.threads > 1)
    std::stable_sort(works.begin(), works.end(), [](const Job& a, const Job& b) {
      return a.loc->chrom != b.loc->chrom ? a.loc->chrom < b.loc->chrom : a.loc->tss < b.loc->tss;
    });
  std::vector<std::vector<int32_t>> keeps;
  bool mixed = false;
  for (size_t w = 0; w < works.size(); ++w) {
    Job jb = works[w];
    jb.work = static_cast<int>(w);
    // the LM takes every gene through the complete-case checks; the LMM with
    // the shared basis takes a gene that keeps every sample as it is, and one
    // with missing values through the checks on its own sample set
    // (src/scan_cis.cpp:111-120, src/scan.cpp:259-269)
    std::vector<int32_t> keep;
    const bool ok = gene_ready(st, gene_y(st, jb.gene), true, &keep);
    const bool full = keep.size() == st.samples.size();
    if (!ok && !(model == "lmm" && full)) continue;
    mixed = mixed || !full;
    jobs.push_back(jb);
    keeps.push_back(std::move(keep));
  }
  info("cis " + model + ": " + std::to_string(jobs.size()) + " genes");
  if (jobs.empty()) return;
  const double pthr = opt.pval_cis;
  if (mixed) {
    // per-gene sample sets: the genes of each set scan on its sample view
    // (scan_by_keep), results in job order; pairs by gene, then SNP
    if (opt.perm > 0)
      die("phenotype or covariate values missing for some samples: gene-level permutations take the case where "
          "every gene keeps every analysis sample");
    Trace tr;
    KeepScan K = scan_by_keep(st, model, jobs, keeps, 2, pthr);
    tr.mark("cis " + model + ": device scans of the gene sample sets");
    std::vector<size_t> order(K.R.pairs.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
      const eqtl_pair &x = K.R.pairs[a], &y = K.R.pairs[b];
      return x.gene != y.gene ? x.gene < y.gene : x.snp < y.snp;
    });
    emit(st, jobs, K.R, "cis", pthr, order, out, regions, nullptr, opt.threads > 1 ? works.size() : 0, &K.n_job,
         &K.af_job);
    return;
  }
  // the device scan takes the genes in window order (a banded tile list);
  // results come back to the output order
  std::vector<size_t> dev_order(jobs.size());
  std::iota(dev_order.begin(), dev_order.end(), 0);
  std::vector<std::string> keys(jobs.size());
  for (size_t j = 0; j < jobs.size(); ++j) keys[j] = chrom_key(jobs[j].loc->chrom);
  std::stable_sort(dev_order.begin(), dev_order.end(), [&](size_t a, size_t b) {
    return keys[a] != keys[b] ? keys[a] < keys[b] : jobs[a].loc->start < jobs[b].loc->start;
  });
  std::vector<Job> jobs_dev(jobs.size());
  for (size_t j = 0; j < jobs.size(); ++j) jobs_dev[j] = jobs[dev_order[j]];
  Trace tr;
  ScanResult R = device_scan(st, model, jobs_dev, 2, pthr, 0.0);
  tr.mark("cis " + model + ": device scan");
  {
    std::vector<eqtl_gene_result> genes(R.genes.size());
    std::vector<double> delta(R.delta.size());
    for (size_t j = 0; j < dev_order.size(); ++j) {
      genes[dev_order[j]] = R.genes[j];
      delta[dev_order[j]] = R.delta[j];
    }
    R.genes.swap(genes);
    R.delta.swap(delta);
    for (auto& q : R.pairs) q.gene = static_cast<int32_t>(dev_order[q.gene]);
    for (auto& q : R.cands) q.gene = static_cast<int32_t>(dev_order[q.gene]);
  }
  std::vector<PermOut> perms;
  if (opt.perm > 0) {
    std::vector<PermGene> pg(jobs.size());
    for (size_t j = 0; j < jobs.size(); ++j) {
      pg[j].name = st.genes[jobs[j].gene];
      pg[j].y = gene_y(st, jobs[j].gene);
      pg[j].obs_min_p = R.genes[j].best_p;
      pg[j].active = R.genes[j].n_tested > 0;
    }
    for (size_t j = 0; j < jobs.size(); ++j) pg[j].window = jobs[j].loc;  // permutations scan the window
    perms = run_permutations(st, model, pg, R.delta);
    tr.mark("cis " + model + ": permutations");
  }
  std::vector<size_t> order(R.pairs.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    const eqtl_pair &x = R.pairs[a], &y = R.pairs[b];
    return x.gene != y.gene ? x.gene < y.gene : x.snp < y.snp;
  });
  emit(st, jobs, R, "cis", pthr, order, out, regions, opt.perm > 0 ? &perms : nullptr,
       opt.threads > 1 ? works.size() : 0);
}

// Whether every finite value is a non-negative integer (within 1e-8) and one
// is present (looks_like_counts, src/model_lm.cpp:8-17).
static bool looks_like_counts(const std::vector<double>& y) {
  int seen = 0;
  for (double v : y) {
    if (!std::isfinite(v)) continue;
    ++seen;
    if (v < 0 || std::fabs(v - std::floor(v)) > 1e-8) return false;
  }
  return seen > 0;
}

void run_glm(const Study& st, const std::string& scope, ScopeFiles& out, std::vector<RegionRow>& regions) {
  const Options& opt = *st.opt;
  const bool have_gff = !opt.gff.empty();
  // cis with -t > 1 runs the per-thread driver: the raw counts are checked
  // before --pheno-norm, and the genes go in (chromosome, TSS) order
  const bool par_cis = scope == "cis" && opt.threads > 1 && have_gff;
  const size_t n = st.samples.size();
  std::vector<Job> works, jobs;
  for (size_t g = 0; g < st.genes.size(); ++g) {
    Job jb;
    jb.gene = static_cast<int>(g);
    if (have_gff) {
      auto it = st.annot.find(st.genes[g]);
      if (it != st.annot.end()) jb.loc = &it->second;
      else if (scope != "gw") continue;
    }
    if (scope != "gw" && !jb.loc) continue;
    const std::vector<double> y = gene_y(st, jb.gene);
    const std::vector<double> raw(st.Y.begin() + g * n, st.Y.begin() + (g + 1) * n);
    if (!looks_like_counts(par_cis ? raw : y)) {
      warn("skip non-count gene for glm: " + st.genes[g]);
      continue;
    }
    works.push_back(jb);
  }
  if (par_cis)
    std::stable_sort(works.begin(), works.end(), [](const Job& a, const Job& b) {
      return a.loc->chrom != b.loc->chrom ? a.loc->chrom < b.loc->chrom : a.loc->tss < b.loc->tss;
    });
  for (size_t w = 0; w < works.size(); ++w) {
    Job jb = works[w];
    jb.work = static_cast<int>(w);
    if (!gene_ready(st, gene_y(st, jb.gene), true)) continue;
    jobs.push_back(jb);
  }
  info(scope + " glm: " + std::to_string(jobs.size()) + " genes");
  if (jobs.empty()) return;
  const double pthr = scope == "cis" ? opt.pval_cis : opt.pval_trans;
  const int mode = scope == "cis" ? 2 : scope == "trans" ? 1 : 0;
  // cis: the device takes the genes in window order (a banded tile list)
  std::vector<size_t> dev_order(jobs.size());
  std::iota(dev_order.begin(), dev_order.end(), 0);
  if (mode == 2) {
    std::vector<std::string> keys(jobs.size());
    for (size_t j = 0; j < jobs.size(); ++j) keys[j] = chrom_key(jobs[j].loc->chrom);
    std::stable_sort(dev_order.begin(), dev_order.end(), [&](size_t a, size_t b) {
      return keys[a] != keys[b] ? keys[a] < keys[b] : jobs[a].loc->start < jobs[b].loc->start;
    });
  }
  std::vector<Job> jobs_dev(jobs.size());
  for (size_t j = 0; j < jobs.size(); ++j) jobs_dev[j] = jobs[dev_order[j]];
  Trace tr;
  ScanResult R = device_scan(st, "glm", jobs_dev, mode, pthr, 0.0);
  tr.mark(scope + " glm: device scan");
  {
    std::vector<eqtl_gene_result> genes(R.genes.size());
    std::vector<double> phi(R.phi.size());
    std::vector<uint8_t> conv(R.conv.size());
    for (size_t j = 0; j < dev_order.size(); ++j) {
      genes[dev_order[j]] = R.genes[j];
      phi[dev_order[j]] = R.phi[j];
      conv[dev_order[j]] = R.conv[j];
    }
    R.genes.swap(genes);
    R.phi.swap(phi);
    R.conv.swap(conv);
    for (auto& q : R.pairs) q.gene = static_cast<int32_t>(dev_order[q.gene]);
  }
  std::vector<PermOut> perms;
  if (opt.perm > 0) {
    // the observed null means, back in output order
    std::vector<double> mu_dev(jobs.size() * n), mu(jobs.size() * n);
    st.dev->check(eqtl_glm_mu(st.dev->ctx, mu_dev.data()), "GLM null means");
    for (size_t j = 0; j < dev_order.size(); ++j)
      std::copy(mu_dev.begin() + j * n, mu_dev.begin() + (j + 1) * n, mu.begin() + dev_order[j] * n);
    std::vector<PermGene> pg(jobs.size());
    for (size_t j = 0; j < jobs.size(); ++j) {
      // the reference caches every tested SNP's dosages for its permutations
      // and stops past 25,000,000 values (include/eqtl/scan_cis.hpp:58-61)
      if (R.genes[j].n_tested > 1 && static_cast<int64_t>(R.genes[j].n_tested - 1) * static_cast<int64_t>(n) >
                                         25'000'000)
        die("cis perm: too many SNPs in cis window for gene " + st.genes[jobs[j].gene] + " — reduce --window");
      pg[j].name = st.genes[jobs[j].gene];
      pg[j].obs_min_p = R.genes[j].best_p;
      pg[j].active = R.genes[j].n_tested > 0;
      pg[j].mu.assign(mu.begin() + j * n, mu.begin() + (j + 1) * n);
      pg[j].phi = R.phi[j];
      pg[j].scan_mode = mode;
      pg[j].window = mode == 0 ? nullptr : jobs[j].loc;
    }
    perms = run_permutations(st, "glm", pg, {});
    tr.mark(scope + " glm: permutations");
  }
  std::vector<size_t> order(R.pairs.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    const eqtl_pair &x = R.pairs[a], &y = R.pairs[b];
    return x.gene != y.gene ? x.gene < y.gene : x.snp < y.snp;
  });
  emit(st, jobs, R, scope, pthr, order, out, regions, opt.perm > 0 ? &perms : nullptr,
       par_cis ? works.size() : 0);
}

}  // namespace eqtl_host
