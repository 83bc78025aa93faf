// Gene-level permutations (include/eqtl/scan_cis.hpp:68-176 for cis,
// src/scan_perm.cpp:11-142 for the trans/gw stage 2).
#pragma once
#include "scan.hpp"

namespace eqtl_host {

// Per-gene outputs of one device scan.
struct ScanResult {
  int n = 0;
  std::vector<eqtl_gene_result> genes;
  std::vector<eqtl_pair> pairs, cands;
  std::vector<double> delta;  // LMM: REML delta per gene
  std::vector<double> phi;    // GLM: NB dispersion per gene
  std::vector<uint8_t> conv;  // GLM: null fit converged
};

struct PermGene {
  std::string name;
  std::vector<double> y;            // the gene's phenotype (after --pheno-norm)
  double obs_min_p = 1.0;           // observed min p over the gene's tested SNPs
  bool active = false;              // gene takes part in the permutations
  const GeneLoc* window = nullptr;  // cis: permutations test the gene's window
  std::vector<int64_t> snps;        // trans/gw stage 2: the top-K kept SNPs
  // NB-GLM: permutations resample counts from the observed null fit and
  // test every SNP of the scope (scan_mode 0 gw, 1 trans, 2 cis; window =
  // the gene's location for 1 and 2)
  std::vector<double> mu;
  double phi = 0.0;
  int scan_mode = -1;
};

struct PermOut {
  bool done = false;
  double p_emp = NAN;
  BetaFit beta;
};

// One device scan of explicit phenotype columns Y [cols][n] (Y empty: the
// columns resident on the device, drawn by eqtl_pheno_permute): scope mode 0
// gw, 1 trans, 2 cis with per-column windows (null = no location); LMM
// columns may already be rotated into the eigenbasis. X_view: the covariates
// of the current sample view (eqtl_geno_subset), column-major [n_view, p];
// null = every analysis sample.
ScanResult scan_columns(const Study& st, const std::string& model, const std::vector<double>& Y, size_t cols,
                        const std::vector<const GeneLoc*>& windows, int mode, double pthr, double perm_thr,
                        bool rotated, const std::vector<double>* X_view = nullptr);

std::vector<PermOut> run_permutations(const Study& st, const std::string& model, const std::vector<PermGene>& genes,
                                      const std::vector<double>& delta);

}  // namespace eqtl_host
