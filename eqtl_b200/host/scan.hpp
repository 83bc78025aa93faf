// Scan drivers of the host program: one device context, the genotypes
// resident on it, and the per-(model, scope) drivers that call the C ABI and
// turn its per-gene results and refined pairs into output rows.
#pragma once
#include "host.hpp"

namespace eqtl_host {

struct Device {
  eqtl_ctx* ctx = nullptr;
  Device();
  ~Device();
  Device(const Device&) = delete;
  Device& operator=(const Device&) = delete;
  void check(int rc, const std::string& what) const;
};

// The .bed decoded on the device for the analysis samples
// (eqtl_geno_load_bed); kept[k] = .bim row of kept SNP k.
struct Genotypes {
  const Device& dev;
  int n = 0;
  std::vector<int64_t> kept;
  Genotypes(const Device& d, const Plink& P, const std::vector<int32_t>& sample_col, const Options& opt);
  // Reference allele frequency of each listed kept SNP over the analysis
  // samples: (sum of imputed dosages in sample order / n) / 2, clamped to
  // [0, 1] (subset_maf_or_nan, src/scan_common.cpp:133-151).
  // n_view: the samples of the current device view (eqtl_geno_subset); 0 =
  // every analysis sample.
  std::unordered_map<int64_t, double> af(std::vector<int64_t> kept_idx, int n_view = 0) const;
};

struct Study {
  const Options* opt = nullptr;
  const Plink* plink = nullptr;
  std::vector<std::string> samples, genes;
  std::vector<double> Y;  // gene-major [G][n]
  std::vector<double> Y_int;  // --pheno-norm int: Y with every gene transformed (eqtl_pheno_int)
  std::vector<double> X;  // column-major [n, p]
  int p = 1;
  std::unordered_map<std::string, GeneLoc> annot;
  const Device* dev = nullptr;
  const Genotypes* geno = nullptr;
  // LMM permutations: the device eigenbasis on the host (Q column-major,
  // column j = eigenvector j; lambda clipped at 0)
  std::vector<double> basis_Q, basis_lambda;
  // genes whose phenotype or covariates miss some samples (per-gene keep
  // sets): the full GRM on the host, sliced to each keep set for its basis
  std::vector<double> K_full;
};

void run_trans(const Study& st, const std::string& model, const std::string& scope, ScopeFiles& out,
               std::vector<RegionRow>& regions);
void run_cis(const Study& st, const std::string& model, ScopeFiles& out, std::vector<RegionRow>& regions);
// NB-GLM, gene-outer in every scope (src/scan.cpp:227-300; cis with -t > 1
// src/scan_cis.cpp:18-115): genes in phenotype order (cis with -t > 1: by
// chromosome and TSS), pairs per gene in SNP order.
void run_glm(const Study& st, const std::string& scope, ScopeFiles& out, std::vector<RegionRow>& regions);

}  // namespace eqtl_host
