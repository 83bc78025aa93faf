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
};

struct PermGene {
  std::string name;
  std::vector<double> y;        // the gene's phenotype (after --pheno-norm)
  double obs_min_p = 1.0;       // observed min p over the gene's tested SNPs
  bool active = false;          // gene takes part in the permutations
  std::vector<int64_t> snps;    // kept-SNP indices the permutations test
};

struct PermOut {
  bool done = false;
  double p_emp = NAN;
  BetaFit beta;
};

std::vector<PermOut> run_permutations(const Study& st, const std::string& model, const std::vector<PermGene>& genes,
                                      const std::vector<double>& delta);

}  // namespace eqtl_host
