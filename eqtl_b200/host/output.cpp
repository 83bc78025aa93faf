// The reference's three output files per (model, scope) (src/output.cpp:8-110,
// named {out}.{model}.{scope}.{pairs,top,region}.tsv at src/scan.cpp:140-145):
//   pairs / top: gene snp chrom pos ref alt af beta se stat p r2 n tss_dist scope
//   region:      gene chrom tss n_tested n_sig acat_p q_bh p_emp p_beta beta_shape1 beta_shape2
// Reals print as %.10g; tss_dist, q_bh, p_emp and p_beta print NA when absent
// or not finite.
#include "host.hpp"

namespace eqtl_host {

ScopeFiles::ScopeFiles(const std::string& prefix, bool glm) {
  pairs = std::fopen((prefix + ".pairs.tsv").c_str(), "w");
  top = std::fopen((prefix + ".top.tsv").c_str(), "w");
  region = std::fopen((prefix + ".region.tsv").c_str(), "w");
  if (!pairs || !top || !region) die("cannot open output for " + prefix);
  // write_pairs_header (src/output.cpp:8-13): GLM files add phi, glm_converged
  const char* header = glm ? "gene\tsnp\tchrom\tpos\tref\talt\taf\tbeta\tse\tstat\tp\tr2\tn\ttss_dist\tscope\tphi\t"
                             "glm_converged\n"
                           : "gene\tsnp\tchrom\tpos\tref\talt\taf\tbeta\tse\tstat\tp\tr2\tn\ttss_dist\tscope\n";
  std::fputs(header, pairs);
  std::fputs(header, top);
  std::fputs("gene\tchrom\ttss\tn_tested\tn_sig\tacat_p\tq_bh\tp_emp\tp_beta\tbeta_shape1\tbeta_shape2\n", region);
}

ScopeFiles::~ScopeFiles() {
  for (FILE* f : {pairs, top, region})
    if (f) std::fclose(f);
}

void write_pair(FILE* f, const PairRow& r, const std::string& scope) {
  std::fprintf(f, "%s\t%s\t%s\t%lld\t%s\t%s\t%.10g\t%.10g\t%.10g\t%.10g\t%.10g\t%.10g\t%d\t", r.gene.c_str(),
               r.snp.c_str(), r.chrom.c_str(), static_cast<long long>(r.pos), r.ref.c_str(), r.alt.c_str(), r.af,
               r.beta, r.se, r.t, r.p, r.r2, r.n);
  if (r.has_tss) std::fprintf(f, "%.10g", r.tss_dist);
  else std::fputs("NA", f);
  std::fprintf(f, "\t%s", scope.c_str());
  if (r.glm) std::fprintf(f, "\t%.10g\t%d", r.phi, r.converged);
  std::fputc('\n', f);
}

void write_region(FILE* f, const RegionRow& r) {
  auto na = [](double v, char* buf) {
    if (std::isfinite(v)) std::snprintf(buf, 32, "%.10g", v);
    else std::snprintf(buf, 32, "NA");
    return buf;
  };
  char q[32], pe[32], pb[32];
  std::fprintf(f, "%s\t%s\t%lld\t%d\t%d\t%.10g\t%s\t%s\t%s\t%.10g\t%.10g\n", r.gene.c_str(), r.chrom.c_str(),
               static_cast<long long>(r.tss), r.n_tested, r.n_sig, r.acat, na(r.q, q), na(r.p_emp, pe),
               na(r.p_beta, pb), r.s1, r.s2);
}

}  // namespace eqtl_host
