// eqtl: the reference program's command line (src/main.cpp, src/scan.cpp)
// for PLINK or VCF (GT or DS) input and the LM / LMM / NB-GLM models, with every scan run
// on the B200 through libeqtl_cuda. The orchestration follows run_eqtl_geno
// (src/scan.cpp:50-312): analysis samples = phenotype samples present in the
// .fam, in phenotype order; one GRM (computed or -k) shared by the LMM
// scopes; per (model, scope) the pairs / top / region files; BH over the
// scope's genes.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <memory>
#include <numeric>
#include <unordered_set>

#include "host.hpp"
#include "scan.hpp"

namespace eqtl_host {

Device::Device() {
  if (eqtl_open(0, &ctx) != EQTL_OK || !ctx) die("no usable B200 (eqtl_open failed)");
}
Device::~Device() {
  if (ctx) eqtl_close(ctx);
}
void Device::check(int rc, const std::string& what) const {
  if (rc != EQTL_OK) die(what + ": " + eqtl_last_error(ctx));
}

namespace {

std::vector<int32_t> sample_columns(const Plink& P, const std::vector<std::string>& samples) {
  std::unordered_map<std::string, int32_t> at;
  for (size_t i = 0; i < P.fam_iid.size(); ++i) at.emplace(P.fam_iid[i], static_cast<int32_t>(i));
  std::vector<int32_t> col;
  for (const auto& s : samples) col.push_back(at.at(s));
  return col;
}

// Phenotype samples that are in the .fam, in phenotype order (intersect_order).
std::vector<std::string> overlap(const std::vector<std::string>& pheno, const Plink& P) {
  std::unordered_set<std::string> fam(P.fam_iid.begin(), P.fam_iid.end());
  std::vector<std::string> out;
  for (const auto& s : pheno)
    if (fam.count(s)) out.push_back(s);
  return out;
}

// PLINK or VCF genotypes of the run (-b / -v); a VCF's calls are parsed on
// the device, which `dev` then holds.
Plink read_genotypes(const Options& opt, VcfInfo& vi, std::unique_ptr<Device>& dev) {
  if (opt.vcf.empty()) return read_plink(opt.bfile);
  return read_vcf(opt.vcf, vi, [&]() {
    if (!dev) dev = std::make_unique<Device>();
    return dev->ctx;
  });
}

// Options for the device decode: a VCF has been filtered on the host with
// the reference's VCF rules (vcf_filter), so the device applies none.
Options device_filters(const Options& opt) {
  if (opt.vcf.empty()) return opt;
  Options o = opt;
  o.max_miss = 1.0;
  o.miss_filter = false;
  o.maf = 0.0;
  return o;
}

int run_make_grm(const Options& opt) {
  VcfInfo vi;
  std::unique_ptr<Device> devp;
  Plink P = read_genotypes(opt, vi, devp);
  std::vector<std::string> samples = P.fam_iid;
  if (!opt.pheno.empty()) {
    samples = overlap(load_pheno(opt.pheno).samples, P);
    if (samples.empty()) die("no overlapping samples for GRM");
  }
  if (!opt.vcf.empty()) vcf_filter(P, vi, sample_columns(P, samples), opt);
  if (!devp) devp = std::make_unique<Device>();
  Device& dev = *devp;
  Genotypes geno(dev, P, sample_columns(P, samples), device_filters(opt));
  const int n = static_cast<int>(samples.size());
  std::vector<double> K(static_cast<size_t>(n) * n);
  std::vector<int32_t> N(static_cast<size_t>(n) * (n + 1) / 2);
  int64_t m_used = 0;
  dev.check(eqtl_grm(dev.ctx, K.data(), N.data(), &m_used), "GRM");
  write_grm(opt.out, samples, K, N);
  info("wrote GRM " + opt.out + ".grm.id/.grm.bin/.grm.N.bin (" + std::to_string(m_used) + " SNPs)");
  return 0;
}

int run_scan(const Options& opt) {
  VcfInfo vi;
  std::unique_ptr<Device> devp;
  Plink P = read_genotypes(opt, vi, devp);
  Pheno ph = load_pheno(opt.pheno);
  Study st;
  st.opt = &opt;
  st.plink = &P;
  st.samples = overlap(ph.samples, P);
  if (st.samples.empty()) die("no overlapping samples between pheno and genotypes");
  const size_t n = st.samples.size(), G = ph.genes.size();
  {
    std::unordered_map<std::string, size_t> row;
    for (size_t i = 0; i < ph.samples.size(); ++i) row.emplace(ph.samples[i], i);
    st.genes = ph.genes;
    st.Y.resize(n * G);  // gene-major [G][n]
    for (size_t i = 0; i < n; ++i) {
      const double* r = &ph.Y[row.at(st.samples[i]) * G];
      for (size_t g = 0; g < G; ++g) st.Y[g * n + i] = r[g];
    }
  }
  st.X = load_covar(opt.covar, st.samples, st.p);
  const bool have_gff = !opt.gff.empty();
  if (have_gff) {
    st.annot = load_gff(opt.gff, opt.gff_id_key);
    size_t matched = 0;
    for (const auto& g : st.genes) matched += st.annot.count(g);
    info("pheno genes matched to GFF: " + std::to_string(matched) + "/" + std::to_string(G));
    if (matched == 0) die("no phenotype gene IDs match the GFF annotation (check --gff-id-key and ID format)");
  } else {
    info("no GFF: mode ignored; genome-wide all-pairs (gw)");
  }
  std::vector<std::string> scopes;
  if (!have_gff) scopes = {"gw"};
  else if (opt.mode == "all") scopes = {"cis", "trans"};
  else scopes = {opt.mode};
  {
    const std::string probe = opt.out + ".probe";
    FILE* f = std::fopen(probe.c_str(), "w");
    if (!f) die("cannot write to output prefix: " + opt.out);
    std::fclose(f);
    std::remove(probe.c_str());
  }
  // a cis scan of a VCF needs its index, as the reference's region queries do
  // (src/scan.cpp:92-98); the records themselves are read in file order
  if (!opt.vcf.empty() && std::find(scopes.begin(), scopes.end(), "cis") != scopes.end() &&
      !vcf_has_index(opt.vcf))
    die("cis mode requires an indexed genotype file; for VCF run: tabix -p vcf <file>.vcf.gz");

  if (!opt.vcf.empty()) vcf_filter(P, vi, sample_columns(P, st.samples), opt);
  if (!devp) devp = std::make_unique<Device>();
  Device& dev = *devp;
  if (opt.pheno_int) {  // every gene's rank-based inverse normal transform, on the device
    st.Y_int = st.Y;
    dev.check(eqtl_pheno_int(dev.ctx, st.Y_int.data(), static_cast<int32_t>(n), static_cast<int32_t>(G)),
              "--pheno-norm int");
  }
  Genotypes geno(dev, P, sample_columns(P, st.samples), device_filters(opt));
  st.dev = &dev;
  st.geno = &geno;
  if (std::find(opt.models.begin(), opt.models.end(), "lmm") != opt.models.end()) {
    // genes that miss some samples get the basis of their own slice of the
    // GRM (build_gene_ready, src/scan_common.cpp:41-63), and the scans of the
    // other genes the shared basis back: both on the host
    bool missing = false;
    for (double v : st.Y) missing = missing || !std::isfinite(v);
    for (double v : st.X) missing = missing || !std::isfinite(v);
    // the permutations rebuild LMM phenotypes through the basis on the host
    const bool host_basis = opt.perm > 0 || missing;
    if (host_basis) {
      st.basis_Q.resize(n * n);
      st.basis_lambda.resize(n);
    }
    double* lam = host_basis ? st.basis_lambda.data() : nullptr;
    double* Q = host_basis ? st.basis_Q.data() : nullptr;
    // --fast: the GRM's small off-diagonal entries are zeroed before the
    // eigendecomposition (sparsify_grm, src/model_lmm.cpp:88-104)
    const double thr = opt.fast ? 1e-4 : 0.0;
    int64_t zeroed = 0;
    if (const char* bf = std::getenv("EQTL_LMM_BASIS")) {
      // an eigenbasis computed elsewhere (for example by the reference's own
      // eigensolver, whose eigenvector signs its LMM permutations depend on)
      std::vector<double> lam_in(n), Q_in(n * n);
      FILE* fp = std::fopen(bf, "rb");
      if (!fp) die(std::string("EQTL_LMM_BASIS: cannot open ") + bf);
      const size_t got = std::fread(lam_in.data(), sizeof(double), n, fp) +
                         std::fread(Q_in.data(), sizeof(double), n * n, fp);
      const bool extra = std::fgetc(fp) != EOF;
      std::fclose(fp);
      if (got != n + n * n || extra)
        die("EQTL_LMM_BASIS: expected " + std::to_string(n) + " eigenvalues and a " + std::to_string(n) + " x " +
            std::to_string(n) + " eigenvector matrix (float64)");
      for (double& l : lam_in) l = std::max(l, 0.0);
      dev.check(eqtl_lmm_set_basis(dev.ctx, Q_in.data(), lam_in.data(), static_cast<int32_t>(n)), "LMM basis");
      if (host_basis) {
        st.basis_Q = Q_in;
        st.basis_lambda = lam_in;
      }
      info(std::string("LMM eigenbasis read from ") + bf);
    } else if (!opt.grm.empty()) {
      std::vector<double> K = slice_grm(load_grm(opt.grm), st.samples);
      dev.check(eqtl_lmm_basis_fast(dev.ctx, K.data(), static_cast<int32_t>(n), thr, lam, Q, &zeroed), "LMM basis");
      if (missing) st.K_full = std::move(K);
    } else {
      info("computing GRM from genotypes (overlap samples)");
      dev.check(eqtl_lmm_basis_fast(dev.ctx, nullptr, static_cast<int32_t>(n), thr, lam, Q, &zeroed), "LMM basis");
    }
    if (opt.fast)
      info("fast: GRM sparse approx thr=" + std::to_string(thr) + " zeroed " + std::to_string(zeroed) +
           " off-diagonal entries");
    if (missing && st.K_full.empty()) {
      st.K_full.resize(n * n);
      std::vector<int32_t> N(n * (n + 1) / 2);
      int64_t m_used = 0;
      dev.check(eqtl_grm(dev.ctx, st.K_full.data(), N.data(), &m_used), "GRM");
    }
  }
  for (const auto& model : opt.models) {
    for (const auto& scope : scopes) {
      ScopeFiles out(opt.out + "." + model + "." + scope, model == "glm");
      std::vector<RegionRow> regions;
      if (model == "glm") run_glm(st, scope, out, regions);
      else if (scope == "cis") run_cis(st, model, out, regions);
      else run_trans(st, model, scope, out, regions);
      std::vector<double> acat;
      for (const auto& r : regions) acat.push_back(r.acat);
      const std::vector<double> q = bh_adjust(acat);
      for (size_t i = 0; i < regions.size(); ++i) {
        regions[i].q = q[i];
        write_region(out.region, regions[i]);
      }
    }
  }
  return 0;
}

}  // namespace
}  // namespace eqtl_host

int main(int argc, char** argv) {
  using namespace eqtl_host;
  try {
    Options opt;
    const int rc = parse_options(argc, argv, opt);
    if (rc == 2) return 0;
    if (rc != 0) return 1;
    if (opt.run_fission) return run_fission(opt);
    return opt.make_grm ? run_make_grm(opt) : run_scan(opt);
  } catch (const Fatal& e) {
    std::cerr << "[E] " << e.what() << '\n';
    return 1;
  } catch (const std::exception& e) {
    std::cerr << "[E] " << e.what() << '\n';
    return 1;
  }
}
