// Host side of the eqtl drop-in: the command line of the reference program
// (src/options.cpp) for PLINK input and the LM / LMM models, its input
// readers, the scan drivers that call libeqtl_cuda through the C ABI, and the
// pairs / top / region TSV writers (src/output.cpp:8-110). Everything here is
// plain C++17; all association arithmetic runs on the device.
#pragma once
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "eqtl_b200.h"

namespace eqtl_host {

// Fatal input or usage error; main prints "[E] <what>" and exits 1, like the
// reference's die() (src/util.cpp:15-19, src/main.cpp:13-20).
struct Fatal : std::runtime_error {
  using std::runtime_error::runtime_error;
};
[[noreturn]] void die(const std::string& msg);
void info(const std::string& msg);
void warn(const std::string& msg);

// Opt-in phase timings: with EQTL_TRACE set, mark() prints the wall time
// since the previous mark to stderr.
struct Trace {
  bool on = std::getenv("EQTL_TRACE") != nullptr;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  void mark(const std::string& what) {
    if (!on) return;
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[eqtl trace] %s %.1f ms\n", what.c_str(),
                 std::chrono::duration<double, std::milli>(now - t).count());
    t = now;
  }
};

// ------------------------------------------------------------------ options
struct Options {
  std::string bfile, vcf, pheno, out = "eqtl_out", gff, covar, grm, gff_id_key;
  bool make_grm = false;
  std::string mode = "all";              // cis | trans | all | gw
  std::vector<std::string> models{"lmm"};
  int window = 1000000;
  double pval_cis = 1e-5, pval_trans = 1e-5;
  bool miss_filter = false;              // --miss-hand filter
  double max_miss = 0.8, maf = 0.0;
  bool pheno_int = false;                // --pheno-norm int
  bool fast = false;                     // --fast: sparse GRM before the LMM eigenbasis
  int threads = 1;
  int perm = 0;
  double perm_trans_thr = 1e-5;
  int perm_trans_top = 1000;
  int seed = -1;
  bool disable_beta_approx = false;
  bool perm_device = false;              // --perm-rng device: LM/LMM permutations drawn on the GPU
  // the fission subcommand (src/options.cpp:104-109, 237-252)
  bool run_fission = false;
  int peer_factors = 10;
  double fission_epsilon = 0.5;
  int fission_max_iter = 1000;
  double fission_tol = 1e-3;
};
// eqtl fission: data thinning of the phenotype table and PEER factors of Y1
// (src/fission.cpp:277-393).
int run_fission(const Options& opt);
// Returns 0 to run, 2 after --help / --version, 1 on a usage error.
int parse_options(int argc, char** argv, Options& opt);

// ------------------------------------------------------------------- inputs
struct Plink {
  std::vector<std::string> fam_iid;
  std::vector<std::string> chrom, id, a1, a2;  // .bim columns 1, 2, 5, 6
  std::vector<int64_t> pos;                    // .bim column 4
  int n_file = 0;
  int64_t bytes_per_snp = 0;
  std::vector<uint8_t> rows;                   // .bed payload, SNP-major
  bool dense = false;                          // dosage rows in ds instead of rows (VCF with DS)
  std::vector<float> ds;                       // [m][n_file] ALT dosages, NaN = missing call
};
Plink read_plink(const std::string& prefix);

// VCF input (vcf.cpp): GT calls as .bed 2-bit rows (ALT counted), or, when
// the header defines an ID "DS", FP32 dosage rows taken from FORMAT/DS where
// a record carries it and from GT elsewhere; plus what the reference's
// ploidy-aware filters need.
struct VcfInfo {
  std::vector<uint8_t> hap_chrom;               // per record: X, Y or MT (every call carries one allele)
  std::vector<std::vector<int32_t>> hap_calls;  // per record elsewhere: file columns with a haploid call
  int64_t n_multi = 0;                          // records skipped as not biallelic
};
// The calls are parsed on the device of the context that `ctx()` returns
// (opened when first needed).
Plink read_vcf(const std::string& path, VcfInfo& vi, const std::function<eqtl_ctx*()>& ctx);
// Keeps the records that pass the reference's VCF filters over the analysis
// samples `cols` (file columns): calls present, missing fraction, ploidy-
// aware allele frequency not monomorphic, --miss-hand filter, --maf.
void vcf_filter(Plink& P, const VcfInfo& vi, const std::vector<int32_t>& cols, const Options& opt);
// True when <path>.tbi or <path>.csi is a tabix / CSI index (its magic bytes
// after decompression); the index content itself is not used.
bool vcf_has_index(const std::string& path);

struct Pheno {
  std::vector<std::string> samples, genes;
  std::vector<double> Y;  // [samples][genes], row-major as in the file
};
Pheno load_pheno(const std::string& path);

// Covariates for the analysis samples, column-major [n, p], intercept first
// unless a column is already constant 1 (src/pheno.cpp:89-196).
std::vector<double> load_covar(const std::string& path, const std::vector<std::string>& samples, int& p);

struct GeneLoc {
  std::string chrom;
  int64_t start = 0, end = 0, tss = 0;
};
std::unordered_map<std::string, GeneLoc> load_gff(const std::string& path, const std::string& id_key);

// Chromosome names compare after dropping a "chr" prefix and leading zeros
// (chrom_equal, src/util.cpp:68-87); ids are assigned per normalised name.
std::string chrom_key(const std::string& c);

struct GrmFile {
  std::vector<std::string> ids;
  std::vector<double> K;  // [n, n]
};
GrmFile load_grm(const std::string& prefix);
std::vector<double> slice_grm(const GrmFile& g, const std::vector<std::string>& samples);
void write_grm(const std::string& prefix, const std::vector<std::string>& ids, const std::vector<double>& K,
               const std::vector<int32_t>& N_packed);

// --------------------------------------------------------------- statistics
double acat_p(double tan_sum, int used);                       // AcatAcc::p
std::vector<double> bh_adjust(const std::vector<double>& p);   // src/scan_common.cpp:201-217
uint64_t fnv1a64(const std::string& s);
uint32_t fnv1a32(const std::string& s);
uint32_t perm_seed(int seed_opt, int b, const std::string& gene);
double p_emp(double T_obs, const std::vector<double>& T_perm);
struct BetaFit {
  double p = NAN, s1 = NAN, s2 = NAN;
};
BetaFit beta_approx(const std::vector<double>& perm_min_p, double obs_min_p);

// -------------------------------------------------------------------- output
struct PairRow {
  std::string gene, snp, chrom, ref, alt;
  int64_t pos = 0;
  double af = 0, beta = 0, se = 0, t = 0, p = 1, r2 = 0;
  int n = 0;
  bool has_tss = false;
  double tss_dist = 0;
  bool glm = false;  // NB-GLM rows carry phi and glm_converged
  double phi = 0;
  int converged = 1;
};
struct RegionRow {
  std::string gene, chrom;
  int64_t tss = 0;
  int n_tested = 0, n_sig = 0;
  double acat = 1.0, q = NAN, p_emp = NAN, p_beta = NAN, s1 = 0, s2 = 0;
};
struct ScopeFiles {
  FILE* pairs = nullptr;
  FILE* top = nullptr;
  FILE* region = nullptr;
  ScopeFiles(const std::string& prefix, bool glm = false);
  ~ScopeFiles();
};
void write_pair(FILE* f, const PairRow& r, const std::string& scope);
void write_region(FILE* f, const RegionRow& r);

}  // namespace eqtl_host
