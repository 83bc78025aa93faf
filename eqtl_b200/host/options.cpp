// Command line of the reference program (src/options.cpp:145-179): the same
// long and short flags, defaults and range checks, for the LM / LMM / NB-GLM
// models, with PLINK (-b) or VCF (-v, GT or DS) genotypes. The flags of paths
// outside the device scan (the GLMM model) are recognised and refused with a
// message instead of being silently ignored. `eqtl fission ...` selects the fission subcommand.
#include <getopt.h>

#include <algorithm>
#include <cstdlib>
#include <iostream>

#include "host.hpp"

namespace eqtl_host {

[[noreturn]] void die(const std::string& msg) { throw Fatal(msg); }
void info(const std::string& msg) { std::cerr << "[I] " << msg << '\n'; }
void warn(const std::string& msg) { std::cerr << "[W] " << msg << '\n'; }

namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
  while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
  return s.substr(a, b - a);
}

std::vector<std::string> parse_models(const std::string& s) {
  std::vector<std::string> out;
  size_t i = 0;
  while (i <= s.size()) {
    size_t j = s.find(',', i);
    if (j == std::string::npos) j = s.size();
    const std::string t = trim(s.substr(i, j - i));
    if (!t.empty()) {
      if (t == "glmm") die("--model glmm is outside the device scan (lm|lmm|glm are supported)");
      if (t != "lm" && t != "lmm" && t != "glm") die("invalid --model value: " + t + " (lm|glm|lmm|glmm)");
      out.push_back(t);
    }
    i = j + 1;
  }
  if (out.empty()) die("empty --model");
  return out;
}

void print_help() {
  std::cout << "Program: eqtl (expression QTL mapping, B200 device scan)\n"
               "\n"
               "Usage:   eqtl [options]\n"
               "         eqtl fission [options]   # data fission + PEER factor estimation\n"
               "\n"
               "Input options:\n"
               "    -v, --vcf FILE         genotypes VCF (GT or DS; plain or bgzip/gzip)\n"
               "    -b, --bfile PREFIX     PLINK bed/bim/fam prefix\n"
               "    -e, --pheno FILE       phenotype matrix (col1=sample)\n"
               "    -g, --gff FILE         GFF3 gene annotation (TSS)\n"
               "    -c, --covar FILE       covariates\n"
               "    -k, --grm PREFIX       relatedness matrix (.grm.id/.grm.bin)\n"
               "        --gff-id-key STR   GFF attribute for gene id\n"
               "\n"
               "Analysis options:\n"
               "        --make-grm         write relatedness matrix and exit\n"
               "    -m, --mode STR         cis|trans|all|gw  [all]\n"
               "        --model STR        lm|lmm|glm[,...]  [lmm]\n"
               "    -w, --window INT       cis flank around gene body (bp)  [1000000]\n"
               "        --pval-cis FLOAT   cis output p threshold  [1e-5]\n"
               "        --pval-trans FLOAT trans/gw output p threshold  [1e-5]\n"
               "        --miss-hand STR    filter|impute missing GT  [impute]\n"
               "        --max-miss FLOAT   drop SNP if missing fraction > value  [0.8]\n"
               "        --maf FLOAT        min MAF on analysis samples  [0=off]\n"
               "        --pheno-norm STR   per-gene phenotype normalization none|int  [none]\n"
               "        --fast             sparse GRM approx (LMM); glm/glmm: fix null phi/sigma2\n"
               "\n"
               "Fission options (subcommand: eqtl fission ...):\n"
               "    -c, --covar FILE       residualize known covars from Y1 before PEER\n"
               "        --peer-factors INT number of PEER factors to estimate  [10]\n"
               "        --epsilon FLOAT    thinning fraction (0,1)  [0.5]\n"
               "        --fission-max-iter INT  max PEER iterations  [1000]\n"
               "        --fission-tol FLOAT     PEER convergence tolerance  [1e-3]\n"
               "\n"
               "Permutation options:\n"
               "        --perm INT         gene-level permutations  [0=off]\n"
               "        --perm-trans-thr FLOAT  trans/gw: stage-2 if obs min-p < thr  [1e-5]\n"
               "        --perm-trans-top INT    trans/gw: top-K SNPs for stage-2 perm  [1000]\n"
               "        --seed INT         permutation / fission seed\n"
               "        --disable-beta-approx  omit beta-approximated p\n"
               "        --perm-rng STR     host: the reference's shuffles (std::mt19937, exact);\n"
               "                           device: LM/LMM permutations drawn on the GPU (Philox)  [host]\n"
               "\n"
               "Output options:\n"
               "    -o, --out PREFIX       output prefix  [eqtl_out]\n"
               "    -t, --thread INT       threads (cis output order follows the reference's)  [1]\n"
               "    -h, --help             help\n"
               "        --version          version\n";
}

}  // namespace

int parse_options(int argc, char** argv, Options& opt) {
  if (argc == 1) {
    print_help();
    return 2;
  }
  // subcommand: eqtl fission [...]
  int start = 1;
  if (argc >= 2 && std::string(argv[1]) == "fission") {
    opt.run_fission = true;
    start = 2;
  }
  enum {
    kGffIdKey = 1001, kMakeGrm, kModel, kPvalCis, kPvalTrans, kMissHand, kFast, kPerm, kSeed, kNoBeta, kVersion,
    kMaxMiss, kMaf, kPeerFactors, kEpsilon, kFissionMaxIter, kFissionTol, kPermThr = 1020, kPermTop, kPhenoNorm, kPermRng
  };
  static struct option long_opts[] = {{"vcf", required_argument, nullptr, 'v'},
                                      {"bfile", required_argument, nullptr, 'b'},
                                      {"pheno", required_argument, nullptr, 'e'},
                                      {"out", required_argument, nullptr, 'o'},
                                      {"gff", required_argument, nullptr, 'g'},
                                      {"covar", required_argument, nullptr, 'c'},
                                      {"grm", required_argument, nullptr, 'k'},
                                      {"gff-id-key", required_argument, nullptr, kGffIdKey},
                                      {"make-grm", no_argument, nullptr, kMakeGrm},
                                      {"mode", required_argument, nullptr, 'm'},
                                      {"model", required_argument, nullptr, kModel},
                                      {"window", required_argument, nullptr, 'w'},
                                      {"pval-cis", required_argument, nullptr, kPvalCis},
                                      {"pval-trans", required_argument, nullptr, kPvalTrans},
                                      {"miss-hand", required_argument, nullptr, kMissHand},
                                      {"max-miss", required_argument, nullptr, kMaxMiss},
                                      {"maf", required_argument, nullptr, kMaf},
                                      {"pheno-norm", required_argument, nullptr, kPhenoNorm},
                                      {"fast", no_argument, nullptr, kFast},
                                      {"thread", required_argument, nullptr, 't'},
                                      {"threads", required_argument, nullptr, 't'},
                                      {"perm", required_argument, nullptr, kPerm},
                                      {"permutations", required_argument, nullptr, kPerm},
                                      {"perm-trans-thr", required_argument, nullptr, kPermThr},
                                      {"perm-trans-top", required_argument, nullptr, kPermTop},
                                      {"seed", required_argument, nullptr, kSeed},
                                      {"perm-rng", required_argument, nullptr, kPermRng},
                                      {"disable-beta-approx", no_argument, nullptr, kNoBeta},
                                      {"peer-factors", required_argument, nullptr, kPeerFactors},
                                      {"epsilon", required_argument, nullptr, kEpsilon},
                                      {"fission-max-iter", required_argument, nullptr, kFissionMaxIter},
                                      {"fission-tol", required_argument, nullptr, kFissionTol},
                                      {"help", no_argument, nullptr, 'h'},
                                      {"version", no_argument, nullptr, kVersion},
                                      {nullptr, 0, nullptr, 0}};
  bool help = false, version = false;
  optind = start;
  int c, idx;
  while ((c = getopt_long(argc, argv, "v:b:e:o:g:c:k:m:w:t:h", long_opts, &idx)) != -1) {
    const std::string a = optarg ? optarg : "";
    switch (c) {
      case 'v': opt.vcf = a; break;
      case 'b': opt.bfile = a; break;
      case 'e': opt.pheno = a; break;
      case 'o': opt.out = a; break;
      case 'g': opt.gff = a; break;
      case 'c': opt.covar = a; break;
      case 'k': opt.grm = a; break;
      case 'm':
        if (a == "cis" || a == "trans" || a == "all" || a == "gw") opt.mode = a;
        else if (a == "gwas") opt.mode = "gw";
        else die("invalid --mode: " + a + " (cis|trans|all|gw)");
        break;
      case 'w': opt.window = std::atoi(a.c_str()); break;
      case 't': opt.threads = std::max(1, std::atoi(a.c_str())); break;
      case 'h': help = true; break;
      case kGffIdKey: opt.gff_id_key = a; break;
      case kMakeGrm: opt.make_grm = true; break;
      case kModel: opt.models = parse_models(a); break;
      case kPvalCis: opt.pval_cis = std::atof(a.c_str()); break;
      case kPvalTrans: opt.pval_trans = std::atof(a.c_str()); break;
      case kMissHand:
        if (a == "filter") opt.miss_filter = true;
        else if (a == "impute") opt.miss_filter = false;
        else die("invalid --miss-hand (filter|impute)");
        break;
      case kFast: opt.fast = true; break;
      case kPerm: opt.perm = std::atoi(a.c_str()); break;
      case kPermThr:
        opt.perm_trans_thr = std::atof(a.c_str());
        if (opt.perm_trans_thr <= 0 || opt.perm_trans_thr > 1) die("--perm-trans-thr must be in (0,1]");
        break;
      case kPermTop:
        opt.perm_trans_top = std::atoi(a.c_str());
        if (opt.perm_trans_top < 1) die("--perm-trans-top must be >= 1");
        break;
      case kSeed: opt.seed = std::atoi(a.c_str()); break;
      case kPermRng:
        if (a == "host") opt.perm_device = false;
        else if (a == "device") opt.perm_device = true;
        else die("invalid --perm-rng (host|device)");
        break;
      case kNoBeta: opt.disable_beta_approx = true; break;
      case kVersion: version = true; break;
      case kMaxMiss:
        opt.max_miss = std::atof(a.c_str());
        if (opt.max_miss < 0.0 || opt.max_miss > 1.0) die("--max-miss must be in [0,1]");
        break;
      case kMaf:
        opt.maf = std::atof(a.c_str());
        if (opt.maf < 0.0 || opt.maf > 0.5) die("--maf must be in [0,0.5]");
        break;
      case kPeerFactors:
        opt.peer_factors = std::atoi(a.c_str());
        if (opt.peer_factors < 1) die("--peer-factors must be >= 1");
        break;
      case kEpsilon:
        opt.fission_epsilon = std::atof(a.c_str());
        if (opt.fission_epsilon <= 0.0 || opt.fission_epsilon >= 1.0) die("--epsilon must be in (0,1)");
        break;
      case kFissionMaxIter:
        opt.fission_max_iter = std::atoi(a.c_str());
        if (opt.fission_max_iter < 1) die("--fission-max-iter must be >= 1");
        break;
      case kFissionTol:
        opt.fission_tol = std::atof(a.c_str());
        if (opt.fission_tol <= 0.0) die("--fission-tol must be > 0");
        break;
      case kPhenoNorm:
        if (a == "none" || a == "off") opt.pheno_int = false;
        else if (a == "int" || a == "rank") opt.pheno_int = true;
        else die("invalid --pheno-norm (none|int)");
        break;
      default: return 1;
    }
  }
  if (help) {
    print_help();
    return 2;
  }
  if (version) {
    std::cout << "eqtl 0.1.0 (eqtl_b200)\n";
    return 2;
  }
  if (opt.run_fission) {
    if (opt.pheno.empty()) {
      std::cerr << "[E] fission requires -e/--pheno\n";
      return 1;
    }
    return 0;
  }
  if (opt.vcf.empty() == opt.bfile.empty()) {
    if (opt.vcf.empty()) std::cerr << "[E] need exactly one of -v/--vcf or -b/--bfile\n";
    else std::cerr << "[E] use only one of -v/--vcf or -b/--bfile\n";
    return 1;
  }
  if (!opt.make_grm && opt.pheno.empty()) {
    std::cerr << "[E] missing -e/--pheno (or use --make-grm)\n";
    return 1;
  }
  if (opt.window < 0) die("--window must be >= 0");
  // src/options.cpp:288-299: INT output is continuous, the count models need raw counts
  if (opt.pheno_int && std::find(opt.models.begin(), opt.models.end(), "glm") != opt.models.end())
    die("--pheno-norm int is incompatible with count model glm (apply INT only for lm/lmm; count models need raw "
        "integer counts)");
  return 0;
}

}  // namespace eqtl_host
