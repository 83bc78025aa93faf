// Internal host-side declarations of libeqtl_cuda: the context object behind
// the C ABI, device buffer ownership, and the launchers each .cu file
// provides. Nothing here crosses the ABI.
#pragma once
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/eqtl_b200.h"

namespace eqtl {

// Thrown inside the library, converted to a status code at the ABI boundary.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define EQTL_CUDA(call)                                                                          \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      throw ::eqtl::Error(EQTL_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

#define EQTL_CHECK(cond, code, msg)                         \
  do {                                                      \
    if (!(cond)) throw ::eqtl::Error((code), (msg));        \
  } while (0)

// Opt-in host trace: with EQTL_TRACE set in the environment, mark() prints
// the host time since the previous mark to stderr. Phases that end in a
// stream synchronisation include the device time they waited for.
struct HostTrace {
  bool on;
  const char* scope;
  std::chrono::steady_clock::time_point t;
  explicit HostTrace(const char* s) : on(std::getenv("EQTL_TRACE") != nullptr), scope(s) {
    if (on) t = std::chrono::steady_clock::now();
  }
  void mark(const char* what) {
    if (!on) return;
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[eqtl trace] %s %s %.3f ms\n", scope, what,
                 std::chrono::duration<double, std::milli>(now - t).count());
    t = now;
  }
};

// Device buffer that keeps its allocation: alloc() only reallocates when
// the requested count exceeds the capacity, so per-call workspaces held by
// the context cost no cudaMalloc / cudaFree after the first call.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;    // elements in use
  size_t cap = 0;  // elements allocated
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = cap = 0;
  }
  void alloc(size_t count) {
    if (count <= cap && p) {
      n = count;
      return;
    }
    release();
    if (count == 0) return;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      throw Error(EQTL_E_NOMEM, "device allocation of " + std::to_string(count * sizeof(T)) +
                                    " bytes failed: " + cudaGetErrorString(e));
    }
    n = cap = count;
  }
  void zero(cudaStream_t s) {
    if (p) EQTL_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  void upload(const T* h, size_t count, cudaStream_t s) {
    alloc(count);
    if (count) EQTL_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void download(T* h, size_t count, cudaStream_t s) const {
    if (count) EQTL_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
};

// Device view of the uploaded genotype rows, in one of two forms: PLINK
// 2-bit SNP-major rows (bed, bps bytes each; 00 -> 2 A1 alleles, 10 -> 1,
// 11 -> 0, 01 -> missing) or FP32 dosage rows (ds, ld values each, the ALT
// dosage of a VCF's FORMAT/DS or GT; a value that is not finite is missing).
// dosage() is the dosage of file column c of row s, NaN when missing.
struct GenoRows {
  const uint8_t* bed = nullptr;
  int64_t bps = 0;
  const float* ds = nullptr;
  int64_t ld = 0;
#ifdef __CUDACC__
  __device__ __forceinline__ double dosage(int64_t s, int c) const {
    if (ds) {
      const float v = __ldg(ds + s * ld + c);
      return isfinite(v) ? static_cast<double>(v) : __longlong_as_double(0x7ff8000000000000LL);
    }
    const uint32_t b = __ldg(bed + s * bps + (c >> 2));
    const uint32_t pair = (b >> ((c & 3) * 2)) & 3u;
    return pair == 1u ? __longlong_as_double(0x7ff8000000000000LL)
                      : static_cast<double>((0x00010002u >> (pair * 8)) & 0xFFu);
  }
#endif
};

// Decoded genotypes resident on the device (one .bed or dosage load).
struct Geno {
  int64_t m_all = 0;      // SNP rows uploaded
  int64_t m = 0;          // SNPs kept by decode (rows of every SNP-side operand)
  int n = 0;              // analysis samples
  int n_file = 0;         // .fam samples
  int64_t bytes_per_snp = 0;
  int k_pad = 0;          // n rounded up to a multiple of 64
  DevBuf<uint8_t> bed;    // [m_all, bytes_per_snp] (2-bit rows)
  bool dense = false;     // rows are FP32 dosages in ds instead of bed
  DevBuf<float> ds;       // [m_all, n_file] FP32 dosages (dense rows)
  DevBuf<int32_t> col;    // [n] .fam column per analysis sample
  bool col_identity = false;  // col[i] == i for every analysis sample
  DevBuf<int32_t> n_miss; // [m_all]
  DevBuf<double> s1;      // [m_all] sum of the non-missing dosages
  DevBuf<double> s2;      // [m_all] sum of their squares
  DevBuf<uint8_t> pass;   // [m_all]
  DevBuf<double> af;      // [m_all]
  DevBuf<double> mu;      // [m_all] imputation mean
  DevBuf<int64_t> kept;   // [m] row index of kept SNP
  DevBuf<__half> gc_hi, gc_lo;  // [m, k_pad] (dosage - mean) * kGcScale, hi/lo FP16
  // Sample view (eqtl_geno_subset): n, col and the operands above cover
  // either every analysis sample of the load (n_full, col_full_h) or a
  // subset of them; the kept SNPs and imputation means stay the load's.
  int n_full = 0;
  std::vector<int32_t> col_full_h;
  bool subset = false;
  // per-SNP sums of the imputed dosage and its square over a subset view
  // ([m_all]), with zero missing counts, for the per-gene SNP gate
  DevBuf<double> vs1, vs2;
  DevBuf<int32_t> vzero;
  const double* gate_s1() const { return subset ? vs1.p : s1.p; }
  const double* gate_s2() const { return subset ? vs2.p : s2.p; }
  const int32_t* gate_nmiss() const { return subset ? vzero.p : n_miss.p; }
  std::vector<int64_t> kept_h;
  std::vector<double> mu_h, af_h;
  std::vector<int32_t> n_miss_h;
  GenoRows rows() const {
    GenoRows r;
    if (dense) {
      r.ds = ds.p;
      r.ld = n_file;
    } else {
      r.bed = bed.p;
      r.bps = bytes_per_snp;
    }
    return r;
  }
};

// Rotated genotypes for the LMM scans: Gt = Q^T (g - mean), Gt^2, hi/lo.
struct Rotated {
  int64_t m = 0;
  int k_pad = 0;
  DevBuf<__half> gt_hi, gt_lo, gt2_hi, gt2_lo;
  // Exact unrotated SNP operand of the LMM scan (geno_raw_operand): row r =
  // c_r * dosage (or c_r * (2 - dosage)) in FP16, every value an integer
  // below 4096, missing calls and padding column n at c_r times the imputed
  // mean; a gene-side vector v holding -sum(v) at column n gives
  // v . (dosage - mean) = alpha[r] * (v . row).
  DevBuf<__half> raw;
  DevBuf<float> alpha;
  int64_t raw_m = -1;      // SNPs the operand was built for (-1: not built)
  bool raw_exact = false;  // every kept SNP representable exactly
  // FP32 copies of Gt and Gt^2 for the plain FP32 CUDA-core comparator
  DevBuf<float> gt32, gt2_32;
  // split-BF16 scans: Gt and Gt^2 re-split into BF16 hi + lo (bits of
  // __nv_bfloat16 in 16-bit storage), for the rotation of bf16_m SNPs
  DevBuf<__half> bgt_hi, bgt_lo, bgt2_hi, bgt2_lo;
  int64_t bf16_m = -1;
};

// Phenotypes / covariates resident on the device (eqtl_pheno_load).
struct PhenoDev {
  int n = 0, G = 0, p = 0;
  DevBuf<double> Y;   // [G][n]
  DevBuf<double> X;   // [p][n]
  std::vector<double> X_h;
};

// Per-call workspaces reused across calls (capacity grows, never shrinks).
struct Workspace {
  DevBuf<double> Ytil, Xtil, Ys, XtY, XtXinv, delta, chi0, ainv, a00L, rss, gtg, inv_gtg, af_sub, inv_yty, yty;
  DevBuf<__half> ops_hi[34], ops_lo[34];  // gene-side operands, one per accumulator (dev::kMaxAcc)
  DevBuf<__half> opsb_hi[34], opsb_lo[34];  // the same re-split into BF16 hi + lo (split-BF16 LMM scans)
  DevBuf<__half*> ops_ptr;
  DevBuf<float> unscale, gscale, inv_gtg_f;
  DevBuf<uint8_t> ok;
  DevBuf<double> graw, gt;
  // device-drawn permutations: per-gene base vectors, sort keys, offsets
  DevBuf<double> perm_base, perm_xb0, perm_dinv;
  DevBuf<uint64_t> perm_gkey;
  DevBuf<unsigned long long> perm_keys, perm_sorted;
  DevBuf<int> perm_off;
  DevBuf<uint8_t> perm_temp;
  DevBuf<eqtl_pair> refined;
  DevBuf<double> tiny_p;
  DevBuf<int2> tile_list;
  DevBuf<__half> q_hi, q_lo;  // rotation: split eigenvector operand
  DevBuf<int> ref_snps, ref_col;
  DevBuf<int2> ref_pairs;
  // batched REML (p > 3): covariate pair products, per-round weights and sums
  DevBuf<double> rb_P, rb_dlt, rb_W, rb_WY, rb_A, rb_B, rb_ld, rb_ydy;
  DevBuf<double> rb_Wg, rb_Xw, rb_Ag, rb_Lg, rb_ldx, rb_ldD, rb_Bg, rb_Yg;  // grid phase
  DevBuf<uint8_t> rb_state;
  DevBuf<unsigned int> rb_active;
  // NB-GLM null fits: per gene and sample mu, w = mu / (1 + phi mu) and
  // r = (y - mu) / (1 + phi mu); per gene phi, sum r and flags
  DevBuf<double> glm_mu, glm_w, glm_r, glm_phi, glm_rsum;
  DevBuf<float> glm_rsum_f, snp_mean;
  DevBuf<uint8_t> glm_ok, glm_counts;
  // per-gene scan outputs + candidates
  DevBuf<double> acat;
  DevBuf<int> used, tested;
  DevBuf<unsigned long long> best;
  DevBuf<int2> cand;
  DevBuf<unsigned int> count;
  // windows
  DevBuf<int32_t> win_gc, win_sc;
  DevBuf<int64_t> win_glo, win_ghi, win_sp;
  DevBuf<int32_t> win_bc;            // Windows::blk_chrom
  DevBuf<int64_t> win_blo, win_bhi;  // Windows::blk_lo / blk_hi
  DevBuf<float> tt_h, tt_L, tt_c1, tt_lt, tt_c1q, tt_ltq;
  double tt_df = -1;
  // GRM operands and accumulators, eigen-solver scratch
  DevBuf<uint8_t> grm_use;
  DevBuf<double> grm_mean, grm_isd, grm_A, eig_work;
  DevBuf<int2> grm_tiles;  // lower-triangle tile list of the GRM contraction
  DevBuf<unsigned long long> grm_count;  // SNPs the GRM uses
  DevBuf<unsigned long long> raw_inexact;  // SNPs the exact LMM operand cannot hold
  DevBuf<double> lmm_w, lmm_uv;            // [n, G (p + 1)]: w o (r~, X~_k) and Q times them
  // per-call scratch kept with the context, so warm calls allocate nothing:
  // the GRM and its joint-missing counts of eqtl_grm / eqtl_lmm_basis, the
  // --fast sparsification count, the covariate coefficients of the LM prep
  DevBuf<double> basis_K, resid_C;
  DevBuf<int32_t> basis_N;
  DevBuf<unsigned long long> sparsify_cnt;
  // interpolated LMM scan (lmm_lr_prepare): node log-deltas and deltas, the
  // node pass's gene-side operands, its FP32 table [m][lr_kb] with the column
  // maxima and scales, the split SNP-side table and the genes' coefficients
  DevBuf<double> lr_a, lr_delta, lr_zero, lr_w, lr_uv;
  DevBuf<__half> lr_ops_hi[4], lr_ops_lo[4];
  DevBuf<__half*> lr_ops_ptr;
  DevBuf<float> lr_unscale, lr_val, lr_sigma;
  DevBuf<unsigned int> lr_colmax;
  DevBuf<__half> lr_phi, lr_plo, lr_chi, lr_clo;
  int lr_kn = 0, lr_kb = 0;
  int lr_nodes = 0;  // node deltas of the most recent LMM scan (0: direct form)
  DevBuf<float> ops32[4];                  // FP32 gene-side operands of the CUDA-core comparator
  DevBuf<const float*> ops32_ptr;
  DevBuf<__half> grm_zh, grm_zl, grm_mk;
  DevBuf<int> grm_J, eig_info;
};

struct LmmBasisDev {
  int n = 0;
  DevBuf<double> Q;        // [n, n] column-major (column j = eigenvector j)
  DevBuf<double> lambda;   // [n]
  std::vector<double> Q_h, lambda_h;
};

}  // namespace eqtl

// Per-stage device timing: CUDA events recorded on the context stream around
// each stage of the last call (see eqtl_stage_ms).
struct StageTimer {
  cudaEvent_t start[EQTL_N_STAGES] = {};
  cudaEvent_t stop[EQTL_N_STAGES] = {};
  bool used[EQTL_N_STAGES] = {};
};

struct eqtl_ctx {
  int device = 0;
  StageTimer timer;
  uint64_t launches = 0;  // kernels launched by the library since eqtl_open
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  uint32_t* d_status = nullptr;  // device status word of the last tile launch
  void* cublas = nullptr;        // cublasHandle_t
  void* cusolver = nullptr;      // cusolverDnHandle_t
  std::string last_error;
  eqtl::Geno geno;
  eqtl::Rotated rot;
  eqtl::Rotated glm_ops;  // NB-GLM SNP operands: centred dosages gc and gc^2 (not rotated)
  eqtl::LmmBasisDev basis;
  eqtl::PhenoDev pheno;
  eqtl::Workspace ws;
  bool have_basis = false;
  int precision = EQTL_PREC_SPLIT_F16;
  std::vector<int> host_mark;  // per-kept-SNP scratch of the refinement's index
};

namespace eqtl {

// scale applied to centred dosages before the FP16 split (exact power of two)
constexpr float kGcScale = 64.0f;

// -- geno.cu
void geno_load(eqtl_ctx* ctx, const uint8_t* rows, int64_t m, int64_t bytes_per_snp, int n_file,
               const int32_t* sample_col, int n, int miss_hand, double max_miss, double maf_min);
void geno_load_dosage(eqtl_ctx* ctx, const float* ds, int64_t m, int n_file, const int32_t* sample_col, int n,
                      int miss_hand, double max_miss, double maf_min);

void geno_dosage(eqtl_ctx* ctx, int64_t lo, int64_t hi, double* out_host);
// Rank-based inverse normal transform of each of the G columns of Y_host
// [G][n], in place (computed on the device).
void pheno_int(eqtl_ctx* ctx, double* Y_host, int n, int G);
// VCF sample columns of R records parsed on the device (see vcf_parse.cu).
void vcf_parse(eqtl_ctx* ctx, const char* text, int64_t text_len, const int64_t* beg, const int64_t* end,
               const int32_t* gt_at, const int32_t* ds_at, int64_t R, int n_file, int dense, uint8_t* codes_out,
               float* ds_out, uint8_t* hap_out, uint8_t* flag_out);
// PEER factors of Y_host [n, G] (column-major) from the starting X0 [n, K]
// and W0 [G, K]; returns the iterations run.
int peer_factors(eqtl_ctx* ctx, const double* Y_host, int n, int G, int K, int max_iter, double tol,
                 const double* X0, const double* W0, double* X_out);
void geno_dosage_rows(eqtl_ctx* ctx, const int64_t* rows, int64_t k, double* out_host);
void pheno_load(eqtl_ctx* ctx, const double* Y, const double* X, int n, int G, int p);
// Resident phenotypes = G * B permuted columns drawn on the device (perm.cu).
void pheno_permute(eqtl_ctx* ctx, const double* base, const double* xb0, const double* dinv,
                   const uint64_t* gene_key, int n, int G, int B, uint64_t seed, const double* X, int p,
                   double* Y_out);

// -- scan drivers
void scan_trans_lm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                   eqtl_gene_result* genes, std::vector<eqtl_pair>& pairs, std::vector<eqtl_pair>& cands);

void scan_trans_lmm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X, double* delta_out,
                    eqtl_gene_result* genes, std::vector<eqtl_pair>& pairs, std::vector<eqtl_pair>& cands);
void scan_trans_lmm_simt(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                         double* delta_out, eqtl_gene_result* genes, std::vector<eqtl_pair>& pairs,
                         std::vector<eqtl_pair>& cands);

// -- grm.cu / lmm.cu
template <class T>
struct DevBuf;
int64_t grm_compute(eqtl_ctx* ctx, DevBuf<double>& K, DevBuf<int32_t>& Npk);
// Eigenbasis of the device GRM K_dev; with sparsify_thr > 0 the off-diagonal
// entries below it in magnitude are zeroed first (--fast), *zeroed = count.
void lmm_basis_from_grm(eqtl_ctx* ctx, const double* K_dev, int n, double sparsify_thr = 0.0,
                        int64_t* zeroed = nullptr);
void lmm_set_basis(eqtl_ctx* ctx, const double* Q, const double* lambda, int n);
void lmm_rotate(eqtl_ctx* ctx);
int64_t grm_noalloc(eqtl_ctx* ctx, const uint8_t* bed, int64_t m, int64_t bps, const int32_t* col, int n,
                    int miss_hand, double max_miss, double maf_min, double* K, int32_t* Npk);
void grm_noalloc_prepare(eqtl_ctx* ctx);
bool geno_raw_operand(eqtl_ctx* ctx);
void geno_expand(eqtl_ctx* ctx);
// Restricts the genotype view to the analysis samples idx[0..n_sub) (null:
// every analysis sample again).
void geno_subset(eqtl_ctx* ctx, const int32_t* idx, int n_sub);
void solver_release(eqtl_ctx* ctx);
void test_pairs_lm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                   const std::vector<int2>& todo, eqtl_pair* out);
// NB-GLM score-test scan (model_glm.cpp) of every (gene, kept SNP) pair in
// scope; phi_out / converged_out per gene.
void scan_glm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X, double* phi_out,
              uint8_t* converged_out, eqtl_gene_result* genes, std::vector<eqtl_pair>& pairs,
              std::vector<eqtl_pair>& cands);
void test_pairs_lmm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                    const std::vector<int2>& todo, eqtl_pair* out, double* delta_out);

// -- stage timing (capi.cu)
void stage_begin(eqtl_ctx* ctx, int stage);
void stage_end(eqtl_ctx* ctx, int stage);
struct StageScope {
  eqtl_ctx* c;
  int s;
  StageScope(eqtl_ctx* ctx, int stage) : c(ctx), s(stage) { stage_begin(c, s); }
  ~StageScope() { stage_end(c, s); }
};

// -- status check after a tile launch (capi.cu)
void check_tile_status(eqtl_ctx* ctx, const char* what);

}  // namespace eqtl
