/*
 * libeqtl_cuda: B200 (sm_100a) kernels for the eqtl association-scan hot
 * path behind a plain C ABI.
 *
 * The reference eqtl program (WWz33/eqtl) has no plugin or FFI layer: its
 * hot path is a set of C++ functions called from the scan orchestrator
 * (src/scan.cpp:164-226). Each entry point below replaces one of those
 * functions for the shared-keep case (every gene analysed on the same
 * complete-case sample set) and cites it. Conventions:
 *   - every function returns EQTL_OK (0) or a negative EQTL_E_* code and
 *     never throws; eqtl_last_error() describes the last failure;
 *   - all buffers are caller-owned HOST memory with explicit sizes; device
 *     state (decoded genotypes, eigenbasis, rotated genotypes) lives in the
 *     context and is reused across calls;
 *   - matrices are column-major: Y[g * n + i] is sample i of gene g,
 *     X[k * n + i] is sample i of covariate k, Q[j * n + i] is entry i of
 *     eigenvector j;
 *   - SNP indices in results are positions in the list of SNPs kept by
 *     eqtl_geno_load_bed (0 .. n_kept-1), in .bim order.
 */
#ifndef EQTL_B200_H
#define EQTL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EQTL_OK 0
#define EQTL_E_ARG (-1)         /* invalid argument */
#define EQTL_E_CUDA (-2)        /* CUDA runtime / library error */
#define EQTL_E_NOMEM (-3)       /* device allocation failed */
#define EQTL_E_STATE (-4)       /* call order violated (e.g. scan before load) */
#define EQTL_E_DEVICE (-5)      /* a device-side bounded wait expired */
#define EQTL_E_UNSUPPORTED (-6) /* input outside what the device path handles */
#define EQTL_E_OVERFLOW (-7)    /* result buffer too small (see *_count outputs) */
#define EQTL_E_INTERNAL (-8)

#define EQTL_MISS_FILTER 0 /* --miss-hand filter */
#define EQTL_MISS_IMPUTE 1 /* --miss-hand impute */

/* Arithmetic of the tensor-core contractions (FP32 accumulation always). */
#define EQTL_PREC_SPLIT_F16 0  /* operands as FP16 hi+lo pairs, 3 products */
#define EQTL_PREC_SPLIT_BF16 1 /* operands as BF16 hi+lo pairs, 3 products */
#define EQTL_PREC_FP32_SIMT 2  /* plain FP32 CUDA-core kernels (comparator) */

/* Pipeline stages timed with CUDA events (eqtl_stage_ms). */
#define EQTL_STAGE_DECODE 0 /* .bed decode + FP16 expansion */
#define EQTL_STAGE_GRM 1    /* GRM contraction + division */
#define EQTL_STAGE_EIGEN 2  /* eigendecomposition */
#define EQTL_STAGE_ROTATE 3 /* spectral rotation of the genotypes */
#define EQTL_STAGE_PREP 4   /* per-gene prep (residualisation / REML) */
#define EQTL_STAGE_SCAN 5   /* tensor-core scan kernel (all launches of the call) */
#define EQTL_STAGE_REFINE 6 /* FP64 refinement of candidate pairs */
#define EQTL_N_STAGES 7

typedef struct eqtl_ctx eqtl_ctx;

/* ---------------------------------------------------------------- context */
int eqtl_open(int device, eqtl_ctx** out);
void eqtl_close(eqtl_ctx* ctx);
const char* eqtl_last_error(const eqtl_ctx* ctx);
int eqtl_set_precision(eqtl_ctx* ctx, int precision);
/* Device time (ms, CUDA events on the context's stream) of `stage` in the
 * most recent call that ran it; EQTL_E_STATE if it has not run. */
int eqtl_stage_ms(eqtl_ctx* ctx, int stage, double* ms);
/* Number of kernels the library has launched on this context. */
int eqtl_launch_count(eqtl_ctx* ctx, uint64_t* count);
/* How the most recent LMM scan (p <= 2, split FP16) formed gg and a_k:
 * *nodes = 0 directly (K = n); otherwise interpolated between *nodes node
 * deltas, K = *node_cols per accumulator. EQTL_LMM_FORM=direct|lr in the
 * environment fixes the form (default: interpolated from 256 genes on, in
 * dense scans). */
int eqtl_lmm_form(eqtl_ctx* ctx, int32_t* nodes, int32_t* node_cols);
/* The cudaStream_t all work of this context is issued on (for callers that
 * time or order their own work against it). */
int eqtl_stream(eqtl_ctx* ctx, void** stream);

/* ---------------------------------------------------------- genotype load
 * Replaces PlinkBed::decode_row + for_each_range_pos
 * (src/plink_bed.cpp:263-320, 327-352; LUT :221-224; sample order :245-255).
 * rows: m SNP-major .bed records of bytes_per_snp bytes (the file after its
 * 3 magic bytes). sample_col[i] = .fam column of analysis sample i.
 * Outputs per input SNP: keep_out (1 = passes the missingness / allele-
 * frequency / MAF filters of decode_row), af_out (A1 frequency of the
 * non-missing calls = SnpRec.maf), n_miss_out. The kept SNPs stay decoded
 * and mean-imputed on the device for the scans. */
int eqtl_geno_load_bed(eqtl_ctx* ctx, const uint8_t* rows, int64_t m, int64_t bytes_per_snp, int32_t n_file,
                       const int32_t* sample_col, int32_t n, int32_t miss_hand, double max_miss, double maf_min,
                       uint8_t* keep_out, double* af_out, int32_t* n_miss_out, int64_t* n_kept_out);

/* The same load from dosage rows: replaces VcfSession::parse_record's
 * FORMAT/DS and GT dosages (src/vcf_session.cpp:193-258) for a VCF read on
 * the host. ds: m SNP-major rows of n_file FP32 ALT dosages (row s, file
 * sample j at ds[s * n_file + j]); a value that is not finite (NaN for ".")
 * is a missing call, every other value is used as it is. The filters and
 * outputs are those of eqtl_geno_load_bed, with af = mean / 2 of the
 * non-missing dosages (a caller that needs the reference's ploidy-aware VCF
 * filters applies them itself and passes max_miss 1, maf_min 0). Every
 * other call treats the loaded SNPs as it treats .bed SNPs. */
int eqtl_geno_load_dosage(eqtl_ctx* ctx, const float* ds, int64_t m, int32_t n_file, const int32_t* sample_col,
                          int32_t n, int32_t miss_hand, double max_miss, double maf_min, uint8_t* keep_out,
                          double* af_out, int32_t* n_miss_out, int64_t* n_kept_out);

/* VCF sample columns parsed on the device (VcfSession::parse_record's
 * per-call loop, src/vcf_session.cpp:193-258). text [text_len]: decompressed
 * VCF text; per record r (n_rec of them): the sample columns lie in
 * [beg[r], end[r]) (the 10th column to the end of the line), gt_at[r] / ds_at[r]
 * give the FORMAT position of GT and of the DS field to use (ds_at -1: GT).
 * dense 0: codes_out [n_rec][ceil(n_file/4)] 2-bit .bed codes of the GT
 * calls (ALT counted); dense 1: ds_out [n_rec][n_file] FP32 dosages (DS
 * values, or GT counts), NaN = missing. hap_out [n_rec][ceil(n_file/8)]: one
 * bit per GT call carrying a single allele. flag_out [n_rec]: 1 = fewer
 * sample columns than n_file, 2 = a call outside the parser's exact fast
 * paths (the caller parses such records itself). */
int eqtl_vcf_parse(eqtl_ctx* ctx, const char* text, int64_t text_len, const int64_t* beg, const int64_t* end,
                   const int32_t* gt_at, const int32_t* ds_at, int64_t n_rec, int32_t n_file, int32_t dense,
                   uint8_t* codes_out, float* ds_out, uint8_t* hap_out, uint8_t* flag_out);

/* Decoded, mean-imputed dosages of kept SNPs [lo, hi) as FP64, row-major
 * [hi - lo, n] (SnpRec.dosage after src/plink_bed.cpp:298-302). */
int eqtl_geno_dosage(eqtl_ctx* ctx, int64_t lo, int64_t hi, double* out);

/* Per-gene sample subsets (the reference's per-gene keep sets,
 * build_gene_ready, src/scan_common.cpp:11-65, and the trans/gw paths for
 * genes whose keep sets differ, src/scan_trans_lm.cpp:121-151,
 * src/scan_trans_lmm.cpp:192-228). Restricts the loaded genotypes to the
 * analysis samples idx[0..n_sub) (positions in the sample order of the
 * load, increasing); idx == NULL restores every analysis sample. The kept
 * SNPs, their imputation means and the load's filters stay those of the
 * whole sample set, as the reference imputes each SNP before it subsets it;
 * the per-SNP gate (subset_maf_or_nan) and every scan, refinement and
 * dosage call that follows use the subset (n = n_sub). The rotated LMM
 * operands are dropped: install the subset's basis (eqtl_lmm_basis with the
 * GRM sliced to the subset) before an LMM scan. eqtl_grm refuses a subset
 * view; the NB-GLM scan too. */
int eqtl_geno_subset(eqtl_ctx* ctx, const int32_t* idx, int32_t n_sub);

/* The same for k kept-SNP indices rows[0..k): out [k, n]. The host driver
 * prints each pair's af from these (subset_maf_or_nan,
 * src/scan_common.cpp:133-151, sums the dosages in sample order). */
int eqtl_geno_dosage_rows(eqtl_ctx* ctx, const int64_t* rows, int64_t k, double* out);

/* Evaluates the device Student-t tail (the device form of p_from_t,
 * src/util.cpp:259-264, through the df-specific interpolation tables) for n
 * values of t at residual df. mode bit 0: read the tables from shared memory
 * as the scan kernels do. mode bit 1 clear: the full tail, giving -log10 p,
 * the ACAT term tan((1/2 - p) pi) and flags. mode bit 1 set: the scan
 * epilogues' ACAT screen, giving |t| in place of -log10 p, the term, and the
 * same flags. Flag bit 0: term added on the device; bit 1: pair deferred to
 * the host's FP64 / long-double path (p < 1e-14, and t within a few 1e-6 of
 * 0 where the reference's p is quantised by the ulp of df); bit 2: deferred
 * for the latter reason. For validation. */
int eqtl_t_tail(eqtl_ctx* ctx, double df, const float* t, int64_t n, int32_t mode, float* neglog10p,
                double* term, uint8_t* flags);

/* ------------------------------------------------------------- phenotypes
 * Keeps the phenotype matrix Y [n, n_genes] (after the caller's per-gene
 * preparation: complete-case subset, optional --pheno-norm int) and the
 * covariate matrix X [n, p] (intercept included, src/pheno.cpp:171-193)
 * resident on the device. The scan entry points use them when called with
 * Y == NULL and X == NULL, so repeated scans need no host transfer. */
int eqtl_pheno_load(eqtl_ctx* ctx, const double* Y, const double* X, int32_t n, int32_t n_genes, int32_t p);

/* Permuted null phenotypes drawn on the device: the throughput mode of the
 * gene-level permutations (include/eqtl/scan_cis.hpp:102-147 for cis,
 * src/scan_perm.cpp:80-132 for trans/gw stage 2). The reference shuffles
 * each gene's null base vector with std::mt19937 + std::shuffle on the host;
 * here permutation b of gene g is the order of the keys
 * Philox4x32-10(counter = (b, i / 4, gene_key[g]), key = seed) (word i % 4)
 * of its samples i (Salmon et al., SC 2011), so the draws are independent
 * and uniform but not the reference's sequences. The resident phenotypes
 * (as after eqtl_pheno_load) become n_genes * n_perm columns, column
 * g * n_perm + b:
 *   LM  (xb0 == dinv == NULL)  base[g][perm(i)]
 *   LMM                        xb0[g][i] + base[g][perm(i)] / sqrt(max(dinv[g][i], 1e-12))
 * base, xb0, dinv [n_genes][n]; X [n, p] becomes the resident covariates.
 * Scan the columns with Y == X == NULL (y_rotated = 1 for the LMM form, whose
 * columns are in the eigenbasis). Y_out, if not NULL, receives the columns
 * [n_genes * n_perm][n] (for validation). At most 2^31 values per call. */
int eqtl_pheno_permute(eqtl_ctx* ctx, const double* base, const double* xb0, const double* dinv,
                       const uint64_t* gene_key, int32_t n, int32_t n_genes, int32_t n_perm, uint64_t seed,
                       const double* X, int32_t p, double* Y_out);

/* --pheno-norm int on the device: replaces inverse_normal_transform
 * (src/util.cpp:177-206, with qnorm_inv :132-171) for every column of
 * Y [n, n_cols] (column-major, host memory), in place. Per column the finite
 * values get average ranks (ties share them) and become
 * qnorm_inv((rank - 1/2) / n_finite); values that are not finite are left as
 * they are, as is a column with at most one finite value. */
int eqtl_pheno_int(eqtl_ctx* ctx, double* Y, int32_t n, int32_t n_cols);

/* ------------------------------------------------------------- fission
 * Replaces peer_factors (src/fission.cpp:203-275): PEER variational factor
 * analysis of Y [n, n_genes] (column-major host memory; each gene is centred
 * over its values that are not NaN, NaN counts as 0) with K factors, from
 * the starting factors X0 [n, K] and loadings W0 [n_genes, K] (column-major;
 * the reference draws X0 then W0, column by column, from
 * std::normal_distribution on std::mt19937(seed + 1)). Iterates the W,
 * Alpha, X and Eps updates until the mean squared residual moves by less
 * than 1e-8 or tol, at most max_iter times. X_out [n, K] receives the
 * factors, iters_out (optional) the iterations run. 1 <= K <= 96 and
 * K < min(n, n_genes). */
int eqtl_peer(eqtl_ctx* ctx, const double* Y, int32_t n, int32_t n_genes, int32_t K, int32_t max_iter, double tol,
              const double* X0, const double* W0, double* X_out, int32_t* iters_out);

/* ------------------------------------------------------- scan result types */
typedef struct {
  int32_t n_tested;      /* finite tests counted (GeneSummary.n_tested) */
  int32_t acat_used;     /* p-values entering ACAT (AcatAcc.used) */
  double acat_tan_sum;   /* sum of tan((0.5 - p) pi) (AcatAcc.tan_sum) */
  int64_t best_snp;      /* kept-SNP index of the smallest p, -1 if none */
  double best_p, best_beta, best_se, best_t, best_r2;
} eqtl_gene_result;

typedef struct {
  int64_t snp;  /* kept-SNP index */
  int32_t gene; /* gene (column of Y) */
  int32_t reserved;
  double beta, se, t, p, r2;
} eqtl_pair;

typedef struct {
  int32_t n;             /* samples: rows of Y and X */
  int32_t n_genes;       /* columns of Y */
  int32_t p;             /* covariate columns of X, intercept included */
  int32_t exclude_cis;   /* scope: 0 = gw (every SNP), 1 = trans (skip each gene's
                          * cis window), 2 = cis (only each gene's window) */
  double pthr;           /* pairs with p <= pthr are returned */
  double perm_thr;       /* candidates with p < perm_thr are returned (0 = none) */
  const int32_t* gene_chrom; /* [n_genes] chromosome id, -1 = no location */
  const int64_t* gene_lo;    /* [n_genes] window start (1-based, inclusive) */
  const int64_t* gene_hi;    /* [n_genes] window end (inclusive) */
  const int32_t* snp_chrom;  /* [n_kept] chromosome id of each kept SNP */
  const int64_t* snp_pos;    /* [n_kept] position of each kept SNP */
  int32_t y_rotated;         /* LMM only: 1 = Y is already in the eigenbasis
                              * (Q'y), as for permuted null phenotypes */
} eqtl_scan_params;

/* ------------------------------------------------------------ trans/gw LM
 * Replaces scan_lm_snp_outer (src/scan_trans_lm.cpp:41-163) on the shared-
 * keep path: prep_lm per gene (src/model_lm.cpp:19-30), gty = Y_s g_s and
 * hit_from_gty for every (SNP, gene) (:77-120), ACAT / n_tested / best
 * (include/eqtl/scan_trans.hpp:86-102). Y [n, n_genes], X [n, p], or both
 * NULL to use the phenotypes resident from eqtl_pheno_load.
 * genes[n_genes] receives the per-gene summary; pairs (p <= pthr) come back
 * sorted by (snp, gene) like the reference's pair file; cands (p <
 * perm_thr, the stage-2 permutation candidates) sorted by (gene, p). The
 * counts are always written; EQTL_E_OVERFLOW if a capacity was too small. */
int eqtl_scan_trans_lm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                       eqtl_gene_result* genes, eqtl_pair* pairs, int64_t pair_cap, int64_t* n_pairs,
                       eqtl_pair* cands, int64_t cand_cap, int64_t* n_cands);

/* --------------------------------------------------------------------- GRM
 * Replaces compute_grm (src/grm.cpp:113-224) for the loaded genotypes and
 * the analysis samples: K_out [n, n] (row-major, symmetric, FP64) and the
 * per-pair non-missing marker counts N_packed_out [n(n+1)/2] (row-major
 * lower triangle incl. diagonal, the .grm.N.bin order); m_used_out = SNPs
 * used. Either output may be NULL. */
int eqtl_grm(eqtl_ctx* ctx, double* K_out, int32_t* N_packed_out, int64_t* m_used_out);

/* ---------------------------------------------------- allocation-free GRM
 * No counterpart in the reference. The GRM of eqtl_geno_load_bed +
 * eqtl_grm with the same arguments, computed from caller-owned DEVICE
 * buffers without allocating device memory, for callers that cannot
 * allocate once running (a process that reserves its device memory up
 * front, e.g. a service sharing the GPU under a fixed budget). Inputs:
 * bed_dev = m SNP rows of bytes_per_snp bytes (.bed payload after the
 * 3-byte header), sample_col_dev = n analysis-sample columns. Outputs:
 * K_dev [n, n] row-major, N_packed_dev [n(n+1)/2] (may be NULL),
 * m_used_out (host, may be NULL). Equal to eqtl_grm up to the FP64
 * summation order of K; N bit-exact.
 *   - all scratch is one static device array of
 *     EQTL_GRM_NOALLOC_SCRATCH_BYTES in the library image; n is limited to
 *     EQTL_GRM_NOALLOC_MAX_N (larger n: EQTL_E_UNSUPPORTED), m is not (SNPs
 *     go through in passes of EQTL_GRM_NOALLOC_CHUNK);
 *   - eqtl_open resolves the array's address (cudaGetSymbolAddress, with
 *     the device current) and loads the kernels of this call, so that the
 *     array and the kernel images are in place before the call is first
 *     made: open the context while device memory can still be allocated,
 *     and before any stream capture;
 *   - the call returns once its work on the context's stream has finished
 *     (the outputs are ready to use): it synchronises the stream, so it
 *     cannot itself be recorded in a stream capture;
 *   - the accumulators and counters are zeroed at the start of every call
 *     on the context's stream; K is exactly symmetric (the lower triangle
 *     is summed, the upper one mirrors it);
 *   - the scratch is shared by every context on the device: overlapping
 *     calls (other threads, contexts or streams) race; serialise them. */
#define EQTL_GRM_NOALLOC_MAX_N 512
#define EQTL_GRM_NOALLOC_CHUNK 2048
#define EQTL_GRM_NOALLOC_SCRATCH_BYTES 9472256
int eqtl_grm_noalloc(eqtl_ctx* ctx, const uint8_t* bed_dev, int64_t m, int64_t bytes_per_snp,
                     const int32_t* sample_col_dev, int32_t n, int32_t miss_hand, double max_miss, double maf_min,
                     double* K_dev, int32_t* N_packed_dev, int64_t* m_used_out);

/* ------------------------------------------------------------- eigenbasis
 * Replaces make_lmm_basis (src/model_lmm.cpp:106-113): eigendecomposition of
 * the GRM K [n, n] (row-major; NULL = compute the GRM of the loaded
 * genotypes first) on the device, eigenvalues clipped at 0. The basis stays
 * resident for the LMM scans. lambda_out [n] ascending and Q_out [n, n]
 * (column j = eigenvector j) are optional. */
int eqtl_lmm_basis(eqtl_ctx* ctx, const double* K, int32_t n, double* lambda_out, double* Q_out);

/* The same with --fast (sparsify_grm, src/model_lmm.cpp:88-104, applied at
 * src/scan_trans_lmm.cpp:103, src/scan_cis.cpp:60, src/scan_common.cpp:56):
 * off-diagonal entries of K below sparsify_thr in magnitude (1e-4 in the
 * reference) are set to 0 before the eigendecomposition; zeroed_out
 * (optional) receives how many were. */
int eqtl_lmm_basis_fast(eqtl_ctx* ctx, const double* K, int32_t n, double sparsify_thr, double* lambda_out,
                        double* Q_out, int64_t* zeroed_out);

/* Installs an eigenbasis computed elsewhere (LmmBasis, include/eqtl/models.hpp
 * :43-46). Eigenvector signs are arbitrary; statistics do not depend on
 * them, but LMM permutations (which shuffle residuals in eigen-coordinates,
 * include/eqtl/scan_cis.hpp:77-87) do, so supplying the reference's own basis
 * reproduces its permutation p-values exactly. */
int eqtl_lmm_set_basis(eqtl_ctx* ctx, const double* Q, const double* lambda, int32_t n);

/* Rotates the loaded genotypes into the eigenbasis, Gt = Q'(g - mean) for
 * every kept SNP (the per-SNP g~ = Q'g of src/scan_trans_lmm.cpp:168, done
 * once for all SNPs); eqtl_scan_trans_lmm reuses it while the genotypes and
 * basis are unchanged, and runs it itself when needed. */
int eqtl_lmm_rotate(eqtl_ctx* ctx);

/* ----------------------------------------------------------- trans/gw LMM
 * Replaces scan_lmm_snp_outer (src/scan_trans_lmm.cpp:82-251) on the
 * shared-keep path, including prep_lmm's REML delta per gene
 * (src/model_lmm.cpp:39-86,124-153) and the bordered-Schur Wald test per
 * (SNP, gene) (src/scan_trans_lmm.cpp:11-40). Needs an eigenbasis of size n.
 * delta_out [n_genes] (optional) receives each gene's REML delta. Outputs as
 * for eqtl_scan_trans_lm. The tensor-core form handles p <= 2 covariate
 * columns; EQTL_PREC_FP32_SIMT selects the plain FP32 CUDA-core form. */
int eqtl_scan_trans_lmm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                        double* delta_out, eqtl_gene_result* genes, eqtl_pair* pairs, int64_t pair_cap,
                        int64_t* n_pairs, eqtl_pair* cands, int64_t cand_cap, int64_t* n_cands);

/* ---------------------------------------------------------------- NB GLM
 * Replaces the gene-outer NB-GLM scan (src/scan.cpp:227-300, per gene
 * include/eqtl/scan_cis.hpp:15-66) on the shared-keep path: prep_glm_nb's
 * null fit per gene (IRLS with moment dispersion, src/model_glm.cpp:28-96)
 * and test_glm_nb's score test per (gene, SNP) (:98-132), for every kept SNP
 * in the gene's scope (prm->exclude_cis as for the other scans). Y holds
 * counts (non-negative integers; other values fail with EQTL_E_ARG, as
 * prep_glm_nb dies). Outputs as for eqtl_scan_trans_lm, with eqtl_pair.t the
 * score statistic z and p two-sided normal; phi_out [n_genes] and
 * converged_out [n_genes] (optional) receive each gene's dispersion and
 * whether its null fit succeeded (a failed fit tests no SNP). Needs
 * EQTL_PREC_SPLIT_F16 and 1 <= p <= 32. */
int eqtl_scan_glm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X, double* phi_out,
                  uint8_t* converged_out, eqtl_gene_result* genes, eqtl_pair* pairs, int64_t pair_cap,
                  int64_t* n_pairs, eqtl_pair* cands, int64_t cand_cap, int64_t* n_cands);

/* The null fits of the most recent eqtl_scan_glm call: mu_out [n, n_genes]
 * (column-major) receives each gene's fitted means, which the reference's
 * GLM permutations resample from (include/eqtl/scan_cis.hpp:115-127). */
int eqtl_glm_mu(eqtl_ctx* ctx, double* mu_out);

/* -------------------------------------------------------------- pair tests
 * FP64 tests of explicit (column of Y, kept SNP) pairs with the scans' own
 * per-column prep: LM (EQTL_MODEL_LM) residualises each column on X
 * (prep_lm, src/model_lm.cpp:19-30); LMM (EQTL_MODEL_LMM) runs the full null
 * fit of each column with the resident eigenbasis, REML delta included
 * (prep_lmm, src/model_lmm.cpp:124-153). This is test_one_p with a fresh
 * prep_null per column, the inner loop of the gene-level permutations
 * (include/eqtl/scan_cis.hpp:150-163, src/scan_perm.cpp:118-126): the host
 * passes the permuted phenotypes as columns. out[i] gets beta, se, t, p, r2
 * of pair i; p is NaN when the SNP fails the subset gate on the analysis
 * samples (src/scan_common.cpp:133-151), which the reference never tests.
 * delta_out [n_genes] (LMM, may be NULL) receives each column's delta. Only
 * prm->n, n_genes and p are read. */
#define EQTL_MODEL_LM 0
#define EQTL_MODEL_LMM 1
int eqtl_test_pairs(eqtl_ctx* ctx, int32_t model, const eqtl_scan_params* prm, const double* Y, const double* X,
                    const int32_t* pair_col, const int64_t* pair_snp, int64_t n_pairs, eqtl_pair* out,
                    double* delta_out);

#ifdef __cplusplus
}
#endif

#endif /* EQTL_B200_H */
