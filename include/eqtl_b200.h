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

typedef struct eqtl_ctx eqtl_ctx;

/* ---------------------------------------------------------------- context */
int eqtl_open(int device, eqtl_ctx** out);
void eqtl_close(eqtl_ctx* ctx);
const char* eqtl_last_error(const eqtl_ctx* ctx);
int eqtl_set_precision(eqtl_ctx* ctx, int precision);

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

/* Decoded, mean-imputed dosages of kept SNPs [lo, hi) as FP64, row-major
 * [hi - lo, n] (SnpRec.dosage after src/plink_bed.cpp:298-302). */
int eqtl_geno_dosage(eqtl_ctx* ctx, int64_t lo, int64_t hi, double* out);

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
  int32_t exclude_cis;   /* 1 = trans scope: skip each gene's cis window */
  double pthr;           /* pairs with p <= pthr are returned */
  double perm_thr;       /* candidates with p < perm_thr are returned (0 = none) */
  const int32_t* gene_chrom; /* [n_genes] chromosome id, -1 = no location */
  const int64_t* gene_lo;    /* [n_genes] window start (1-based, inclusive) */
  const int64_t* gene_hi;    /* [n_genes] window end (inclusive) */
  const int32_t* snp_chrom;  /* [n_kept] chromosome id of each kept SNP */
  const int64_t* snp_pos;    /* [n_kept] position of each kept SNP */
} eqtl_scan_params;

/* ------------------------------------------------------------ trans/gw LM
 * Replaces scan_lm_snp_outer (src/scan_trans_lm.cpp:41-163) on the shared-
 * keep path: prep_lm per gene (src/model_lm.cpp:19-30), gty = Y_s g_s and
 * hit_from_gty for every (SNP, gene) (:77-120), ACAT / n_tested / best
 * (include/eqtl/scan_trans.hpp:86-102). Y [n, n_genes], X [n, p].
 * genes[n_genes] receives the per-gene summary; pairs (p <= pthr) come back
 * sorted by (snp, gene) like the reference's pair file; cands (p <
 * perm_thr, the stage-2 permutation candidates) sorted by (gene, p). The
 * counts are always written; EQTL_E_OVERFLOW if a capacity was too small. */
int eqtl_scan_trans_lm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                       eqtl_gene_result* genes, eqtl_pair* pairs, int64_t pair_cap, int64_t* n_pairs,
                       eqtl_pair* cands, int64_t cand_cap, int64_t* n_cands);

#ifdef __cplusplus
}
#endif

#endif /* EQTL_B200_H */
