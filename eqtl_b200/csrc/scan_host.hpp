// Host-side plumbing shared by the scan drivers: tensor-map setup and tile
// launches, per-gene output buffers (with candidate-overflow retry), window
// tables, the device t table, and the FP64 finishing arithmetic applied to
// refined pairs. Included only by .cu files.
#pragma once
#include <algorithm>
#include <cstring>
#include <functional>
#include <vector>

#include "internal.hpp"
#include "scan_common.cuh"
#include "tile_gemm.cuh"
#include "tstat.hpp"

namespace eqtl {

// -- covariate algebra (host FP64)
std::vector<double> xtx_inverse(const double* X, int n, int p);  // (X'X)^-1, row-major p x p
// Y[n, G] <- Y - X (XtXinv X'Y), on the device (cuBLAS DGEMM). XtY: scratch [p, G].
void residualize_genes(eqtl_ctx* ctx, const double* dX, const double* dXtXinv, int n, int p, int G, double* dY,
                       double* dXtY);

// Splits refined pairs into the pair list (p <= pthr, sorted by snp then
// gene) and stage-2 candidates (p < perm_thr, sorted by gene, p, snp), and
// sets each gene's best from the refined pairs (smallest p, lowest snp).
void finish_scan(const eqtl_scan_params* prm, eqtl_gene_result* genes, const std::vector<eqtl_pair>& refined,
                 std::vector<eqtl_pair>& pairs, std::vector<eqtl_pair>& cands);

// Uploads the scan windows into the context workspace; returns the device
// view (mode none when the caller gave no windows).
dev::Windows upload_windows(eqtl_ctx* ctx, const eqtl_scan_params* prm, int64_t m, int mode);

// Device t-tail table for `df`, cached in the context workspace.
// Device tables of the two-sided t tail with `df` residual degrees of
// freedom, or of the normal tail (normal = true; df is then ignored).
dev::TTable device_ttable(eqtl_ctx* ctx, double df, bool normal = false);
bool cis_tile_list(eqtl_ctx* ctx, const eqtl_scan_params* prm, int64_t m, int NT, const int2*& list, int& n_list);

// Resolves the phenotypes of a scan call: uploads (Y, X) when given,
// otherwise checks the resident ones match the call's shape.
const PhenoDev& resolve_pheno(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X);

// Per-gene outputs of one scan launch + candidate buffer (context workspace).
struct ScanOutputs {
  eqtl_ctx* ctx;
  int G;
  DevBuf<double>& acat;
  DevBuf<int>& used;
  DevBuf<int>& tested;
  DevBuf<unsigned long long>& best;
  DevBuf<int2>& cand;
  DevBuf<unsigned int>& count;
  unsigned int cap;
  unsigned int n_cand = 0;
  ScanOutputs(eqtl_ctx* c, int genes, int64_t m, int64_t cap_hint);
  void reset();
  // runs `launch` until every candidate fitted in the buffer
  void run(const std::function<void(dev::GeneOut)>& launch);
  // downloads per-gene sums into genes[] and returns the (gene, snp) pairs to
  // refine: all candidates plus each gene's best SNP
  // refine: all candidates plus each gene's best SNP; with `tiny`, the pairs
  // deferred only for 0 < |t| < tiny_t go there instead of todo / deferred
  void collect(eqtl_gene_result* genes, std::vector<int2>& todo, std::vector<int2>& deferred,
               std::vector<int2>* tiny = nullptr);
};

// Adds, for every deferred (gene, snp) pair, the reference's long-double ACAT
// term tan((0.5L - p) pi_L) computed from the refined FP64 p
// (src/stats_extra.cpp:16-22; p <= 0 -> 1e-300).
// `refined` is sorted by (gene, snp), as ScanOutputs::collect orders the
// pairs it hands to the refinement.
void add_deferred_acat(eqtl_gene_result* genes, const std::vector<eqtl_pair>& refined,
                       const std::vector<int2>& deferred);

// Adds the reference's long-double ACAT term and `used` count of each pair
// whose FP64 p (p_pairs[i]) enters ACAT (src/stats_extra.cpp:16-22).
void add_acat_terms(eqtl_gene_result* genes, const std::vector<int2>& pairs, const std::vector<double>& p_pairs);

// Candidate-buffer size: three times the pairs expected under the null at the
// larger of the two thresholds, at least 2^16.
inline int64_t expected_candidates(const eqtl_scan_params* prm, int64_t m) {
  const double thr = std::max(prm->pthr, prm->perm_thr);
  const double e = 3.0 * static_cast<double>(m) * prm->n_genes * std::min(1.0, thr) + 65536.0;
  return static_cast<int64_t>(std::min(e, static_cast<double>(1 << 26)));
}

void make_map_2d(CUtensorMap* map, const void* base, uint64_t rows, uint64_t k_pad, uint32_t box_rows, bool bf16);
int sm_count(eqtl_ctx* ctx);

// Per-accumulator K ranges and operand K extents of one tile launch: an
// accumulator j with end[j] > 0 runs over the K chunks [beg[j], end[j]) of
// its own operands instead of the whole K (ksplit 1, no sub-ranges).
struct TileK {
  int beg[dev::kMaxAcc] = {};
  int end[dev::kMaxAcc] = {};
  int k_a[dev::kMaxAcc] = {};  // K extent of accumulator j's gene-side operand (0: k_pad)
  int k_b[2] = {};             // K extent of SNP-side pair b (0: k_pad)
};

// Launches the persistent tile kernel for NACC accumulators. a_*[j] are the
// gene-side hi/lo operands of accumulator j ([rows_a, k_pad]); b_*[0..1] the
// SNP-side pairs ([rows_b, k_pad]); bsel[j] picks the pair, prod[j] the
// products. tiles: optional explicit tile list (device pointer) + count.
// BL: where the SNP-side lo parts go (dev::kBLoStage; kBLoNone: exact SNP
// operands, no product may have bit 2, and more ring stages fit). kc_sub:
// K chunks per sub-range (0: none; single-group epilogues only). tk:
// per-accumulator K ranges (TileK; null: every accumulator over all of K).
template <int NT, int NACC, class EpiParams, int BL = dev::kBLoStage>
void launch_tile_n(eqtl_ctx* ctx, bool bf16, const EpiParams& ep, const __half* const* a_hi,
                   const __half* const* a_lo, int64_t rows_a, const __half* const* b_hi, const __half* const* b_lo,
                   int64_t rows_b, int k_pad, const int* bsel, const int* prod, const int2* tile_list = nullptr,
                   int n_tile_list = 0, int ksplit = 1, int n_acc = NACC, int kc_sub = 0,
                   const TileK* tk = nullptr);

}  // namespace eqtl

// ----------------------------------------------------------------- template
namespace eqtl {

template <class EpiParams>
struct EpiOf;

template <int NT, int NACC, class EpiParams, int BL>
void launch_tile_n(eqtl_ctx* ctx, bool bf16, const EpiParams& ep, const __half* const* a_hi,
                   const __half* const* a_lo, int64_t rows_a, const __half* const* b_hi, const __half* const* b_lo,
                   int64_t rows_b, int k_pad, const int* bsel, const int* prod, const int2* tile_list,
                   int n_tile_list, int ksplit, int n_acc, int kc_sub, const TileK* tk) {
  using Epi = typename EpiOf<EpiParams>::type;
  using C = dev::TileCfg<NT, NACC, BL>;
  dev::TileMaps maps;
  std::memset(&maps, 0, sizeof(maps));
  EQTL_CHECK(n_acc >= 1 && n_acc <= dev::kMaxAcc && (n_acc == NACC || Epi::kGrouped), EQTL_E_INTERNAL,
             "tile kernel: accumulator count");
  for (int j = 0; j < n_acc; ++j) {
    const int ka = tk && tk->k_a[j] > 0 ? tk->k_a[j] : k_pad;
    make_map_2d(&maps.a[2 * j], a_hi[j], rows_a, ka, dev::kTileM, bf16);
    make_map_2d(&maps.a[2 * j + 1], a_lo[j], rows_a, ka, dev::kTileM, bf16);
  }
  int npairs = 0;
  for (int j = 0; j < n_acc; ++j) npairs = std::max(npairs, bsel[j] + 1);
  for (int b = 0; b < npairs; ++b) {
    const int kb = tk && tk->k_b[b] > 0 ? tk->k_b[b] : k_pad;
    make_map_2d(&maps.b[2 * b], b_hi[b], rows_b, kb, NT, bf16);
    make_map_2d(&maps.b[2 * b + 1], b_lo[b], rows_b, kb, NT, bf16);
  }
  for (int b = npairs; b < 2; ++b) {
    maps.b[2 * b] = maps.b[0];
    maps.b[2 * b + 1] = maps.b[1];
  }
  dev::TileShape sh{};
  sh.rows_a = static_cast<int>(rows_a);
  sh.rows_b = static_cast<int>(rows_b);
  sh.kchunks = k_pad / dev::kChunkK;
  sh.n_acc = n_acc;
  sh.n_groups = (n_acc + NACC - 1) / NACC;
  for (int j = 0; j < dev::kMaxAcc; ++j) {
    sh.bsel[j] = j < n_acc ? bsel[j] : 0;
    sh.prod[j] = j < n_acc ? prod[j] : 0;
    if (tk && j < n_acc && tk->end[j] > 0) {
      // the range lies inside both operands' K extents and is not empty
      const int ka = tk->k_a[j] > 0 ? tk->k_a[j] : k_pad, kb = tk->k_b[sh.bsel[j]] > 0 ? tk->k_b[sh.bsel[j]] : k_pad;
      EQTL_CHECK(tk->beg[j] >= 0 && tk->beg[j] < tk->end[j] && tk->end[j] * dev::kChunkK <= std::min(ka, kb) &&
                     ksplit == 1 && kc_sub == 0,
                 EQTL_E_INTERNAL, "tile kernel: accumulator K range");
      sh.kc_beg[j] = tk->beg[j];
      sh.kc_end[j] = tk->end[j];
    } else {
      EQTL_CHECK(!tk || j >= n_acc || ((tk->k_a[j] <= 0 || tk->k_a[j] == k_pad) &&
                                       (tk->k_b[sh.bsel[j]] <= 0 || tk->k_b[sh.bsel[j]] == k_pad)),
                 EQTL_E_INTERNAL, "tile kernel: an accumulator over all of K needs operands of K extent k_pad");
    }
    EQTL_CHECK(BL != dev::kBLoNone || !(sh.prod[j] & 2), EQTL_E_INTERNAL,
               "tile kernel: hi*lo product without SNP-side lo parts");
  }
  sh.tiles_a = static_cast<int>((rows_a + dev::kTileM - 1) / dev::kTileM);
  sh.tiles_b = static_cast<int>((rows_b + NT - 1) / NT);
  sh.tile_list = tile_list;
  sh.ksplit = std::max(1, std::min(ksplit, sh.kchunks));
  sh.kc_per_split = (sh.kchunks + sh.ksplit - 1) / sh.ksplit;
  sh.ksplit = (sh.kchunks + sh.kc_per_split - 1) / sh.kc_per_split;  // no empty ranges
  sh.n_tiles = (tile_list ? n_tile_list : sh.tiles_a * sh.tiles_b) * sh.ksplit;
  EQTL_CHECK(kc_sub >= 0 && (kc_sub == 0 || (!Epi::kGrouped && !dev::IsTwoPhase<Epi>::value)), EQTL_E_INTERNAL,
             "tile kernel: K sub-ranges need a single-group epilogue");
  sh.kc_sub = kc_sub;
  // gene-side tiles per raster group: keep the group's A operands (hi+lo of
  // every accumulator) within ~48 MB of L2
  {
    const double a_bytes = static_cast<double>(n_acc) * 2.0 * dev::kTileM * k_pad * 2.0;
    sh.group_a = std::max(1, std::min(sh.tiles_a, static_cast<int>(48e6 / a_bytes)));
  }
  sh.status = ctx->d_status;
  if (sh.n_tiles == 0) return;
  EQTL_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream));
  const int grid = std::min(sh.n_tiles, sm_count(ctx));
  ++ctx->launches;
  const int smem = C::SMEM_BYTES + Epi::kSmemBytes;
  EQTL_CHECK(smem <= 232448, EQTL_E_INTERNAL, "tile kernel shared memory over the 227 KB limit");
  if (bf16) {
    auto kern = dev::tile_kernel<NT, NACC, 1u, Epi, BL>;
    EQTL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    kern<<<grid, dev::kTileThreads, smem, ctx->stream>>>(maps, sh, ep);
  } else {
    auto kern = dev::tile_kernel<NT, NACC, 0u, Epi, BL>;
    EQTL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    kern<<<grid, dev::kTileThreads, smem, ctx->stream>>>(maps, sh, ep);
  }
  EQTL_CUDA(cudaGetLastError());
  check_tile_status(ctx, "tile kernel");
}

}  // namespace eqtl
