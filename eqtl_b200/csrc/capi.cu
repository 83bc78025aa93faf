// C ABI of libeqtl_cuda and the host-side helpers shared by the scans.
//
// Every exported function catches all C++ exceptions, stores the message
// in ctx->last_error and returns a negative EQTL_E_* code; nothing throws
// across the ABI (the reference's die()/exception path, src/util.cpp:15-19,
// becomes a status code the caller turns into its own "[E] ..." exit).
#include <cublas_v2.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <map>
#include <mutex>

#include "host_par.hpp"
#include "internal.hpp"
#include "scan_host.hpp"
#include "tstat.hpp"

namespace eqtl {

// ------------------------------------------------------------ tensor maps
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  EQTL_CHECK(fn != nullptr, EQTL_E_CUDA, "cuTensorMapEncodeTiled unavailable");
  return fn;
}

// 2-D map over a row-major [rows, k_pad] 16-bit matrix, box = 64 x box_rows,
// 128-byte swizzle (the layout smem_desc_sw128 describes). Rows past `rows`
// read as zeros.
void make_map_2d(CUtensorMap* map, const void* base, uint64_t rows, uint64_t k_pad, uint32_t box_rows, bool bf16) {
  EQTL_CHECK(base != nullptr && rows > 0, EQTL_E_INTERNAL, "make_map_2d: empty operand");
  EQTL_CHECK(k_pad % 64 == 0, EQTL_E_INTERNAL, "make_map_2d: k_pad must be a multiple of 64");
  EQTL_CHECK((reinterpret_cast<uintptr_t>(base) & 15) == 0, EQTL_E_INTERNAL, "make_map_2d: base not 16B aligned");
  const cuuint64_t dims[2] = {k_pad, rows};
  const cuuint64_t strides[1] = {k_pad * 2};
  const cuuint32_t box[2] = {64, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                           const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  EQTL_CHECK(r == CUDA_SUCCESS, EQTL_E_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(r) + ")");
}

int sm_count(eqtl_ctx* ctx) { return ctx->sm_count; }

void stage_begin(eqtl_ctx* ctx, int stage) {
  StageTimer& T = ctx->timer;
  if (!T.start[stage]) {
    EQTL_CUDA(cudaEventCreate(&T.start[stage]));
    EQTL_CUDA(cudaEventCreate(&T.stop[stage]));
  }
  EQTL_CUDA(cudaEventRecord(T.start[stage], ctx->stream));
}

void stage_end(eqtl_ctx* ctx, int stage) {
  StageTimer& T = ctx->timer;
  if (T.stop[stage] && cudaEventRecord(T.stop[stage], ctx->stream) == cudaSuccess) T.used[stage] = true;
}

void check_tile_status(eqtl_ctx* ctx, const char* what) {
  EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
  uint32_t st = 0;
  EQTL_CUDA(cudaMemcpy(&st, ctx->d_status, sizeof(st), cudaMemcpyDeviceToHost));
  if (st != 0) {
    static const char* names[] = {"ok",          "operand stage timeout", "ring slot timeout",
                                  "accumulator commit timeout", "accumulator drain timeout",
                                  "unwind timeout", "bad shape"};
    throw Error(EQTL_E_DEVICE, std::string(what) + ": device wait expired (" +
                                   (st < 7 ? names[st] : "unknown") + ")");
  }
}

// --------------------------------------------------------- covariate math
std::vector<double> xtx_inverse(const double* X, int n, int p) {
  std::vector<double> A(static_cast<size_t>(p) * p, 0.0);
  for (int a = 0; a < p; ++a)
    for (int b = 0; b <= a; ++b) {
      double s = 0;
      for (int i = 0; i < n; ++i) s += X[static_cast<size_t>(a) * n + i] * X[static_cast<size_t>(b) * n + i];
      A[a * p + b] = A[b * p + a] = s;
    }
  // Cholesky A = L L', then inverse column by column
  std::vector<double> L(A);
  for (int j = 0; j < p; ++j) {
    double d = L[j * p + j];
    for (int k = 0; k < j; ++k) d -= L[j * p + k] * L[j * p + k];
    EQTL_CHECK(d > 0, EQTL_E_ARG, "covariate matrix X'X is singular");
    L[j * p + j] = std::sqrt(d);
    for (int i = j + 1; i < p; ++i) {
      double s = L[i * p + j];
      for (int k = 0; k < j; ++k) s -= L[i * p + k] * L[j * p + k];
      L[i * p + j] = s / L[j * p + j];
    }
  }
  std::vector<double> inv(static_cast<size_t>(p) * p, 0.0), y(p), x(p);
  for (int c = 0; c < p; ++c) {
    for (int i = 0; i < p; ++i) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) s -= L[i * p + k] * y[k];
      y[i] = s / L[i * p + i];
    }
    for (int i = p - 1; i >= 0; --i) {
      double s = y[i];
      for (int k = i + 1; k < p; ++k) s -= L[k * p + i] * x[k];
      x[i] = s / L[i * p + i];
    }
    for (int i = 0; i < p; ++i) inv[i * p + c] = x[i];
  }
  return inv;
}

static cublasHandle_t blas(eqtl_ctx* ctx) {
  if (!ctx->cublas) {
    cublasHandle_t h;
    EQTL_CHECK(cublasCreate(&h) == CUBLAS_STATUS_SUCCESS, EQTL_E_CUDA, "cublasCreate failed");
    cublasSetStream(h, ctx->stream);
    ctx->cublas = h;
  }
  return static_cast<cublasHandle_t>(ctx->cublas);
}

#define EQTL_BLAS(call) EQTL_CHECK((call) == CUBLAS_STATUS_SUCCESS, EQTL_E_CUDA, #call " failed")

void residualize_genes(eqtl_ctx* ctx, const double* dX, const double* dXtXinv, int n, int p, int G, double* dY,
                       double* dXtY) {
  cublasHandle_t h = blas(ctx);
  const double one = 1.0, zero = 0.0, mone = -1.0;
  // XtY = X' Y  [p, G]
  EQTL_BLAS(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, p, G, n, &one, dX, n, dY, n, &zero, dXtY, p));
  // C = XtXinv XtY (XtXinv symmetric; row-major == column-major)
  DevBuf<double>& C = ctx->ws.resid_C;
  C.alloc(static_cast<size_t>(p) * G);
  EQTL_BLAS(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, p, G, p, &one, dXtXinv, p, dXtY, p, &zero, C.p, p));
  // Y <- Y - X C
  EQTL_BLAS(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, G, p, &mone, dX, n, C.p, p, &one, dY, n));
  EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
}



void finish_scan(const eqtl_scan_params* prm, eqtl_gene_result* genes, const std::vector<eqtl_pair>& refined,
                 std::vector<eqtl_pair>& pairs, std::vector<eqtl_pair>& cands) {
  pairs.clear();
  cands.clear();
  const int G = prm->n_genes;
  std::vector<const eqtl_pair*> best(G, nullptr);
  for (const eqtl_pair& q : refined) {
    if (q.p <= prm->pthr) pairs.push_back(q);
    if (prm->perm_thr > 0 && std::isfinite(q.p) && q.p < prm->perm_thr) cands.push_back(q);
    const eqtl_pair*& b = best[q.gene];
    if (!b || q.p < b->p || (q.p == b->p && q.snp < b->snp)) b = &q;
  }
  for (int g = 0; g < G; ++g) {
    eqtl_gene_result& r = genes[g];
    if (r.n_tested > 0 && best[g]) {
      r.best_snp = best[g]->snp;
      r.best_p = best[g]->p;
      r.best_beta = best[g]->beta;
      r.best_se = best[g]->se;
      r.best_t = best[g]->t;
      r.best_r2 = best[g]->r2;
    } else {
      r.best_snp = -1;
      r.best_p = 2.0;
      r.best_beta = r.best_se = r.best_t = r.best_r2 = 0.0;
    }
  }
  {
    // (snp, gene) order through 64-bit keys: snp < 2^31, gene < 2^31
    std::vector<uint64_t> key(pairs.size());
    std::vector<uint32_t> idx(pairs.size());
    for (size_t i = 0; i < pairs.size(); ++i) {
      key[i] = (static_cast<uint64_t>(pairs[i].snp) << 32) | static_cast<uint32_t>(pairs[i].gene);
      idx[i] = static_cast<uint32_t>(i);
    }
    radix_sort_u64(key, &idx);
    std::vector<eqtl_pair> sorted(pairs.size());
    for (size_t i = 0; i < idx.size(); ++i) sorted[i] = pairs[idx[i]];
    pairs.swap(sorted);
  }
  std::sort(cands.begin(), cands.end(), [](const eqtl_pair& a, const eqtl_pair& b) {
    if (a.gene != b.gene) return a.gene < b.gene;
    if (a.p != b.p) return a.p < b.p;
    return a.snp < b.snp;
  });
}

void add_deferred_acat(eqtl_gene_result* genes, const std::vector<eqtl_pair>& refined,
                       const std::vector<int2>& deferred) {
  const long double kPiL = 3.14159265358979323846L;
  // terms on every host thread, then added in pair order (the sums do not
  // depend on the thread count)
  std::vector<double> term(deferred.size());
  std::vector<uint8_t> use(deferred.size());
  std::vector<uint8_t> found(deferred.size());
  parallel_for(deferred.size(), [&](size_t i) {
    const int2 d = deferred[i];
    auto it = std::lower_bound(refined.begin(), refined.end(), d, [](const eqtl_pair& q, const int2& k) {
      return q.gene != k.x ? q.gene < k.x : q.snp < static_cast<int64_t>(k.y);
    });
    found[i] = it != refined.end() && it->gene == d.x && it->snp == d.y;
    if (!found[i]) return;
    double p = it->p;
    use[i] = !(!std::isfinite(p) || p < 0.0 || p >= 1.0 - 1e-12);  // AcatAcc::add guards
    if (!use[i]) return;
    if (p <= 0.0) p = 1e-300;
    term[i] = static_cast<double>(std::tan((0.5L - static_cast<long double>(p)) * kPiL));
  });
  for (size_t i = 0; i < deferred.size(); ++i) {
    EQTL_CHECK(found[i], EQTL_E_INTERNAL, "deferred ACAT pair was not refined");
    if (!use[i]) continue;
    genes[deferred[i].x].acat_tan_sum += term[i];
    ++genes[deferred[i].x].acat_used;
  }
}

void add_acat_terms(eqtl_gene_result* genes, const std::vector<int2>& pairs, const std::vector<double>& p_pairs) {
  const long double kPiL = 3.14159265358979323846L;
  // terms on every host thread, then added in pair order (the sums do not
  // depend on the thread count)
  std::vector<double> term(pairs.size());
  std::vector<uint8_t> use(pairs.size());
  parallel_for(pairs.size(), [&](size_t i) {
    double p = p_pairs[i];
    use[i] = !(!std::isfinite(p) || p < 0.0 || p >= 1.0 - 1e-12);  // AcatAcc::add guards
    if (!use[i]) return;
    if (p <= 0.0) p = 1e-300;
    term[i] = static_cast<double>(std::tan((0.5L - static_cast<long double>(p)) * kPiL));
  });
  for (size_t i = 0; i < pairs.size(); ++i) {
    if (!use[i]) continue;
    eqtl_gene_result& g = genes[pairs[i].x];
    g.acat_tan_sum += term[i];
    ++g.acat_used;
  }
}

dev::Windows upload_windows(eqtl_ctx* ctx, const eqtl_scan_params* prm, int64_t m, int mode) {
  dev::Windows w{};
  w.mode = dev::kWinNone;
  if (mode == dev::kWinNone || !prm->gene_chrom || !prm->gene_lo || !prm->gene_hi || !prm->snp_chrom ||
      !prm->snp_pos)
    return w;
  Workspace& ws = ctx->ws;
  ws.win_gc.upload(prm->gene_chrom, prm->n_genes, ctx->stream);
  ws.win_glo.upload(prm->gene_lo, prm->n_genes, ctx->stream);
  ws.win_ghi.upload(prm->gene_hi, prm->n_genes, ctx->stream);
  ws.win_sc.upload(prm->snp_chrom, m, ctx->stream);
  ws.win_sp.upload(prm->snp_pos, m, ctx->stream);
  w.mode = mode;
  w.gene_chrom = ws.win_gc.p;
  w.gene_lo = ws.win_glo.p;
  w.gene_hi = ws.win_ghi.p;
  w.snp_chrom = ws.win_sc.p;
  w.snp_pos = ws.win_sp.p;
  // 16-SNP block bounds, up to one 256-SNP tile past the last padded tile
  const int64_t nb = ((m + 255) / 256 + 1) * 16;
  std::vector<int32_t> bc(static_cast<size_t>(nb), -1);
  std::vector<int64_t> blo(static_cast<size_t>(nb), 0), bhi(static_cast<size_t>(nb), -1);
  for (int64_t b = 0; b * 16 < m; ++b) {
    const int64_t s1 = std::min<int64_t>(m, b * 16 + 16);
    int32_t c = prm->snp_chrom[b * 16];
    int64_t lo = prm->snp_pos[b * 16], hi = lo;
    for (int64_t s = b * 16 + 1; s < s1; ++s) {
      if (prm->snp_chrom[s] != c) c = -1;
      lo = std::min<int64_t>(lo, prm->snp_pos[s]);
      hi = std::max<int64_t>(hi, prm->snp_pos[s]);
    }
    bc[static_cast<size_t>(b)] = c;
    blo[static_cast<size_t>(b)] = lo;
    bhi[static_cast<size_t>(b)] = hi;
  }
  ws.win_bc.upload(bc.data(), bc.size(), ctx->stream);
  ws.win_blo.upload(blo.data(), blo.size(), ctx->stream);
  ws.win_bhi.upload(bhi.data(), bhi.size(), ctx->stream);
  w.blk_chrom = ws.win_bc.p;
  w.blk_lo = ws.win_blo.p;
  w.blk_hi = ws.win_bhi.p;
  return w;
}

// Banded tile list of a cis scan (scope 2): for every tile of 128 genes, the
// SNP tiles of NT kept SNPs that hold some gene's window. Needs the kept
// SNPs grouped by chromosome in position order (as in a sorted .bim); returns
// false otherwise, and the caller runs the full grid masked to the windows.
bool cis_tile_list(eqtl_ctx* ctx, const eqtl_scan_params* prm, int64_t m, int NT, const int2*& list, int& n_list) {
  list = nullptr;
  n_list = 0;
  if (prm->exclude_cis != 2 || !prm->gene_chrom || !prm->snp_chrom || !prm->snp_pos || m == 0) return false;
  // chromosome blocks [first, last) of the kept SNPs, positions non-decreasing
  std::map<int32_t, std::pair<int64_t, int64_t>> block;
  for (int64_t k = 0; k < m; ++k) {
    const int32_t c = prm->snp_chrom[k];
    auto it = block.find(c);
    if (it == block.end()) {
      block.emplace(c, std::make_pair(k, k + 1));
      continue;
    }
    if (it->second.second != k || prm->snp_pos[k] < prm->snp_pos[k - 1]) return false;
    it->second.second = k + 1;
  }
  const int G = prm->n_genes;
  const int tiles_a = (G + dev::kTileM - 1) / dev::kTileM;
  const int64_t tiles_b = (m + NT - 1) / NT;
  std::vector<uint8_t> mark(static_cast<size_t>(tiles_a) * tiles_b, 0);
  for (int g = 0; g < G; ++g) {
    auto it = block.find(prm->gene_chrom[g]);
    if (prm->gene_chrom[g] < 0 || it == block.end()) continue;
    const int64_t* p0 = prm->snp_pos + it->second.first;
    const int64_t* p1 = prm->snp_pos + it->second.second;
    const int64_t k_lo = std::lower_bound(p0, p1, prm->gene_lo[g]) - prm->snp_pos;
    const int64_t k_hi = std::upper_bound(p0, p1, prm->gene_hi[g]) - prm->snp_pos;  // exclusive
    if (k_hi <= k_lo) continue;
    uint8_t* row = &mark[static_cast<size_t>(g / dev::kTileM) * tiles_b];
    for (int64_t tb = k_lo / NT; tb <= (k_hi - 1) / NT; ++tb) row[tb] = 1;
  }
  std::vector<int2> tl;
  for (int ta = 0; ta < tiles_a; ++ta)
    for (int64_t tb = 0; tb < tiles_b; ++tb)
      if (mark[static_cast<size_t>(ta) * tiles_b + tb]) tl.push_back(make_int2(ta, static_cast<int>(tb)));
  n_list = static_cast<int>(tl.size());
  if (n_list == 0) tl.push_back(make_int2(0, 0));  // keeps a valid (unused) device pointer
  ctx->ws.tile_list.upload(tl.data(), tl.size(), ctx->stream);
  list = ctx->ws.tile_list.p;
  return true;
}

dev::TTable device_ttable(eqtl_ctx* ctx, double df, bool normal) {
  EQTL_CHECK(normal || df > 0, EQTL_E_ARG, "residual degrees of freedom must be positive");
  if (normal) df = kZTableD;
  const double key = normal ? -2.0 : df;  // the normal table is cached under -2 (-1: none uploaded)
  static std::mutex mu;
  static std::map<double, TTableHost> cache;
  TTableHost T;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it == cache.end()) it = cache.emplace(key, build_ttable(df, normal)).first;
    T = it->second;
  }
  Workspace& ws = ctx->ws;
  if (ws.tt_df != key) {
    ws.tt_h.upload(T.h.data(), T.h.size(), ctx->stream);
    ws.tt_L.upload(T.L.data(), T.L.size(), ctx->stream);
    ws.tt_c1.upload(T.c1.data(), T.c1.size(), ctx->stream);
    ws.tt_lt.upload(T.lt.data(), T.lt.size(), ctx->stream);
    ws.tt_c1q.upload(T.c1q.data(), T.c1q.size(), ctx->stream);
    ws.tt_ltq.upload(T.ltq.data(), T.ltq.size(), ctx->stream);
    ws.tt_df = key;
  }
  dev::TTable t{};
  t.h = ws.tt_h.p;
  t.L = ws.tt_L.p;
  t.t0 = static_cast<float>(T.t0);
  t.du_inv = static_cast<float>(T.na / (T.t0 * T.t0));
  t.x0 = static_cast<float>(T.x0);
  t.dx_inv = static_cast<float>(T.nb / (T.x_end - T.x0));
  t.x_end = static_cast<float>(T.x_end);
  t.inv_df = static_cast<float>(1.0 / df);
  // deferral band around t = 0: 256 ulps of df in t^2 (the reference's
  // x = df / (df + t^2) is quantised there) widened by 4x the screening
  // error of t for this precision
  static const double kTErr[3] = {2e-6, 6.4e-5, 2e-6};
  const int prec = ctx->precision >= 0 && ctx->precision < 3 ? ctx->precision : 0;
  const double ulp = std::nextafter(df, std::numeric_limits<double>::infinity()) - df;
  t.tiny_t = static_cast<float>(std::sqrt(256.0 * ulp) + 4.0 * kTErr[prec]);
  t.c1 = ws.tt_c1.p;
  t.lt = ws.tt_lt.p;
  t.dl_inv = static_cast<float>(T.nb / (T.x_defer - T.x0));
  t.lt_u = T.lt_u ? 1 : 0;
  t.dlu_inv = T.lt_u ? static_cast<float>(1.0 / T.du_t) : 0.0f;
  EQTL_CHECK(!T.lt_u || (T.na == dev::kTTableNa && T.nq == dev::kTTableNq), EQTL_E_INTERNAL, "screen table sizes");
  t.c1q = T.lt_u ? reinterpret_cast<const float4*>(ws.tt_c1q.p) : nullptr;
  t.ltq = T.lt_u ? reinterpret_cast<const float4*>(ws.tt_ltq.p) : nullptr;
  t.nq = T.nq;
  t.dq_inv = T.lt_u ? static_cast<float>(1.0 / T.du_q) : 0.0f;
  t.uq0 = static_cast<float>(T.uq0);
  t.dqc_inv = static_cast<float>(T.na / T.uq0);
  // round t_defer down so that every pair with p <= 1e-14 is deferred
  t.t_defer = static_cast<float>(T.t_defer * (1.0 - 1e-6));
  t.u0 = static_cast<float>(T.t0 * T.t0);
  t.u_tiny = t.tiny_t * t.tiny_t;
  t.u_defer = static_cast<float>(T.t_defer * T.t_defer * (1.0 - 2e-6));
  t.na = T.na;
  t.nb = T.nb;
  return t;
}

const PhenoDev& resolve_pheno(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X) {
  PhenoDev& P = ctx->pheno;
  if (Y || X) {
    EQTL_CHECK(Y && X, EQTL_E_ARG, "give both Y and X, or neither to use the resident phenotypes");
    pheno_load(ctx, Y, X, prm->n, prm->n_genes, prm->p);
  }
  EQTL_CHECK(P.Y.p && P.n == prm->n && P.G == prm->n_genes && P.p == prm->p, EQTL_E_STATE,
             "no resident phenotypes of this shape (call eqtl_pheno_load or pass Y and X)");
  return P;
}

void pheno_load(eqtl_ctx* ctx, const double* Y, const double* X, int n, int G, int p) {
  EQTL_CHECK(n > 0 && G > 0 && p > 0, EQTL_E_ARG, "pheno_load: bad sizes");
  PhenoDev& P = ctx->pheno;
  P.n = n;
  P.G = G;
  P.p = p;
  P.Y.upload(Y, static_cast<size_t>(n) * G, ctx->stream);
  P.X.upload(X, static_cast<size_t>(n) * p, ctx->stream);
  P.X_h.assign(X, X + static_cast<size_t>(n) * p);
  EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
}

namespace {
// One instantiation per mode (tables in shared memory or read from global
// memory; the t tail or the ACAT screen), so that every table pointer the
// kernel reads has one address space.
template <bool SMEM, bool SCREEN>
__global__ void t_tail_kernel(dev::TTable T, const float* t, int64_t n, float* nl, double* term, uint8_t* flags) {
  extern __shared__ float4 tsm4[];
  dev::TTable tt = T;
  if constexpr (SMEM) {
    float* tsm = reinterpret_cast<float*>(tsm4);
    if constexpr (SCREEN) tt = dev::screen_to_smem(T, tsm, threadIdx.x, blockDim.x);
    else tt = dev::ttable_to_smem(T, tsm, threadIdx.x, blockDim.x);
    __syncthreads();
  }
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if constexpr (SCREEN) {
    const dev::ScreenOut o = dev::acat_screen(t[i], tt);
    nl[i] = o.key;
    term[i] = o.term;
    flags[i] = static_cast<uint8_t>((o.use_acat ? 1 : 0) | (o.deferred ? 2 : 0) | (o.tiny ? 4 : 0));
    return;
  }
  const dev::TailOut o = dev::t_tail(t[i], tt);
  nl[i] = o.neglog10p;
  term[i] = o.term;
  flags[i] = static_cast<uint8_t>((o.use_acat ? 1 : 0) | (o.deferred ? 2 : 0) | (o.tiny ? 4 : 0));
}

__global__ void fill_u64(unsigned long long* p, int n, unsigned long long v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
}  // namespace

ScanOutputs::ScanOutputs(eqtl_ctx* c, int genes, int64_t m, int64_t cap_hint)
    : ctx(c), G(genes), acat(c->ws.acat), used(c->ws.used), tested(c->ws.tested), best(c->ws.best),
      cand(c->ws.cand), count(c->ws.count) {
  acat.alloc(G);
  used.alloc(G);
  tested.alloc(G);
  best.alloc(G);
  count.alloc(1);
  cap = static_cast<unsigned int>(std::min<int64_t>(std::max<int64_t>(cap_hint, 1 << 16), 1 << 26));
  cand.alloc(cap);
  (void)m;
}

void ScanOutputs::reset() {
  EQTL_CUDA(cudaMemsetAsync(acat.p, 0, sizeof(double) * G, ctx->stream));
  EQTL_CUDA(cudaMemsetAsync(used.p, 0, sizeof(int) * G, ctx->stream));
  EQTL_CUDA(cudaMemsetAsync(tested.p, 0, sizeof(int) * G, ctx->stream));
  EQTL_CUDA(cudaMemsetAsync(count.p, 0, sizeof(unsigned int), ctx->stream));
  fill_u64<<<(G + 255) / 256, 256, 0, ctx->stream>>>(best.p, G, ~0ull);
  EQTL_CUDA(cudaGetLastError());
}

void ScanOutputs::run(const std::function<void(dev::GeneOut)>& launch) {
  for (int attempt = 0; attempt < 3; ++attempt) {
    reset();
    dev::GeneOut o{acat.p, used.p, tested.p, best.p, cand.p, count.p, cap};
    launch(o);
    EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
    count.download(&n_cand, 1, ctx->stream);
    EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
    if (n_cand <= cap) return;
    EQTL_CHECK(n_cand <= (1u << 28), EQTL_E_OVERFLOW,
               "scan produced " + std::to_string(n_cand) + " candidate pairs; lower the p threshold");
    cap = n_cand + n_cand / 8;
    cand.alloc(cap);
  }
  throw Error(EQTL_E_INTERNAL, "candidate buffer did not converge");
}

void ScanOutputs::collect(eqtl_gene_result* genes, std::vector<int2>& todo, std::vector<int2>& deferred,
                          std::vector<int2>* tiny) {
  std::vector<double> a(G);
  std::vector<int> u(G), t(G);
  std::vector<unsigned long long> b(G);
  acat.download(a.data(), G, ctx->stream);
  used.download(u.data(), G, ctx->stream);
  tested.download(t.data(), G, ctx->stream);
  best.download(b.data(), G, ctx->stream);
  std::vector<int2> c(n_cand);
  cand.download(c.data(), n_cand, ctx->stream);
  EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
  todo.clear();
  deferred.clear();
  if (tiny) tiny->clear();
  for (const int2& q : c) {
    const uint32_t s = static_cast<uint32_t>(q.y);
    const int2 clean = make_int2(q.x, static_cast<int>(s & ~(dev::kCandDeferred | dev::kCandTiny)));
    if (tiny && (s & dev::kCandTiny)) {
      tiny->push_back(clean);
      continue;
    }
    todo.push_back(clean);
    if (s & dev::kCandDeferred) deferred.push_back(clean);
  }
  for (int g = 0; g < G; ++g) {
    genes[g].n_tested = t[g];
    genes[g].acat_used = u[g];
    genes[g].acat_tan_sum = a[g];
    genes[g].best_snp = -1;
    if (t[g] > 0 && b[g] != ~0ull) todo.push_back(make_int2(g, static_cast<int>(b[g] & 0xFFFFFFFFull)));
  }
  // (gene, snp) order without duplicates, through 64-bit keys
  std::vector<uint64_t> key(todo.size());
  for (size_t i = 0; i < todo.size(); ++i)
    key[i] = (static_cast<uint64_t>(static_cast<uint32_t>(todo[i].x)) << 32) | static_cast<uint32_t>(todo[i].y);
  radix_sort_u64(key);
  key.erase(std::unique(key.begin(), key.end()), key.end());
  todo.resize(key.size());
  for (size_t i = 0; i < key.size(); ++i)
    todo[i] = make_int2(static_cast<int>(key[i] >> 32), static_cast<int>(key[i] & 0xFFFFFFFFull));
}

}  // namespace eqtl

// ===================================================================== ABI
using eqtl::Error;

template <class F>
static int guarded(eqtl_ctx* ctx, F&& f) {
  if (!ctx) return EQTL_E_ARG;
  try {
    EQTL_CUDA(cudaSetDevice(ctx->device));
    f();
    ctx->last_error.clear();
    return EQTL_OK;
  } catch (const Error& e) {
    ctx->last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    ctx->last_error = "host allocation failed";
    return EQTL_E_NOMEM;
  } catch (const std::exception& e) {
    ctx->last_error = e.what();
    return EQTL_E_INTERNAL;
  }
}

extern "C" {

int eqtl_open(int device, eqtl_ctx** out) {
  if (!out) return EQTL_E_ARG;
  *out = nullptr;
  auto* ctx = new (std::nothrow) eqtl_ctx;
  if (!ctx) return EQTL_E_NOMEM;
  ctx->device = device;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev) {
    delete ctx;
    return EQTL_E_CUDA;
  }
  int rc = guarded(ctx, [&] {
    cudaDeviceProp prop;
    EQTL_CUDA(cudaGetDeviceProperties(&prop, device));
    EQTL_CHECK(prop.major == 10 && prop.minor == 0, EQTL_E_UNSUPPORTED,
               std::string("libeqtl_cuda is built for sm_100a (B200); device is ") + prop.name);
    ctx->sm_count = prop.multiProcessorCount;
    EQTL_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    EQTL_CUDA(cudaMalloc(&ctx->d_status, sizeof(uint32_t)));
    EQTL_CUDA(cudaMemset(ctx->d_status, 0, sizeof(uint32_t)));
    // the allocation-free GRM's static scratch and kernels are loaded here,
    // while the caller can still allocate, not in its first call
    eqtl::grm_noalloc_prepare(ctx);
  });
  if (rc != EQTL_OK) {
    eqtl_close(ctx);
    return rc;
  }
  *out = ctx;
  return EQTL_OK;
}

void eqtl_close(eqtl_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->cublas) cublasDestroy(static_cast<cublasHandle_t>(ctx->cublas));
  eqtl::solver_release(ctx);
  if (ctx->d_status) cudaFree(ctx->d_status);
  for (int i = 0; i < EQTL_N_STAGES; ++i) {
    if (ctx->timer.start[i]) cudaEventDestroy(ctx->timer.start[i]);
    if (ctx->timer.stop[i]) cudaEventDestroy(ctx->timer.stop[i]);
  }
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* eqtl_last_error(const eqtl_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int eqtl_set_precision(eqtl_ctx* ctx, int precision) {
  return guarded(ctx, [&] {
    EQTL_CHECK(precision == EQTL_PREC_SPLIT_F16 || precision == EQTL_PREC_SPLIT_BF16 ||
                   precision == EQTL_PREC_FP32_SIMT,
               EQTL_E_ARG, "unknown precision");
    EQTL_CHECK(ctx->geno.m_all == 0, EQTL_E_STATE, "set the precision before loading genotypes");
    ctx->precision = precision;
  });
}

int eqtl_stage_ms(eqtl_ctx* ctx, int stage, double* ms) {
  return guarded(ctx, [&] {
    EQTL_CHECK(stage >= 0 && stage < EQTL_N_STAGES && ms, EQTL_E_ARG, "bad stage");
    EQTL_CHECK(ctx->timer.used[stage], EQTL_E_STATE, "stage has not run");
    EQTL_CUDA(cudaEventSynchronize(ctx->timer.stop[stage]));
    float f = 0;
    EQTL_CUDA(cudaEventElapsedTime(&f, ctx->timer.start[stage], ctx->timer.stop[stage]));
    *ms = f;
  });
}

int eqtl_launch_count(eqtl_ctx* ctx, uint64_t* count) {
  return guarded(ctx, [&] {
    EQTL_CHECK(count, EQTL_E_ARG, "null output");
    *count = ctx->launches;
  });
}

int eqtl_lmm_form(eqtl_ctx* ctx, int32_t* nodes, int32_t* node_cols) {
  return guarded(ctx, [&] {
    EQTL_CHECK(nodes && node_cols, EQTL_E_ARG, "null output");
    *nodes = ctx->ws.lr_nodes;
    *node_cols = ctx->ws.lr_nodes > 0 ? ctx->ws.lr_kn : 0;
  });
}

int eqtl_stream(eqtl_ctx* ctx, void** stream) {
  return guarded(ctx, [&] {
    EQTL_CHECK(stream, EQTL_E_ARG, "null output");
    *stream = static_cast<void*>(ctx->stream);
  });
}

int eqtl_lmm_rotate(eqtl_ctx* ctx) {
  return guarded(ctx, [&] {
    ctx->rot.m = 0;
    eqtl::lmm_rotate(ctx);
  });
}

int eqtl_geno_load_bed(eqtl_ctx* ctx, const uint8_t* rows, int64_t m, int64_t bytes_per_snp, int32_t n_file,
                       const int32_t* sample_col, int32_t n, int32_t miss_hand, double max_miss, double maf_min,
                       uint8_t* keep_out, double* af_out, int32_t* n_miss_out, int64_t* n_kept_out) {
  return guarded(ctx, [&] {
    EQTL_CHECK((rows || m == 0) && sample_col, EQTL_E_ARG, "null input");
    eqtl::geno_load(ctx, rows, m, bytes_per_snp, n_file, sample_col, n, miss_hand, max_miss, maf_min);
    const eqtl::Geno& g = ctx->geno;
    if (keep_out) {
      std::fill(keep_out, keep_out + m, 0);
      for (int64_t s : g.kept_h) keep_out[s] = 1;
    }
    if (af_out) std::copy(g.af_h.begin(), g.af_h.end(), af_out);
    if (n_miss_out) std::copy(g.n_miss_h.begin(), g.n_miss_h.end(), n_miss_out);
    if (n_kept_out) *n_kept_out = g.m;
  });
}

int eqtl_geno_load_dosage(eqtl_ctx* ctx, const float* ds, int64_t m, int32_t n_file, const int32_t* sample_col,
                          int32_t n, int32_t miss_hand, double max_miss, double maf_min, uint8_t* keep_out,
                          double* af_out, int32_t* n_miss_out, int64_t* n_kept_out) {
  return guarded(ctx, [&] {
    EQTL_CHECK((ds || m == 0) && sample_col, EQTL_E_ARG, "null input");
    eqtl::geno_load_dosage(ctx, ds, m, n_file, sample_col, n, miss_hand, max_miss, maf_min);
    const eqtl::Geno& g = ctx->geno;
    if (keep_out) {
      std::fill(keep_out, keep_out + m, 0);
      for (int64_t s : g.kept_h) keep_out[s] = 1;
    }
    if (af_out) std::copy(g.af_h.begin(), g.af_h.end(), af_out);
    if (n_miss_out) std::copy(g.n_miss_h.begin(), g.n_miss_h.end(), n_miss_out);
    if (n_kept_out) *n_kept_out = g.m;
  });
}

int eqtl_vcf_parse(eqtl_ctx* ctx, const char* text, int64_t text_len, const int64_t* beg, const int64_t* end,
                   const int32_t* gt_at, const int32_t* ds_at, int64_t n_rec, int32_t n_file, int32_t dense,
                   uint8_t* codes_out, float* ds_out, uint8_t* hap_out, uint8_t* flag_out) {
  return guarded(ctx, [&] {
    EQTL_CHECK((text || text_len == 0) && ((beg && end && gt_at && ds_at && hap_out && flag_out) || n_rec == 0),
               EQTL_E_ARG, "null input");
    EQTL_CHECK(dense ? (ds_out != nullptr || n_rec == 0) : (codes_out != nullptr || n_rec == 0), EQTL_E_ARG,
               "null output");
    eqtl::vcf_parse(ctx, text, text_len, beg, end, gt_at, ds_at, n_rec, n_file, dense, codes_out, ds_out, hap_out,
                    flag_out);
  });
}

int eqtl_geno_dosage(eqtl_ctx* ctx, int64_t lo, int64_t hi, double* out) {
  return guarded(ctx, [&] {
    EQTL_CHECK(out || hi == lo, EQTL_E_ARG, "null output");
    eqtl::geno_dosage(ctx, lo, hi, out);
  });
}

int eqtl_test_pairs(eqtl_ctx* ctx, int32_t model, const eqtl_scan_params* prm, const double* Y, const double* X,
                    const int32_t* pair_col, const int64_t* pair_snp, int64_t n_pairs, eqtl_pair* out,
                    double* delta_out) {
  return guarded(ctx, [&] {
    EQTL_CHECK(prm && ((pair_col && pair_snp && out) || n_pairs == 0), EQTL_E_ARG, "null input");
    EQTL_CHECK(model == EQTL_MODEL_LM || model == EQTL_MODEL_LMM, EQTL_E_ARG, "model must be EQTL_MODEL_LM or _LMM");
    std::vector<int2> todo(static_cast<size_t>(n_pairs));
    for (int64_t i = 0; i < n_pairs; ++i) {
      EQTL_CHECK(pair_snp[i] >= 0 && pair_snp[i] < (int64_t(1) << 31), EQTL_E_ARG, "pair SNP index out of range");
      todo[i] = make_int2(pair_col[i], static_cast<int>(pair_snp[i]));
    }
    if (model == EQTL_MODEL_LM) {
      eqtl::test_pairs_lm(ctx, prm, Y, X, todo, out);
    } else {
      EQTL_CHECK(ctx->have_basis, EQTL_E_STATE, "the LMM needs an eigenbasis (eqtl_lmm_basis)");
      eqtl::test_pairs_lmm(ctx, prm, Y, X, todo, out, delta_out);
    }
  });
}

int eqtl_geno_dosage_rows(eqtl_ctx* ctx, const int64_t* rows, int64_t k, double* out) {
  return guarded(ctx, [&] {
    EQTL_CHECK((rows && out) || k == 0, EQTL_E_ARG, "null input");
    eqtl::geno_dosage_rows(ctx, rows, k, out);
  });
}

int eqtl_t_tail(eqtl_ctx* ctx, double df, const float* t, int64_t n, int32_t use_smem, float* neglog10p,
                double* term, uint8_t* flags) {
  return guarded(ctx, [&] {
    EQTL_CHECK(t && neglog10p && term && flags && n >= 0, EQTL_E_ARG, "null input");
    if (n == 0) return;
    const eqtl::dev::TTable T = eqtl::device_ttable(ctx, df);
    eqtl::DevBuf<float> dt, dn;
    eqtl::DevBuf<double> dterm;
    eqtl::DevBuf<uint8_t> dfl;
    dt.upload(t, n, ctx->stream);
    dn.alloc(n);
    dterm.alloc(n);
    dfl.alloc(n);
    ++ctx->launches;
    const unsigned grid = static_cast<unsigned>((n + 255) / 256);
    const size_t sm = eqtl::dev::kTTableSmemBytes;
    switch (use_smem & 3) {
      case 0: eqtl::t_tail_kernel<false, false><<<grid, 256, 0, ctx->stream>>>(T, dt.p, n, dn.p, dterm.p, dfl.p); break;
      case 1: eqtl::t_tail_kernel<true, false><<<grid, 256, sm, ctx->stream>>>(T, dt.p, n, dn.p, dterm.p, dfl.p); break;
      case 2: eqtl::t_tail_kernel<false, true><<<grid, 256, 0, ctx->stream>>>(T, dt.p, n, dn.p, dterm.p, dfl.p); break;
      default: eqtl::t_tail_kernel<true, true><<<grid, 256, sm, ctx->stream>>>(T, dt.p, n, dn.p, dterm.p, dfl.p); break;
    }
    EQTL_CUDA(cudaGetLastError());
    dn.download(neglog10p, n, ctx->stream);
    dterm.download(term, n, ctx->stream);
    dfl.download(flags, n, ctx->stream);
    EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int eqtl_geno_subset(eqtl_ctx* ctx, const int32_t* idx, int32_t n_sub) {
  return guarded(ctx, [&] { eqtl::geno_subset(ctx, idx, n_sub); });
}

int eqtl_pheno_load(eqtl_ctx* ctx, const double* Y, const double* X, int32_t n, int32_t n_genes, int32_t p) {
  return guarded(ctx, [&] {
    EQTL_CHECK(Y && X, EQTL_E_ARG, "null input");
    eqtl::pheno_load(ctx, Y, X, n, n_genes, p);
  });
}

int eqtl_pheno_permute(eqtl_ctx* ctx, const double* base, const double* xb0, const double* dinv,
                       const uint64_t* gene_key, int32_t n, int32_t n_genes, int32_t n_perm, uint64_t seed,
                       const double* X, int32_t p, double* Y_out) {
  return guarded(ctx, [&] {
    EQTL_CHECK(base && gene_key && X, EQTL_E_ARG, "null input");
    eqtl::pheno_permute(ctx, base, xb0, dinv, gene_key, n, n_genes, n_perm, seed, X, p, Y_out);
  });
}

int eqtl_peer(eqtl_ctx* ctx, const double* Y, int32_t n, int32_t n_genes, int32_t K, int32_t max_iter, double tol,
              const double* X0, const double* W0, double* X_out, int32_t* iters_out) {
  return guarded(ctx, [&] {
    EQTL_CHECK(Y && X0 && W0 && X_out, EQTL_E_ARG, "null input");
    const int it = eqtl::peer_factors(ctx, Y, n, n_genes, K, max_iter, tol, X0, W0, X_out);
    if (iters_out) *iters_out = it;
  });
}

int eqtl_pheno_int(eqtl_ctx* ctx, double* Y, int32_t n, int32_t n_cols) {
  return guarded(ctx, [&] {
    EQTL_CHECK(Y, EQTL_E_ARG, "null input");
    eqtl::pheno_int(ctx, Y, n, n_cols);
  });
}

int eqtl_grm(eqtl_ctx* ctx, double* K_out, int32_t* N_packed_out, int64_t* m_used_out) {
  return guarded(ctx, [&] {
    eqtl::DevBuf<double>& K = ctx->ws.basis_K;
    eqtl::DevBuf<int32_t>& N = ctx->ws.basis_N;
    const int64_t mu = eqtl::grm_compute(ctx, K, N);
    const int n = ctx->geno.n;
    if (K_out) K.download(K_out, static_cast<size_t>(n) * n, ctx->stream);
    if (N_packed_out) N.download(N_packed_out, static_cast<size_t>(n) * (n + 1) / 2, ctx->stream);
    EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
    if (m_used_out) *m_used_out = mu;
  });
}

int eqtl_grm_noalloc(eqtl_ctx* ctx, const uint8_t* bed_dev, int64_t m, int64_t bytes_per_snp,
                     const int32_t* sample_col_dev, int32_t n, int32_t miss_hand, double max_miss, double maf_min,
                     double* K_dev, int32_t* N_packed_dev, int64_t* m_used_out) {
  return guarded(ctx, [&] {
    const int64_t mu = eqtl::grm_noalloc(ctx, bed_dev, m, bytes_per_snp, sample_col_dev, n, miss_hand, max_miss,
                                         maf_min, K_dev, N_packed_dev);
    if (m_used_out) *m_used_out = mu;
  });
}

int eqtl_lmm_basis(eqtl_ctx* ctx, const double* K, int32_t n, double* lambda_out, double* Q_out) {
  return eqtl_lmm_basis_fast(ctx, K, n, 0.0, lambda_out, Q_out, nullptr);
}

int eqtl_lmm_basis_fast(eqtl_ctx* ctx, const double* K, int32_t n, double sparsify_thr, double* lambda_out,
                        double* Q_out, int64_t* zeroed_out) {
  return guarded(ctx, [&] {
    EQTL_CHECK(sparsify_thr >= 0.0, EQTL_E_ARG, "sparsify threshold must be >= 0");
    eqtl::DevBuf<double>& dK = ctx->ws.basis_K;
    if (K) {
      EQTL_CHECK(n > 0, EQTL_E_ARG, "n must be positive");
      dK.upload(K, static_cast<size_t>(n) * n, ctx->stream);
    } else {
      eqtl::grm_compute(ctx, dK, ctx->ws.basis_N);
      n = ctx->geno.n;
    }
    eqtl::lmm_basis_from_grm(ctx, dK.p, n, sparsify_thr, zeroed_out);
    if (lambda_out) std::copy(ctx->basis.lambda_h.begin(), ctx->basis.lambda_h.end(), lambda_out);
    if (Q_out) {
      ctx->basis.Q.download(Q_out, static_cast<size_t>(n) * n, ctx->stream);
      EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
    }
  });
}

int eqtl_lmm_set_basis(eqtl_ctx* ctx, const double* Q, const double* lambda, int32_t n) {
  return guarded(ctx, [&] {
    EQTL_CHECK(Q && lambda && n > 0, EQTL_E_ARG, "null basis");
    eqtl::lmm_set_basis(ctx, Q, lambda, n);
  });
}

int eqtl_scan_trans_lmm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                        double* delta_out, eqtl_gene_result* genes, eqtl_pair* pairs, int64_t pair_cap,
                        int64_t* n_pairs, eqtl_pair* cands, int64_t cand_cap, int64_t* n_cands) {
  return guarded(ctx, [&] {
    EQTL_CHECK(prm && genes, EQTL_E_ARG, "null input");
    std::vector<eqtl_pair> pv, cv;
    if (ctx->precision == EQTL_PREC_FP32_SIMT)
      eqtl::scan_trans_lmm_simt(ctx, prm, Y, X, delta_out, genes, pv, cv);
    else
      eqtl::scan_trans_lmm(ctx, prm, Y, X, delta_out, genes, pv, cv);
    if (n_pairs) *n_pairs = static_cast<int64_t>(pv.size());
    if (n_cands) *n_cands = static_cast<int64_t>(cv.size());
    EQTL_CHECK(static_cast<int64_t>(pv.size()) <= pair_cap && static_cast<int64_t>(cv.size()) <= cand_cap,
               EQTL_E_OVERFLOW, "result buffer too small");
    if (!pv.empty()) std::copy(pv.begin(), pv.end(), pairs);
    if (!cv.empty()) std::copy(cv.begin(), cv.end(), cands);
  });
}

int eqtl_scan_glm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X, double* phi_out,
                  uint8_t* converged_out, eqtl_gene_result* genes, eqtl_pair* pairs, int64_t pair_cap,
                  int64_t* n_pairs, eqtl_pair* cands, int64_t cand_cap, int64_t* n_cands) {
  return guarded(ctx, [&] {
    EQTL_CHECK(prm && genes, EQTL_E_ARG, "null input");
    std::vector<eqtl_pair> pv, cv;
    eqtl::scan_glm(ctx, prm, Y, X, phi_out, converged_out, genes, pv, cv);
    if (n_pairs) *n_pairs = static_cast<int64_t>(pv.size());
    if (n_cands) *n_cands = static_cast<int64_t>(cv.size());
    EQTL_CHECK(static_cast<int64_t>(pv.size()) <= pair_cap && static_cast<int64_t>(cv.size()) <= cand_cap,
               EQTL_E_OVERFLOW, "result buffer too small");
    if (!pv.empty()) std::copy(pv.begin(), pv.end(), pairs);
    if (!cv.empty()) std::copy(cv.begin(), cv.end(), cands);
  });
}

int eqtl_glm_mu(eqtl_ctx* ctx, double* mu_out) {
  return guarded(ctx, [&] {
    EQTL_CHECK(mu_out, EQTL_E_ARG, "null output");
    EQTL_CHECK(ctx->ws.glm_mu.p && ctx->ws.glm_mu.n > 0, EQTL_E_STATE, "no GLM scan has run");
    ctx->ws.glm_mu.download(mu_out, ctx->ws.glm_mu.n, ctx->stream);
    EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int eqtl_scan_trans_lm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                       eqtl_gene_result* genes, eqtl_pair* pairs, int64_t pair_cap, int64_t* n_pairs,
                       eqtl_pair* cands, int64_t cand_cap, int64_t* n_cands) {
  return guarded(ctx, [&] {
    EQTL_CHECK(prm && genes, EQTL_E_ARG, "null input");
    EQTL_CHECK(ctx->precision != EQTL_PREC_FP32_SIMT, EQTL_E_UNSUPPORTED,
               "the FP32 CUDA-core comparator is available for the LMM scan only");
    std::vector<eqtl_pair> pv, cv;
    eqtl::scan_trans_lm(ctx, prm, Y, X, genes, pv, cv);
    if (n_pairs) *n_pairs = static_cast<int64_t>(pv.size());
    if (n_cands) *n_cands = static_cast<int64_t>(cv.size());
    EQTL_CHECK(static_cast<int64_t>(pv.size()) <= pair_cap && static_cast<int64_t>(cv.size()) <= cand_cap,
               EQTL_E_OVERFLOW, "result buffer too small");
    if (!pv.empty()) std::copy(pv.begin(), pv.end(), pairs);
    if (!cv.empty()) std::copy(cv.begin(), cv.end(), cands);
  });
}

}  // extern "C"
