// K4: trans/gw LM scan (and the LM half of the cis scan).
//
// Restates scan_lm_snp_outer's shared-keep path (src/scan_trans_lm.cpp:41-120)
// as one persistent tcgen05 launch over gene x SNP tiles:
//   prep      y_s = y - X (X'X)^-1 X'y, yty = |y_s|^2 per gene (cuBLAS DGEMM,
//             src/model_lm.cpp:19-30); gtg_s = |g - X (X'X)^-1 X'g|^2 per SNP
//             in FP64 (residualize_g, :11-19);
//   contract  gty[g, s] = y_s . g_s on the tensor cores: y_s and the centred
//             dosage both as FP16 hi/lo pairs, FP32 accumulate (centring is
//             free: y_s is orthogonal to the intercept);
//   epilogue  hit_from_gty's t (:21-36) in FP64, the Student-t tail from the
//             df table, ACAT / n_tested / best-SNP key per gene, and
//             compaction of candidate pairs |t| >= t_cand;
//   refine    every candidate (and each gene's best SNP) recomputed in FP64
//             from the exact decoded dosages, so printed rows use the
//             reference's formulas at FP64.
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <memory>

#include "internal.hpp"
#include "scan_common.cuh"
#include "scan_host.hpp"
#include "tstat.hpp"

namespace eqtl {
namespace dev {

struct LmEpiParams {
  int G;
  int64_t m;
  const double* inv_yty;   // [G] 1 / yty (0 when yty == 0)
  const float* gscale;     // [G] gene-side factor of the accumulator -> gty
  // [m, padded to 16] per SNP, in FP32: a^2 / gtg with a the SNP-side factor
  // of the accumulator -> gty (0 where gtg < 1e-12: tested with p = 1; -1
  // where the SNP is not tested: subset gate, src/scan_common.cpp:133-151,
  // and the padding)
  const float* igs;
  Windows win;
  float df;
  float t_cand;
  TTable tt;
  GeneOut out;
};

struct LmEpi {
  static constexpr bool kGrouped = false;
  using Params = LmEpiParams;
  static constexpr int kSmemBytes = kTTableSmemBytes;
  const Params& P;
  float* tsm;
  TTable tt;
  int gene = 0;
  int64_t snp0 = 0;
  bool gvalid = false;
  float w = 0;   // gscale^2 / yty
  float u_cand;  // t_cand^2
  GeneAcc acc;

  __device__ LmEpi(const Params& p, const TileShape&, uint8_t* smem)
      : P(p), tsm(reinterpret_cast<float*>(smem)), tt(p.tt), u_cand(p.t_cand * p.t_cand) {}
  __device__ void init(int tid, int nthr) {
    if (tsm) tt = screen_to_smem(P.tt, tsm, tid, nthr);
  }
  __device__ void begin_tile(int g, int64_t s0) {
    gene = g;
    snp0 = s0;
    gvalid = g < P.G;
    acc.reset();
    if (gvalid) {
      const float gs = P.gscale[g];
      w = gs * gs * static_cast<float>(P.inv_yty[g]);
      acc.load_window(P.win, g);
    }
  }
  // t^2 = df r / (1 - r), r = gty^2 / (gtg yty) = acc^2 (a^2 / gtg) (gscale^2 / yty)
  // (hit_from_gty algebra), screened in FP32 without branches and without t
  // itself; printed statistics come from the FP64 refinement.
  template <int NACC>
  __device__ void chunk(int c, const float (&v)[NACC][16]) {
    const int64_t s0 = snp0 + c;
    if (!gvalid || s0 >= P.m) return;
    // the 16 SNPs' factors: s0 is a multiple of 16 and the array is padded
    float igv[16];
    const float4* ig4 = reinterpret_cast<const float4*>(P.igs + s0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 v4 = __ldg(ig4 + q);
      igv[4 * q] = v4.x;
      igv[4 * q + 1] = v4.y;
      igv[4 * q + 2] = v4.z;
      igv[4 * q + 3] = v4.w;
    }
    if (tt.lt_u) {  // uniform across the launch
      // a gw scan (no windows), and a trans scan on a chunk clear of every
      // lane's gene window, skip the per-pair window test; the vote keeps
      // the warp on one path
      if (P.win.mode == kWinNone)
        chunk_cubic<false>(s0, v[0], igv);
      else if (P.win.mode == kWinExclude && __all_sync(__activemask(), acc.chunk_clear(P.win, s0)))
        chunk_cubic<false>(s0, v[0], igv);
      else
        chunk_cubic<true>(s0, v[0], igv);
      return;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int64_t s = s0 + j;
      const bool valid = igv[j] >= 0.0f && acc.in_scope(P.win, s);
      const float ig = valid ? igv[j] * w : 0.0f;
      const float r = v[0][j] * v[0][j] * ig;
      const float omr = 1.0f - r;
      const float u = (ig > 0.0f && omr > 0.0f) ? P.df * __fdividef(r, omr) : 0.0f;  // t^2
      const ScreenOut o = acat_screen_u(u, tt);
      acc.add_screen(o, s, valid);
      if (valid && (u >= u_cand || o.deferred)) emit_candidate(P.out, gene, s, o.deferred, o.tiny);
    }
    acc.end_chunk();
  }
  // The same screen with the per-interval cubics (screen16_cubic): u is
  // never NaN here (a pair outside the scan or with p = 1 has u = 0).
  template <bool WIN>
  __device__ void chunk_cubic(int64_t s0, const float (&v)[16], const float (&igv)[16]) {
    float u[16];
    bool valid[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      valid[j] = igv[j] >= 0.0f && (!WIN || acc.in_scope(P.win, s0 + j));
      const float ig = valid[j] ? igv[j] * w : 0.0f;
      const float r = v[j] * v[j] * ig;
      const float omr = 1.0f - r;
      u[j] = (ig > 0.0f && omr > 0.0f) ? P.df * __fdividef(r, omr) : 0.0f;  // t^2
    }
    screen16_cubic(tt, u, valid, u_cand, P.out, gene, s0, acc);
  }
  __device__ void end_tile() {
    if (gvalid) acc.flush(P.out, gene);
  }
  __device__ void finish() {}
};

// The epilogue's per-SNP factor (LmEpiParams::igs) for the padded range
// [0, count): alpha^2 / gtg (alpha null: 1) where the SNP is tested, -1
// elsewhere.
__global__ void lm_igs_kernel(const double* __restrict__ inv_gtg, const uint8_t* __restrict__ ok,
                              const float* __restrict__ alpha, int64_t m, int64_t count, float* out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float v = -1.0f;
    if (i < m && ok[i]) {
      const double a = alpha ? static_cast<double>(alpha[i]) : 1.0;
      v = static_cast<float>(a * a * inv_gtg[i]);
    }
    out[i] = v;
  }
}

// ---------------------------------------------------------------- prep
// One block per gene: yty, power-of-two scale, FP16/BF16 hi/lo rows.
template <class T>
__global__ void gene_split_kernel(const double* __restrict__ Ys, int n, int k_pad, int G, T* hi, T* lo,
                                  float* gscale, double* yty_out, double* inv_yty, float snp_scale) {
  const int g = blockIdx.x;
  if (g >= G) return;
  const double* y = Ys + static_cast<int64_t>(g) * n;
  __shared__ double red[32];
  __shared__ double redm[32];
  double ss = 0, mx = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = y[i];
    ss += v * v;
    mx = fmax(mx, fabs(v));
  }
  for (int o = 16; o; o >>= 1) {
    ss += __shfl_xor_sync(0xffffffffu, ss, o);
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = ss;
    redm[threadIdx.x >> 5] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < (blockDim.x >> 5); ++w) {
      a += red[w];
      b = fmax(b, redm[w]);
    }
    red[0] = a;
    redm[0] = b;
  }
  __syncthreads();
  const double yty = red[0];
  const double mxv = redm[0];
  // scale so the largest |entry| lands in [2^10, 2^11): no FP16 overflow,
  // lo parts stay normal
  int e = 0;
  if (mxv > 0) e = 10 - static_cast<int>(floor(log2(mxv)));
  const double sc = ldexp(1.0, e);
  for (int k = threadIdx.x; k < k_pad; k += blockDim.x) {
    const double v = k < n ? y[k] * sc : 0.0;
    T h, l;
    if constexpr (sizeof(T) == 2 && std::is_same<T, __half>::value) {
      h = __double2half(v);
      l = __double2half(v - static_cast<double>(__half2float(h)));
    } else {
      h = __double2bfloat16(v);
      l = __double2bfloat16(v - static_cast<double>(__bfloat162float(h)));
    }
    hi[static_cast<int64_t>(g) * k_pad + k] = h;
    lo[static_cast<int64_t>(g) * k_pad + k] = l;
  }
  if (threadIdx.x == 0) {
    gscale[g] = static_cast<float>(1.0 / (sc * snp_scale));
    yty_out[g] = yty;
    inv_yty[g] = yty > 0 ? 1.0 / yty : 0.0;
  }
}

constexpr int kMaxP = 32;

// One warp per kept SNP: FP64 |g_s|^2 with the exact decoded dosage, and the
// subset gate on the analysis samples.
__global__ void snp_gtg_kernel(GenoRows src, const int32_t* __restrict__ col, int n,
                               const int64_t* __restrict__ kept, int64_t m, const double* __restrict__ mu,
                               const int32_t* __restrict__ n_miss, const double* __restrict__ s1,
                               const double* __restrict__ s2, const double* __restrict__ X, int p,
                               const double* __restrict__ XtXinv, double* gtg_out, double* inv_gtg, uint8_t* ok,
                               double* af_sub) {
  const int lane = threadIdx.x & 31;
  const int64_t r = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= m) return;
  const int64_t s = kept[r];
  const double mus = mu[s];
  double gg = 0;
  double v[kMaxP];
#pragma unroll
  for (int k = 0; k < kMaxP; ++k) v[k] = 0;
  for (int i = lane; i < n; i += 32) {
    const double d = src.dosage(s, __ldg(col + i));
    const double gc = isnan(d) ? 0.0 : d - mus;
    gg += gc * gc;
#pragma unroll
    for (int k = 0; k < kMaxP; ++k)
      if (k < p) v[k] += __ldg(X + static_cast<int64_t>(k) * n + i) * gc;
  }
  for (int o = 16; o; o >>= 1) {
    gg += __shfl_xor_sync(0xffffffffu, gg, o);
#pragma unroll
    for (int k = 0; k < kMaxP; ++k)
      if (k < p) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  }
  if (lane) return;
  double q = 0;
  for (int a = 0; a < p; ++a) {
    double t = 0;
    for (int b = 0; b < p; ++b) t += XtXinv[a * p + b] * v[b];
    q += v[a] * t;
  }
  const double gtg = gg - q;
  gtg_out[r] = gtg;
  inv_gtg[r] = gtg < 1e-12 ? 0.0 : 1.0 / gtg;
  // subset_maf_or_nan on the imputed vector: sum = s1 + k mu, sum2 = s2 + k mu^2
  const int k = n_miss[s];
  const double sum = s1[s] + k * mus;
  const double sum2 = s2[s] + k * mus * mus;
  double af = (sum / n) / 2.0;
  af = fmin(fmax(af, 0.0), 1.0);
  const double maf = af > 0.5 ? 1.0 - af : af;
  const double var = sum2 / n - (sum / n) * (sum / n);
  ok[r] = (maf < 1e-12 || var < 1e-12) ? 0 : 1;
  af_sub[r] = af;
}

// One warp per pair: FP64 gty = sum_i (g_i - mu) y_s[i] (y_s sums to zero).
// One warp per (gene, snp) pair: gty from the exact decoded dosage in FP64,
// then the pair's printed statistics (hit_from_gty, src/scan_trans_lm.cpp:21-36).
__global__ void lm_refine_kernel(GenoRows src, const int32_t* __restrict__ col, int n,
                                 const int64_t* __restrict__ kept, const double* __restrict__ mu,
                                 const double* __restrict__ Ys, const double* __restrict__ gtg,
                                 const double* __restrict__ yty, double df, const int2* __restrict__ pairs,
                                 int n_pairs, eqtl_pair* out) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= n_pairs) return;
  const int2 pr = pairs[w];
  const int64_t s = kept[pr.y];
  const double mus = mu[s];
  const double* y = Ys + static_cast<int64_t>(pr.x) * n;
  double acc = 0;
  for (int i = lane; i < n; i += 32) {
    const double d = src.dosage(s, __ldg(col + i));
    const double gc = isnan(d) ? 0.0 : d - mus;
    acc += gc * y[i];
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) {
    eqtl_pair q;
    q.snp = pr.y;
    q.gene = pr.x;
    q.reserved = 0;
    lm_stats_fp64(gtg[pr.y], acc, yty[pr.x], df, q);
    out[w] = q;
  }
}

}  // namespace dev

template <>
struct EpiOf<dev::LmEpiParams> {
  using type = dev::LmEpi;
};

using namespace dev;

// FP64 statistics of (gene, kept SNP) pairs against the current LM prep
// (ws.Ys, ws.yty, ws.gtg): gty from the exact decoded dosage, one warp per pair.
static std::vector<eqtl_pair> lm_refine_pairs(eqtl_ctx* ctx, double df, const std::vector<int2>& todo) {
  Geno& g = ctx->geno;
  Workspace& ws = ctx->ws;
  cudaStream_t st = ctx->stream;
  const int n = g.n;
  std::vector<eqtl_pair> refined(todo.size());
  if (!todo.empty()) {
    ws.ref_pairs.upload(todo.data(), todo.size(), st);
    ws.refined.alloc(todo.size());
    ++ctx->launches;
    lm_refine_kernel<<<static_cast<unsigned>((todo.size() + 7) / 8), 256, 0, st>>>(
        g.rows(), g.col.p, n, g.kept.p, g.mu.p, ws.Ys.p, ws.gtg.p, ws.yty.p, df, ws.ref_pairs.p,
        static_cast<int>(todo.size()), ws.refined.p);
    EQTL_CUDA(cudaGetLastError());
    ws.refined.download(refined.data(), todo.size(), st);
    EQTL_CUDA(cudaStreamSynchronize(st));
  }
  return refined;
}

void scan_trans_lm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                   eqtl_gene_result* genes, std::vector<eqtl_pair>& pairs, std::vector<eqtl_pair>& cands) {
  Geno& g = ctx->geno;
  Workspace& ws = ctx->ws;
  EQTL_CHECK(g.m_all > 0, EQTL_E_STATE, "scan_trans_lm: no genotypes loaded");
  const int n = prm->n, G = prm->n_genes, p = prm->p;
  EQTL_CHECK(n == g.n, EQTL_E_ARG, "scan_trans_lm: n differs from the loaded genotypes");
  EQTL_CHECK(G > 0 && p > 0 && p <= kMaxP, EQTL_E_ARG, "scan_trans_lm: need 1 <= p <= 32 and genes > 0");
  EQTL_CHECK(g.m < (int64_t(1) << 30), EQTL_E_UNSUPPORTED, "scan_trans_lm: more than 2^30 kept SNPs");
  EQTL_CHECK(prm->y_rotated == 0, EQTL_E_ARG, "y_rotated applies to the LMM only");
  cudaStream_t st = ctx->stream;
  const double df = static_cast<double>(n - p - 1);
  const PhenoDev& ph = resolve_pheno(ctx, prm, Y, X);

  // ---- covariate algebra (host, p x p) and gene prep (device DGEMMs)
  std::unique_ptr<StageScope> prep_timer(new StageScope(ctx, EQTL_STAGE_PREP));
  std::vector<double> XtXinv = xtx_inverse(ph.X_h.data(), n, p);
  ws.XtXinv.upload(XtXinv.data(), XtXinv.size(), st);
  ws.Ys.alloc(static_cast<size_t>(n) * G);
  EQTL_CUDA(cudaMemcpyAsync(ws.Ys.p, ph.Y.p, sizeof(double) * n * G, cudaMemcpyDeviceToDevice, st));
  ws.XtY.alloc(static_cast<size_t>(p) * G);
  residualize_genes(ctx, ph.X.p, ws.XtXinv.p, n, p, G, ws.Ys.p, ws.XtY.p);  // Ys <- Y - X beta

  const int k_pad = g.k_pad;
  DevBuf<__half>& a_hi = ws.ops_hi[0];
  DevBuf<__half>& a_lo = ws.ops_lo[0];
  a_hi.alloc(static_cast<size_t>(G) * k_pad);
  a_lo.alloc(static_cast<size_t>(G) * k_pad);
  ws.gscale.alloc(G);
  ws.inv_yty.alloc(G);
  ws.yty.alloc(G);
  const bool bf16 = ctx->precision == EQTL_PREC_SPLIT_BF16;
  // FP16 scans read the exact integer-scaled dosages (one slice; the
  // centring is implicit: the residualised y_s sum to zero, X holding the
  // intercept), so two products per test (y hi and lo against them)
  // instead of three against the split centred dosages
  const bool raw = !bf16 && geno_raw_operand(ctx);
  ++ctx->launches;
  if (bf16)
    gene_split_kernel<__nv_bfloat16><<<G, 256, 0, st>>>(ws.Ys.p, n, k_pad, G,
                                                        reinterpret_cast<__nv_bfloat16*>(a_hi.p),
                                                        reinterpret_cast<__nv_bfloat16*>(a_lo.p), ws.gscale.p,
                                                        ws.yty.p, ws.inv_yty.p, kGcScale);
  else
    gene_split_kernel<__half><<<G, 256, 0, st>>>(ws.Ys.p, n, k_pad, G, a_hi.p, a_lo.p, ws.gscale.p, ws.yty.p,
                                                 ws.inv_yty.p, raw ? 1.0f : kGcScale);
  EQTL_CUDA(cudaGetLastError());

  // ---- per-SNP FP64 residual sum of squares + subset gate
  const int64_t m = g.m;
  ws.gtg.alloc(std::max<int64_t>(m, 1));
  ws.inv_gtg.alloc(std::max<int64_t>(m, 1));
  ws.af_sub.alloc(std::max<int64_t>(m, 1));
  ws.ok.alloc(static_cast<size_t>(((m + 255) / 256 + 1) * 256));  // the epilogue reads 16 flags per chunk, up to the last tile's end
  EQTL_CUDA(cudaMemsetAsync(ws.ok.p, 0, ws.ok.n, st));
  if (m > 0) {
    ++ctx->launches;
    snp_gtg_kernel<<<static_cast<unsigned>((m + 7) / 8), 256, 0, st>>>(
        g.rows(), g.col.p, n, g.kept.p, m, g.mu.p, g.gate_nmiss(), g.gate_s1(), g.gate_s2(), ph.X.p, p,
        ws.XtXinv.p, ws.gtg.p, ws.inv_gtg.p, ws.ok.p, ws.af_sub.p);
    EQTL_CUDA(cudaGetLastError());
  }

  // ---- thresholds, windows and t table
  double t_cand = t_critical(prm->pthr, df);
  if (prm->perm_thr > 0) t_cand = std::min(t_cand, t_critical(prm->perm_thr, df));
  LmEpiParams ep{};
  ep.G = G;
  ep.m = m;
  ep.inv_yty = ws.inv_yty.p;
  ep.gscale = ws.gscale.p;
  // per-SNP factors, padded to the end of the last tile of 256 SNPs
  const int64_t m_pad = ((m + 255) / 256 + 1) * 256;
  ws.inv_gtg_f.alloc(static_cast<size_t>(m_pad));
  ++ctx->launches;
  lm_igs_kernel<<<static_cast<unsigned>(std::min<int64_t>((m_pad + 255) / 256, 4096)), 256, 0, st>>>(
      ws.inv_gtg.p, ws.ok.p, raw ? ctx->rot.alpha.p : nullptr, m, m_pad, ws.inv_gtg_f.p);
  EQTL_CUDA(cudaGetLastError());
  ep.igs = ws.inv_gtg_f.p;
  ep.win = upload_windows(ctx, prm, m, prm->exclude_cis == 2 ? kWinInclude : prm->exclude_cis ? kWinExclude : kWinNone);
  ep.df = static_cast<float>(df);
  ep.t_cand = static_cast<float>(t_cand * (1.0 - 1e-3));
  ep.tt = device_ttable(ctx, df);
  prep_timer.reset();

  ScanOutputs so(ctx, G, m, expected_candidates(prm, m));
  const int2* tiles = nullptr;  // cis: banded tile list
  int n_tiles = 0;
  cis_tile_list(ctx, prm, m, 256, tiles, n_tiles);
  std::unique_ptr<StageScope> scan_timer(new StageScope(ctx, EQTL_STAGE_SCAN));
  if (m > 0) {
    so.run([&](GeneOut out) {
      ep.out = out;
      const __half* ah[1] = {a_hi.p};
      const __half* al[1] = {a_lo.p};
      const int bsel[1] = {0};
      if (raw) {
        const __half* bh[1] = {ctx->rot.raw.p};
        const int prod[1] = {5};
        launch_tile_n<256, 1, LmEpiParams, dev::kBLoNone>(ctx, false, ep, ah, al, G, bh, bh, m, k_pad, bsel, prod,
                                                          tiles, n_tiles);
      } else {
        const __half* bh[1] = {g.gc_hi.p};
        const __half* bl[1] = {g.gc_lo.p};
        const int prod[1] = {7};
        launch_tile_n<256, 1>(ctx, bf16, ep, ah, al, G, bh, bl, m, k_pad, bsel, prod, tiles, n_tiles);
      }
    });
  }
  scan_timer.reset();

  // ---- refine candidates + per-gene best in FP64
  StageScope refine_timer(ctx, EQTL_STAGE_REFINE);
  HostTrace tr("scan_trans_lm");
  std::vector<int2> todo, deferred;
  so.collect(genes, todo, deferred);
  tr.mark("collect");
  std::vector<eqtl_pair> refined = lm_refine_pairs(ctx, df, todo);
  tr.mark("refine pairs (device + download)");
  add_deferred_acat(genes, refined, deferred);
  tr.mark("deferred ACAT terms");
  finish_scan(prm, genes, refined, pairs, cands);
  tr.mark("finish");
  if (tr.on)
    std::fprintf(stderr, "[eqtl trace] scan_trans_lm counts: refined %zu deferred %zu\n", todo.size(),
                 deferred.size());
}

// FP64 tests of explicit (column of Y, kept SNP) pairs with the scan's prep:
// Y residualised on X, gtg and the subset gate per SNP; a SNP that fails the
// gate gets p = NaN (it is never tested in the reference).
void test_pairs_lm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                   const std::vector<int2>& todo, eqtl_pair* out) {
  Geno& g = ctx->geno;
  Workspace& ws = ctx->ws;
  EQTL_CHECK(g.m_all > 0, EQTL_E_STATE, "test_pairs: no genotypes loaded");
  const int n = prm->n, G = prm->n_genes, p = prm->p;
  EQTL_CHECK(n == g.n, EQTL_E_ARG, "test_pairs: n differs from the loaded genotypes");
  EQTL_CHECK(G > 0 && p > 0 && p <= kMaxP, EQTL_E_ARG, "test_pairs: need 1 <= p <= 32 and columns > 0");
  for (const int2& q : todo)
    EQTL_CHECK(q.x >= 0 && q.x < G && q.y >= 0 && q.y < g.m, EQTL_E_ARG, "test_pairs: pair index out of range");
  cudaStream_t st = ctx->stream;
  const double df = static_cast<double>(n - p - 1);
  const PhenoDev& ph = resolve_pheno(ctx, prm, Y, X);
  std::vector<double> XtXinv = xtx_inverse(ph.X_h.data(), n, p);
  ws.XtXinv.upload(XtXinv.data(), XtXinv.size(), st);
  ws.Ys.alloc(static_cast<size_t>(n) * G);
  EQTL_CUDA(cudaMemcpyAsync(ws.Ys.p, ph.Y.p, sizeof(double) * n * G, cudaMemcpyDeviceToDevice, st));
  ws.XtY.alloc(static_cast<size_t>(p) * G);
  residualize_genes(ctx, ph.X.p, ws.XtXinv.p, n, p, G, ws.Ys.p, ws.XtY.p);
  const int k_pad = g.k_pad;
  ws.ops_hi[0].alloc(static_cast<size_t>(G) * k_pad);
  ws.ops_lo[0].alloc(static_cast<size_t>(G) * k_pad);
  ws.gscale.alloc(G);
  ws.inv_yty.alloc(G);
  ws.yty.alloc(G);
  ++ctx->launches;
  gene_split_kernel<__half><<<G, 256, 0, st>>>(ws.Ys.p, n, k_pad, G, ws.ops_hi[0].p, ws.ops_lo[0].p, ws.gscale.p,
                                               ws.yty.p, ws.inv_yty.p, kGcScale);
  EQTL_CUDA(cudaGetLastError());
  const int64_t m = g.m;
  ws.gtg.alloc(std::max<int64_t>(m, 1));
  ws.inv_gtg.alloc(std::max<int64_t>(m, 1));
  ws.af_sub.alloc(std::max<int64_t>(m, 1));
  ws.ok.alloc(static_cast<size_t>(((m + 255) / 256 + 1) * 256));
  EQTL_CUDA(cudaMemsetAsync(ws.ok.p, 0, ws.ok.n, st));
  if (m > 0) {
    ++ctx->launches;
    snp_gtg_kernel<<<static_cast<unsigned>((m + 7) / 8), 256, 0, st>>>(
        g.rows(), g.col.p, n, g.kept.p, m, g.mu.p, g.gate_nmiss(), g.gate_s1(), g.gate_s2(), ph.X.p, p,
        ws.XtXinv.p, ws.gtg.p, ws.inv_gtg.p, ws.ok.p, ws.af_sub.p);
    EQTL_CUDA(cudaGetLastError());
  }
  std::vector<uint8_t> ok(static_cast<size_t>(m));
  ws.ok.download(ok.data(), static_cast<size_t>(m), st);
  const std::vector<eqtl_pair> refined = lm_refine_pairs(ctx, df, todo);
  for (size_t i = 0; i < todo.size(); ++i) {
    out[i] = refined[i];
    if (!ok[todo[i].y]) out[i].p = std::numeric_limits<double>::quiet_NaN();
  }
}

}  // namespace eqtl
