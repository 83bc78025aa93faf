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
  const float* gscale;     // [G] accumulator -> gty factor
  const double* inv_gtg;   // [m] 1 / gtg (0 marks gtg < 1e-12: p = 1)
  const uint8_t* snp_ok;   // [m] subset gate (src/scan_common.cpp:133-151)
  Windows win;
  float df;
  float t_cand;
  TTable tt;
  GeneOut out;
};

struct LmEpi {
  using Params = LmEpiParams;
  const Params& P;
  int gene = 0;
  int64_t snp0 = 0;
  bool gvalid = false;
  double inv_yty = 0;
  float gs = 0;
  GeneAcc acc;

  __device__ LmEpi(const Params& p, const TileShape&) : P(p) {}
  __device__ void begin_tile(int g, int64_t s0) {
    gene = g;
    snp0 = s0;
    gvalid = g < P.G;
    acc.reset();
    if (gvalid) {
      inv_yty = P.inv_yty[g];
      gs = P.gscale[g];
      acc.load_window(P.win, g);
    }
  }
  template <int NACC>
  __device__ void chunk(int c, const float (&v)[NACC][16]) {
    if (!gvalid) return;
#pragma unroll 4
    for (int j = 0; j < 16; ++j) {
      const int64_t s = snp0 + c + j;
      if (s >= P.m) break;
      if (!__ldg(P.snp_ok + s)) continue;
      if (!acc.in_scope(P.win, s)) continue;
      const double ig = __ldg(P.inv_gtg + s);
      float t = 0.0f;
      if (ig > 0.0) {
        // t^2 = df r / (1 - r), r = gty^2 / (gtg yty)  (hit_from_gty algebra)
        const double num = static_cast<double>(v[0][j]) * gs;
        const double r = num * num * ig * inv_yty;
        const double omr = 1.0 - r;
        if (omr > 0.0) {
          const float t2 = P.df * static_cast<float>(r) / static_cast<float>(omr);
          t = copysignf(sqrtf(t2), static_cast<float>(num));
        }
      }
      const TailOut o = t_tail(t, P.tt);
      acc.add(o, s);
      if (fabsf(t) >= P.t_cand || o.deferred) emit_candidate(P.out, gene, s, o.deferred);
    }
  }
  __device__ void end_tile() {
    if (gvalid) acc.flush(P.out, gene);
  }
  __device__ void finish() {}
};

// ---------------------------------------------------------------- prep
// One block per gene: yty, power-of-two scale, FP16/BF16 hi/lo rows.
template <class T>
__global__ void gene_split_kernel(const double* __restrict__ Ys, int n, int k_pad, int G, T* hi, T* lo,
                                  float* gscale, double* inv_yty, float snp_scale) {
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
    inv_yty[g] = yty > 0 ? 1.0 / yty : 0.0;
  }
}

__device__ __forceinline__ int bed_code_dev(const uint8_t* row, int col) {
  const uint32_t b = __ldg(row + (col >> 2));
  const uint32_t pair = (b >> ((col & 3) * 2)) & 3u;
  return static_cast<int>(static_cast<int8_t>((0x0001FF02u >> (pair * 8)) & 0xFFu));
}

constexpr int kMaxP = 32;

// One warp per kept SNP: FP64 |g_s|^2 with the exact decoded dosage, and the
// subset gate on the analysis samples.
__global__ void snp_gtg_kernel(const uint8_t* __restrict__ bed, int64_t bps, const int32_t* __restrict__ col,
                               int n, const int64_t* __restrict__ kept, int64_t m, const double* __restrict__ mu,
                               const int32_t* __restrict__ n_miss, const int32_t* __restrict__ s1,
                               const int32_t* __restrict__ s2, const double* __restrict__ X, int p,
                               const double* __restrict__ XtXinv, double* gtg_out, double* inv_gtg, uint8_t* ok,
                               double* af_sub) {
  const int lane = threadIdx.x & 31;
  const int64_t r = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= m) return;
  const int64_t s = kept[r];
  const uint8_t* row = bed + s * bps;
  const double mus = mu[s];
  double gg = 0;
  double v[kMaxP];
#pragma unroll
  for (int k = 0; k < kMaxP; ++k) v[k] = 0;
  for (int i = lane; i < n; i += 32) {
    const int c = bed_code_dev(row, __ldg(col + i));
    const double gc = c < 0 ? 0.0 : static_cast<double>(c) - mus;
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
  const double sum = static_cast<double>(s1[s]) + k * mus;
  const double sum2 = static_cast<double>(s2[s]) + k * mus * mus;
  double af = (sum / n) / 2.0;
  af = fmin(fmax(af, 0.0), 1.0);
  const double maf = af > 0.5 ? 1.0 - af : af;
  const double var = sum2 / n - (sum / n) * (sum / n);
  ok[r] = (maf < 1e-12 || var < 1e-12) ? 0 : 1;
  af_sub[r] = af;
}

// One warp per pair: FP64 gty = sum_i (g_i - mu) y_s[i] (y_s sums to zero).
__global__ void lm_refine_kernel(const uint8_t* __restrict__ bed, int64_t bps, const int32_t* __restrict__ col,
                                 int n, const int64_t* __restrict__ kept, const double* __restrict__ mu,
                                 const double* __restrict__ Ys, const int2* __restrict__ pairs, int n_pairs,
                                 double* gty) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= n_pairs) return;
  const int2 pr = pairs[w];
  const int64_t s = kept[pr.y];
  const uint8_t* row = bed + s * bps;
  const double mus = mu[s];
  const double* y = Ys + static_cast<int64_t>(pr.x) * n;
  double acc = 0;
  for (int i = lane; i < n; i += 32) {
    const int c = bed_code_dev(row, __ldg(col + i));
    const double gc = c < 0 ? 0.0 : static_cast<double>(c) - mus;
    acc += gc * y[i];
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) gty[w] = acc;
}

}  // namespace dev

template <>
struct EpiOf<dev::LmEpiParams> {
  using type = dev::LmEpi;
};

using namespace dev;

void scan_trans_lm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                   eqtl_gene_result* genes, std::vector<eqtl_pair>& pairs, std::vector<eqtl_pair>& cands) {
  Geno& g = ctx->geno;
  EQTL_CHECK(g.m_all > 0 || g.m == 0, EQTL_E_STATE, "scan_trans_lm: no genotypes loaded");
  const int n = prm->n, G = prm->n_genes, p = prm->p;
  EQTL_CHECK(n == g.n, EQTL_E_ARG, "scan_trans_lm: n differs from the loaded genotypes");
  EQTL_CHECK(G > 0 && p > 0 && p <= kMaxP, EQTL_E_ARG, "scan_trans_lm: need 1 <= p <= 32 and genes > 0");
  cudaStream_t st = ctx->stream;
  const double df = static_cast<double>(n - p - 1);

  // ---- covariate algebra (host, p x p) and gene prep (device DGEMMs)
  std::unique_ptr<StageScope> prep_timer(new StageScope(ctx, EQTL_STAGE_PREP));
  std::vector<double> XtXinv = xtx_inverse(X, n, p);
  DevBuf<double> dX, dXtXinv, dY, dXtY;
  dX.upload(X, static_cast<size_t>(n) * p, st);
  dXtXinv.upload(XtXinv.data(), XtXinv.size(), st);
  dY.upload(Y, static_cast<size_t>(n) * G, st);
  dXtY.alloc(static_cast<size_t>(p) * G);
  residualize_genes(ctx, dX.p, dXtXinv.p, n, p, G, dY.p, dXtY.p);  // dY <- Y_s

  const int k_pad = g.k_pad;
  DevBuf<__half> a_hi, a_lo;
  a_hi.alloc(static_cast<size_t>(G) * k_pad);
  a_lo.alloc(static_cast<size_t>(G) * k_pad);
  DevBuf<float> gscale;
  DevBuf<double> inv_yty;
  gscale.alloc(G);
  inv_yty.alloc(G);
  const bool bf16 = ctx->precision == EQTL_PREC_SPLIT_BF16;
  ++ctx->launches;
  if (bf16)
    gene_split_kernel<__nv_bfloat16><<<G, 256, 0, st>>>(dY.p, n, k_pad, G, reinterpret_cast<__nv_bfloat16*>(a_hi.p),
                                                        reinterpret_cast<__nv_bfloat16*>(a_lo.p), gscale.p, inv_yty.p,
                                                        kGcScale);
  else
    gene_split_kernel<__half><<<G, 256, 0, st>>>(dY.p, n, k_pad, G, a_hi.p, a_lo.p, gscale.p, inv_yty.p, kGcScale);
  EQTL_CUDA(cudaGetLastError());

  // ---- per-SNP FP64 residual sum of squares + subset gate
  const int64_t m = g.m;
  DevBuf<double> gtg, inv_gtg, af_sub;
  DevBuf<uint8_t> ok;
  gtg.alloc(m);
  inv_gtg.alloc(m);
  af_sub.alloc(m);
  ok.alloc(m);
  if (m > 0) {
    ++ctx->launches;
    snp_gtg_kernel<<<static_cast<unsigned>((m + 7) / 8), 256, 0, st>>>(
        g.bed.p, g.bytes_per_snp, g.col.p, n, g.kept.p, m, g.mu.p, g.n_miss.p, g.s1.p, g.s2.p, dX.p, p, dXtXinv.p,
        gtg.p, inv_gtg.p, ok.p, af_sub.p);
    EQTL_CUDA(cudaGetLastError());
  }

  // ---- windows
  ScanWindows wins;
  upload_windows(ctx, prm, m, wins);

  // ---- thresholds and t table
  double t_cand = t_critical(prm->pthr, df);
  if (prm->perm_thr > 0) t_cand = std::min(t_cand, t_critical(prm->perm_thr, df));
  const float t_cand_f = static_cast<float>(t_cand * (1.0 - 1e-3));
  DeviceTTable tt(ctx, df);

  prep_timer.reset();
  ScanOutputs so(ctx, G, m, expected_candidates(prm, m));
  std::unique_ptr<StageScope> scan_timer(new StageScope(ctx, EQTL_STAGE_SCAN));
  LmEpiParams ep{};
  ep.G = G;
  ep.m = m;
  ep.inv_yty = inv_yty.p;
  ep.gscale = gscale.p;
  ep.inv_gtg = inv_gtg.p;
  ep.snp_ok = ok.p;
  ep.win = wins.view(prm->exclude_cis ? kWinExclude : kWinNone);
  ep.df = static_cast<float>(df);
  ep.t_cand = t_cand_f;
  ep.tt = tt.view();

  if (m > 0) {
    so.run([&](GeneOut out) {
      ep.out = out;
      const __half* ah[1] = {a_hi.p};
      const __half* al[1] = {a_lo.p};
      const __half* bh[1] = {g.gc_hi.p};
      const __half* bl[1] = {g.gc_lo.p};
      const int bsel[1] = {0}, prod[1] = {7};
      launch_tile_n<256, 1>(ctx, bf16, ep, ah, al, G, bh, bl, m, k_pad, bsel, prod);
    });
  }

  scan_timer.reset();
  // ---- refine candidates + per-gene best in FP64
  StageScope refine_timer(ctx, EQTL_STAGE_REFINE);
  std::vector<int2> todo, deferred;
  so.collect(genes, todo, deferred);
  std::vector<double> gtg_h(m);
  gtg.download(gtg_h.data(), m, st);
  std::vector<double> yty_h(G);
  gene_yty(ctx, dY.p, n, G, yty_h);
  EQTL_CUDA(cudaStreamSynchronize(st));
  std::vector<double> gty(todo.size());
  if (!todo.empty()) {
    DevBuf<int2> dt;
    DevBuf<double> dg;
    dt.upload(todo.data(), todo.size(), st);
    dg.alloc(todo.size());
    ++ctx->launches;
    lm_refine_kernel<<<static_cast<unsigned>((todo.size() + 7) / 8), 256, 0, st>>>(
        g.bed.p, g.bytes_per_snp, g.col.p, n, g.kept.p, g.mu.p, dY.p, dt.p, static_cast<int>(todo.size()), dg.p);
    EQTL_CUDA(cudaGetLastError());
    dg.download(gty.data(), todo.size(), st);
    EQTL_CUDA(cudaStreamSynchronize(st));
  }
  std::vector<eqtl_pair> refined(todo.size());
  for (size_t i = 0; i < todo.size(); ++i) {
    eqtl_pair& q = refined[i];
    q.gene = todo[i].x;
    q.snp = todo[i].y;
    q.reserved = 0;
    lm_stats_fp64(gtg_h[q.snp], gty[i], yty_h[q.gene], df, q);
  }
  add_deferred_acat(genes, refined, deferred);
  finish_scan(prm, genes, refined, pairs, cands);
}

}  // namespace eqtl
