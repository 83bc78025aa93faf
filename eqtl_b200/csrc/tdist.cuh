// Device Student-t tail for the scan epilogues.
//
// Every scan of one keep-set has a single residual df, so the host tabulates
// the two-sided p once (TTableHost, tstat.hpp) and the epilogue interpolates:
//   |t| <= t0 : 1 - p = |t| h(t^2)        (h analytic; cubic Lagrange in u = t^2)
//   |t| >  t0 : ln p  = L(s), s = log1p(t^2/df)   (cubic Lagrange in s)
// Node k of each table sits at (k-1) steps from the region start, so the
// four nodes around any point in range exist. The result feeds
//   * screening: -log10 p for the per-gene best key and threshold tests;
//   * ACAT: tan((1/2 - p) pi), skipped for p >= 1 - 1e-12 like the
//     reference's AcatAcc::add (src/stats_extra.cpp:16-22).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace eqtl {
namespace dev {

struct TTable {
  const float* h;  // na + 4 nodes
  const float* L;  // nb + 4 nodes
  float du_inv;    // na / t0^2
  float s0, ds_inv, s_end;
  float inv_df;
  float t0;
  int na, nb;
};

__device__ __forceinline__ float lagrange4(const float* y, float x, int n_int) {
  // x in node-step units from the region start; clamp into [0, n_int)
  x = fminf(fmaxf(x, 0.0f), static_cast<float>(n_int) - 1e-3f);
  const int i = static_cast<int>(x);
  const float f = x - static_cast<float>(i);
  const float* q = y + i;  // q[0] = node i-1 (stored with +1 offset)
  const float y0 = __ldg(q), y1 = __ldg(q + 1), y2 = __ldg(q + 2), y3 = __ldg(q + 3);
  const float fm1 = f - 1.0f, fm2 = f - 2.0f, fp1 = f + 1.0f;
  const float w0 = -f * fm1 * fm2 * (1.0f / 6.0f);
  const float w1 = fp1 * fm1 * fm2 * 0.5f;
  const float w2 = -fp1 * f * fm2 * 0.5f;
  const float w3 = fp1 * f * fm1 * (1.0f / 6.0f);
  return fmaf(w0, y0, fmaf(w1, y1, fmaf(w2, y2, w3 * y3)));
}

struct TailOut {
  float neglog10p;   // -log10 p (>= 0); capped where the FP64 reference p underflows
  double term;       // tan((1/2 - p) pi)
  bool use_acat;     // p < 1 - 1e-12
  bool deferred;     // p < 1e-14: term left to the host (see below)
};

// The reference evaluates tan((0.5L - p) * pi) in 80-bit long double
// (src/stats_extra.cpp:20). For tiny p that expression is quantised by the
// long-double spacing near 0.5 (2^-65) and, below p ~ 2.7e-20, rounds to
// tan(0.5L * pi_L), a huge NEGATIVE value because pi_L exceeds pi. To stay a
// drop-in, the epilogue does not add terms for p < 1e-14; it counts them
// in `used`, emits the pair as a flagged candidate, and the host adds the
// reference's long-double term from the pair's FP64-refined p.
constexpr float kDeferNegLog10P = 14.0f;

constexpr float kLn10 = 2.302585092994046f;
constexpr double kPiD = 3.141592653589793;

__device__ __forceinline__ TailOut t_tail(float t, const TTable& T) {
  TailOut o;
  o.deferred = false;
  const float at = fabsf(t);
  if (!(at == at)) {  // NaN t: p = 1 (src/util.cpp:260)
    o.neglog10p = 0.0f;
    o.term = 0.0;
    o.use_acat = false;
    return o;
  }
  if (at <= T.t0) {
    const float h = lagrange4(T.h, at * at * T.du_inv, T.na + 1);
    const float q = at * h;  // 1 - p, accurate for tiny |t|
    o.neglog10p = -log1pf(-q) * (1.0f / kLn10);
    o.use_acat = q > 1e-12f;
    if (q < 0.5f) {
      // p > 1/2: tan((1/2-p) pi) = -cot(pi q)
      float sq, cq;
      sincospif(q, &sq, &cq);
      o.term = -static_cast<double>(cq) / static_cast<double>(sq);
    } else {
      const float p = 1.0f - q;
      float sp, cp;
      sincospif(p, &sp, &cp);
      o.term = static_cast<double>(cp) / static_cast<double>(sp);
    }
    return o;
  }
  const float s = log1pf(at * at * T.inv_df);
  if (s >= T.s_end) {
    // beyond the table: the FP64 reference p underflows to (near) zero
    o.neglog10p = 323.3f;
    o.term = 0.0;
    o.use_acat = true;
    o.deferred = true;
    return o;
  }
  const float L = lagrange4(T.L, (s - T.s0) * T.ds_inv, T.nb + 1);
  o.neglog10p = fminf(-L * (1.0f / kLn10), 323.3f);
  o.use_acat = true;
  if (o.neglog10p > kDeferNegLog10P) {
    o.term = 0.0;
    o.deferred = true;
  } else if (L < -6.907755f) {  // p < 1e-3: cot(pi p) = 1/(pi p) - pi p / 3 - ...
    double pd = exp(static_cast<double>(L));
    pd = fmax(pd, 1e-300);
    o.term = 1.0 / (kPiD * pd) - kPiD * pd / 3.0;
  } else {
    const float p = __expf(L);
    float sp, cp;
    sincospif(p, &sp, &cp);
    o.term = static_cast<double>(cp) / static_cast<double>(sp);
  }
  return o;
}

// Monotone 64-bit key for "smallest p, then lowest SNP index": atomicMin
// over keys picks the reference's best (strict < keeps the first SNP).
__device__ __forceinline__ unsigned long long best_key(float neglog10p, uint32_t snp) {
  // larger -log10 p is better -> invert the (non-negative) float bits
  const uint32_t b = __float_as_uint(fmaxf(neglog10p, 0.0f));
  return (static_cast<unsigned long long>(~b) << 32) | snp;
}

}  // namespace dev
}  // namespace eqtl
