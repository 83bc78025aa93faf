// Device Student-t tail for the scan epilogues.
//
// Every scan of one keep-set has a single residual df, so the host tabulates
// the two-sided p once (TTableHost, tstat.hpp) and the epilogue interpolates:
//   |t| <= t0 : 1 - p = |t| h(t^2)        (h analytic; cubic Lagrange in u = t^2)
//   |t| >  t0 : ln p  = L(x), x = sqrt(log1p(t^2/df))   (cubic Lagrange in x;
//               ln p is analytic in x: |t| ~ sqrt(df) x at the start of the
//               range and ln p ~ -(df/2) x^2 far out, so the cubic is exact
//               to FP32 rounding where a grid in s would meet a sqrt(s)
//               singularity)
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

constexpr int kTTableNa = 512;   // central intervals (TTableHost::na)
constexpr int kTTableNb = 4096;  // tail intervals (TTableHost::nb)
constexpr int kTTableNq = 1024;  // tail intervals of the per-interval cubics (TTableHost::nq)
constexpr int kTTableNodeBytes = (kTTableNa + 4 + kTTableNb + 4) * 4;
constexpr int kTTableCubicBytes = (kTTableNa + kTTableNq) * 16;
constexpr int kTTableSmemBytes = kTTableNodeBytes > kTTableCubicBytes ? kTTableNodeBytes : kTTableCubicBytes;

struct TTable {
  const float* h;  // na + 4 nodes
  const float* L;  // nb + 4 nodes
  float du_inv;    // na / t0^2
  float x0, dx_inv, x_end;  // tail grid in x = sqrt(log1p(t^2/df))
  float tiny_t;             // 0 < |t| < tiny_t: deferred (see below)
  float inv_df;
  float t0;
  int na, nb;
  // ACAT screening of the scan epilogues (acat_screen): |t| tan((1/2 - p) pi)
  // on the central u grid, ln tan((1/2 - p) pi) on x in [x0, x(t_defer)]
  const float* c1;  // na + 4 nodes
  const float* lt;  // nb + 4 nodes
  float dl_inv;     // nb / (x(t_defer) - x0)
  int lt_u;         // 1: lt holds the term itself on u in [u0, u_defer] (dlu_inv = nb / that range)
  float dlu_inv;
  // with lt_u, the screen's per-interval cubics (a0, a1, a2, a3): c1q over
  // u in [0, uq0] (na intervals, dqc_inv per unit of u), ltq over u in
  // [uq0, u_defer] (nq intervals, dq_inv)
  const float4* c1q;
  const float4* ltq;
  float uq0, dqc_inv, dq_inv;
  int nq;
  float t_defer;    // |t| >= t_defer (p <= 1e-14): the term is left to the host
  // the same thresholds on u = t^2 (the scan epilogues screen t^2 directly)
  float u0;         // t0^2
  float u_tiny;     // tiny_t^2
  float u_defer;    // t_defer^2, rounded down
};

__device__ __forceinline__ float lagrange4(const float* y, float x, int n_int) {
  // x in node-step units from the region start; clamp into [0, n_int)
  x = fminf(fmaxf(x, 0.0f), static_cast<float>(n_int) - 1e-3f);
  const int i = static_cast<int>(x);
  const float f = x - static_cast<float>(i);
  const float* q = y + i;  // q[0] = node i-1 (stored with +1 offset); global or shared
  const float y0 = q[0], y1 = q[1], y2 = q[2], y3 = q[3];
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
  bool use_acat;     // p < 1 - 1e-12 and not deferred: term added on the device
  bool deferred;     // p < 1e-14 or 0 < |t| < tiny_t: left to the host (see below)
  bool tiny;         // deferred because 0 < |t| < tiny_t
};

// The reference evaluates tan((0.5L - p) * pi) in 80-bit long double
// (src/stats_extra.cpp:20). For tiny p that expression is quantised by the
// long-double spacing near 0.5 (2^-65) and, below p ~ 2.7e-20, rounds to
// tan(0.5L * pi_L), a huge NEGATIVE value because pi_L exceeds pi.
// At the other end, the reference's x = df / (df + t^2) (src/util.cpp:261)
// rounds to exactly 1 for t^2 below half an ulp of df, so p = 1 and the pair
// leaves ACAT, while just above it 1 - p is quantised by the ulp; the term
// there is ~ -1 / (0.8 pi |t|), so the gene's ACAT hinges on it. To stay a
// drop-in, the epilogue adds neither kind: it emits the pair as a flagged
// candidate, and the host refines it in FP64 with the reference's
// arithmetic and adds the long-double term (and its `used` count) when the
// refined p enters ACAT. tiny_t = sqrt(256 ulp(df)) plus four times the
// screening error of t, so every pair the reference quantises is caught.
constexpr float kDeferNegLog10P = 14.0f;

constexpr float kLn10 = 2.302585092994046f;
constexpr double kPiD = 3.141592653589793;

// One branch-free path for every lane (a warp's lanes are different genes,
// so |t| straddles t0 within a warp): the lane picks its table, interpolates
// once, and derives m = min(p, 1-p) with full relative precision (1-p from
// the central table, p from the tail table), so tan((1/2-p) pi) =
// +-cot(pi m) is one sincospi and one division.
__device__ __forceinline__ TailOut t_tail(float t, const TTable& T) {
  TailOut o;
  const float at = fabsf(t);
  const bool nan_t = !(at == at);
  const bool central = at <= T.t0;
  const float u = at * at;
  const float xs = sqrtf(log1pf(u * T.inv_df));
  const bool beyond = !central && xs >= T.x_end;
  const float x = central ? u * T.du_inv : (xs - T.x0) * T.dx_inv;
  const float y = lagrange4(central ? T.h : T.L, x, central ? T.na + 1 : T.nb + 1);
  // central: y = h (1-p = |t| h); tail: y = ln p
  const float q = at * y;
  const float lnp = central ? log1pf(-q) : y;
  const float p = central ? 1.0f - q : __expf(y);
  const bool p_small = !central || q >= 0.5f;        // p <= 1/2: m = p
  const float mm = p_small ? p : q;
  float sm, cm;
  sincospif(mm, &sm, &cm);
  const float cot = __fdividef(cm, sm);
  o.neglog10p = nan_t ? 0.0f : fminf(-lnp * (1.0f / kLn10), 323.3f);
  const bool tiny = at > 0.0f && at < T.tiny_t;
  o.tiny = !nan_t && tiny;
  o.deferred = !nan_t && (beyond || tiny || o.neglog10p > kDeferNegLog10P);
  o.use_acat = !nan_t && !o.deferred && (central ? q > 1e-12f : true);
  o.term = (nan_t || o.deferred || !o.use_acat) ? 0.0 : static_cast<double>(p_small ? cot : -cot);
  if (beyond) o.neglog10p = 323.3f;
  return o;
}

// What the scan epilogues need of each pair: the ACAT term, whether it
// enters ACAT on the device, and whether the host takes it over. Same rules
// as t_tail, without -log10 p, and from u = t^2 alone (no square root per
// pair): the best SNP is keyed on u (p falls as u grows at one df),
// deferral for p <= 1e-14 is u >= u_defer, for |t| near 0 0 < u < u_tiny.
// One table lookup:
//   central  tan((1/2 - p) pi) = c1(u) / |t| = c1(u) rsqrt(u)
//   tail     tan((1/2 - p) pi) = lt(u)                      (T.lt_u, short tails)
// (with T.lt_u both as per-interval cubics: one 16-byte load and three FMAs)
//            tan((1/2 - p) pi) = exp(lt(sqrt(log1p(u / df))))  (otherwise)
struct ScreenOut {
  float term;     // tan((1/2 - p) pi) when use_acat, else 0
  float key;      // best-SNP score: u for the scans (|t| through acat_screen); 0 for NaN
  bool use_acat;  // p < 1 - 1e-12 and not deferred
  bool deferred;  // p <= 1e-14 or 0 < |t| < tiny_t
  bool tiny;      // deferred because 0 < |t| < tiny_t
};

__device__ __forceinline__ ScreenOut acat_screen_u(float u, const TTable& T) {
  ScreenOut o;
  const bool nan_u = !(u == u);
  const bool tiny = u > 0.0f && u < T.u_tiny;
  o.tiny = !nan_u && tiny;
  o.deferred = !nan_u && (tiny || u >= T.u_defer);
  o.use_acat = !nan_u && !o.deferred && u > 0.0f;
  o.key = nan_u ? 0.0f : u;
  float term;
  if (T.lt_u) {  // uniform across the launch
    const bool central = u <= T.uq0;
    float x = central ? u * T.dqc_inv : (u - T.uq0) * T.dq_inv;
    x = fminf(fmaxf(x, 0.0f), static_cast<float>(central ? T.na : T.nq) - 1e-3f);
    const int i = static_cast<int>(x);
    const float f = x - static_cast<float>(i);
    const float4 a = (central ? T.c1q : T.ltq)[i];
    const float y = fmaf(fmaf(fmaf(a.w, f, a.z), f, a.y), f, a.x);
    term = central ? y * rsqrtf(u) : y;
  } else {
    const bool central = u <= T.u0;
    float x;
    const float xs = sqrtf(log1pf(u * T.inv_df));
    x = central ? u * T.du_inv : (xs - T.x0) * T.dl_inv;
    const float y = lagrange4(central ? T.c1 : T.lt, x, central ? T.na + 1 : T.nb + 1);
    term = central ? y * rsqrtf(u) : __expf(y);
  }
  o.term = o.use_acat ? term : 0.0f;
  return o;
}

// The screen of one t (the t_tail ABI's screen mode): key = |t|.
__device__ __forceinline__ ScreenOut acat_screen(float t, const TTable& T) {
  ScreenOut o = acat_screen_u(t * t, T);
  const float at = fabsf(t);
  o.key = at == at ? at : 0.0f;
  return o;
}

// Copies the screening tables into shared memory (cooperatively, by `nthr`
// threads) and returns a view of them; the caller synchronises before use.
// (With lt_u the per-interval cubics, else the node tables; `sm` 16-byte
// aligned, kTTableSmemBytes.)
__device__ __forceinline__ TTable screen_to_smem(const TTable& T, float* sm, int tid, int nthr) {
  TTable o = T;
  if (T.lt_u) {
    float4* q = reinterpret_cast<float4*>(sm);
    for (int i = tid; i < T.na; i += nthr) q[i] = T.c1q[i];
    for (int i = tid; i < T.nq; i += nthr) q[T.na + i] = T.ltq[i];
    o.c1q = q;
    o.ltq = q + T.na;
    return o;
  }
  const int nc = T.na + 4, nl = T.nb + 4;
  for (int i = tid; i < nc; i += nthr) sm[i] = T.c1[i];
  for (int i = tid; i < nl; i += nthr) sm[nc + i] = T.lt[i];
  o.c1 = sm;
  o.lt = sm + nc;
  return o;
}

// Copies the t_tail tables into shared memory (cooperatively, by `nthr`
// threads) and returns a view of them; the caller synchronises before use.
__device__ __forceinline__ TTable ttable_to_smem(const TTable& T, float* sm, int tid, int nthr) {
  const int nh = T.na + 4, nl = T.nb + 4;
  for (int i = tid; i < nh; i += nthr) sm[i] = T.h[i];
  for (int i = tid; i < nl; i += nthr) sm[nh + i] = T.L[i];
  TTable o = T;
  o.h = sm;
  o.L = sm + nh;
  return o;
}

// Monotone 64-bit key for "smallest p, then lowest SNP index": atomicMin
// over keys picks the reference's best (strict < keeps the first SNP). The
// score is any non-negative quantity that grows as p falls: -log10 p, or |t|
// within one gene (one df).
__device__ __forceinline__ unsigned long long best_key(float score, uint32_t snp) {
  // larger score is better -> invert the (non-negative) float bits
  const uint32_t b = __float_as_uint(fmaxf(score, 0.0f));
  return (static_cast<unsigned long long>(~b) << 32) | snp;
}

}  // namespace dev
}  // namespace eqtl
