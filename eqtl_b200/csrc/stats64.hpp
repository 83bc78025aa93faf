// FP64 per-pair statistics, compiled for host and device alike, so the
// refinement kernels print exactly what the host formulas give:
//   * the two-sided Student-t p through the regularised incomplete beta
//     function (Lentz's continued fraction with the reference's constants:
//     maxit 200, eps 3e-12, fpmin 1e-30; src/util.cpp:209-264), including
//     its x = df / (df + t^2) arithmetic, which gives p = 1 exactly where x
//     rounds to 1;
//   * the LM pair statistics of hit_from_gty (src/scan_trans_lm.cpp:21-36);
//   * the LMM bordered-Schur Wald test from gg, yg, a (test_lmm_gtil,
//     src/scan_trans_lmm.cpp:11-40).
#pragma once
#include <math.h>

#include "../../include/eqtl_b200.h"

#if defined(__CUDACC__)
#define EQTL_HD __host__ __device__ __forceinline__
#else
#define EQTL_HD inline
#endif

namespace eqtl {

EQTL_HD double incbeta_cf(double a, double b, double x) {
  const int kMaxIt = 200;
  const double kEps = 3e-12, kTiny = 1e-30;
  const double qab = a + b, qap = a + 1.0, qam = a - 1.0;
  double c = 1.0;
  double d = 1.0 - qab * x / qap;
  if (fabs(d) < kTiny) d = kTiny;
  d = 1.0 / d;
  double h = d;
  for (int m = 1; m <= kMaxIt; ++m) {
    const int m2 = 2 * m;
    double aa = m * (b - m) * x / ((qam + m2) * (a + m2));
    d = 1.0 + aa * d;
    if (fabs(d) < kTiny) d = kTiny;
    c = 1.0 + aa / c;
    if (fabs(c) < kTiny) c = kTiny;
    d = 1.0 / d;
    h *= d * c;
    aa = -(a + m) * (qab + m) * x / ((a + m2) * (qap + m2));
    d = 1.0 + aa * d;
    if (fabs(d) < kTiny) d = kTiny;
    c = 1.0 + aa / c;
    if (fabs(c) < kTiny) c = kTiny;
    d = 1.0 / d;
    const double del = d * c;
    h *= del;
    if (fabs(del - 1.0) < kEps) break;
  }
  return h;
}

// I_x(a, b)
EQTL_HD double incbeta(double a, double b, double x) {
  if (x < 0 || x > 1) return NAN;
  if (x == 0 || x == 1) return x;
  const double lbeta = lgamma(a) + lgamma(b) - lgamma(a + b);
  const double front = exp(log(x) * a + log(1 - x) * b - lbeta) / a;
  if (x < (a + 1) / (a + b + 2)) return front * incbeta_cf(a, b, x);
  return 1.0 - front * incbeta_cf(b, a, 1 - x) * a / b;
}

EQTL_HD double t_two_sided_p(double t, double df) {
  if (!isfinite(t) || df <= 0) return 1.0;
  const double x = df / (df + t * t);
  const double p = incbeta(0.5 * df, 0.5, x);
  return fmin(1.0, fmax(0.0, p));
}

// Inverse of the standard normal CDF as qnorm_inv computes it
// (src/util.cpp:132-171): Acklam's published rational approximation (central
// region p in [0.02425, 0.97575], tails in sqrt(-2 ln p)), with the
// coefficient digits the reference carries (they differ from the published
// ones in the last places; the Halley step absorbs that, but parity wants the
// same starting point), then one Halley step on Phi(v) - p. p is clamped to
// [1e-15, 1 - 1e-15].
EQTL_HD double normal_quantile(double p) {
  const double a[6] = {-39.6968302866538, 220.9460984245205, -275.9285104469687,
                       138.3577518678900, -30.6647980661472, 2.506628277459239};
  const double b[5] = {-54.4760987982241, 161.5858368580409, -155.6989798598867, 66.8013118877197,
                       -13.28068155278571};
  const double c[6] = {-0.007784894002430293, -0.3223964580411364, -2.4007582771618388,
                       -2.5497325393437340,   4.3746641414649678,  2.9381639826987831};
  const double d[4] = {0.0077846957090414622, 0.32246712907003983, 2.4451341371429960, 3.7544086619074161};
  p = fmin(fmax(p, 1e-15), 1.0 - 1e-15);
  const double target = p;
  const bool upper = p > 0.5;
  if (upper) p = 1.0 - p;
  double v;
  if (p < 0.02425) {
    const double q = sqrt(-2.0 * log(p));
    v = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
        ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
  } else {
    const double q = p - 0.5, r = q * q;
    v = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
        (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
  }
  if (upper) v = -v;
  const double cdf = 0.5 * erfc(-v / sqrt(2.0));
  const double phi = exp(-0.5 * v * v) / sqrt(2.0 * 3.14159265358979323846);
  if (phi > 1e-300) {
    const double f = cdf - target;
    const double den = 2.0 * phi * phi + f * v * phi;
    if (den != 0.0) v -= 2.0 * f * phi / den;
  }
  return v;
}

// Two-sided normal tail P(|Z| > |z|) = erfc(|z| / sqrt 2), clipped to
// [0, 1]; 1 for a z that is not finite (pnorm_two_sided, src/util.cpp:116-123).
EQTL_HD double z_two_sided_p(double z) {
  if (!isfinite(z)) return 1.0;
  const double p = erfc(fabs(z) / sqrt(2.0));
  return fmin(1.0, fmax(0.0, p));
}

// NB-GLM score test of one pair (test_glm_nb, src/model_glm.cpp:98-132) from
// U = g'r, gwg = g'Wg, the quadratic form xAx = (X'Wg)' (X'WX)^-1 (X'Wg) and
// the SNP's dosage variance over the samples: beta = U / info,
// se = 1 / sqrt(info), stat = U / sqrt(info), with info = gwg - xAx; p = 1
// (the rest 0) for gvar or info below 1e-12.
EQTL_HD void glm_stats_fp64(double U, double gwg, double xAx, double gvar, eqtl_pair& q) {
  q.beta = q.se = q.t = q.r2 = 0.0;
  q.p = 1.0;
  if (gvar < 1e-12) return;
  const double info = gwg - xAx;
  if (info < 1e-12) return;
  q.beta = U / info;
  q.se = 1.0 / sqrt(info);
  q.t = U / sqrt(info);
  q.p = z_two_sided_p(q.t);
}

// LM pair from gtg = |g_s|^2, gty = g_s . y_s, yty = |y_s|^2.
EQTL_HD void lm_stats_fp64(double gtg, double gty, double yty, double df, eqtl_pair& q) {
  q.beta = q.se = q.t = q.r2 = 0.0;
  q.p = 1.0;
  if (gtg < 1e-12 || df <= 0) return;
  q.beta = gty / gtg;
  const double rss = yty - q.beta * gty;
  const double s2 = fmax(rss / df, 0.0);
  q.se = sqrt(s2 / gtg);
  q.t = q.se > 0 ? q.beta / q.se : 0.0;
  q.p = t_two_sided_p(q.t, df);
  q.r2 = yty > 0 ? 1.0 - rss / yty : 0.0;
}

// LMM pair from its Wald numerator NUM = yg - a'chi0 and Schur denominator
// S = gg - a'A00^-1 a (the tail of lmm_stats_fp64).
EQTL_HD void lmm_stats_num_s(double num, double S, double rss_null, double df, eqtl_pair& q) {
  q.beta = q.se = q.t = q.r2 = 0.0;
  q.p = 1.0;
  if (S <= 1e-15) return;
  const double bg = num / S;
  double qq = rss_null - S * bg * bg;
  if (qq < 0) qq = 0;
  const double sigma2 = df > 0 ? qq / df : 1.0;
  q.beta = bg;
  q.se = sqrt(fmax(sigma2 / S, 0.0));
  q.t = q.se > 0 ? q.beta / q.se : 0.0;
  q.p = t_two_sided_p(q.t, df);
  q.r2 = rss_null > 1e-15 ? fmax(0.0, 1.0 - qq / rss_null) : 0.0;
}

// LMM pair from gg = Gt'W Gt, yg = Gt'W y~, a = X~'W Gt and the gene's null
// fit (chi0, L = lower Cholesky factor of X~'W X~ row-major, rss_null; L = 0
// where that matrix was not positive definite). a'A00^-1 a is |z|^2 with
// L z = a, a solve as in the reference (src/scan_trans_lmm.cpp:26,
// src/model_lmm.cpp:179): with a badly conditioned A00 an explicit inverse
// loses cond(A00) eps there, the triangular solve only sqrt(cond(A00)) eps,
// and S = gg - a'A00^-1 a can cancel by orders of magnitude.
constexpr int kStatsMaxP = 32;
EQTL_HD void lmm_stats_fp64(double gg, double yg, const double* a, const double* chi0, const double* L,
                            double rss_null, int p, double df, eqtl_pair& q) {
  q.beta = q.se = q.t = q.r2 = 0.0;
  q.p = 1.0;
  if (gg < 1e-12) return;
  double aTu = 0, aTchi = 0;
  if (p > 0 && L[0] > 0) {
    double z[kStatsMaxP];
    for (int x = 0; x < p; ++x) {
      double t = a[x];
      for (int y = 0; y < x; ++y) t -= L[x * p + y] * z[y];
      z[x] = t / L[x * p + x];
      aTu += z[x] * z[x];
    }
  }
  for (int x = 0; x < p; ++x) aTchi += a[x] * chi0[x];
  const double S = gg - aTu;
  if (S <= 1e-15) return;
  const double bg = (yg - aTchi) / S;
  double qq = rss_null - S * bg * bg;
  if (qq < 0) qq = 0;
  const double sigma2 = df > 0 ? qq / df : 1.0;
  q.beta = bg;
  q.se = sqrt(fmax(sigma2 / S, 0.0));
  q.t = q.se > 0 ? q.beta / q.se : 0.0;
  q.p = t_two_sided_p(q.t, df);
  q.r2 = rss_null > 1e-15 ? fmax(0.0, 1.0 - qq / rss_null) : 0.0;
}

}  // namespace eqtl
