// FP64 statistics shared by the host side of the library and the CLI:
// Student-t two-sided p-value through the regularised incomplete beta
// function (Lentz's continued fraction with the same constants as the
// reference: maxit 200, eps 3e-12, fpmin 1e-30; src/util.cpp:209-264), and
// the construction of the interpolation tables the device epilogues use to
// screen t statistics (see tdist.cuh).
#pragma once
#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

namespace eqtl {

inline double incbeta_cf(double a, double b, double x) {
  const int kMaxIt = 200;
  const double kEps = 3e-12, kTiny = 1e-30;
  const double qab = a + b, qap = a + 1.0, qam = a - 1.0;
  double c = 1.0;
  double d = 1.0 - qab * x / qap;
  if (std::fabs(d) < kTiny) d = kTiny;
  d = 1.0 / d;
  double h = d;
  for (int m = 1; m <= kMaxIt; ++m) {
    const int m2 = 2 * m;
    double aa = m * (b - m) * x / ((qam + m2) * (a + m2));
    d = 1.0 + aa * d;
    if (std::fabs(d) < kTiny) d = kTiny;
    c = 1.0 + aa / c;
    if (std::fabs(c) < kTiny) c = kTiny;
    d = 1.0 / d;
    h *= d * c;
    aa = -(a + m) * (qab + m) * x / ((a + m2) * (qap + m2));
    d = 1.0 + aa * d;
    if (std::fabs(d) < kTiny) d = kTiny;
    c = 1.0 + aa / c;
    if (std::fabs(c) < kTiny) c = kTiny;
    d = 1.0 / d;
    const double del = d * c;
    h *= del;
    if (std::fabs(del - 1.0) < kEps) break;
  }
  return h;
}

// I_x(a, b)
inline double incbeta(double a, double b, double x) {
  if (x < 0 || x > 1) return std::numeric_limits<double>::quiet_NaN();
  if (x == 0 || x == 1) return x;
  const double lbeta = std::lgamma(a) + std::lgamma(b) - std::lgamma(a + b);
  const double front = std::exp(std::log(x) * a + std::log(1 - x) * b - lbeta) / a;
  if (x < (a + 1) / (a + b + 2)) return front * incbeta_cf(a, b, x);
  return 1.0 - front * incbeta_cf(b, a, 1 - x) * a / b;
}

inline double t_two_sided_p(double t, double df) {
  if (!std::isfinite(t) || df <= 0) return 1.0;
  const double x = df / (df + t * t);
  const double p = incbeta(0.5 * df, 0.5, x);
  return std::min(1.0, std::max(0.0, p));
}

inline double beta_cdf(double x, double a, double b) {
  if (a <= 0 || b <= 0) return std::numeric_limits<double>::quiet_NaN();
  if (x <= 0) return 0;
  if (x >= 1) return 1;
  return incbeta(a, b, x);
}

// |t| at which the two-sided p equals pthr (bisection on the monotone tail).
inline double t_critical(double pthr, double df) {
  if (!(pthr > 0)) return std::numeric_limits<double>::infinity();
  if (pthr >= 1) return 0.0;
  double lo = 0.0, hi = 1.0;
  while (t_two_sided_p(hi, df) > pthr && hi < 1e8) hi *= 2;
  for (int i = 0; i < 200; ++i) {
    const double mid = 0.5 * (lo + hi);
    if (t_two_sided_p(mid, df) > pthr) lo = mid;
    else hi = mid;
  }
  return hi;
}

// Interpolation tables for the device t tail (layout documented in tdist.cuh).
struct TTableHost {
  double df = 0;
  double t0 = 1.0;               // central / tail boundary in |t|
  int na = 512;                  // central intervals over u = t^2 in [0, t0^2]
  int nb = 4096;                 // tail intervals over s = log1p(t^2/df)
  double s0 = 0, s_end = 0;
  std::vector<float> h;          // na + 4 nodes: h(u) = (1 - p) / |t|, node k at u = (k-1) du
  std::vector<float> L;          // nb + 4 nodes: ln p at s = s0 + (k-1) ds
};

inline double t_density_const(double df) {
  return std::exp(std::lgamma(0.5 * (df + 1)) - std::lgamma(0.5 * df)) / std::sqrt(df * M_PI);
}

// Gauss-Legendre nodes/weights on [-1, 1] by Newton iteration on P_n.
inline void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      const double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1e-15) break;
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

// h(u) = 2 c \int_0^1 (1 + x^2 u / df)^{-(df+1)/2} dx, so that 1 - p = |t| h(t^2);
// analytic in u (also slightly below 0). Composite 4 x 24-point Gauss-Legendre.
inline double central_h(double u, double df) {
  static std::vector<double> xg, wg;
  if (xg.empty()) gauss_legendre(24, xg, wg);
  const double c = t_density_const(df);
  double acc = 0;
  for (int seg = 0; seg < 4; ++seg) {
    const double a = 0.25 * seg, hw = 0.125;
    for (size_t i = 0; i < xg.size(); ++i) {
      const double xx = a + hw + hw * xg[i];
      acc += hw * wg[i] * std::pow(1.0 + xx * xx * u / df, -0.5 * (df + 1));
    }
  }
  return 2.0 * c * acc;
}

inline TTableHost build_ttable(double df) {
  TTableHost T;
  T.df = df;
  const double du = (T.t0 * T.t0) / T.na;
  T.h.resize(T.na + 4);
  for (int k = 0; k < T.na + 4; ++k) T.h[k] = static_cast<float>(central_h((k - 1) * du, df));
  T.s0 = std::log1p(T.t0 * T.t0 / df);
  // s where ln p falls below ln(1e-320): beyond it the reference's p underflows.
  double s_hi = T.s0 + 1.0;
  auto lnp = [&](double s) {
    const double t = std::sqrt(df * std::expm1(s));
    const double p = t_two_sided_p(t, df);
    return p > 0 ? std::log(p) : -1e30;
  };
  while (lnp(s_hi) > std::log(1e-320) && s_hi < 1e4) s_hi = T.s0 + 2 * (s_hi - T.s0);
  T.s_end = s_hi;
  const double ds = (T.s_end - T.s0) / T.nb;
  T.L.resize(T.nb + 4);
  for (int k = 0; k < T.nb + 4; ++k) {
    const double s = T.s0 + (k - 1) * ds;
    double v;
    if (s <= T.s0 - 0.5 * ds) {
      // below the tail's first node: extend smoothly from the exact value
      const double t = std::sqrt(std::max(df * std::expm1(s), 0.0));
      v = std::log(t_two_sided_p(t, df));
    } else {
      v = lnp(s);
      if (v < -1e29) v = T.L[k - 1] + (T.L[k - 1] - T.L[k - 2]);  // past underflow: extrapolate
    }
    T.L[k] = static_cast<float>(v);
  }
  return T;
}

}  // namespace eqtl
