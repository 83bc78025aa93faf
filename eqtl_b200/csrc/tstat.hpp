// Host-side statistics shared by the library and the CLI: the beta CDF and
// t critical values on top of the FP64 tail in stats64.hpp, and the
// construction of the interpolation tables the device epilogues use to
// screen t statistics (see tdist.cuh).
#pragma once
#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "stats64.hpp"

namespace eqtl {

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
  while (t_two_sided_p(hi, df) > pthr && hi < 1e30) hi *= 2;  // df = 1: p = 1e-14 at |t| ~ 6e13
  for (int i = 0; i < 200; ++i) {
    const double mid = 0.5 * (lo + hi);
    if (t_two_sided_p(mid, df) > pthr) lo = mid;
    else hi = mid;
  }
  return hi;
}

// |z| at which the two-sided normal p equals pthr.
inline double z_critical(double pthr) {
  if (!(pthr > 0)) return std::numeric_limits<double>::infinity();
  if (pthr >= 1) return 0.0;
  double lo = 0.0, hi = 1.0;
  while (z_two_sided_p(hi) > pthr && hi < 1e30) hi *= 2;
  for (int i = 0; i < 200; ++i) {
    const double mid = 0.5 * (lo + hi);
    if (z_two_sided_p(mid) > pthr) lo = mid;
    else hi = mid;
  }
  return hi;
}

// The tail variable of a normal table: x = sqrt(log1p(z^2 / kZTableD)). Any
// scale works (ln p is analytic in x); this one spreads z in [1, 38] over x
// in [0.01, 0.37].
constexpr double kZTableD = 1e4;

// Interpolation tables for the device t tail (layout documented in tdist.cuh).
// A table built with normal = true holds the two-sided normal tail instead
// (the NB-GLM score statistic), with df = kZTableD as the tail scale.
struct TTableHost {
  bool normal = false;
  double df = 0;
  double t0 = 1.0;               // central / tail boundary in |t|
  int na = 512;                  // central intervals over u = t^2 in [0, t0^2]
  int nb = 4096;                 // tail intervals over x = sqrt(log1p(t^2/df)) in [x0, x_end]
  double x0 = 0, x_end = 0;
  // ACAT screening tables of the scan epilogues (tdist.cuh, acat_screen):
  std::vector<float> c1;   // na + 4 nodes on the central u grid: |t| * tan((1/2 - p) pi)
  std::vector<float> lt;   // nb + 4 nodes on x in [x0, x_defer]: ln tan((1/2 - p) pi); with lt_u, the
                           // term tan((1/2 - p) pi) itself on u = t^2 in [t0^2, t_defer^2]
  bool lt_u = false;       // the tail table is linear in u (short tails: df large enough, or normal)
  double du_t = 0;         // its u step
  // With lt_u, the screen reads per-interval cubics instead of nodes: four
  // coefficients (a0, a1, a2, a3) per interval, y = a0 + a1 f + a2 f^2 + a3 f^3
  // at the fraction f of the interval (one 16-byte load per pair):
  // (their own split at u = uq0: the term is far from exponential in u just
  // above t0 = 1, where a cubic on the tail's coarser step would be off by
  // up to 4e-5 at df = 30)
  double uq0 = 4.0;
  std::vector<float> c1q;  // na intervals on u in [0, uq0]: |t| * tan((1/2 - p) pi)
  std::vector<float> ltq;  // nq intervals on u in [uq0, t_defer^2]: tan((1/2 - p) pi)
  int nq = 1024;
  double du_q = 0;
  double x_defer = 0;      // tail grid end: x at p = 1e-14
  double t_defer = 0;      // |t| with p = 1e-14: beyond it the term is left to the host
  std::vector<float> h;          // na + 4 nodes: h(u) = (1 - p) / |t|, node k at u = (k-1) du
  std::vector<float> L;          // nb + 4 nodes: ln p at x = x0 + (k-1) dx
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

// z cot z as a function of w = z^2 (even in z, analytic in w; y coth y for w < 0).
inline double zcotz(double w) {
  if (std::fabs(w) < 1e-8) return 1.0 - w / 3.0 - w * w / 45.0;
  if (w > 0) {
    const double z = std::sqrt(w);
    return z * std::cos(z) / std::sin(z);
  }
  const double y = std::sqrt(-w);
  return y * std::cosh(y) / std::sinh(y);
}

// The normal counterpart of central_h: 1 - p = |z| h(z^2) with
// h(u) = 2 phi0 \int_0^1 exp(-x^2 u / 2) dx, phi0 = 1 / sqrt(2 pi).
inline double central_h_normal(double u) {
  static std::vector<double> xg, wg;
  if (xg.empty()) gauss_legendre(24, xg, wg);
  double acc = 0;
  for (int seg = 0; seg < 4; ++seg) {
    const double a = 0.25 * seg, hw = 0.125;
    for (size_t i = 0; i < xg.size(); ++i) {
      const double xx = a + hw + hw * xg[i];
      acc += hw * wg[i] * std::exp(-0.5 * xx * xx * u);
    }
  }
  return 2.0 * acc / std::sqrt(2.0 * M_PI);
}

// Coefficients of the cubic through (-1, y0), (0, y1), (1, y2), (2, y3) in
// powers of f (the interval between the middle nodes is f in [0, 1]).
inline void cubic_coeffs(double y0, double y1, double y2, double y3, float* a) {
  a[0] = static_cast<float>(y1);
  a[1] = static_cast<float>(-y0 / 3.0 - y1 / 2.0 + y2 - y3 / 6.0);
  a[2] = static_cast<float>(0.5 * (y0 + y2) - y1);
  a[3] = static_cast<float>((y3 - y0) / 6.0 + 0.5 * (y1 - y2));
}

inline TTableHost build_ttable(double df, bool normal = false) {
  TTableHost T;
  T.normal = normal;
  if (normal) df = kZTableD;
  T.df = df;
  auto pfun = [&](double t) { return normal ? z_two_sided_p(t) : t_two_sided_p(t, df); };
  auto hfun = [&](double u) { return normal ? central_h_normal(u) : central_h(u, df); };
  // p(t0) < 1/2 keeps the tail's tan term away from 0 (df = 1 has p(1) = 1/2)
  T.t0 = !normal && df < 1.5 ? 1.5 : 1.0;
  const double du = (T.t0 * T.t0) / T.na;
  T.h.resize(T.na + 4);
  for (int k = 0; k < T.na + 4; ++k) T.h[k] = static_cast<float>(hfun((k - 1) * du));
  T.x0 = std::sqrt(std::log1p(T.t0 * T.t0 / df));
  auto lnp = [&](double x) {
    const double t = std::sqrt(df * std::expm1(x * x));
    const double p = pfun(t);
    return p > 0 ? std::log(p) : -1e30;
  };
  // x_end: where ln p reaches ln(1e-320) (beyond it the reference's p
  // underflows), capped at |t| = 1e19, past which the FP32 t^2 of the
  // epilogue overflows (small df). Pairs beyond x_end are deferred to the
  // FP64 refinement. Bracket by doubling, then bisect so the nodes span
  // only the range in use.
  const double kLnFloor = std::log(1e-320);
  const double x_cap = std::sqrt(std::log1p(1e38 / df));
  if (lnp(x_cap) > kLnFloor) {
    T.x_end = x_cap;
  } else {
    double lo = T.x0, hi = std::min(T.x0 + 1.0, x_cap);
    while (lnp(hi) > kLnFloor) {
      lo = hi;
      hi = std::min(T.x0 + 2 * (hi - T.x0), x_cap);
    }
    for (int it = 0; it < 80; ++it) {
      const double mid = 0.5 * (lo + hi);
      (lnp(mid) > kLnFloor ? lo : hi) = mid;
    }
    T.x_end = hi;
  }
  const double dx = (T.x_end - T.x0) / T.nb;
  T.L.resize(T.nb + 4);
  for (int k = 0; k < T.nb + 4; ++k) {
    double v = lnp(T.x0 + (k - 1) * dx);
    if (v < -1e29) v = 2.0 * T.L[k - 1] - T.L[k - 2];  // past underflow: extrapolate
    T.L[k] = static_cast<float>(v);
  }
  // ACAT screening. Central: 1 - p = |t| h(u), so |t| tan((1/2 - p) pi) =
  // -|t| cot(pi |t| h) = -(z cot z) / (pi h) with z^2 = pi^2 u h^2, analytic
  // in u (also at the node below 0). Tail: ln tan((1/2 - p) pi) = ln cot(pi p),
  // smooth in x up to p = 1e-14, past which the host adds the term.
  auto c1fun = [&](double u) {
    const double h = hfun(u);
    return -zcotz(M_PI * M_PI * u * h * h) / (M_PI * h);
  };
  T.c1.resize(T.na + 4);
  for (int k = 0; k < T.na + 4; ++k) T.c1[k] = static_cast<float>(c1fun((k - 1) * du));
  T.t_defer = normal ? z_critical(1e-14) : t_critical(1e-14, df);
  T.x_defer = std::sqrt(std::log1p(T.t_defer * T.t_defer / df));
  T.lt.resize(T.nb + 4);
  // Where the tail up to p = 1e-14 is short in u (t_defer^2 within ~200 of
  // t0^2: df above ~30, and the normal tail), the term itself is smooth
  // enough in u for the cubic (it grows about as exp(u / 2), 0.05 per step
  // at most), and the epilogue's grid position is one FMA of u; longer
  // tails keep the x grid of ln tan((1/2 - p) pi).
  const double du_t = (T.t_defer * T.t_defer - T.t0 * T.t0) / T.nb;
  if (du_t <= 0.05) {
    T.lt_u = true;
    T.du_t = du_t;
    auto term = [&](double u) {
      const double p = pfun(std::sqrt(u));
      return std::cos(M_PI * p) / std::sin(M_PI * p);
    };
    for (int k = 0; k < T.nb + 4; ++k) T.lt[k] = static_cast<float>(term(T.t0 * T.t0 + (k - 1) * du_t));
    // the per-interval cubics: above uq0 the term grows about as exp(u / 2)
    // (fourth derivative ~ 1/16 of it), so at nq = 1024 intervals (u step
    // <= 0.2) the cubic's relative error stays below 1.5e-3 step^4 ~ 3e-6
    const double du_c = T.uq0 / T.na;
    std::vector<double> cd(T.na + 3);
    for (int k = 0; k < T.na + 3; ++k) cd[k] = c1fun((k - 1) * du_c);
    T.c1q.resize(4 * static_cast<size_t>(T.na));
    for (int i = 0; i < T.na; ++i) cubic_coeffs(cd[i], cd[i + 1], cd[i + 2], cd[i + 3], &T.c1q[4 * i]);
    T.du_q = (T.t_defer * T.t_defer - T.uq0) / T.nq;
    std::vector<double> ld(T.nq + 3);
    for (int k = 0; k < T.nq + 3; ++k) ld[k] = term(T.uq0 + (k - 1) * T.du_q);
    T.ltq.resize(4 * static_cast<size_t>(T.nq));
    for (int i = 0; i < T.nq; ++i) cubic_coeffs(ld[i], ld[i + 1], ld[i + 2], ld[i + 3], &T.ltq[4 * i]);
    return T;
  }
  const double dl = (T.x_defer - T.x0) / T.nb;
  for (int k = 0; k < T.nb + 4; ++k) {
    const double x = T.x0 + (k - 1) * dl;
    const double t = std::sqrt(df * std::expm1(x * x));
    const double p = pfun(t);
    T.lt[k] = static_cast<float>(std::log(std::cos(M_PI * p) / std::sin(M_PI * p)));
  }
  return T;
}

}  // namespace eqtl
