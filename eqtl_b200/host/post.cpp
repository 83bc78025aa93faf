// Per-gene statistics computed on the host after the device scans, with the
// reference's definitions:
//   ACAT p        0.5 - atan(mean tan term) / pi in long double, clamped
//                 (AcatAcc::p, src/stats_extra.cpp:24-31)
//   BH q          step-up over the genes of one scope (src/scan_common.cpp:201-217)
//   p_emp         (1 + #{T_perm >= T_obs}) / (1 + B) (src/stats_extra.cpp:39-46)
//   beta approx   method-of-moments start, Nelder-Mead on the beta likelihood
//                 within s1 in [0.1, 10], s2 in [5, 1e6], then I_p(s1, s2)
//                 (src/stats_extra.cpp:79-158)
//   perm seed     (seed or 1) + b * 9973 + fnv1a(gene) (include/eqtl/scan_cis.hpp:106-111)
#include <algorithm>
#include <numeric>

#include "host.hpp"
#include "tstat.hpp"

namespace eqtl_host {

double acat_p(double tan_sum, int used) {
  if (used <= 0) return 1.0;
  const long double kPiL = 3.14159265358979323846264338327950288L;
  const long double T = static_cast<long double>(tan_sum) / static_cast<long double>(used);
  const double ac = 0.5 - static_cast<double>(atanl(T) / kPiL);
  return std::min(std::max(ac, 0.0), 1.0);
}

std::vector<double> bh_adjust(const std::vector<double>& a) {
  const size_t m = a.size();
  std::vector<double> q(m);
  std::vector<size_t> idx(m);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return a[x] < a[y]; });
  double prev = 1.0;
  for (size_t rank = m; rank >= 1; --rank) {
    const size_t j = idx[rank - 1];
    double v = a[j] * static_cast<double>(m) / static_cast<double>(rank);
    v = std::min(std::min(v, prev), 1.0);
    q[j] = v;
    prev = v;
  }
  return q;
}


uint64_t fnv1a64(const std::string& s) {
  uint64_t h = 14695981039346656037ull;
  for (unsigned char ch : s) {
    h ^= ch;
    h *= 1099511628211ull;
  }
  return h;
}

uint32_t fnv1a32(const std::string& s) { return static_cast<uint32_t>(fnv1a64(s)); }

uint32_t perm_seed(int seed_opt, int b, const std::string& gene) {
  const uint64_t base = seed_opt >= 0 ? static_cast<uint64_t>(seed_opt) : 1u;
  return static_cast<uint32_t>(base + static_cast<uint64_t>(b) * 9973u + fnv1a32(gene));
}

double p_emp(double T_obs, const std::vector<double>& T_perm) {
  size_t ge = 0;
  for (double t : T_perm)
    if (t >= T_obs) ++ge;
  return (1.0 + static_cast<double>(ge)) / (1.0 + static_cast<double>(T_perm.size()));
}

namespace {

// Nelder-Mead with the moves of GSL's nmsimplex2 (reflect through the
// centroid of the others, expand, contract, shrink towards the best vertex)
// and its stopping size: the RMS distance of the vertices from their centroid.
struct Simplex2 {
  template <class F>
  static bool minimise(F f, double x[2], const double step[2], double tol, int maxit) {
    double v[3][2] = {{x[0], x[1]}, {x[0] + step[0], x[1]}, {x[0], x[1] + step[1]}};
    double fv[3] = {f(v[0]), f(v[1]), f(v[2])};
    const double P = 3.0;
    double c[2], size;
    auto center_size = [&]() {
      c[0] = (v[0][0] + v[1][0] + v[2][0]) / P;
      c[1] = (v[0][1] + v[1][1] + v[2][1]) / P;
      double s = 0;
      for (int i = 0; i < 3; ++i) s += (v[i][0] - c[0]) * (v[i][0] - c[0]) + (v[i][1] - c[1]) * (v[i][1] - c[1]);
      size = std::sqrt(s / P);
    };
    center_size();
    bool ok = false;
    for (int it = 1;; ++it) {
      int hi = 0, lo = 0, s_hi = 1;
      double dhi = fv[0], dlo = fv[0], ds_hi = fv[1];
      for (int i = 1; i < 3; ++i) {
        const double y = fv[i];
        if (y < dlo) {
          dlo = y;
          lo = i;
        } else if (y > dhi) {
          ds_hi = dhi;
          s_hi = hi;
          dhi = y;
          hi = i;
        } else if (y > ds_hi) {
          ds_hi = y;
          s_hi = i;
        }
      }
      auto move = [&](double coeff, double out[2]) {
        const double alpha = (1 - coeff) * P / (P - 1.0), beta = (P * coeff - 1.0) / (P - 1.0);
        out[0] = alpha * c[0] + beta * v[hi][0];
        out[1] = alpha * c[1] + beta * v[hi][1];
      };
      double xr[2];
      move(-1.0, xr);
      const double fr = f(xr);
      if (std::isfinite(fr) && fr < fv[lo]) {
        double xe[2];
        move(-2.0, xe);
        const double fe = f(xe);
        if (std::isfinite(fe) && fe < fv[lo]) {
          v[hi][0] = xe[0], v[hi][1] = xe[1], fv[hi] = fe;
        } else {
          v[hi][0] = xr[0], v[hi][1] = xr[1], fv[hi] = fr;
        }
        center_size();
      } else if (!std::isfinite(fr) || fr > fv[s_hi]) {
        if (std::isfinite(fr) && fr <= fv[hi]) {
          v[hi][0] = xr[0], v[hi][1] = xr[1], fv[hi] = fr;
          center_size();
        }
        double xk[2];
        move(0.5, xk);
        const double fk = f(xk);
        if (std::isfinite(fk) && fk <= fv[hi]) {
          v[hi][0] = xk[0], v[hi][1] = xk[1], fv[hi] = fk;
        } else {
          for (int i = 0; i < 3; ++i)
            if (i != lo) {
              v[i][0] = 0.5 * (v[i][0] + v[lo][0]);
              v[i][1] = 0.5 * (v[i][1] + v[lo][1]);
              fv[i] = f(v[i]);
            }
        }
        center_size();
      } else {
        v[hi][0] = xr[0], v[hi][1] = xr[1], fv[hi] = fr;
        center_size();
      }
      if (size < tol) {
        ok = true;
        break;
      }
      if (it >= maxit) break;
    }
    int best = 0;
    for (int i = 1; i < 3; ++i)
      if (fv[i] < fv[best]) best = i;
    x[0] = v[best][0];
    x[1] = v[best][1];
    return ok;
  }
};

}  // namespace

BetaFit beta_approx(const std::vector<double>& perm_min_p, double obs_min_p) {
  BetaFit out;
  std::vector<double> x;
  for (double v : perm_min_p)
    if (std::isfinite(v) && v > 0.0 && v < 1.0) x.push_back(v);
  if (x.size() < 10) return out;
  // method of moments
  double mean = 0;
  for (double v : x) mean += v;
  mean /= static_cast<double>(x.size());
  double var = 0;
  for (double v : x) var += (v - mean) * (v - mean);
  var /= static_cast<double>(x.size() - 1);
  if (var <= 0 || mean <= 0 || mean >= 1) return out;
  const double tt = mean * (1.0 - mean) / var - 1.0;
  if (tt <= 0) return out;
  double s1 = mean * tt, s2 = (1.0 - mean) * tt;
  double S1 = 0, S2 = 0;
  for (double v : x) {
    const double xv = v >= 1.0 ? 0.99999999 : v;
    S1 += std::log(xv);
    S2 += std::log(1.0 - xv);
  }
  const double N = static_cast<double>(x.size());
  auto nll = [&](const double* v) {
    const double a = v[0], b = v[1];
    if (!(a >= 0.1 && a <= 10.0 && b >= 5.0 && b <= 1e6)) return 1e300;
    const double lnb = std::lgamma(a) + std::lgamma(b) - std::lgamma(a + b);
    return -((a - 1.0) * S1 + (b - 1.0) * S2 - N * lnb);
  };
  if (s1 > 0 && s2 > 0) {
    double xb[2] = {s1, s2};
    const double step[2] = {s1 / 10.0, s2 / 10.0};
    const bool conv = Simplex2::minimise(nll, xb, step, 0.01, 1000);
    if (conv && std::isfinite(xb[0]) && std::isfinite(xb[1]) && xb[0] >= 0.1 && xb[0] <= 10.0 && xb[1] >= 5.0 &&
        xb[1] <= 1e6) {
      s1 = xb[0];
      s2 = xb[1];
    }
  }
  const double o = std::min(std::max(obs_min_p, 1e-300), 1.0 - 1e-16);
  const double pb = eqtl::beta_cdf(o, s1, s2);
  out.p = std::isfinite(pb) ? pb : NAN;
  out.s1 = s1;
  out.s2 = s2;
  return out;
}

}  // namespace eqtl_host
