// Test infrastructure only: the slice of the GSL multimin API that
// src/stats_extra.cpp:95-126 (beta_fit_ml_simplex) uses, so the reference can
// be compiled here without GSL. The minimiser restates the published
// Nelder-Mead variant GSL ships as `nmsimplex2` (reflection -1, expansion -2,
// one-dimensional contraction 0.5, shrink toward the best vertex; simplex
// size = RMS distance of the vertices from their centroid). GSL itself is not
// vendored by the reference, so p_beta / beta_shape{1,2} are unpinned against
// a real GSL build; the product's fit (eqtl_b200/host/stats.cpp) restates the
// same algorithm.
#pragma once
#include <cmath>
#include <cstddef>
#include <vector>

enum { GSL_SUCCESS = 0, GSL_CONTINUE = -2, GSL_ENOPROG = 27 };

struct gsl_vector {
  size_t size;
  std::vector<double> v;
};
inline gsl_vector* gsl_vector_alloc(size_t n) { return new gsl_vector{n, std::vector<double>(n, 0.0)}; }
inline void gsl_vector_free(gsl_vector* v) { delete v; }
inline double gsl_vector_get(const gsl_vector* v, size_t i) { return v->v[i]; }
inline void gsl_vector_set(gsl_vector* v, size_t i, double x) { v->v[i] = x; }

struct gsl_multimin_function {
  double (*f)(const gsl_vector*, void*);
  size_t n;
  void* params;
};

struct gsl_multimin_fminimizer_type { int unused; };
static const gsl_multimin_fminimizer_type gsl_nmsimplex2_type_shim{0};
static const gsl_multimin_fminimizer_type* gsl_multimin_fminimizer_nmsimplex2 = &gsl_nmsimplex2_type_shim;

struct gsl_multimin_fminimizer {
  size_t n = 0;                    // dimension
  std::vector<std::vector<double>> xs;  // n+1 vertices
  std::vector<double> ys;          // function values
  std::vector<double> center;
  double size = 0;
  gsl_multimin_function* f = nullptr;
  gsl_vector* x = nullptr;         // best vertex (public, like GSL's s->x)
  double fval = 0;
};

inline gsl_multimin_fminimizer* gsl_multimin_fminimizer_alloc(const gsl_multimin_fminimizer_type*, size_t n) {
  auto* s = new gsl_multimin_fminimizer;
  s->n = n;
  s->x = gsl_vector_alloc(n);
  return s;
}
inline void gsl_multimin_fminimizer_free(gsl_multimin_fminimizer* s) {
  gsl_vector_free(s->x);
  delete s;
}

namespace shim_nm {
inline double eval(gsl_multimin_fminimizer* s, const std::vector<double>& p) {
  gsl_vector tmp{s->n, p};
  return s->f->f(&tmp, s->f->params);
}
inline void recompute(gsl_multimin_fminimizer* s) {
  const size_t P = s->n + 1;
  s->center.assign(s->n, 0.0);
  for (size_t i = 0; i < P; ++i)
    for (size_t j = 0; j < s->n; ++j) s->center[j] += s->xs[i][j] / static_cast<double>(P);
  double ss = 0;
  for (size_t i = 0; i < P; ++i) {
    double d2 = 0;
    for (size_t j = 0; j < s->n; ++j) {
      const double d = s->xs[i][j] - s->center[j];
      d2 += d * d;
    }
    ss += d2;
  }
  s->size = std::sqrt(ss / static_cast<double>(P));
}
// Point obtained by moving vertex `corner` with coefficient `coeff` relative to
// the centroid of the other vertices (-1 reflect, -2 expand, 0.5 contract).
inline std::vector<double> corner_move(gsl_multimin_fminimizer* s, double coeff, size_t corner) {
  const double P = static_cast<double>(s->n + 1);
  const double alpha = (1.0 - coeff) * P / (P - 1.0);
  const double beta = (P * coeff - 1.0) / (P - 1.0);
  std::vector<double> xc(s->n);
  for (size_t j = 0; j < s->n; ++j) xc[j] = alpha * s->center[j] + beta * s->xs[corner][j];
  return xc;
}
inline void set_best(gsl_multimin_fminimizer* s) {
  size_t lo = 0;
  for (size_t i = 1; i < s->ys.size(); ++i)
    if (s->ys[i] < s->ys[lo]) lo = i;
  s->x->v = s->xs[lo];
  s->fval = s->ys[lo];
}
}  // namespace shim_nm

inline int gsl_multimin_fminimizer_set(gsl_multimin_fminimizer* s, gsl_multimin_function* f, const gsl_vector* x,
                                       const gsl_vector* step) {
  s->f = f;
  const size_t n = s->n;
  s->xs.assign(n + 1, x->v);
  for (size_t i = 0; i < n; ++i) s->xs[i + 1][i] += step->v[i];
  s->ys.resize(n + 1);
  for (size_t i = 0; i <= n; ++i) s->ys[i] = shim_nm::eval(s, s->xs[i]);
  shim_nm::recompute(s);
  shim_nm::set_best(s);
  return GSL_SUCCESS;
}

inline int gsl_multimin_fminimizer_iterate(gsl_multimin_fminimizer* s) {
  const size_t P = s->n + 1;
  auto& y = s->ys;
  size_t hi = 0, lo = 0, s_hi = 1;
  double dhi = y[0], dlo = y[0], ds_hi = y[1];
  for (size_t i = 1; i < P; ++i) {
    const double v = y[i];
    if (v < dlo) { dlo = v; lo = i; }
    else if (v > dhi) { ds_hi = dhi; s_hi = hi; dhi = v; hi = i; }
    else if (v > ds_hi) { ds_hi = v; s_hi = i; }
  }
  auto replace = [&](size_t i, const std::vector<double>& p, double v) {
    s->xs[i] = p;
    y[i] = v;
    shim_nm::recompute(s);
  };
  std::vector<double> xr = shim_nm::corner_move(s, -1.0, hi);
  const double vr = shim_nm::eval(s, xr);
  if (std::isfinite(vr) && vr < y[lo]) {
    std::vector<double> xe = shim_nm::corner_move(s, -2.0, hi);
    const double ve = shim_nm::eval(s, xe);
    if (std::isfinite(ve) && ve < y[lo]) replace(hi, xe, ve);
    else replace(hi, xr, vr);
  } else if (!std::isfinite(vr) || vr > y[s_hi]) {
    if (std::isfinite(vr) && vr <= y[hi]) replace(hi, xr, vr);
    std::vector<double> xk = shim_nm::corner_move(s, 0.5, hi);
    const double vk = shim_nm::eval(s, xk);
    if (std::isfinite(vk) && vk <= y[hi]) {
      replace(hi, xk, vk);
    } else {
      for (size_t i = 0; i < P; ++i) {
        if (i == lo) continue;
        for (size_t j = 0; j < s->n; ++j) s->xs[i][j] = 0.5 * (s->xs[i][j] + s->xs[lo][j]);
        y[i] = shim_nm::eval(s, s->xs[i]);
      }
      shim_nm::recompute(s);
    }
  } else {
    replace(hi, xr, vr);
  }
  shim_nm::set_best(s);
  return GSL_SUCCESS;
}

inline double gsl_multimin_fminimizer_size(const gsl_multimin_fminimizer* s) { return s->size; }
inline int gsl_multimin_test_size(double size, double epsabs) {
  return size < epsabs ? GSL_SUCCESS : GSL_CONTINUE;
}
