// LMM path: eigenbasis, spectral rotation (K3), batched REML (K7) and the
// trans/gw LMM scan (K5).
//
// Restates src/model_lmm.cpp and src/scan_trans_lmm.cpp:82-251 on the
// shared-keep path:
//   basis     K = Q diag(lambda) Q', lambda clipped at 0 (make_lmm_basis,
//             src/model_lmm.cpp:106-113) - cuSOLVER syevd, or a basis the
//             caller supplies;
//   rotate    Gt = Q' (g - mean) for every kept SNP on the tensor cores
//             (FP16 hi/lo x hi/lo), written once as FP16 hi/lo pairs of Gt
//             and Gt^2 (the SNP-side operands of the scan);
//   REML      per gene: y~ = Q'y, X~ = Q'X, delta by the reference's grid /
//             golden-section / Newton search on reml_negll
//             (src/model_lmm.cpp:10-86), then dinv, A00, chi0, rss_null
//             (prep_lmm, :124-153) - one CTA per gene, FP64;
//   scan      per (gene, SNP) the bordered-Schur Wald test
//             (src/scan_trans_lmm.cpp:11-40) from three contractions
//               NUM = Gt . (w o r~)      (= yg - a'chi0, r~ = y~ - X~ chi0)
//               a_k = Gt . (w o X~_k)
//               gg  = Gt^2 . w
//             S = gg - a' A00^-1 a, t^2 = df r/(1-r), r = NUM^2/(S rss_null);
//   refine    candidates and each gene's best recomputed in FP64 from raw
//             dosages rotated by cuBLAS DGEMM.
#include <cublas_v2.h>
#include <cusolverDn.h>
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <limits>
#include <memory>
#include <type_traits>

#include "internal.hpp"
#include "scan_host.hpp"
#include "simt_tile.cuh"
#include "tstat.hpp"

namespace eqtl {
namespace dev {

constexpr int kMaxPLmm = 32;
static_assert(kMaxPLmm + 2 <= kMaxAcc, "the grouped LMM scan needs p + 2 accumulators");
static_assert(sizeof(Workspace::ops_hi) / sizeof(Workspace::ops_hi[0]) >= static_cast<size_t>(kMaxAcc),
              "one gene-side operand buffer per accumulator");

// ----------------------------------------------------------- rotation
struct RotEpiParams {
  int n;          // eigen rows (valid)
  int64_t m;      // SNPs
  int k_pad;
  float unscale;  // accumulator -> Gt
  float s1, s2;   // output scales of Gt and Gt^2
  __half *gt_hi, *gt_lo, *gt2_hi, *gt2_lo;
};

struct RotEpi {
  static constexpr bool kGrouped = false;
  using Params = RotEpiParams;
  const Params& P;
  int row = 0;
  int64_t col0 = 0;
  static constexpr int kSmemBytes = 0;
  __device__ RotEpi(const Params& p, const TileShape&, uint8_t*) : P(p) {}
  __device__ void init(int, int) {}
  __device__ void begin_tile(int r, int64_t c0) {
    row = r;
    col0 = c0;
  }
  template <int NACC>
  __device__ void chunk(int c, const float (&v)[NACC][16]) {
    if (row >= P.n) return;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int64_t s = col0 + c + j;
      if (s >= P.m) break;
      const float g = v[0][j] * P.unscale;
      const float a = g * P.s1;
      const float b = g * g * P.s2;
      const __half ah = __float2half_rn(a), bh = __float2half_rn(b);
      const int64_t idx = s * P.k_pad + row;
      P.gt_hi[idx] = ah;
      P.gt_lo[idx] = __float2half_rn(a - __half2float(ah));
      P.gt2_hi[idx] = bh;
      P.gt2_lo[idx] = __float2half_rn(b - __half2float(bh));
    }
  }
  __device__ void end_tile() {}
  __device__ void finish() {}
};

// Qt operand: row j = eigenvector j (column j of column-major Q) * 2^10.
// Q' split into hi + lo rows of T (FP16, or BF16 for the split-BF16 form,
// whose genotype operand is BF16 too)
template <class T>
__global__ void q_split_kernel(const double* __restrict__ Q, int n, int k_pad, T* hi, T* lo) {
  const int j = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k_pad; i += gridDim.x * blockDim.x) {
    const double v = i < n ? Q[static_cast<int64_t>(j) * n + i] * 1024.0 : 0.0;
    if constexpr (std::is_same_v<T, __half>) {
      const __half h = __double2half(v);
      hi[static_cast<int64_t>(j) * k_pad + i] = h;
      lo[static_cast<int64_t>(j) * k_pad + i] = __double2half(v - static_cast<double>(__half2float(h)));
    } else {
      const __nv_bfloat16 h = __double2bfloat16(v);
      hi[static_cast<int64_t>(j) * k_pad + i] = h;
      lo[static_cast<int64_t>(j) * k_pad + i] = __double2bfloat16(v - static_cast<double>(__bfloat162float(h)));
    }
  }
}

// --------------------------------------------------------------- REML
// Packed upper-triangle index of (a, b), a <= b.
__device__ __forceinline__ int tri(int a, int b, int p) { return a * p - a * (a - 1) / 2 + (b - a); }

// Solves A x = b for SPD A (p x p, row-major, Cholesky); returns false if not PD.
__device__ bool chol_solve(const double* A, const double* b, double* x, double* logdet, int p, double* L) {
  for (int j = 0; j < p; ++j) {
    double d = A[j * p + j];
    for (int k = 0; k < j; ++k) d -= L[j * p + k] * L[j * p + k];
    if (!(d > 0)) return false;
    L[j * p + j] = sqrt(d);
    for (int i = j + 1; i < p; ++i) {
      double s = A[i * p + j];
      for (int k = 0; k < j; ++k) s -= L[i * p + k] * L[j * p + k];
      L[i * p + j] = s / L[j * p + j];
    }
  }
  double ld = 0;
  for (int j = 0; j < p; ++j) ld += 2.0 * log(L[j * p + j]);
  *logdet = ld;
  if (b) {
    double y[kMaxPLmm];
    for (int i = 0; i < p; ++i) {
      double s = b[i];
      for (int k = 0; k < i; ++k) s -= L[i * p + k] * y[k];
      y[i] = s / L[i * p + i];
    }
    for (int i = p - 1; i >= 0; --i) {
      double s = y[i];
      for (int k = i + 1; k < p; ++k) s -= L[k * p + i] * x[k];
      x[i] = s / L[i * p + i];
    }
  }
  return true;
}

// optimize_delta (src/model_lmm.cpp:39-86): grid 1e-5..1e5 x2 (and 1.0), 40
// golden-section steps on [best/4, best*4] clipped to [1e-8, 1e6], then up to
// 8 Newton steps on central differences. f(d) returns -loglik and is called
// by every thread of the unit (warp or block) that evaluates it.
template <class F>
__device__ double optimize_delta_dev(F&& f, int df) {
  double d = 1.0;
  if (df <= 0) return d;
  double best_d = 1.0;
  double best_ll = f(1.0);
  for (double dd = 1e-5; dd <= 1e5; dd *= 2.0) {
    const double v = f(dd);
    if (v < best_ll) {
      best_ll = v;
      best_d = dd;
    }
  }
  double lo = best_d / 4.0, hi = best_d * 4.0;
  if (lo < 1e-8) lo = 1e-8;
  if (hi > 1e6) hi = 1e6;
  const double phi = (1.0 + sqrt(5.0)) / 2.0;
  for (int it = 0; it < 40; ++it) {
    const double m1 = hi - (hi - lo) / phi;
    const double m2 = lo + (hi - lo) / phi;
    const double f1 = f(m1);
    const double f2 = f(m2);
    if (f1 < f2) hi = m2;
    else lo = m1;
  }
  d = 0.5 * (lo + hi);
  double cur = f(d);
  for (int it = 0; it < 8; ++it) {
    const double h = fmax(d * 1e-4, 1e-9);
    const double fm = f(d - h);
    const double fp = f(d + h);
    const double g1 = (fp - fm) / (2.0 * h);
    const double g2 = (fp - 2.0 * cur + fm) / (h * h);
    if (!(g2 > 1e-12)) break;
    const double step = g1 / g2;
    const double dn = d - step;
    if (!(dn > 1e-8 && dn < 1e6)) break;
    const double vn = f(dn);
    if (!(vn < cur)) break;
    d = dn;
    cur = vn;
    if (fabs(step) < d * 1e-8) break;
  }
  return d;
}

// prep_lmm caches (src/model_lmm.cpp:124-153) from A = X~'DX~ (p x p,
// row-major), b = X~'Dy~ and y~'Dy~ at the chosen delta; one thread. Besides
// chi0, A^-1 and rss, the lower Cholesky factor of A (row-major, zeros when A
// is not positive definite) for the FP64 pair statistics.
__device__ void reml_caches(double* A, const double* b, double y_dy, int p, int g, double* L, double* e,
                            double* x, double* chi0_out, double* ainv_out, double* rss_out, double* a00L_out) {
  double chi0[kMaxPLmm];
  double ld;
  const bool ok = chol_solve(A, b, chi0, &ld, p, L);
  double rss = y_dy;
  for (int i = 0; i < p; ++i)
    for (int j = 0; j < p; ++j)
      a00L_out[(static_cast<int64_t>(g) * p + i) * p + j] = ok && j <= i ? L[i * p + j] : 0.0;
  if (ok) {
    for (int k = 0; k < p; ++k) rss -= b[k] * chi0[k];
    if (rss < 0) rss = 0;
    for (int c = 0; c < p; ++c) {  // A00^-1 column by column
      for (int i = 0; i < p; ++i) e[i] = (i == c) ? 1.0 : 0.0;
      double dummy;
      chol_solve(A, e, x, &dummy, p, L);
      for (int i = 0; i < p; ++i) ainv_out[(static_cast<int64_t>(g) * p + i) * p + c] = x[i];
    }
  } else {
    for (int k = 0; k < p; ++k) chi0[k] = 0;
    for (int i = 0; i < p * p; ++i) ainv_out[static_cast<int64_t>(g) * p * p + i] = 0;
  }
  rss_out[g] = rss;
  for (int k = 0; k < p; ++k) chi0_out[static_cast<int64_t>(g) * p + k] = chi0[k];
}

// REML -loglik (src/model_lmm.cpp:10-37) for P <= 3 covariate columns,
// evaluated by one warp:
// each lane sums log v, w y^2, w x_a x_b and w y x_a over its samples in
// registers, and xor-shuffle reductions give every lane the same totals
// (IEEE addition is commutative), so there is no shared memory and no block
// barrier. tot = [sum log v, y'Dy, X'DX packed (a <= b), X'Dy].
template <int P>
__device__ __forceinline__ double reml_eval_warp(double delta, const double* __restrict__ yt,
                                                 const double* __restrict__ Xt, const double* __restrict__ lam,
                                                 int n, double* tot) {
  constexpr int NQ = P * (P + 1) / 2;
  constexpr int V = 2 + NQ + P;
  const int lane = threadIdx.x & 31;
  double acc[V];
#pragma unroll
  for (int q = 0; q < V; ++q) acc[q] = 0.0;
  double prod = 1.0;
  int nprod = 0;
  for (int i = lane; i < n; i += 32) {
    double v = delta * lam[i] + 1.0;
    if (v < 1e-12) v = 1e-12;
    const double w = 1.0 / v;
    // sum of log v as the log of products of up to eight factors: every factor
    // lies in [1e-12, 1e36] (larger ones take their own log), so a product
    // stays within [1e-96, 1e288]
    if (v <= 1e36) {
      prod *= v;
      if (++nprod == 8) {
        acc[0] += log(prod);
        prod = 1.0;
        nprod = 0;
      }
    } else {
      acc[0] += log(v);
    }
    const double y = yt[i];
    acc[1] += w * y * y;
    double x[P];
#pragma unroll
    for (int a = 0; a < P; ++a) x[a] = Xt[static_cast<int64_t>(a) * n + i];
#pragma unroll
    for (int a = 0; a < P; ++a) {
#pragma unroll
      for (int b = a; b < P; ++b) acc[2 + a * P - a * (a - 1) / 2 + (b - a)] += w * x[a] * x[b];
      acc[2 + NQ + a] += w * y * x[a];
    }
  }
  acc[0] += log(prod);
#pragma unroll
  for (int q = 0; q < V; ++q) {
    double s = acc[q];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    tot[q] = s;
  }
  // Cholesky of X'DX; q = y'Dy - b'(X'DX)^-1 b as y'Dy - |z|^2 with L z = b
  double L[P][P];
  double logdet_x = 0.0;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    double d = tot[2 + j * P - j * (j - 1) / 2];
#pragma unroll
    for (int k = 0; k < j; ++k) d -= L[j][k] * L[j][k];
    if (!(d > 0)) return 1e300;
    L[j][j] = sqrt(d);
    logdet_x += 2.0 * log(L[j][j]);
#pragma unroll
    for (int i = j + 1; i < P; ++i) {
      double s = tot[2 + j * P - j * (j - 1) / 2 + (i - j)];
#pragma unroll
      for (int k = 0; k < j; ++k) s -= L[i][k] * L[j][k];
      L[i][j] = s / L[j][j];
    }
  }
  double q = tot[1];
  double z[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    double s = tot[2 + NQ + i];
#pragma unroll
    for (int k = 0; k < i; ++k) s -= L[i][k] * z[k];
    z[i] = s / L[i][i];
    q -= z[i] * z[i];
  }
  if (q <= 0) q = 1e-12;
  const double df = static_cast<double>(n - P);
  return 0.5 * (df * log(q / df) + tot[0] + logdet_x);
}

// One warp per gene for P <= 3 (intercept and a few covariates):
// optimize_delta (src/model_lmm.cpp:39-86) and the prep_lmm caches (:124-153).
constexpr int kRemlWarpP = 3;
template <int P>
__global__ void __launch_bounds__(256) reml_warp_kernel(const double* __restrict__ Ytil,
                                                        const double* __restrict__ Xtil,
                                                        const double* __restrict__ lam, int n, int G,
                                                        double* delta_out, double* chi0_out, double* ainv_out,
                                                        double* rss_out, double* a00L_out) {
  constexpr int NQ = P * (P + 1) / 2;
  const int g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (g >= G) return;  // whole warps only: no block barrier follows
  const double* yt = Ytil + static_cast<int64_t>(g) * n;
  double tot[2 + NQ + P];
  auto f = [&](double d) { return reml_eval_warp<P>(d, yt, Xtil, lam, n, tot); };
  const double d = optimize_delta_dev(f, n - P);
  f(d);
  if ((threadIdx.x & 31) == 0) {
    double A[P * P], L[P * P], e[P], x[P];
    for (int a = 0; a < P; ++a)
      for (int b = a; b < P; ++b) A[a * P + b] = A[b * P + a] = tot[2 + a * P - a * (a - 1) / 2 + (b - a)];
    delta_out[g] = d;
    reml_caches(A, tot + 2 + NQ, tot[1], P, g, L, e, x, chi0_out, ainv_out, rss_out, a00L_out);
  }
}

// ------------------------------------------- batched REML (p > kRemlWarpP)
// The same schedule and -loglik for many columns in lockstep. Each round
// evaluates up to two deltas per column (slot s = slot * C + column); the
// sums over the n samples run as FP64 GEMMs shared by all columns,
//   A[q, s] = sum_i P[q, i] W[i, s]     P[q, i] = x~_ai x~_bi (q = tri(a, b))
//   b[a, s] = sum_i x~_ai (W o Y)[i, s]
// with W[i, s] = 1 / max(delta_s lambda_i + 1, 1e-12), and one thread per
// column advances its search (golden section, Newton) between rounds; the
// grid phase, whose deltas every column shares, runs once before them.
enum : int { kRbGolden = 1, kRbCentre, kRbNewtonPair, kRbNewtonStep, kRbFinal, kRbDone };
constexpr int kRbGridN = 35;  // f(1.0), then 1e-5 * 2^k for k = 0..33 (the loop dd <= 1e5, dd *= 2)
constexpr int kRbMaxRounds = 40 + 1 + 2 * 8 + 1;  // golden, centre, Newton, final

struct RemlBatchState {
  int phase, k;
  double best_d, best_ll, lo, hi, d, cur, h, step, dn;
};

// 1e-5 doubled k times is exact, so this is the reference's dd sequence
__device__ __forceinline__ double rb_grid_delta(int j) { return j == 0 ? 1.0 : ldexp(1e-5, j - 1); }

__device__ void rb_propose(const RemlBatchState& s, double& d0, double& d1) {
  d0 = d1 = CUDART_NAN;
  switch (s.phase) {
    case kRbGolden: {
      const double phi = (1.0 + sqrt(5.0)) / 2.0;
      d0 = s.hi - (s.hi - s.lo) / phi;
      d1 = s.lo + (s.hi - s.lo) / phi;
      break;
    }
    case kRbCentre:
    case kRbFinal:
      d0 = s.d;
      break;
    case kRbNewtonPair:
      d0 = s.d - s.h;
      d1 = s.d + s.h;
      break;
    case kRbNewtonStep:
      d0 = s.dn;
      break;
    default:
      break;
  }
}

// P[q + nq i] = x~_ai x~_bi
__global__ void rb_pairs_kernel(const double* __restrict__ Xtil, int n, int p, double* P) {
  const int nq = p * (p + 1) / 2;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < static_cast<int64_t>(nq) * n;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int q = static_cast<int>(t % nq);
    const int i = static_cast<int>(t / nq);
    int a = 0;
    while (tri(a, p - 1, p) < q) ++a;
    const int b = a + (q - tri(a, a, p));
    P[t] = Xtil[static_cast<int64_t>(a) * n + i] * Xtil[static_cast<int64_t>(b) * n + i];
  }
}

// ---- grid phase, shared by all columns: the 35 grid deltas are the same for
// every column, so D_k, X~'D_k X~ (and its Cholesky factor) and sum log v
// are computed once; per column only X~'D_k y and y'D_k y remain (GEMMs).
// Wg[i + n k] = w_k,i, Xw[i + n (k p + a)] = w_k,i x~_ai, ldD[k] = sum_i log v_k,i.
__global__ void rb_grid_weights_kernel(const double* __restrict__ Xtil, const double* __restrict__ lam, int n,
                                       int p, double* Wg, double* Xw, double* ldD) {
  const int k = blockIdx.x;  // grid point
  const double delta = rb_grid_delta(k);
  const int lane = threadIdx.x & 31;
  double acc = 0.0, prod = 1.0;
  int nprod = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double v = delta * lam[i] + 1.0;
    if (v < 1e-12) v = 1e-12;
    const double w = 1.0 / v;
    Wg[i + static_cast<int64_t>(n) * k] = w;
    for (int a = 0; a < p; ++a)
      Xw[i + static_cast<int64_t>(n) * (k * p + a)] = w * Xtil[static_cast<int64_t>(a) * n + i];
    if (v <= 1e36) {
      prod *= v;
      if (++nprod == 8) {
        acc += log(prod);
        prod = 1.0;
        nprod = 0;
      }
    } else {
      acc += log(v);
    }
  }
  acc += log(prod);
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double red[32];
  if (lane == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (blockDim.x >> 5); ++w) t += red[w];
    ldD[k] = t;
  }
}

// Lg[k] = Cholesky factor of X~'D_k X~ (row-major, lower), ldx[k] its log
// determinant, or ldx[k] = NaN when it is not positive definite.
__global__ void rb_grid_chol_kernel(const double* __restrict__ Ag, int p, double* Lg, double* ldx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kRbGridN) return;
  const int nq = p * (p + 1) / 2;
  double* L = Lg + static_cast<int64_t>(k) * p * p;
  const double* Ac = Ag + static_cast<int64_t>(k) * nq;
  double ld = 0.0;
  for (int j = 0; j < p; ++j) {
    double d = Ac[tri(j, j, p)];
    for (int q = 0; q < j; ++q) d -= L[j * p + q] * L[j * p + q];
    if (!(d > 0)) {
      ldx[k] = CUDART_NAN;
      return;
    }
    L[j * p + j] = sqrt(d);
    ld += 2.0 * log(L[j * p + j]);
    for (int i = j + 1; i < p; ++i) {
      double v = Ac[tri(j, i, p)];
      for (int q = 0; q < j; ++q) v -= L[i * p + q] * L[j * p + q];
      L[i * p + j] = v / L[j * p + j];
    }
  }
  ldx[k] = ld;
}

// Per column: the 35 grid -logliks in the reference's order (f(1.0) first,
// strict <), then the golden-section bracket; proposes the first round.
// Bg[(k p + a) + 35 p c] = x~_a' D_k y_c, Yg[k + 35 c] = y_c' D_k y_c.
__global__ void rb_grid_advance_kernel(int C, int p, int df, const double* __restrict__ Lg,
                                       const double* __restrict__ ldx, const double* __restrict__ ldD,
                                       const double* __restrict__ Bg, const double* __restrict__ Yg,
                                       RemlBatchState* st, double* dlt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  RemlBatchState s{};
  s.d = 1.0;
  if (df <= 0) {
    s.phase = kRbFinal;
  } else {
    const double dfd = static_cast<double>(df);
    for (int k = 0; k < kRbGridN; ++k) {
      double v = 1e300;
      const double lx = ldx[k];
      if (lx == lx) {
        const double* L = Lg + static_cast<int64_t>(k) * p * p;
        const double* b = Bg + static_cast<int64_t>(kRbGridN) * p * c + static_cast<int64_t>(k) * p;
        double z[kMaxPLmm];
        double q = Yg[k + static_cast<int64_t>(kRbGridN) * c];
        for (int i = 0; i < p; ++i) {
          double t = b[i];
          for (int j = 0; j < i; ++j) t -= L[i * p + j] * z[j];
          z[i] = t / L[i * p + i];
          q -= z[i] * z[i];
        }
        if (q <= 0) q = 1e-12;
        v = 0.5 * (dfd * log(q / dfd) + ldD[k] + lx);
      }
      if (k == 0) {
        s.best_ll = v;
        s.best_d = 1.0;
      } else if (v < s.best_ll) {
        s.best_ll = v;
        s.best_d = rb_grid_delta(k);
      }
    }
    s.lo = s.best_d / 4.0;
    s.hi = s.best_d * 4.0;
    if (s.lo < 1e-8) s.lo = 1e-8;
    if (s.hi > 1e6) s.hi = 1e6;
    s.phase = kRbGolden;
  }
  st[c] = s;
  rb_propose(s, dlt[c], dlt[C + c]);
}

// One warp per slot: W, W o y, sum log v (log of eight-factor products, as in
// reml_eval_warp) and y'Dy. Slots with no delta (NaN) are skipped.
__global__ void __launch_bounds__(256) rb_weights_kernel(const double* __restrict__ Ytil,
                                                         const double* __restrict__ lam, int n, int C,
                                                         const double* __restrict__ dlt, double* W, double* WY,
                                                         double* ld, double* ydy) {
  const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (s >= 2 * C) return;
  const double delta = dlt[s];
  if (!(delta == delta)) return;
  const double* y = Ytil + static_cast<int64_t>(s % C) * n;
  double* w_out = W + static_cast<int64_t>(s) * n;
  double* wy_out = WY + static_cast<int64_t>(s) * n;
  double acc_ld = 0.0, acc_y = 0.0, prod = 1.0;
  int nprod = 0;
  for (int i = lane; i < n; i += 32) {
    double v = delta * lam[i] + 1.0;
    if (v < 1e-12) v = 1e-12;
    const double w = 1.0 / v;
    if (v <= 1e36) {
      prod *= v;
      if (++nprod == 8) {
        acc_ld += log(prod);
        prod = 1.0;
        nprod = 0;
      }
    } else {
      acc_ld += log(v);
    }
    const double yi = y[i];
    w_out[i] = w;
    wy_out[i] = w * yi;
    acc_y += w * yi * yi;
  }
  acc_ld += log(prod);
  for (int o = 16; o; o >>= 1) {
    acc_ld += __shfl_xor_sync(0xffffffffu, acc_ld, o);
    acc_y += __shfl_xor_sync(0xffffffffu, acc_y, o);
  }
  if (lane == 0) {
    ld[s] = acc_ld;
    ydy[s] = acc_y;
  }
}

// -loglik of slot s from its sums; A is unpacked into Af (p x p, row-major).
__device__ double rb_negll(const double* __restrict__ Acol, const double* __restrict__ bcol, double y_dy,
                           double logdet_d, int p, int df, double* Af, double* L) {
  for (int a = 0; a < p; ++a)
    for (int b = a; b < p; ++b) Af[a * p + b] = Af[b * p + a] = Acol[tri(a, b, p)];
  double beta[kMaxPLmm];
  double logdet_x = 0.0;
  if (!chol_solve(Af, bcol, beta, &logdet_x, p, L)) return 1e300;
  double q = y_dy;
  for (int k = 0; k < p; ++k) q -= bcol[k] * beta[k];
  if (q <= 0) q = 1e-12;
  const double dfd = static_cast<double>(df);
  return 0.5 * (dfd * log(q / dfd) + logdet_d + logdet_x);
}

// One thread per column: reads the round's -loglik values, advances the
// search exactly as optimize_delta_dev does, and proposes the next round's
// deltas; in the final round writes delta and the prep_lmm caches.
// PMAX bounds p for the per-thread p x p scratch (p <= 16 keeps the stack
// frame small; 17..32 use the larger instance).
template <int PMAX>
__global__ void rb_advance_kernel(int C, int g0, int p, int df, const double* __restrict__ A,
                                  const double* __restrict__ B, const double* __restrict__ ld,
                                  const double* __restrict__ ydy, RemlBatchState* st, double* dlt,
                                  unsigned int* active, double* delta_out, double* chi0_out, double* ainv_out,
                                  double* rss_out, double* a00L_out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  RemlBatchState s = st[c];
  if (s.phase == kRbDone) return;
  const int nq = p * (p + 1) / 2;
  double Af[PMAX * PMAX], L[PMAX * PMAX];
  auto f = [&](int slot) {
    const int si = slot * C + c;
    return rb_negll(A + static_cast<int64_t>(si) * nq, B + static_cast<int64_t>(si) * p, ydy[si], ld[si], p, df,
                    Af, L);
  };
  switch (s.phase) {
    case kRbGolden: {
      const double phi = (1.0 + sqrt(5.0)) / 2.0;
      const double m1 = s.hi - (s.hi - s.lo) / phi;
      const double m2 = s.lo + (s.hi - s.lo) / phi;
      const double f1 = f(0);
      const double f2 = f(1);
      if (f1 < f2) s.hi = m2;
      else s.lo = m1;
      if (++s.k == 40) {
        s.d = 0.5 * (s.lo + s.hi);
        s.phase = kRbCentre;
      }
      break;
    }
    case kRbCentre:
      s.cur = f(0);
      s.k = 0;
      s.h = fmax(s.d * 1e-4, 1e-9);
      s.phase = kRbNewtonPair;
      break;
    case kRbNewtonPair: {
      const double fm = f(0);
      const double fp = f(1);
      const double g1 = (fp - fm) / (2.0 * s.h);
      const double g2 = (fp - 2.0 * s.cur + fm) / (s.h * s.h);
      s.phase = kRbFinal;
      if (g2 > 1e-12) {
        s.step = g1 / g2;
        s.dn = s.d - s.step;
        if (s.dn > 1e-8 && s.dn < 1e6) s.phase = kRbNewtonStep;
      }
      break;
    }
    case kRbNewtonStep: {
      const double vn = f(0);
      s.phase = kRbFinal;
      if (vn < s.cur) {
        s.d = s.dn;
        s.cur = vn;
        if (!(fabs(s.step) < s.d * 1e-8) && ++s.k < 8) {
          s.h = fmax(s.d * 1e-4, 1e-9);
          s.phase = kRbNewtonPair;
        }
      }
      break;
    }
    case kRbFinal: {
      const int si = c;  // slot 0
      const double* Acol = A + static_cast<int64_t>(si) * nq;
      for (int a = 0; a < p; ++a)
        for (int b = a; b < p; ++b) Af[a * p + b] = Af[b * p + a] = Acol[tri(a, b, p)];
      double e[kMaxPLmm], x[kMaxPLmm];
      delta_out[g0 + c] = s.d;
      reml_caches(Af, B + static_cast<int64_t>(si) * p, ydy[si], p, g0 + c, L, e, x, chi0_out, ainv_out, rss_out,
                  a00L_out);
      s.phase = kRbDone;
      break;
    }
    default:
      break;
  }
  st[c] = s;
  rb_propose(s, dlt[c], dlt[C + c]);
  if (s.phase != kRbDone) atomicAdd(active, 1u);
}

// Gene-side operands, one block per gene: rows (w o r~), (w o X~_k), w, each
// FP16 hi/lo with its own power-of-two scale; unscale[] = factors that turn
// the accumulators back into NUM, a_k, gg.
__global__ void lmm_gene_ops_kernel(const double* __restrict__ Ytil, const double* __restrict__ Xtil,
                                    const double* __restrict__ lam, const double* __restrict__ delta,
                                    const double* __restrict__ chi0, int n, int p, int G, int k_pad, float s1,
                                    float s2, __half* const* hi, __half* const* lo, float* unscale) {
  const int g = blockIdx.x;
  if (g >= G) return;
  const int nops = p + 2;
  __shared__ double mx[kMaxPLmm + 2][8];
  __shared__ double sc[kMaxPLmm + 2];
  const double d = delta[g];
  const double* yt = Ytil + static_cast<int64_t>(g) * n;
  double c0[kMaxPLmm];
  for (int k = 0; k < p; ++k) c0[k] = chi0[static_cast<int64_t>(g) * p + k];
  auto value = [&](int op, int i) -> double {
    if (i >= n) return 0.0;
    double v = d * lam[i] + 1.0;
    if (v < 1e-12) v = 1e-12;
    const double w = 1.0 / v;
    if (op == 0) {
      double r = yt[i];
      for (int k = 0; k < p; ++k) r -= Xtil[static_cast<int64_t>(k) * n + i] * c0[k];
      return w * r;
    }
    if (op <= p) return w * Xtil[static_cast<int64_t>(op - 1) * n + i];
    return w;
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int op = 0; op < nops; ++op) {
    double m = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(value(op, i)));
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) mx[op][warp] = m;
  }
  __syncthreads();
  if (threadIdx.x < nops) {
    double m = 0;
    for (int w = 0; w < (blockDim.x >> 5); ++w) m = fmax(m, mx[threadIdx.x][w]);
    int e = 0;
    if (m > 0) e = 10 - static_cast<int>(floor(log2(m)));
    sc[threadIdx.x] = ldexp(1.0, e);
    const double side = threadIdx.x == nops - 1 ? s2 : s1;
    unscale[static_cast<int64_t>(g) * nops + threadIdx.x] = static_cast<float>(1.0 / (ldexp(1.0, e) * side));
  }
  __syncthreads();
  for (int op = 0; op < nops; ++op) {
    const double s = sc[op];
    for (int i = threadIdx.x; i < k_pad; i += blockDim.x) {
      const double v = value(op, i) * s;
      const __half h = __double2half(v);
      hi[op][static_cast<int64_t>(g) * k_pad + i] = h;
      lo[op][static_cast<int64_t>(g) * k_pad + i] = __double2half(v - static_cast<double>(__half2float(h)));
    }
  }
}

// Gene-side vectors of the exact-operand scan, one block per gene, in
// eigen-coordinates: column (p + 1) g of W is w o r~ and column
// (p + 1) g + 1 + k is w o X~_k, with w = 1 / max(delta lambda + 1, 1e-12);
// Q W then holds u = Q (w o r~) and v_k = Q (w o X~_k).
__global__ void lmm_uv_w_kernel(const double* __restrict__ Ytil, const double* __restrict__ Xtil,
                                const double* __restrict__ lam, const double* __restrict__ delta,
                                const double* __restrict__ chi0, int n, int p, int G, double* W) {
  const int g = blockIdx.x;
  if (g >= G) return;
  const double d = delta[g];
  const double* yt = Ytil + static_cast<int64_t>(g) * n;
  const double* c0 = chi0 + static_cast<int64_t>(g) * p;
  double* out = W + static_cast<int64_t>(g) * (p + 1) * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double v = d * lam[i] + 1.0;
    if (v < 1e-12) v = 1e-12;
    double r = yt[i];
    for (int k = 0; k < p; ++k) {
      const double x = Xtil[static_cast<int64_t>(k) * n + i];
      r -= x * c0[k];
      out[static_cast<int64_t>(1 + k) * n + i] = x / v;
    }
    out[i] = r / v;
  }
}

// Gene-side operands of the exact-operand scan, one block per gene: rows u,
// v_0 .. v_{p-1} (columns of UV = Q W) and w, each FP16 hi/lo with its own
// power-of-two scale. unscale[] turns accumulators back into NUM, a_k (the
// SNP operand carries no scale of its own) and gg (against Gt^2 at s2).
// u and v_k are scaled to a largest entry in [8, 16), so that minus their sum
// (at most 16 n <= 32768) fits FP16 as well: it goes to column n, where the
// SNP operand holds its imputed mean, which centres each SNP inside the
// contraction.
__global__ void lmm_gene_ops_raw_kernel(const double* __restrict__ UV, const double* __restrict__ lam,
                                        const double* __restrict__ delta, int n, int p, int G, int k_pad, float s2,
                                        __half* const* hi, __half* const* lo, float* unscale) {
  const int g = blockIdx.x;
  if (g >= G) return;
  const int nops = p + 2;
  __shared__ double mx[kMaxPLmm + 2][8];
  __shared__ double sc[kMaxPLmm + 2];
  __shared__ double part[8];
  const double d = delta[g];
  const double* uv = UV + static_cast<int64_t>(g) * (p + 1) * n;
  auto value = [&](int op, int i) -> double {
    if (i >= n) return 0.0;
    if (op <= p) return uv[static_cast<int64_t>(op) * n + i];
    double v = d * lam[i] + 1.0;
    if (v < 1e-12) v = 1e-12;
    return 1.0 / v;
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int op = 0; op < nops; ++op) {
    double m = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(value(op, i)));
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) mx[op][warp] = m;
  }
  __syncthreads();
  if (threadIdx.x < nops) {
    double m = 0;
    for (int w = 0; w < (blockDim.x >> 5); ++w) m = fmax(m, mx[threadIdx.x][w]);
    const bool centred = threadIdx.x < nops - 1;  // u and v_k
    int e = 0;
    if (m > 0) e = (centred ? 3 : 10) - static_cast<int>(floor(log2(m)));
    sc[threadIdx.x] = ldexp(1.0, e);
    const double side = centred ? 1.0 : s2;
    unscale[static_cast<int64_t>(g) * nops + threadIdx.x] = static_cast<float>(1.0 / (ldexp(1.0, e) * side));
  }
  __syncthreads();
  for (int op = 0; op < nops; ++op) {
    const double s = sc[op];
    __half* h_row = hi[op] + static_cast<int64_t>(g) * k_pad;
    __half* l_row = lo[op] + static_cast<int64_t>(g) * k_pad;
    double sum = 0.0;
    for (int i = threadIdx.x; i < k_pad; i += blockDim.x) {
      const double v = value(op, i) * s;
      const __half h = __double2half(v);
      const __half l = __double2half(v - static_cast<double>(__half2float(h)));
      h_row[i] = h;
      l_row[i] = l;
      sum += static_cast<double>(__half2float(h)) + static_cast<double>(__half2float(l));
    }
    if (op > p) break;  // w is not centred
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) part[warp] = sum;
    __syncthreads();  // every thread's writes of column n (zero) are done too
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (blockDim.x >> 5); ++w) t += part[w];
      const __half h = __double2half(-t);
      h_row[n] = h;
      l_row[n] = __double2half(-t - static_cast<double>(__half2float(h)));
    }
    __syncthreads();
  }
}

// ------------------------------------------------------- scan epilogue
template <int P>
struct LmmEpiParams {
  int G;
  int64_t m;
  const float* unscale;     // [G][P+2]
  const double* ainv;       // [G][P][P]
  const double* rss_null;   // [G]
  const uint8_t* snp_ok;    // [m]
  Windows win;
  float df;
  float t_cand;
  TTable tt;
  GeneOut out;
  // NB-GLM scan only (GlmEpiParams): per kept SNP the imputation mean (the
  // SNP operand is centred), per gene sum_i r_i and the null fit's success
  const float* snp_mean;    // [m, padded to 16 + 16]
  const float* rsum;        // [G]
  const uint8_t* gene_ok;   // [G]
  // exact-operand LMM scan only (LmmRawEpiParams): per kept SNP the factor
  // alpha of the raw operand (Rotated::raw)
  const float* snp_alpha;   // [m, padded to 256 + 256]
};
// The same fields select the NB-GLM score-test epilogue (LmmEpi<P, true>).
template <int P>
struct GlmEpiParams : LmmEpiParams<P> {};
// ... and the LMM scan on the exact unrotated SNP operand (LmmEpi<P, false, true>).
template <int P>
struct LmmRawEpiParams : LmmEpiParams<P> {};
// ... and the same with gg and a_k interpolated between node deltas
// (LmmEpi<P, false, true, true>): a_k then carries no SNP factor alpha.
template <int P>
struct LmmLrEpiParams : LmmEpiParams<P> {};

// Accumulator order of the tile: [gg, a_0 .. a_{P-1}, NUM] (the gene-side
// operands w, w o X~_k, w o r~ against Gt^2, Gt, Gt). The epilogue is
// two-phase: S = gg - a' A00^-1 a of every pair of the warp's chunks first,
// which frees the gg and a slots for the next tile's MMAs, then NUM and the
// rest of the statistic.
//
// GLM = true is the NB-GLM score test on the same accumulators (unrotated
// centred dosages gc against w, w o x_k and r of the gene's null fit):
// info = S, U = NUM + mean_s * sum_i r_i, and the screened statistic is
// z^2 = U^2 / info against the normal tables.
//
// RAW = true: NUM and a_k come from the exact unrotated SNP operand
// (Rotated::raw) against the gene-side vectors u = Q (w o r~) and
// v_k = Q (w o X~_k), since Gt . (w o r~) = g . Q (w o r~); the operands
// centre each SNP themselves (padding column n), so x = alpha_s * acc.
//
// LR = true (with RAW): gg and a_k come from the node-interpolated operands
// (lmm_lr_scan), which hold each SNP's factor alpha already; NUM as RAW.
template <int P, bool GLM = false, bool RAW = false, bool LR = false>
struct LmmEpi {
  static_assert(!(GLM && RAW), "the exact-operand form is the LMM scan's");
  static_assert(!LR || RAW, "the interpolated form reads NUM from the exact operand");
  static constexpr bool kGrouped = false;
  static constexpr bool kTwoPhase = true;
  static constexpr int kPhase1 = P + 1;  // gg and a_k
  static constexpr int kMaxChunks = 2;   // 16-column chunks per warp and tile
  using Params = std::conditional_t<
      GLM, GlmEpiParams<P>,
      std::conditional_t<LR, LmmLrEpiParams<P>, std::conditional_t<RAW, LmmRawEpiParams<P>, LmmEpiParams<P>>>>;
  static constexpr int kSmemBytes = kTTableSmemBytes;
  const Params& Pr;
  float* tsm;
  TTable tt;
  int gene = 0;
  int64_t snp0 = 0;
  bool gvalid = false;
  float u[P + 2];  // unscale of [NUM, a_0 .. a_{P-1}, gg] (the gene-ops order)
  float ai[P][P];
  float inv_rss = 0;
  float rs = 0;  // GLM: sum_i r_i of the gene
  // S per pair of the warp's two chunks (0 where gg < 1e-12); two named
  // arrays picked by a select, so they stay in registers for a runtime ci
  float S0[16], S1[16];
  float u_cand;  // t_cand^2
  GeneAcc acc;
  __device__ LmmEpi(const Params& p, const TileShape&, uint8_t* smem)
      : Pr(p), tsm(reinterpret_cast<float*>(smem)), tt(p.tt), u_cand(p.t_cand * p.t_cand) {}
  __device__ void init(int tid, int nthr) {
    if (tsm) tt = screen_to_smem(Pr.tt, tsm, tid, nthr);
  }
  __device__ void begin_tile(int g, int64_t s0) {
    gene = g;
    snp0 = s0;
    gvalid = g < Pr.G;
    if constexpr (GLM) gvalid = gvalid && Pr.gene_ok[g];  // a failed null fit tests nothing
    acc.reset();
    if (gvalid) {
      if constexpr (GLM) rs = Pr.rsum[g];
#pragma unroll
      for (int k = 0; k < P + 2; ++k) u[k] = Pr.unscale[static_cast<int64_t>(g) * (P + 2) + k];
#pragma unroll
      for (int a = 0; a < P; ++a)
#pragma unroll
        for (int b = 0; b < P; ++b) ai[a][b] = static_cast<float>(Pr.ainv[(static_cast<int64_t>(g) * P + a) * P + b]);
      if constexpr (!GLM) {
        const double r = Pr.rss_null[g];
        inv_rss = r > 0 ? static_cast<float>(1.0 / r) : 0.0f;
      }
      acc.load_window(Pr.win, g);
    }
  }
  // Screening arithmetic in FP32 (the accumulators carry ~1e-7 relative
  // error already); printed statistics come from the FP64 refinement.
  // Phase 1: v = [gg, a_0 .. a_{P-1}] of 16 pairs.
  template <int N>
  __device__ void pre_chunk(int ci, int c, const float (&v)[N][16]) {
    static_assert(N == P + 1, "phase-1 accumulators");
    float al[16];  // RAW: alpha of each SNP (the array is padded past the last tile)
    if constexpr (RAW && !LR) load16(Pr.snp_alpha + snp0 + c, al);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const float gg = v[0][j] * u[P + 1];
      float S = gg;
      float a[P];
      float us = 1.0f;
      if constexpr (RAW && !LR) us = al[j];
#pragma unroll
      for (int k = 0; k < P; ++k) a[k] = v[1 + k][j] * (us * u[1 + k]);
#pragma unroll
      for (int x = 0; x < P; ++x)
#pragma unroll
        for (int y = 0; y < P; ++y) S = fmaf(-a[x] * ai[x][y], a[y], S);
      const float Sj = gg < 1e-12f ? 0.0f : S;  // gg < 1e-12: p = 1 (S fails the S > 1e-15 test)
      if (ci == 0) S0[j] = Sj;
      else S1[j] = Sj;
    }
  }
  // Phase 2: v = [NUM] of the same 16 pairs. The 16 pairs share one
  // branch-free tail evaluation, so their table lookups overlap.
  template <int N>
  __device__ void post_chunk(int ci, int c, const float (&v)[N][16]) {
    static_assert(N == 1, "phase-2 accumulators");
    const int64_t s0 = snp0 + c;
    if (!gvalid || s0 >= Pr.m) return;
    uint32_t okw[4];
    load_flags16(Pr.snp_ok + s0, okw);
    float al[16];
    if constexpr (RAW) load16(Pr.snp_alpha + s0, al);
    if (!GLM && tt.lt_u) {  // uniform across the launch
      // a gw scan (no windows), and a trans scan on a chunk clear of every
      // lane's gene window, skip the per-pair window test; the vote keeps
      // the warp on one path
      if (Pr.win.mode == kWinNone)
        post_cubic<false>(ci, s0, v[0], okw, al);
      else if (Pr.win.mode == kWinExclude && __all_sync(__activemask(), acc.chunk_clear(Pr.win, s0)))
        post_cubic<false>(ci, s0, v[0], okw, al);
      else
        post_cubic<true>(ci, s0, v[0], okw, al);
      return;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int64_t s = s0 + j;
      const bool valid = flag16(okw, j) && s < Pr.m && acc.in_scope(Pr.win, s);
      float num = v[0][j] * u[0];
      if constexpr (RAW) num *= al[j];
      const float S = ci == 0 ? S0[j] : S1[j];
      float u;
      if constexpr (GLM) {
        const float U = fmaf(__ldg(Pr.snp_mean + s), rs, num);
        u = S > 1e-15f ? __fdividef(U * U, S) : 0.0f;  // z^2
      } else {
        const float r = num * __fdividef(num, S) * inv_rss;
        const float omr = 1.0f - r;
        const bool ok_stat = S > 1e-15f && omr > 0.0f;
        u = ok_stat ? Pr.df * __fdividef(r, omr) : 0.0f;  // t^2
      }
      const ScreenOut o = acat_screen_u(u, tt);
      acc.add_screen(o, s, valid);
      if (valid && (u >= u_cand || o.deferred)) emit_candidate(Pr.out, gene, s, o.deferred, o.tiny);
    }
    acc.end_chunk();
  }
  // Phase 2 with the per-interval cubics (screen16_cubic). The SNP flags are
  // zero past the last kept SNP, so they also mask the padding.
  template <bool WIN>
  __device__ void post_cubic(int ci, int64_t s0, const float (&v)[16], const uint32_t (&okw)[4],
                             const float (&al)[16]) {
    float uu[16];
    bool valid[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      valid[j] = flag16(okw, j) && (!WIN || acc.in_scope(Pr.win, s0 + j));
      float num = v[j] * u[0];
      if constexpr (RAW) num *= al[j];
      const float S = ci == 0 ? S0[j] : S1[j];
      const float r = num * __fdividef(num, S) * inv_rss;
      const float omr = 1.0f - r;
      uu[j] = S > 1e-15f && omr > 0.0f ? Pr.df * __fdividef(r, omr) : 0.0f;  // t^2, never NaN
      if (!valid[j]) uu[j] = 0.0f;
    }
    screen16_cubic(tt, uu, valid, u_cand, Pr.out, gene, s0, acc);
  }
  // Both phases at once (the CUDA-core comparator): v in the tile's order.
  template <int NACC>
  __device__ void chunk(int c, const float (&v)[NACC][16]) {
    static_assert(NACC == P + 2, "accumulators");
    float v1[P + 1][16];
#pragma unroll
    for (int k = 0; k < P + 1; ++k)
#pragma unroll
      for (int j = 0; j < 16; ++j) v1[k][j] = v[k][j];
    pre_chunk<P + 1>(0, c, v1);
    float v2[1][16];
#pragma unroll
    for (int j = 0; j < 16; ++j) v2[0][j] = v[P + 1][j];
    post_chunk<1>(0, c, v2);
  }
  __device__ void end_tile() {
    if (gvalid) acc.flush(Pr.out, gene);
  }
  __device__ void finish() {}
};

// ------------------------------------- node-interpolated gg and a_k (p <= 2)
// The weights w_i = 1 / (1 + delta lambda_i) of a gene enter gg and a_k only
// through delta, and as functions of a = ln(delta) they are analytic in a
// strip of half-width pi around the real axis. So on an interval of a of
// length <= 3, the Lagrange interpolant through 12 Chebyshev-Lobatto nodes
// reproduces every w_i to 1.1e-7 relative at worst (where delta lambda_i is
// near 8), below the 2^-22 to which the FP16 hi/lo pair holds w itself, and
// far closer on shorter intervals; with it
//     gg(s, g) = sum_j l_j(a_g) gg(s, node j),   a_k likewise,
// where gg(s, node j) is the contraction for a "node gene" of delta_j. The
// node pass computes those for the <= 128 nodes that cover the scan's genes
// (one gene-side tile), and the scan then forms gg and a_k with K = the node
// count instead of n. The Lebesgue constants keep |l_j| sums below ~5, so the
// interpolation adds at most a few FP32 roundings.

// Node pass epilogue: rows = nodes, accumulators [gg, a_0 .. a_{P-1}] of
// every kept SNP in FP32 (gg as the scan forms it, a_k with the SNP's alpha)
// into val[s][kind * kn + node] (kind 0 = gg, 1 + k = a_k), and per column
// the largest magnitude (colmax, FP32 bits; non-negative floats order as
// unsigned integers).
template <int P>
struct LmmNodeEpiParams {
  int n_nodes;
  int64_t m;
  int kn, kb;               // node columns per kind (64 or 128); kb = (P + 1) kn
  const float* unscale;     // [nodes][P + 2] in the gene-ops order [NUM, a_0 .., gg]
  const float* snp_alpha;   // [m, padded to 256 + 256]
  float* val;               // [m][kb]
  unsigned int* colmax;     // [kb]
};

template <int P>
struct LmmNodeEpi {
  static constexpr bool kGrouped = false;
  static constexpr int kSmemBytes = 0;
  using Params = LmmNodeEpiParams<P>;
  const Params& Pr;
  int node = 0;
  int64_t snp0 = 0;
  bool valid = false;
  float u[P + 1];   // unscale of [gg, a_0 ..]
  float mx[P + 1];  // largest magnitude of each kind over the tile
  __device__ LmmNodeEpi(const Params& p, const TileShape&, uint8_t*) : Pr(p) {}
  __device__ void init(int, int) {}
  __device__ void begin_tile(int g, int64_t s0) {
    node = g;
    snp0 = s0;
    valid = g < Pr.n_nodes;
#pragma unroll
    for (int k = 0; k <= P; ++k) mx[k] = 0.0f;
    if (valid) {
      u[0] = Pr.unscale[static_cast<int64_t>(g) * (P + 2) + P + 1];
#pragma unroll
      for (int k = 0; k < P; ++k) u[1 + k] = Pr.unscale[static_cast<int64_t>(g) * (P + 2) + 1 + k];
    }
  }
  template <int N>
  __device__ void chunk(int c, const float (&v)[N][16]) {
    static_assert(N == P + 1, "node pass accumulators");
    const int64_t s0 = snp0 + c;
    if (!valid || s0 >= Pr.m) return;
    float al[16];
    load16(Pr.snp_alpha + s0, al);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int64_t s = s0 + j;
      if (s < Pr.m) {
        float* row = Pr.val + s * Pr.kb + node;
        const float gg = v[0][j] * u[0];
        row[0] = gg;
        mx[0] = fmaxf(mx[0], fabsf(gg));
#pragma unroll
        for (int k = 0; k < P; ++k) {
          const float a = v[1 + k][j] * (u[1 + k] * al[j]);
          row[static_cast<int64_t>(1 + k) * Pr.kn] = a;
          mx[1 + k] = fmaxf(mx[1 + k], fabsf(a));
        }
      }
    }
  }
  __device__ void end_tile() {
    if (!valid) return;
#pragma unroll
    for (int k = 0; k <= P; ++k)
      if (mx[k] > 0.0f) atomicMax(Pr.colmax + k * Pr.kn + node, __float_as_uint(mx[k]));
  }
  __device__ void finish() {}
};

// Scale of each node column: a power of two that takes its largest value
// into [2^14, 2^15) (0 for a column that is zero throughout, and for the
// padding columns).
__global__ void lr_sigma_kernel(const unsigned int* __restrict__ colmax, int kb, float* sigma) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kb) return;
  const float mx = __uint_as_float(colmax[i]);
  sigma[i] = mx > 0.0f ? ldexpf(1.0f, min(14 - ilogbf(mx), 100)) : 0.0f;
}

// The SNP-side operand of the interpolated accumulators: val * sigma of its
// column as FP16 hi + lo, four values per thread (kb is a multiple of 64).
// Columns of scale 0 are written as 0 without reading val (padding columns
// are never written by the node pass).
__global__ void lr_split_kernel(const float* __restrict__ val, int64_t total, int kb,
                                const float* __restrict__ sigma, __half* hi, __half* lo) {
  const int64_t n4 = total / 4;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n4;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int c0 = static_cast<int>((4 * i) % kb);
    float x[4];
    const float4 sg = *reinterpret_cast<const float4*>(sigma + c0);
    const float sv[4] = {sg.x, sg.y, sg.z, sg.w};
    const bool any = sv[0] != 0.0f || sv[1] != 0.0f || sv[2] != 0.0f || sv[3] != 0.0f;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (any) v = reinterpret_cast<const float4*>(val)[i];
    const float vv[4] = {v.x, v.y, v.z, v.w};
    uint32_t hw[2], lw[2];
#pragma unroll
    for (int t = 0; t < 4; ++t) x[t] = sv[t] != 0.0f ? vv[t] * sv[t] : 0.0f;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const __half h0 = __float2half_rn(x[2 * t]), h1 = __float2half_rn(x[2 * t + 1]);
      const __half l0 = __float2half_rn(x[2 * t] - __half2float(h0));
      const __half l1 = __float2half_rn(x[2 * t + 1] - __half2float(h1));
      hw[t] = static_cast<uint32_t>(__half_as_ushort(h0)) | (static_cast<uint32_t>(__half_as_ushort(h1)) << 16);
      lw[t] = static_cast<uint32_t>(__half_as_ushort(l0)) | (static_cast<uint32_t>(__half_as_ushort(l1)) << 16);
    }
    reinterpret_cast<uint2*>(hi)[i] = make_uint2(hw[0], hw[1]);
    reinterpret_cast<uint2*>(lo)[i] = make_uint2(lw[0], lw[1]);
  }
}

constexpr int kLrNodes = 12;     // Chebyshev-Lobatto nodes per interval of ln(delta)
constexpr double kLrSpan = 3.0;  // longest interval of ln(delta)

// Gene-side operands of the interpolated accumulators, one thread per gene:
// the Lagrange weights l_j(a) of the gene's interval (a = ln delta, nodes
// node_a[base .. base + kLrNodes), base = q (kLrNodes - 1)) over each kind's
// column scale, times a power of two per gene and kind, as FP16 hi + lo at
// [g][kind * kn + base + j] (rows zeroed beforehand), and that power's
// inverse as the unscale of gg (kind 0) and a_k (kind 1 + k).
__global__ void lr_coef_kernel(const double* __restrict__ delta, int G, const double* __restrict__ node_a,
                               double a0, double h, int nint, const float* __restrict__ sigma, int kn, int kb,
                               int P, __half* hi, __half* lo, float* unscale) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  double a = log(fmax(delta[g], 1e-300));
  if (!(a == a)) a = a0;
  int q = static_cast<int>(floor((a - a0) / h));
  q = q < 0 ? 0 : (q >= nint ? nint - 1 : q);
  const int base = q * (kLrNodes - 1);
  double l[kLrNodes];
#pragma unroll
  for (int j = 0; j < kLrNodes; ++j) {
    double t = 1.0;
#pragma unroll
    for (int i = 0; i < kLrNodes; ++i)
      if (i != j) t *= (a - node_a[base + i]) / (node_a[base + j] - node_a[base + i]);
    l[j] = t;
  }
  for (int kind = 0; kind <= P; ++kind) {
    const float* sg = sigma + kind * kn + base;
    double mx = 0.0;
#pragma unroll
    for (int j = 0; j < kLrNodes; ++j)
      if (sg[j] != 0.0f) mx = fmax(mx, fabs(l[j] / static_cast<double>(sg[j])));
    const double sc = mx > 0.0 ? ldexp(1.0, 10 - ilogb(mx)) : 1.0;
    __half* hr = hi + static_cast<int64_t>(g) * kb + kind * kn + base;
    __half* lr = lo + static_cast<int64_t>(g) * kb + kind * kn + base;
#pragma unroll
    for (int j = 0; j < kLrNodes; ++j) {
      const double y = sg[j] != 0.0f ? l[j] / static_cast<double>(sg[j]) * sc : 0.0;
      const __half hv = __double2half(y);
      hr[j] = hv;
      lr[j] = __double2half(y - static_cast<double>(__half2float(hv)));
    }
    unscale[static_cast<int64_t>(g) * (P + 2) + (kind == 0 ? P + 1 : kind)] = static_cast<float>(1.0 / sc);
  }
}

// ---------------------------------------- any number of covariates (p >= 3)
// With A00 = X~'W X~ and U U' = A00^-1 (Cholesky of the REML kernel's ainv),
// a' A00^-1 a = |U' a|^2 and U' a = Gt'(w o X~U): each covariate column
// becomes one plain accumulator a~_k = Gt'(w o (X~U)_k), and
//     S = gg - sum_k a~_k^2.
// The p + 2 accumulators [NUM, gg, a~_0 .. a~_{p-1}] exceed what TMEM holds
// for one tile, so the tile kernel runs them in groups of four; this
// epilogue keeps NUM and the running S of its 16 pairs across the groups.
__global__ void lmm_gene_ops_orth_kernel(const double* __restrict__ Ytil, const double* __restrict__ Xtil,
                                         const double* __restrict__ lam, const double* __restrict__ delta,
                                         const double* __restrict__ chi0, const double* __restrict__ ainv, int n,
                                         int p, int G, int k_pad, float s1, float s2, __half* const* hi,
                                         __half* const* lo, float* unscale) {
  const int g = blockIdx.x;
  if (g >= G) return;
  const int nops = p + 2;
  __shared__ double mx[kMaxPLmm + 2][8];
  __shared__ double sc[kMaxPLmm + 2];
  __shared__ double U[kMaxPLmm * kMaxPLmm];  // lower Cholesky factor of ainv[g]
  if (threadIdx.x == 0) {
    const double* A = ainv + static_cast<int64_t>(g) * p * p;
    for (int j = 0; j < p; ++j) {
      double d = A[j * p + j];
      for (int k = 0; k < j; ++k) d -= U[j * p + k] * U[j * p + k];
      d = d > 0 ? sqrt(d) : 0.0;  // A00 is positive definite wherever REML succeeded
      U[j * p + j] = d;
      for (int i = j + 1; i < p; ++i) {
        double v = A[i * p + j];
        for (int k = 0; k < j; ++k) v -= U[i * p + k] * U[j * p + k];
        U[i * p + j] = d > 0 ? v / d : 0.0;
      }
      for (int i = 0; i < j; ++i) U[i * p + j] = 0.0;
    }
  }
  __syncthreads();
  const double d = delta[g];
  const double* yt = Ytil + static_cast<int64_t>(g) * n;
  const double* c0 = chi0 + static_cast<int64_t>(g) * p;
  auto value = [&](int op, int i) -> double {
    if (i >= n) return 0.0;
    double v = d * lam[i] + 1.0;
    if (v < 1e-12) v = 1e-12;
    const double w = 1.0 / v;
    if (op == 1) return w;
    double r = 0;
    if (op == 0) {
      r = yt[i];
      for (int k = 0; k < p; ++k) r -= Xtil[static_cast<int64_t>(k) * n + i] * c0[k];
    } else {
      const int k = op - 2;
      for (int l = k; l < p; ++l) r += Xtil[static_cast<int64_t>(l) * n + i] * U[l * p + k];
    }
    return w * r;
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int op = 0; op < nops; ++op) {
    double m = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(value(op, i)));
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) mx[op][warp] = m;
  }
  __syncthreads();
  if (threadIdx.x < nops) {
    double m = 0;
    for (int w = 0; w < (blockDim.x >> 5); ++w) m = fmax(m, mx[threadIdx.x][w]);
    int e = 0;
    if (m > 0) e = 10 - static_cast<int>(floor(log2(m)));
    sc[threadIdx.x] = ldexp(1.0, e);
    const double side = threadIdx.x == 1 ? s2 : s1;  // gg pairs with Gt^2, the rest with Gt
    unscale[static_cast<int64_t>(g) * nops + threadIdx.x] = static_cast<float>(1.0 / (ldexp(1.0, e) * side));
  }
  __syncthreads();
  for (int op = 0; op < nops; ++op) {
    const double s = sc[op];
    for (int i = threadIdx.x; i < k_pad; i += blockDim.x) {
      const double v = value(op, i) * s;
      const __half h = __double2half(v);
      hi[op][static_cast<int64_t>(g) * k_pad + i] = h;
      lo[op][static_cast<int64_t>(g) * k_pad + i] = __double2half(v - static_cast<double>(__half2float(h)));
    }
  }
}

struct LmmGroupEpiParams {
  int G;
  int64_t m;
  int n_acc;                // p + 2
  const float* unscale;     // [G][n_acc]: NUM, gg, a~_0 .. a~_{p-1}
  const double* rss_null;   // [G]
  const uint8_t* snp_ok;    // [m]
  Windows win;
  float df;
  float t_cand;
  TTable tt;
  GeneOut out;
  const float* snp_mean;    // GLM only, as in LmmEpiParams
  const float* rsum;
  const uint8_t* gene_ok;
};
struct GlmGroupEpiParams : LmmGroupEpiParams {};

// GLM = true: the NB-GLM score test, as in LmmEpi.
template <bool GLM>
struct LmmGroupEpiT {
  static constexpr bool kGrouped = true;
  static constexpr int kTileN = 64;  // one 16-column chunk per epilogue thread
  using Params = std::conditional_t<GLM, GlmGroupEpiParams, LmmGroupEpiParams>;
  static constexpr int kSmemBytes = kTTableSmemBytes;
  const Params& Pr;
  float* tsm;
  TTable tt;
  int gene = 0;
  int64_t snp0 = 0;
  bool gvalid = false;
  float inv_rss = 0;
  float rs = 0;  // GLM: sum_i r_i of the gene
  float num[16], S[16];
  float u_cand;  // t_cand^2
  GeneAcc acc;
  __device__ LmmGroupEpiT(const Params& p, const TileShape&, uint8_t* smem)
      : Pr(p), tsm(reinterpret_cast<float*>(smem)), tt(p.tt), u_cand(p.t_cand * p.t_cand) {}
  __device__ void init(int tid, int nthr) {
    if (tsm) tt = screen_to_smem(Pr.tt, tsm, tid, nthr);
  }
  __device__ void begin_tile(int g, int64_t s0) {
    gene = g;
    snp0 = s0;
    gvalid = g < Pr.G;
    if constexpr (GLM) gvalid = gvalid && Pr.gene_ok[g];
    acc.reset();
    if (gvalid) {
      if constexpr (GLM) {
        rs = Pr.rsum[g];
      } else {
        const double r = Pr.rss_null[g];
        inv_rss = r > 0 ? static_cast<float>(1.0 / r) : 0.0f;
      }
      acc.load_window(Pr.win, g);
    }
  }
  // accumulator j of this tile for the 16 columns at c
  __device__ void acc_chunk(int j, int c, const float (&v)[16]) {
    if (!gvalid) return;
    const float us = Pr.unscale[static_cast<int64_t>(gene) * Pr.n_acc + j];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const float x = v[i] * us;
      if (j == 0) {
        num[i] = x;
      } else if (j == 1) {
        S[i] = x < 1e-12f ? -INFINITY : x;  // gg < 1e-12: p = 1
      } else {
        S[i] = fmaf(-x, x, S[i]);
      }
    }
  }
  // after the last group: the 16 pairs' t, tail and per-gene updates
  __device__ void finish_chunk(int c) {
    const int64_t s0 = snp0 + c;
    if (!gvalid || s0 >= Pr.m) return;
    uint32_t okw[4];
    load_flags16(Pr.snp_ok + s0, okw);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int64_t s = s0 + j;
      const bool valid = flag16(okw, j) && s < Pr.m && acc.in_scope(Pr.win, s);
      float u;
      if constexpr (GLM) {
        const float U = fmaf(__ldg(Pr.snp_mean + s), rs, num[j]);
        u = S[j] > 1e-15f ? __fdividef(U * U, S[j]) : 0.0f;  // z^2
      } else {
        const float r = num[j] * __fdividef(num[j], S[j]) * inv_rss;
        const float omr = 1.0f - r;
        const bool ok_stat = S[j] > 1e-15f && omr > 0.0f;
        u = ok_stat ? Pr.df * __fdividef(r, omr) : 0.0f;  // t^2
      }
      const ScreenOut o = acat_screen_u(u, tt);
      acc.add_screen(o, s, valid);
      if (valid && (u >= u_cand || o.deferred)) emit_candidate(Pr.out, gene, s, o.deferred, o.tiny);
    }
    acc.end_chunk();
  }
  __device__ void end_tile() {
    if (gvalid) acc.flush(Pr.out, gene);
  }
  __device__ void finish() {}
};

using LmmGroupEpi = LmmGroupEpiT<false>;
using GlmGroupEpi = LmmGroupEpiT<true>;

// subset gate for the LMM scan (src/scan_common.cpp:133-151)
__global__ void snp_gate_kernel(const int64_t* __restrict__ kept, int64_t m, int n, const double* __restrict__ mu,
                                const int32_t* __restrict__ n_miss, const double* __restrict__ s1,
                                const double* __restrict__ s2, uint8_t* ok) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const int64_t s = kept[r];
  const double mus = mu[s];
  const int k = n_miss[s];
  const double sum = s1[s] + k * mus;
  const double sum2 = s2[s] + k * mus * mus;
  double af = (sum / n) / 2.0;
  af = fmin(fmax(af, 0.0), 1.0);
  const double maf = af > 0.5 ? 1.0 - af : af;
  const double var = sum2 / n - (sum / n) * (sum / n);
  ok[r] = (maf < 1e-12 || var < 1e-12) ? 0 : 1;
}

// raw dosages of listed kept SNPs, column-major [n, u]
__global__ void raw_dosage_kernel(GenoRows src, const int32_t* __restrict__ col, int n,
                                  const int64_t* __restrict__ kept, const double* __restrict__ mu,
                                  const int* __restrict__ snps, int u, double* out) {
  const int64_t tot = static_cast<int64_t>(u) * n;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < tot;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(e / n);
    const int i = static_cast<int>(e - static_cast<int64_t>(c) * n);
    const int64_t s = kept[snps[c]];
    const double d = src.dosage(s, col[i]);
    out[e] = isnan(d) ? mu[s] : d;
  }
}

// One warp per (gene, snp) pair from the FP64 rotated raw dosage Gt = Q'g:
// gg = Gt'W Gt, yg = Gt'W y~, a = X~'W Gt with W = diag(1 / (delta lambda + 1)),
// then the pair's printed statistics (test_lmm_gtil, src/scan_trans_lmm.cpp:11-40).
__global__ void lmm_refine_kernel(const double* __restrict__ Gt, int n, const int* __restrict__ pair_col,
                                  const int2* __restrict__ pairs, int n_pairs, const double* __restrict__ Ytil,
                                  const double* __restrict__ Xtil, int p, const double* __restrict__ lam,
                                  const double* __restrict__ delta, const double* __restrict__ chi0,
                                  const double* __restrict__ a00L, const double* __restrict__ rss, double df,
                                  eqtl_pair* out) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= n_pairs) return;
  const int g = pairs[w].x;
  const double* gt = Gt + static_cast<int64_t>(pair_col[w]) * n;
  const double* yt = Ytil + static_cast<int64_t>(g) * n;
  const double d = delta[g];
  double gg = 0, yg = 0, a[kMaxPLmm];
  for (int k = 0; k < p; ++k) a[k] = 0;
  for (int i = lane; i < n; i += 32) {
    double v = d * lam[i] + 1.0;
    if (v < 1e-12) v = 1e-12;
    const double dg = gt[i] / v;
    gg += dg * gt[i];
    yg += dg * yt[i];
    for (int k = 0; k < p; ++k) a[k] += Xtil[static_cast<int64_t>(k) * n + i] * dg;
  }
  for (int o = 16; o; o >>= 1) {
    gg += __shfl_xor_sync(0xffffffffu, gg, o);
    yg += __shfl_xor_sync(0xffffffffu, yg, o);
    for (int k = 0; k < p; ++k) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
  }
  if (lane == 0) {
    eqtl_pair q;
    q.snp = pairs[w].y;
    q.gene = g;
    q.reserved = 0;
    lmm_stats_fp64(gg, yg, a, chi0 + static_cast<int64_t>(g) * p, a00L + static_cast<int64_t>(g) * p * p, rss[g],
                   p, df, q);
    out[w] = q;
  }
}

// ------------------------------------------------- tiny-|t| pairs in FP64
// Pairs screened with 0 < |t| < tiny_t need an FP64 t only to place them
// against the reference's x = df / (df + t^2) quantisation and to form their
// ACAT term; relative accuracy ~1e-8 is ample. So instead of rotating their
// raw dosages (n^2 per SNP):
//   NUM = g_raw . u,   u = Q (w o r~) for the gene (one DGEMM per scan),
//   S   = Gt'W Gt - a'A00^-1 a from the stored FP16 hi/lo rotated genotypes
//         (centred; S does not see the centring) accumulated in FP64.
__global__ void lmm_wr_kernel(const double* __restrict__ Ytil, const double* __restrict__ Xtil,
                              const double* __restrict__ lam, const double* __restrict__ delta,
                              const double* __restrict__ chi0, int n, int p, int G, double* wr) {
  const int g = blockIdx.x;
  if (g >= G) return;
  const double d = delta[g];
  const double* yt = Ytil + static_cast<int64_t>(g) * n;
  const double* c0 = chi0 + static_cast<int64_t>(g) * p;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double v = d * lam[i] + 1.0;
    if (v < 1e-12) v = 1e-12;
    double r = yt[i];
    for (int k = 0; k < p; ++k) r -= Xtil[static_cast<int64_t>(k) * n + i] * c0[k];
    wr[static_cast<int64_t>(g) * n + i] = r / v;
  }
}

__global__ void lmm_tiny_kernel(GenoRows src, const int32_t* __restrict__ col, int n, int k_pad, const int64_t* __restrict__ kept, const double* __restrict__ mu,
                                const double* __restrict__ U, int64_t u_stride, const __half* __restrict__ gt_hi,
                                const __half* __restrict__ gt_lo, double inv_s1, const double* __restrict__ Xtil,
                                int p, const double* __restrict__ lam, const double* __restrict__ delta,
                                const double* __restrict__ ainv, const double* __restrict__ rss, double df,
                                const int2* __restrict__ pairs, int n_pairs, double* p_out) {
  const int lane = threadIdx.x & 31;
  const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= n_pairs) return;
  const int g = pairs[w].x;
  const int64_t r = pairs[w].y;
  const int64_t s = kept[r];
  const double mus = mu[s];
  const double* u = U + static_cast<int64_t>(g) * u_stride;
  const __half* gh = gt_hi + r * k_pad;
  const __half* gl = gt_lo + r * k_pad;
  const double d = delta[g];
  double num = 0, gg = 0, a[kMaxPLmm];
  for (int k = 0; k < p; ++k) a[k] = 0;
  for (int i = lane; i < n; i += 32) {
    const double dose = src.dosage(s, col[i]);
    num += (isnan(dose) ? mus : dose) * u[i];
    double v = d * lam[i] + 1.0;
    if (v < 1e-12) v = 1e-12;
    const double gt = (static_cast<double>(__half2float(gh[i])) + static_cast<double>(__half2float(gl[i]))) * inv_s1;
    const double dg = gt / v;
    gg += dg * gt;
    for (int k = 0; k < p; ++k) a[k] += Xtil[static_cast<int64_t>(k) * n + i] * dg;
  }
  for (int o = 16; o; o >>= 1) {
    num += __shfl_xor_sync(0xffffffffu, num, o);
    gg += __shfl_xor_sync(0xffffffffu, gg, o);
    for (int k = 0; k < p; ++k) a[k] += __shfl_xor_sync(0xffffffffu, a[k], o);
  }
  if (lane == 0) {
    eqtl_pair q;
    double S = -1.0;
    if (!(gg < 1e-12)) {
      const double* A = ainv + static_cast<int64_t>(g) * p * p;
      double aTu = 0;
      for (int x = 0; x < p; ++x) {
        double ux = 0;
        for (int y = 0; y < p; ++y) ux += A[x * p + y] * a[y];
        aTu += a[x] * ux;
      }
      S = gg - aTu;
    }
    lmm_stats_num_s(num, S, rss[g], df, q);
    p_out[w] = q.p;
  }
}

}  // namespace dev

template <>
struct EpiOf<dev::RotEpiParams> {
  using type = dev::RotEpi;
};
template <>
struct EpiOf<dev::LmmEpiParams<1>> {
  using type = dev::LmmEpi<1>;
};
template <>
struct EpiOf<dev::LmmEpiParams<2>> {
  using type = dev::LmmEpi<2>;
};
template <>
struct EpiOf<dev::LmmRawEpiParams<1>> {
  using type = dev::LmmEpi<1, false, true>;
};
template <>
struct EpiOf<dev::LmmLrEpiParams<1>> {
  using type = dev::LmmEpi<1, false, true, true>;
};
template <>
struct EpiOf<dev::LmmLrEpiParams<2>> {
  using type = dev::LmmEpi<2, false, true, true>;
};
template <>
struct EpiOf<dev::LmmNodeEpiParams<1>> {
  using type = dev::LmmNodeEpi<1>;
};
template <>
struct EpiOf<dev::LmmNodeEpiParams<2>> {
  using type = dev::LmmNodeEpi<2>;
};
template <>
struct EpiOf<dev::LmmRawEpiParams<2>> {
  using type = dev::LmmEpi<2, false, true>;
};
template <>
struct EpiOf<dev::LmmGroupEpiParams> {
  using type = dev::LmmGroupEpi;
};
template <>
struct EpiOf<dev::GlmEpiParams<1>> {
  using type = dev::LmmEpi<1, true>;
};
template <>
struct EpiOf<dev::GlmEpiParams<2>> {
  using type = dev::LmmEpi<2, true>;
};
template <>
struct EpiOf<dev::GlmGroupEpiParams> {
  using type = dev::GlmGroupEpi;
};

using namespace dev;

static cublasHandle_t blas_of(eqtl_ctx* ctx) {
  if (!ctx->cublas) {
    cublasHandle_t h;
    EQTL_CHECK(cublasCreate(&h) == CUBLAS_STATUS_SUCCESS, EQTL_E_CUDA, "cublasCreate failed");
    cublasSetStream(h, ctx->stream);
    ctx->cublas = h;
  }
  return static_cast<cublasHandle_t>(ctx->cublas);
}

// ------------------------------------------------------------------ basis
// --fast (sparsify_grm, src/model_lmm.cpp:88-104): off-diagonal entries of K
// below `thr` in magnitude become 0; the count of zeroed entries goes to *zeroed.
__global__ void sparsify_kernel(double* K, int n, double thr, unsigned long long* zeroed) {
  const int64_t total = static_cast<int64_t>(n) * n;
  unsigned long long c = 0;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = e / n, j = e - i * n;
    if (i != j && fabs(K[e]) < thr) {
      K[e] = 0.0;
      ++c;
    }
  }
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(zeroed, c);
}

void lmm_basis_from_grm(eqtl_ctx* ctx, const double* K_dev, int n, double sparsify_thr, int64_t* zeroed) {
  cudaStream_t st = ctx->stream;
  StageScope timer(ctx, EQTL_STAGE_EIGEN);
  LmmBasisDev& B = ctx->basis;
  B.n = n;
  B.Q.alloc(static_cast<size_t>(n) * n);
  B.lambda.alloc(n);
  EQTL_CUDA(cudaMemcpyAsync(B.Q.p, K_dev, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, st));
  if (sparsify_thr > 0) {
    DevBuf<unsigned long long>& cnt = ctx->ws.sparsify_cnt;
    cnt.alloc(1);
    cnt.zero(st);
    ++ctx->launches;
    const int64_t total = static_cast<int64_t>(n) * n;
    sparsify_kernel<<<static_cast<unsigned>(std::min<int64_t>((total + 255) / 256, 1184)), 256, 0, st>>>(
        B.Q.p, n, sparsify_thr, cnt.p);
    EQTL_CUDA(cudaGetLastError());
    unsigned long long c = 0;
    cnt.download(&c, 1, st);
    EQTL_CUDA(cudaStreamSynchronize(st));
    if (zeroed) *zeroed = static_cast<int64_t>(c);
  }
  if (!ctx->cusolver) {
    cusolverDnHandle_t hc;
    EQTL_CHECK(cusolverDnCreate(&hc) == CUSOLVER_STATUS_SUCCESS, EQTL_E_CUDA, "cusolverDnCreate failed");
    ctx->cusolver = hc;
  }
  cusolverDnHandle_t h = static_cast<cusolverDnHandle_t>(ctx->cusolver);
  cusolverDnSetStream(h, st);
  int lwork = 0;
  cusolverStatus_t cs = cusolverDnDsyevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, B.Q.p, n,
                                                    B.lambda.p, &lwork);
  DevBuf<double>& work = ctx->ws.eig_work;
  DevBuf<int>& info = ctx->ws.eig_info;
  if (cs == CUSOLVER_STATUS_SUCCESS) {
    work.alloc(std::max(lwork, 1));
    info.alloc(1);
    cs = cusolverDnDsyevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, B.Q.p, n, B.lambda.p, work.p, lwork,
                          info.p);
  }
  int info_h = 0;
  if (cs == CUSOLVER_STATUS_SUCCESS) {
    info.download(&info_h, 1, st);
    EQTL_CUDA(cudaStreamSynchronize(st));
  }
  EQTL_CHECK(cs == CUSOLVER_STATUS_SUCCESS && info_h == 0, EQTL_E_CUDA, "GRM eigen decomposition failed");
  B.lambda_h.resize(n);
  B.lambda.download(B.lambda_h.data(), n, st);
  EQTL_CUDA(cudaStreamSynchronize(st));
  for (double& l : B.lambda_h) l = std::max(l, 0.0);  // cwiseMax(0.0)
  B.lambda.upload(B.lambda_h.data(), n, st);
  B.Q_h.clear();
  ctx->have_basis = true;
  ctx->rot.m = 0;  // rotated genotypes belong to the previous basis
}

void solver_release(eqtl_ctx* ctx) {
  if (ctx->cusolver) cusolverDnDestroy(static_cast<cusolverDnHandle_t>(ctx->cusolver));
  ctx->cusolver = nullptr;
}

void lmm_set_basis(eqtl_ctx* ctx, const double* Q, const double* lambda, int n) {
  LmmBasisDev& B = ctx->basis;
  B.n = n;
  B.Q.upload(Q, static_cast<size_t>(n) * n, ctx->stream);
  B.lambda_h.assign(lambda, lambda + n);
  for (double& l : B.lambda_h) l = std::max(l, 0.0);
  B.lambda.upload(B.lambda_h.data(), n, ctx->stream);
  EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->have_basis = true;
  ctx->rot.m = 0;
}

// --------------------------------------------------------------- rotation
static void output_scales(int n, float& s1, float& s2) {
  // |Gt| <= |g - mean|_2 <= 2 sqrt(n); |Gt^2| <= 4 n: keep both below ~3e4
  s1 = std::ldexp(1.0f, static_cast<int>(std::floor(std::log2(30000.0 / (2.0 * std::sqrt(static_cast<double>(n)))))));
  s2 = std::ldexp(1.0f, static_cast<int>(std::floor(std::log2(30000.0 / (4.0 * n)))));
}

void lmm_rotate(eqtl_ctx* ctx) {
  Geno& g = ctx->geno;
  Rotated& R = ctx->rot;
  EQTL_CHECK(ctx->have_basis && ctx->basis.n == g.n, EQTL_E_STATE, "rotation needs an eigenbasis of size n");
  if (R.m == g.m && R.k_pad == g.k_pad && R.gt_hi.p) return;
  R.bf16_m = -1;
  cudaStream_t st = ctx->stream;
  StageScope timer(ctx, EQTL_STAGE_ROTATE);
  const int n = g.n, k_pad = g.k_pad;
  const int64_t m = g.m;
  DevBuf<__half>& qh = ctx->ws.q_hi;
  DevBuf<__half>& ql = ctx->ws.q_lo;
  ++ctx->launches;
  qh.alloc(static_cast<size_t>(n) * k_pad);
  ql.alloc(static_cast<size_t>(n) * k_pad);
  // split-BF16 contexts hold the genotype operand in BF16, so Q' is split
  // in BF16 too and the rotation runs on BF16 pairs
  const bool bf16 = ctx->precision == EQTL_PREC_SPLIT_BF16;
  if (bf16)
    q_split_kernel<__nv_bfloat16><<<dim3((k_pad + 255) / 256, n), 256, 0, st>>>(
        ctx->basis.Q.p, n, k_pad, reinterpret_cast<__nv_bfloat16*>(qh.p), reinterpret_cast<__nv_bfloat16*>(ql.p));
  else
    q_split_kernel<__half><<<dim3((k_pad + 255) / 256, n), 256, 0, st>>>(ctx->basis.Q.p, n, k_pad, qh.p, ql.p);
  EQTL_CUDA(cudaGetLastError());
  const size_t elems = static_cast<size_t>(m) * k_pad;
  R.gt_hi.alloc(elems);
  R.gt_lo.alloc(elems);
  R.gt2_hi.alloc(elems);
  R.gt2_lo.alloc(elems);
  R.gt_hi.zero(st);
  R.gt_lo.zero(st);
  R.gt2_hi.zero(st);
  R.gt2_lo.zero(st);
  RotEpiParams ep{};
  ep.n = n;
  ep.m = m;
  ep.k_pad = k_pad;
  ep.unscale = 1.0f / (kGcScale * 1024.0f);
  output_scales(n, ep.s1, ep.s2);
  ep.gt_hi = R.gt_hi.p;
  ep.gt_lo = R.gt_lo.p;
  ep.gt2_hi = R.gt2_hi.p;
  ep.gt2_lo = R.gt2_lo.p;
  if (m > 0) {
    const __half* ah[1] = {qh.p};
    const __half* al[1] = {ql.p};
    const __half* bh[1] = {g.gc_hi.p};
    const __half* bl[1] = {g.gc_lo.p};
    const int bsel[1] = {0}, prod[1] = {7};
    launch_tile_n<256, 1>(ctx, bf16, ep, ah, al, n, bh, bl, m, k_pad, bsel, prod);
  }
  if (ctx->precision == EQTL_PREC_FP32_SIMT && m > 0) {
    // the FP32 form keeps its SNP-side operands in FP32
    R.gt32.alloc(elems);
    R.gt2_32.alloc(elems);
    ctx->launches += 2;
    sum_split_kernel<<<1184, 256, 0, st>>>(R.gt_hi.p, R.gt_lo.p, static_cast<int64_t>(elems), R.gt32.p);
    sum_split_kernel<<<1184, 256, 0, st>>>(R.gt2_hi.p, R.gt2_lo.p, static_cast<int64_t>(elems), R.gt2_32.p);
    EQTL_CUDA(cudaGetLastError());
  }
  R.m = m;
  R.k_pad = k_pad;
}

// ------------------------------------------------------------------- REML
// Per-gene REML prep into the context workspace (ws.Ytil, Xtil, delta, chi0,
// ainv, rss) from the resident phenotypes.
// out[i] = x[i]^2
__global__ void square_kernel(const double* __restrict__ x, int64_t count, double* out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = x[i] * x[i];
}

// Batched REML for p > kRemlWarpP over ws.Ytil / ws.Xtil into ws.delta,
// chi0, ainv, rss: columns in chunks whose per-round buffers stay near 2 GB.
static void reml_batched(eqtl_ctx* ctx, int n, int p, int G) {
  Workspace& ws = ctx->ws;
  cudaStream_t st = ctx->stream;
  cublasHandle_t h = blas_of(ctx);
  const int nq = p * (p + 1) / 2;
  const int df = n - p;
  ws.rb_P.alloc(static_cast<size_t>(nq) * n);
  ++ctx->launches;
  rb_pairs_kernel<<<1184, 256, 0, st>>>(ws.Xtil.p, n, p, ws.rb_P.p);
  EQTL_CUDA(cudaGetLastError());
  // grid-phase quantities shared by every column
  {
    const int K = kRbGridN;
    ws.rb_Wg.alloc(static_cast<size_t>(n) * K);
    ws.rb_Xw.alloc(static_cast<size_t>(n) * K * p);
    ws.rb_Ag.alloc(static_cast<size_t>(nq) * K);
    ws.rb_Lg.alloc(static_cast<size_t>(K) * p * p);
    ws.rb_ldx.alloc(K);
    ws.rb_ldD.alloc(K);
    ctx->launches += 2;
    rb_grid_weights_kernel<<<K, 256, 0, st>>>(ws.Xtil.p, ctx->basis.lambda.p, n, p, ws.rb_Wg.p, ws.rb_Xw.p,
                                             ws.rb_ldD.p);
    EQTL_CUDA(cudaGetLastError());
    const double one = 1.0, zero = 0.0;
    EQTL_CHECK(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, nq, K, n, &one, ws.rb_P.p, nq, ws.rb_Wg.p, n, &zero,
                           ws.rb_Ag.p, nq) == CUBLAS_STATUS_SUCCESS,
               EQTL_E_CUDA, "REML grid X'DX failed");
    rb_grid_chol_kernel<<<1, 64, 0, st>>>(ws.rb_Ag.p, p, ws.rb_Lg.p, ws.rb_ldx.p);
    EQTL_CUDA(cudaGetLastError());
  }
  const int cmax = std::max(1024, static_cast<int>((int64_t(1) << 26) / std::max(n, 1)));
  for (int g0 = 0; g0 < G; g0 += cmax) {
    const int C = std::min(cmax, G - g0);
    const size_t slots = 2 * static_cast<size_t>(C);
    ws.rb_state.alloc(sizeof(RemlBatchState) * C);
    ws.rb_dlt.alloc(slots);
    ws.rb_W.alloc(slots * n);
    ws.rb_WY.alloc(slots * n);
    ws.rb_A.alloc(slots * nq);
    ws.rb_B.alloc(slots * p);
    ws.rb_ld.alloc(slots);
    ws.rb_ydy.alloc(slots);
    ws.rb_active.alloc(1);
    RemlBatchState* state = reinterpret_cast<RemlBatchState*>(ws.rb_state.p);
    const double* Y = ws.Ytil.p + static_cast<int64_t>(g0) * n;
    const unsigned cblocks = static_cast<unsigned>((C + 127) / 128);
    const double one = 1.0, zero = 0.0;
    // grid phase: X~'D_k y for all columns as one GEMM over the stacked
    // w_k o X~ (35 p rows), y'D_k y as one GEMM over y o y
    {
      const int K = kRbGridN;
      ws.rb_Bg.alloc(static_cast<size_t>(K) * p * C);
      ws.rb_Yg.alloc(static_cast<size_t>(K) * C);
      ctx->launches += 1;
      square_kernel<<<1184, 256, 0, st>>>(Y, static_cast<int64_t>(n) * C, ws.rb_WY.p);
      EQTL_CUDA(cudaGetLastError());
      EQTL_CHECK(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, K * p, C, n, &one, ws.rb_Xw.p, n, Y, n, &zero,
                             ws.rb_Bg.p, K * p) == CUBLAS_STATUS_SUCCESS,
                 EQTL_E_CUDA, "REML grid X'Dy failed");
      EQTL_CHECK(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, K, C, n, &one, ws.rb_Wg.p, n, ws.rb_WY.p, n, &zero,
                             ws.rb_Yg.p, K) == CUBLAS_STATUS_SUCCESS,
                 EQTL_E_CUDA, "REML grid y'Dy failed");
      ++ctx->launches;
      rb_grid_advance_kernel<<<cblocks, 128, 0, st>>>(C, p, df, ws.rb_Lg.p, ws.rb_ldx.p, ws.rb_ldD.p, ws.rb_Bg.p,
                                                       ws.rb_Yg.p, state, ws.rb_dlt.p);
      EQTL_CUDA(cudaGetLastError());
    }
    for (int round = 0; round < kRbMaxRounds; ++round) {
      ctx->launches += 2;
      rb_weights_kernel<<<static_cast<unsigned>((slots + 7) / 8), 256, 0, st>>>(
          Y, ctx->basis.lambda.p, n, C, ws.rb_dlt.p, ws.rb_W.p, ws.rb_WY.p, ws.rb_ld.p, ws.rb_ydy.p);
      EQTL_CUDA(cudaGetLastError());
      EQTL_CHECK(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, nq, static_cast<int>(slots), n, &one, ws.rb_P.p, nq,
                             ws.rb_W.p, n, &zero, ws.rb_A.p, nq) == CUBLAS_STATUS_SUCCESS,
                 EQTL_E_CUDA, "REML X'DX failed");
      EQTL_CHECK(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, p, static_cast<int>(slots), n, &one, ws.Xtil.p, n,
                             ws.rb_WY.p, n, &zero, ws.rb_B.p, p) == CUBLAS_STATUS_SUCCESS,
                 EQTL_E_CUDA, "REML X'Dy failed");
      EQTL_CUDA(cudaMemsetAsync(ws.rb_active.p, 0, sizeof(unsigned int), st));
      auto advance = p <= 16 ? rb_advance_kernel<16> : rb_advance_kernel<kMaxPLmm>;
      advance<<<cblocks, 128, 0, st>>>(C, g0, p, df, ws.rb_A.p, ws.rb_B.p, ws.rb_ld.p, ws.rb_ydy.p, state,
                                       ws.rb_dlt.p, ws.rb_active.p, ws.delta.p, ws.chi0.p, ws.ainv.p, ws.rss.p,
                                       ws.a00L.p);
      EQTL_CUDA(cudaGetLastError());
      // the golden phase runs the same number of rounds for every column;
      // from the Newton phase on, stop once no column is left
      if (round >= 40) {
        unsigned int left = 0;
        ws.rb_active.download(&left, 1, st);
        EQTL_CUDA(cudaStreamSynchronize(st));
        if (left == 0) break;
      }
    }
  }
}

void lmm_prep(eqtl_ctx* ctx, const PhenoDev& ph, bool y_rotated) {
  const int n = ph.n, G = ph.G, p = ph.p;
  EQTL_CHECK(ctx->have_basis && ctx->basis.n == n, EQTL_E_STATE, "LMM prep needs an eigenbasis of size n");
  EQTL_CHECK(p >= 1 && p <= kMaxPLmm, EQTL_E_UNSUPPORTED, "the device LMM handles 1 <= p <= 32 covariate columns");
  cudaStream_t st = ctx->stream;
  Workspace& ws = ctx->ws;
  cublasHandle_t h = blas_of(ctx);
  ws.Ytil.alloc(static_cast<size_t>(n) * G);
  ws.Xtil.alloc(static_cast<size_t>(n) * p);
  const double one = 1.0, zero = 0.0;
  if (y_rotated) {
    EQTL_CUDA(cudaMemcpyAsync(ws.Ytil.p, ph.Y.p, sizeof(double) * n * G, cudaMemcpyDeviceToDevice, st));
  } else {
    EQTL_CHECK(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, n, G, n, &one, ctx->basis.Q.p, n, ph.Y.p, n, &zero,
                           ws.Ytil.p, n) == CUBLAS_STATUS_SUCCESS,
               EQTL_E_CUDA, "Q'Y failed");
  }
  EQTL_CHECK(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, n, p, n, &one, ctx->basis.Q.p, n, ph.X.p, n, &zero, ws.Xtil.p,
                         n) == CUBLAS_STATUS_SUCCESS,
             EQTL_E_CUDA, "Q'X failed");
  ws.delta.alloc(G);
  ws.chi0.alloc(static_cast<size_t>(G) * p);
  ws.ainv.alloc(static_cast<size_t>(G) * p * p);
  ws.a00L.alloc(static_cast<size_t>(G) * p * p);
  ws.rss.alloc(G);
  ++ctx->launches;
  if (p <= kRemlWarpP) {
    const unsigned blocks = static_cast<unsigned>((G + 7) / 8);
    auto args = [&](auto kern) {
      kern<<<blocks, 256, 0, st>>>(ws.Ytil.p, ws.Xtil.p, ctx->basis.lambda.p, n, G, ws.delta.p, ws.chi0.p,
                                   ws.ainv.p, ws.rss.p, ws.a00L.p);
    };
    if (p == 1) args(reml_warp_kernel<1>);
    else if (p == 2) args(reml_warp_kernel<2>);
    else args(reml_warp_kernel<3>);
    EQTL_CUDA(cudaGetLastError());
    return;
  }
  reml_batched(ctx, n, p, G);
}

// ------------------------------------------------------------------- scan
// hi + lo of an FP16 pair operand, re-split into BF16 hi + lo (the split-BF16
// form of the scans: ~16 significant bits instead of ~22)
__global__ void resplit_bf16_kernel(const __half* __restrict__ hi, const __half* __restrict__ lo, int64_t count,
                                    __nv_bfloat16* bhi, __nv_bfloat16* blo) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float v = __half2float(hi[i]) + __half2float(lo[i]);
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    bhi[i] = h;
    blo[i] = __float2bfloat16_rn(v - __bfloat162float(h));
  }
}

static void resplit_bf16(eqtl_ctx* ctx, const __half* hi, const __half* lo, int64_t count, DevBuf<__half>& bhi,
                         DevBuf<__half>& blo) {
  bhi.alloc(static_cast<size_t>(std::max<int64_t>(count, 1)));
  blo.alloc(static_cast<size_t>(std::max<int64_t>(count, 1)));
  if (count <= 0) return;
  ++ctx->launches;
  resplit_bf16_kernel<<<static_cast<unsigned>(std::min<int64_t>((count + 255) / 256, int64_t(ctx->sm_count) * 32)),
                        256, 0, ctx->stream>>>(hi, lo, count, reinterpret_cast<__nv_bfloat16*>(bhi.p),
                                               reinterpret_cast<__nv_bfloat16*>(blo.p));
  EQTL_CUDA(cudaGetLastError());
}

// The split-BF16 SNP-side operands of the rotation (once per rotation).
static void rot_bf16(eqtl_ctx* ctx, Rotated& R) {
  if (R.bf16_m == R.m && R.bgt_hi.p) return;
  const int64_t elems = R.m * R.k_pad;
  resplit_bf16(ctx, R.gt_hi.p, R.gt_lo.p, elems, R.bgt_hi, R.bgt_lo);
  resplit_bf16(ctx, R.gt2_hi.p, R.gt2_lo.p, elems, R.bgt2_hi, R.bgt2_lo);
  R.bf16_m = R.m;
}

// The split-BF16 gene-side operands: nops pairs of rows x k_pad into
// ws.opsb_hi / opsb_lo; out[j], out[nops + j] point at pair j's hi and lo.
static void gene_ops_bf16(eqtl_ctx* ctx, const __half* const* hi, const __half* const* lo, int nops, int64_t rows,
                          int k_pad, const __half** out) {
  EQTL_CHECK(nops <= dev::kMaxAcc, EQTL_E_INTERNAL, "split-BF16 gene operands");
  for (int j = 0; j < nops; ++j) {
    resplit_bf16(ctx, hi[j], lo[j], rows * k_pad, ctx->ws.opsb_hi[j], ctx->ws.opsb_lo[j]);
    out[j] = ctx->ws.opsb_hi[j].p;
    out[nops + j] = ctx->ws.opsb_lo[j].p;
  }
}

template <int P>
static void lmm_launch_simt(eqtl_ctx* ctx, const LmmEpiParams<P>& ep, const __half* const* ah,
                            const __half* const* al, int G, const __half* const* bh, const __half* const* bl,
                            const int* bsel, const Rotated& R);

template <int P, class EP>
static void lmm_launch(eqtl_ctx* ctx, const EP& ep, const __half* const* ah, const __half* const* al, int G,
                       bool simt, const int2* tiles, int n_tiles, const Rotated& R) {
  // the exact-operand form reads the raw SNP operand (one exact FP16 slice:
  // hi*hi + lo*hi) for NUM and a_k, and Gt^2 for gg as both forms do
  constexpr bool raw = std::is_same_v<EP, LmmRawEpiParams<P>>;
  const __half* bh[2] = {raw ? R.raw.p : R.gt_hi.p, R.gt2_hi.p};
  const __half* bl[2] = {raw ? R.raw.p : R.gt_lo.p, R.gt2_lo.p};
  // tile order [gg, a_0 .. a_{P-1}, NUM] from the gene-ops order [NUM, a.., gg]
  const __half* oh[P + 2];
  const __half* ol[P + 2];
  int bsel[P + 2], prod[P + 2];
  for (int j = 0; j < P + 2; ++j) {
    const int op = j == 0 ? P + 1 : (j == P + 1 ? 0 : j);
    oh[j] = ah[op];
    ol[j] = al[op];
    bsel[j] = j == 0 ? 1 : 0;  // gg reads Gt^2
    prod[j] = raw && j > 0 ? 5 : 7;
  }
  ah = oh;
  al = ol;
  if (!simt && !raw && ctx->precision == EQTL_PREC_SPLIT_BF16) {
    // split-BF16: both sides re-split into BF16 hi + lo, three products each
    const __half* b16[2 * (P + 2)];
    gene_ops_bf16(ctx, ah, al, P + 2, G, R.k_pad, b16);
    Rotated& Rw = const_cast<Rotated&>(R);
    rot_bf16(ctx, Rw);
    const __half* sbh[2] = {Rw.bgt_hi.p, Rw.bgt2_hi.p};
    const __half* sbl[2] = {Rw.bgt_lo.p, Rw.bgt2_lo.p};
    launch_tile_n<128, P + 2>(ctx, true, ep, b16, b16 + (P + 2), G, sbh, sbl, R.m, R.k_pad, bsel, prod, tiles,
                              n_tiles);
    return;
  }
  if (!simt) {
    launch_tile_n<128, P + 2>(ctx, false, ep, ah, al, G, bh, bl, R.m, R.k_pad, bsel, prod, tiles, n_tiles);
    return;
  }
  if constexpr (std::is_same_v<EP, LmmEpiParams<P>>) lmm_launch_simt<P>(ctx, ep, ah, al, G, bh, bl, bsel, R);
}

// the plain FP32 CUDA-core comparator of the LMM scan
// The FP32 operands (ws.ops32 in tile order, Rotated::gt32 / gt2_32) are
// formed before the scan; accumulator 0 (gg) reads Gt^2, the others Gt.
template <int P>
static void lmm_launch_simt(eqtl_ctx* ctx, const LmmEpiParams<P>& ep, const __half* const*, const __half* const*,
                            int G, const __half* const*, const __half* const*, const int* bsel, const Rotated& R) {
  cudaStream_t st = ctx->stream;
  EQTL_CHECK(bsel[0] == 1 && R.gt32.p && R.gt2_32.p, EQTL_E_INTERNAL, "FP32 comparator operands");
  const float* ptrs[P + 2];
  for (int j = 0; j < P + 2; ++j) ptrs[j] = ctx->ws.ops32[j].p;
  DevBuf<const float*>& dptr = ctx->ws.ops32_ptr;
  dptr.upload(ptrs, P + 2, st);
  TileShape sh{};
  using Cfg = SimtCfg<P + 2>;
  auto kern = simt_tile_kernel<P + 2, LmmEpi<P>>;
  EQTL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM_BYTES));
  dim3 grid(static_cast<unsigned>((R.m + kSimtBN - 1) / kSimtBN), static_cast<unsigned>((G + kSimtBM - 1) / kSimtBM));
  ++ctx->launches;
  kern<<<grid, kSimtThreads, Cfg::SMEM_BYTES, st>>>(dptr.p, G, R.gt32.p, R.gt2_32.p, R.m, R.k_pad, sh, ep);
  EQTL_CUDA(cudaGetLastError());
  EQTL_CUDA(cudaStreamSynchronize(st));
}

// FP64 statistics of (gene, kept SNP) pairs against the current LMM prep
// (ws.Ytil, Xtil, delta, chi0, ainv, rss): raw dosages of the SNPs involved,
// Gt = Q'g by DGEMM, then one warp per pair (lmm_refine_kernel).
static std::vector<eqtl_pair> lmm_refine_pairs(eqtl_ctx* ctx, int p, double df, const std::vector<int2>& todo) {
  Geno& g = ctx->geno;
  Workspace& ws = ctx->ws;
  cudaStream_t st = ctx->stream;
  const int n = g.n;
  std::vector<eqtl_pair> refined(todo.size());
  HostTrace tr("lmm_refine_pairs");
  if (!todo.empty()) {
    // distinct SNPs in index order and each pair's column among them, by a
    // marker over the kept SNPs (O(m + pairs), no sort)
    std::vector<int>& mark = ctx->host_mark;
    mark.assign(static_cast<size_t>(g.m), -1);
    for (const int2& q : todo) mark[q.y] = 0;
    std::vector<int> snps;
    for (int64_t s = 0; s < g.m; ++s)
      if (mark[s] == 0) {
        mark[s] = static_cast<int>(snps.size());
        snps.push_back(static_cast<int>(s));
      }
    std::vector<int> pcol(todo.size());
    for (size_t i = 0; i < todo.size(); ++i) pcol[i] = mark[todo[i].y];
    const int u = static_cast<int>(snps.size());
    DevBuf<int>& dsn = ws.ref_snps;
    DevBuf<int>& dpc = ws.ref_col;
    DevBuf<int2>& dtodo = ws.ref_pairs;
    dsn.upload(snps.data(), u, st);
    dpc.upload(pcol.data(), pcol.size(), st);
    dtodo.upload(todo.data(), todo.size(), st);
    tr.mark("host index + upload");
    DevBuf<double>& graw = ws.graw;
    DevBuf<double>& gt = ws.gt;
    graw.alloc(static_cast<size_t>(n) * u);
    gt.alloc(static_cast<size_t>(n) * u);
    ctx->launches += 2;
    raw_dosage_kernel<<<1184, 256, 0, st>>>(g.rows(), g.col.p, n, g.kept.p, g.mu.p, dsn.p, u, graw.p);
    EQTL_CUDA(cudaGetLastError());
    const double one = 1.0, zero = 0.0;
    EQTL_CHECK(cublasDgemm(blas_of(ctx), CUBLAS_OP_T, CUBLAS_OP_N, n, u, n, &one, ctx->basis.Q.p, n, graw.p, n, &zero,
                           gt.p, n) == CUBLAS_STATUS_SUCCESS,
               EQTL_E_CUDA, "Q'g failed");
    ws.refined.alloc(todo.size());
    lmm_refine_kernel<<<static_cast<unsigned>((todo.size() + 7) / 8), 256, 0, st>>>(
        gt.p, n, dpc.p, dtodo.p, static_cast<int>(todo.size()), ws.Ytil.p, ws.Xtil.p, p, ctx->basis.lambda.p,
        ws.delta.p, ws.chi0.p, ws.a00L.p, ws.rss.p, df, ws.refined.p);
    EQTL_CUDA(cudaGetLastError());
    tr.mark("launches");
    ws.refined.download(refined.data(), todo.size(), st);
    EQTL_CUDA(cudaStreamSynchronize(st));
    tr.mark("device work + download");
  }
  return refined;
}

// FP64 p of tiny-|t| pairs against the current LMM prep (see lmm_tiny_kernel).
// U_pre (optional): u = Q (w o r~) of gene g at U_pre + g * u_stride, as the
// exact-operand scan has it already; otherwise it is computed here.
static std::vector<double> lmm_tiny_p(eqtl_ctx* ctx, int p, double df, const std::vector<int2>& tiny,
                                      const double* U_pre = nullptr, int64_t u_stride = 0) {
  Geno& g = ctx->geno;
  Workspace& ws = ctx->ws;
  Rotated& R = ctx->rot;
  cudaStream_t st = ctx->stream;
  const int n = g.n;
  const int G = static_cast<int>(ws.delta.n);
  std::vector<double> out(tiny.size());
  if (tiny.empty()) return out;
  const double* U = U_pre;
  if (!U) {
    ws.graw.alloc(static_cast<size_t>(n) * G);  // w o r~ per gene
    ws.gt.alloc(static_cast<size_t>(n) * G);    // u = Q (w o r~)
    ctx->launches += 1;
    lmm_wr_kernel<<<G, 256, 0, st>>>(ws.Ytil.p, ws.Xtil.p, ctx->basis.lambda.p, ws.delta.p, ws.chi0.p, n, p, G,
                                     ws.graw.p);
    EQTL_CUDA(cudaGetLastError());
    const double one = 1.0, zero = 0.0;
    EQTL_CHECK(cublasDgemm(blas_of(ctx), CUBLAS_OP_N, CUBLAS_OP_N, n, G, n, &one, ctx->basis.Q.p, n, ws.graw.p, n,
                           &zero, ws.gt.p, n) == CUBLAS_STATUS_SUCCESS,
               EQTL_E_CUDA, "Q (w o r) failed");
    U = ws.gt.p;
    u_stride = n;
  }
  ctx->launches += 1;
  float s1, s2;
  output_scales(n, s1, s2);
  ws.ref_pairs.upload(tiny.data(), tiny.size(), st);
  ws.tiny_p.alloc(tiny.size());
  lmm_tiny_kernel<<<static_cast<unsigned>((tiny.size() + 7) / 8), 256, 0, st>>>(
      g.rows(), g.col.p, n, R.k_pad, g.kept.p, g.mu.p, U, u_stride, R.gt_hi.p, R.gt_lo.p, 1.0 / s1,
      ws.Xtil.p, p, ctx->basis.lambda.p, ws.delta.p, ws.ainv.p, ws.rss.p, df, ws.ref_pairs.p,
      static_cast<int>(tiny.size()), ws.tiny_p.p);
  EQTL_CUDA(cudaGetLastError());
  ws.tiny_p.download(out.data(), out.size(), st);
  EQTL_CUDA(cudaStreamSynchronize(st));
  return out;
}

// Which form of the exact-operand scan (p <= 2, dense) forms gg and a_k:
// interpolated between node deltas (lmm_lr_prepare) from 256 genes on, where
// the node pass costs less than it saves, otherwise directly. EQTL_LMM_FORM
// = "direct" or "lr" fixes the form for every gene count.
static bool lmm_lr_wanted(int G) {
  const char* f = std::getenv("EQTL_LMM_FORM");
  if (f && std::strcmp(f, "direct") == 0) return false;
  if (f && std::strcmp(f, "lr") == 0) return true;
  return G >= 256;
}

// Interpolated gg and a_k: Chebyshev-Lobatto nodes over the genes' range of
// ln(delta) (5 equal intervals if that keeps each within kLrSpan, else 11;
// kLrNodes nodes each, neighbours sharing their end node: 56 or 122 nodes),
// the node genes' operands (w and Q (w o X~_k) at each node delta, as
// lmm_gene_ops_raw_kernel forms a gene's), the node pass over every kept
// SNP, then both sides of the scan's gg and a_k accumulators (ws.lr_phi /
// lr_plo: SNP side [m][kb]; ws.lr_chi / lr_clo: gene side [G][kb];
// ws.unscale of gg and a_k). Returns false, leaving the direct form, when
// the intervals would be longer than kLrSpan.
template <int P>
static bool lmm_lr_build(eqtl_ctx* ctx, int n, int G, float s2) {
  Workspace& ws = ctx->ws;
  const Geno& g = ctx->geno;
  const Rotated& R = ctx->rot;
  cudaStream_t st = ctx->stream;
  constexpr int nops = P + 2;
  const int k_pad = g.k_pad;
  const int64_t m = g.m;
  std::vector<double> d(static_cast<size_t>(G));
  ws.delta.download(d.data(), d.size(), st);
  EQTL_CUDA(cudaStreamSynchronize(st));
  double lo = INFINITY, hi = -INFINITY;
  for (double x : d) {
    const double a = std::log(std::max(x, 1e-300));
    if (std::isfinite(a)) {
      lo = std::min(lo, a);
      hi = std::max(hi, a);
    }
  }
  if (!(lo <= hi)) lo = hi = 0.0;
  if (hi - lo < 1e-6) {
    lo -= 0.5;
    hi += 0.5;
  }
  // as many intervals as one or two 64-column chunks of nodes hold (5 or 11)
  const int nint = static_cast<int>(std::ceil((hi - lo) / kLrSpan)) <= 5 ? 5 : 11;
  const double h = (hi - lo) / nint;
  const int nn = nint * (kLrNodes - 1) + 1;
  // intervals longer than kLrSpan (a delta range beyond REML's 1e-8 .. 1e6)
  // would lose the interpolation's accuracy: the direct form then
  if (nn > kTileM || h > kLrSpan * (1.0 + 1e-12)) return false;
  std::vector<double> na(static_cast<size_t>(nn)), nd(static_cast<size_t>(nn));
  for (int q = 0; q < nint; ++q)
    for (int i = 0; i < kLrNodes; ++i)
      na[static_cast<size_t>(q * (kLrNodes - 1) + i)] =
          lo + h * (q + 0.5 * (1.0 - std::cos(M_PI * i / (kLrNodes - 1))));
  for (int j = 0; j < nn; ++j) nd[static_cast<size_t>(j)] = std::exp(na[static_cast<size_t>(j)]);
  const int kn = nn <= 64 ? 64 : 128, kb = (P + 1) * kn;
  ws.lr_kn = kn;
  ws.lr_kb = kb;
  ws.lr_nodes = nn;
  ws.lr_a.upload(na.data(), na.size(), st);
  ws.lr_delta.upload(nd.data(), nd.size(), st);

  // node genes' operands: a zero residual (u = 0), w o X~_k, Q times them
  const size_t cols = static_cast<size_t>(nn) * (P + 1);
  ws.lr_zero.alloc(static_cast<size_t>(nn) * (n + P));
  ws.lr_zero.zero(st);
  ws.lr_w.alloc(static_cast<size_t>(n) * cols);
  ws.lr_uv.alloc(static_cast<size_t>(n) * cols);
  ++ctx->launches;
  lmm_uv_w_kernel<<<nn, 256, 0, st>>>(ws.lr_zero.p, ws.Xtil.p, ctx->basis.lambda.p, ws.lr_delta.p,
                                      ws.lr_zero.p + static_cast<size_t>(nn) * n, n, P, nn, ws.lr_w.p);
  EQTL_CUDA(cudaGetLastError());
  const double one = 1.0, zero = 0.0;
  EQTL_CHECK(cublasDgemm(blas_of(ctx), CUBLAS_OP_N, CUBLAS_OP_N, n, static_cast<int>(cols), n, &one,
                         ctx->basis.Q.p, n, ws.lr_w.p, n, &zero, ws.lr_uv.p, n) == CUBLAS_STATUS_SUCCESS,
             EQTL_E_CUDA, "Q (w o X~) at the node deltas failed");
  ctx->launches += 1;
  __half* nptr[2 * nops];
  for (int k = 0; k < nops; ++k) {
    ws.lr_ops_hi[k].alloc(static_cast<size_t>(nn) * k_pad);
    ws.lr_ops_lo[k].alloc(static_cast<size_t>(nn) * k_pad);
    nptr[k] = ws.lr_ops_hi[k].p;
    nptr[nops + k] = ws.lr_ops_lo[k].p;
  }
  ws.lr_ops_ptr.upload(nptr, 2 * nops, st);
  ws.lr_unscale.alloc(static_cast<size_t>(nn) * nops);
  ++ctx->launches;
  lmm_gene_ops_raw_kernel<<<nn, 256, 0, st>>>(ws.lr_uv.p, ctx->basis.lambda.p, ws.lr_delta.p, n, P, nn, k_pad, s2,
                                              ws.lr_ops_ptr.p, ws.lr_ops_ptr.p + nops, ws.lr_unscale.p);
  EQTL_CUDA(cudaGetLastError());

  // node pass: accumulators [gg, a_0 ..] against Gt^2 and the raw operand
  ws.lr_val.alloc(static_cast<size_t>(m) * kb);
  ws.lr_colmax.alloc(static_cast<size_t>(kb));
  ws.lr_colmax.zero(st);
  if (m > 0) {
    LmmNodeEpiParams<P> ep{};
    ep.n_nodes = nn;
    ep.m = m;
    ep.kn = kn;
    ep.kb = kb;
    ep.unscale = ws.lr_unscale.p;
    ep.snp_alpha = R.alpha.p;
    ep.val = ws.lr_val.p;
    ep.colmax = ws.lr_colmax.p;
    const __half* ah[P + 1];
    const __half* al[P + 1];
    int bsel[P + 1], prod[P + 1];
    ah[0] = ws.lr_ops_hi[P + 1].p;
    al[0] = ws.lr_ops_lo[P + 1].p;
    bsel[0] = 1;
    prod[0] = 7;
    for (int k = 0; k < P; ++k) {
      ah[1 + k] = ws.lr_ops_hi[1 + k].p;
      al[1 + k] = ws.lr_ops_lo[1 + k].p;
      bsel[1 + k] = 0;
      prod[1 + k] = 5;
    }
    const __half* bh[2] = {R.raw.p, R.gt2_hi.p};
    const __half* bl[2] = {R.raw.p, R.gt2_lo.p};
    launch_tile_n<128, P + 1>(ctx, false, ep, ah, al, nn, bh, bl, m, k_pad, bsel, prod);
  }
  ws.lr_sigma.alloc(static_cast<size_t>(kb));
  ++ctx->launches;
  lr_sigma_kernel<<<(kb + 255) / 256, 256, 0, st>>>(ws.lr_colmax.p, kb, ws.lr_sigma.p);
  EQTL_CUDA(cudaGetLastError());
  ws.lr_phi.alloc(std::max<size_t>(1, static_cast<size_t>(m) * kb));
  ws.lr_plo.alloc(std::max<size_t>(1, static_cast<size_t>(m) * kb));
  if (m > 0) {
    ++ctx->launches;
    lr_split_kernel<<<4 * sm_count(ctx), 256, 0, st>>>(ws.lr_val.p, m * kb, kb, ws.lr_sigma.p, ws.lr_phi.p,
                                                       ws.lr_plo.p);
    EQTL_CUDA(cudaGetLastError());
  }
  // genes' coefficients (rows zero outside each gene's nodes)
  ws.lr_chi.alloc(static_cast<size_t>(G) * kb);
  ws.lr_clo.alloc(static_cast<size_t>(G) * kb);
  ws.lr_chi.zero(st);
  ws.lr_clo.zero(st);
  ++ctx->launches;
  lr_coef_kernel<<<(G + 127) / 128, 128, 0, st>>>(ws.delta.p, G, ws.lr_a.p, lo, h, nint, ws.lr_sigma.p, kn, kb, P,
                                                  ws.lr_chi.p, ws.lr_clo.p, ws.unscale.p);
  EQTL_CUDA(cudaGetLastError());
  return true;
}

// lmm_lr_build, or the direct form when its tables do not fit in device
// memory beside the scan's operands (their large buffers are given back).
template <int P>
static bool lmm_lr_prepare(eqtl_ctx* ctx, int n, int G, float s2) {
  try {
    return lmm_lr_build<P>(ctx, n, G, s2);
  } catch (const Error& e) {
    if (e.code != EQTL_E_NOMEM) throw;
    EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
    (void)cudaGetLastError();  // the failed allocation's error, so later launch checks do not see it
    Workspace& ws = ctx->ws;
    ws.lr_val.release();
    ws.lr_phi.release();
    ws.lr_plo.release();
    ws.lr_chi.release();
    ws.lr_clo.release();
    ws.lr_nodes = 0;
    return false;
  }
}

// The scan with interpolated gg and a_k: tile order [gg, a_0 .., NUM]; gg
// and a_k read their kind's node columns of both interpolated operands
// (K chunks [kind c, (kind + 1) c), c = kn / 64), NUM reads u hi + lo
// against the exact raw operand over all of K. ah / al: the gene-ops order
// [NUM, a_0 .., gg] (only NUM's u is read).
template <int P>
static void lmm_launch_lr(eqtl_ctx* ctx, const LmmLrEpiParams<P>& ep, const __half* const* ah,
                          const __half* const* al, int G, const Rotated& R) {
  Workspace& ws = ctx->ws;
  const int kb = ws.lr_kb, c = ws.lr_kn / kChunkK;
  const __half* oh[P + 2];
  const __half* ol[P + 2];
  int bsel[P + 2], prod[P + 2];
  TileK tk;
  for (int j = 0; j <= P; ++j) {
    oh[j] = ws.lr_chi.p;
    ol[j] = ws.lr_clo.p;
    bsel[j] = 1;
    prod[j] = 7;
    tk.beg[j] = j * c;
    tk.end[j] = (j + 1) * c;
    tk.k_a[j] = kb;
  }
  oh[P + 1] = ah[0];
  ol[P + 1] = al[0];
  bsel[P + 1] = 0;
  prod[P + 1] = 5;
  tk.k_b[1] = kb;
  const __half* bh[2] = {R.raw.p, ws.lr_phi.p};
  const __half* bl[2] = {R.raw.p, ws.lr_plo.p};
  launch_tile_n<128, P + 2>(ctx, false, ep, oh, ol, G, bh, bl, R.m, R.k_pad, bsel, prod, nullptr, 0, 1, P + 2, 0,
                            &tk);
}

// Subset gate of every kept SNP on the analysis samples into ws.ok.
static void lmm_gate(eqtl_ctx* ctx) {
  Geno& g = ctx->geno;
  DevBuf<uint8_t>& ok = ctx->ws.ok;
  const int64_t m = g.m;
  ok.alloc(static_cast<size_t>(((m + 255) / 256 + 1) * 256));  // the epilogue reads 16 flags per chunk, up to the last tile's end
  EQTL_CUDA(cudaMemsetAsync(ok.p, 0, ok.n, ctx->stream));
  if (m > 0) {
    ++ctx->launches;
    snp_gate_kernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, ctx->stream>>>(g.kept.p, m, g.n, g.mu.p,
                                                                                     g.gate_nmiss(), g.gate_s1(), g.gate_s2(), ok.p);
    EQTL_CUDA(cudaGetLastError());
  }
}

static void scan_trans_lmm_impl(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                                double* delta_out, eqtl_gene_result* genes, std::vector<eqtl_pair>& pairs,
                                std::vector<eqtl_pair>& cands, bool simt) {
  Geno& g = ctx->geno;
  Workspace& ws = ctx->ws;
  const int n = prm->n, G = prm->n_genes, p = prm->p;
  EQTL_CHECK(g.m_all > 0, EQTL_E_STATE, "scan_trans_lmm: no genotypes loaded");
  EQTL_CHECK(n == g.n, EQTL_E_ARG, "scan_trans_lmm: n differs from the loaded genotypes");
  EQTL_CHECK(G > 0, EQTL_E_ARG, "scan_trans_lmm: no genes");
  EQTL_CHECK(g.m < (int64_t(1) << 30), EQTL_E_UNSUPPORTED, "scan_trans_lmm: more than 2^30 kept SNPs");
  EQTL_CHECK(p >= 1 && p <= kMaxPLmm, EQTL_E_UNSUPPORTED,
             "the LMM scan handles 1 to 32 covariate columns (intercept included)");
  EQTL_CHECK(!(simt && p > 2), EQTL_E_UNSUPPORTED, "the FP32 CUDA-core comparator covers 1 or 2 covariate columns");
  const bool grouped = p > 2;  // accumulators run in groups of four (LmmGroupEpi)
  cudaStream_t st = ctx->stream;
  const double df = static_cast<double>(n - p - 1);
  const PhenoDev& ph = resolve_pheno(ctx, prm, Y, X);
  lmm_rotate(ctx);
  // p <= 2 on the tensor cores: NUM and a_k from the exact unrotated SNP
  // operand when every kept SNP fits it (2-bit rows, FP16 operands)
  const bool raw = !grouped && !simt && ctx->precision == EQTL_PREC_SPLIT_F16 && geno_raw_operand(ctx);
  std::unique_ptr<StageScope> prep_timer(new StageScope(ctx, EQTL_STAGE_PREP));
  lmm_prep(ctx, ph, prm->y_rotated != 0);

  // gene-side operands
  const int k_pad = g.k_pad;
  const int nops = p + 2;
  float s1, s2;
  output_scales(n, s1, s2);
  std::vector<__half*> oph(2 * nops);
  for (int k = 0; k < nops; ++k) {
    ws.ops_hi[k].alloc(static_cast<size_t>(G) * k_pad);
    ws.ops_lo[k].alloc(static_cast<size_t>(G) * k_pad);
    oph[k] = ws.ops_hi[k].p;
    oph[nops + k] = ws.ops_lo[k].p;
  }
  ws.ops_ptr.upload(oph.data(), oph.size(), st);
  DevBuf<float>& unscale = ws.unscale;
  unscale.alloc(static_cast<size_t>(G) * nops);
  ++ctx->launches;
  if (raw) {
    // u = Q (w o r~) and v_k = Q (w o X~_k) in FP64, then their FP16 hi/lo
    const size_t cols = static_cast<size_t>(G) * (p + 1);
    ws.lmm_w.alloc(static_cast<size_t>(n) * cols);
    ws.lmm_uv.alloc(static_cast<size_t>(n) * cols);
    lmm_uv_w_kernel<<<G, 256, 0, st>>>(ws.Ytil.p, ws.Xtil.p, ctx->basis.lambda.p, ws.delta.p, ws.chi0.p, n, p, G,
                                       ws.lmm_w.p);
    EQTL_CUDA(cudaGetLastError());
    const double one = 1.0, zero = 0.0;
    EQTL_CHECK(cublasDgemm(blas_of(ctx), CUBLAS_OP_N, CUBLAS_OP_N, n, static_cast<int>(cols), n, &one,
                           ctx->basis.Q.p, n, ws.lmm_w.p, n, &zero, ws.lmm_uv.p, n) == CUBLAS_STATUS_SUCCESS,
               EQTL_E_CUDA, "Q (w o [r~, X~]) failed");
    ctx->launches += 1;
    lmm_gene_ops_raw_kernel<<<G, 256, 0, st>>>(ws.lmm_uv.p, ctx->basis.lambda.p, ws.delta.p, n, p, G, k_pad, s2,
                                               ws.ops_ptr.p, ws.ops_ptr.p + nops, unscale.p);
  } else if (grouped) {
    lmm_gene_ops_orth_kernel<<<G, 256, 0, st>>>(ws.Ytil.p, ws.Xtil.p, ctx->basis.lambda.p, ws.delta.p, ws.chi0.p,
                                                ws.ainv.p, n, p, G, k_pad, s1, s2, ws.ops_ptr.p,
                                                ws.ops_ptr.p + nops, unscale.p);
  } else {
    lmm_gene_ops_kernel<<<G, 256, 0, st>>>(ws.Ytil.p, ws.Xtil.p, ctx->basis.lambda.p, ws.delta.p, ws.chi0.p, n, p, G,
                                           k_pad, s1, s2, ws.ops_ptr.p, ws.ops_ptr.p + nops, unscale.p);
  }
  EQTL_CUDA(cudaGetLastError());
  // dense scans with the exact operand: gg and a_k interpolated between node
  // deltas when that pays (lmm_lr_wanted)
  bool lr = false;
  ws.lr_nodes = 0;
  if (raw && prm->exclude_cis != 2 && lmm_lr_wanted(G))
    lr = p == 1 ? lmm_lr_prepare<1>(ctx, n, G, s2) : lmm_lr_prepare<2>(ctx, n, G, s2);
  if (simt) {
    // the FP32 form's gene-side operands, in the tile's accumulator order
    // [gg, a_0 .. a_{p-1}, NUM] (the gene-ops order is [NUM, a.., gg])
    for (int j = 0; j < nops; ++j) {
      const int op = j == 0 ? nops - 1 : (j == nops - 1 ? 0 : j);
      ws.ops32[j].alloc(static_cast<size_t>(G) * k_pad);
      ++ctx->launches;
      sum_split_kernel<<<1184, 256, 0, st>>>(ws.ops_hi[op].p, ws.ops_lo[op].p, static_cast<int64_t>(G) * k_pad,
                                             ws.ops32[j].p);
    }
    EQTL_CUDA(cudaGetLastError());
  }

  const int64_t m = g.m;
  lmm_gate(ctx);
  DevBuf<uint8_t>& ok = ws.ok;
  const Windows win = upload_windows(ctx, prm, m, prm->exclude_cis == 2 ? kWinInclude : prm->exclude_cis ? kWinExclude : kWinNone);
  double t_cand = t_critical(prm->pthr, df);
  if (prm->perm_thr > 0) t_cand = std::min(t_cand, t_critical(prm->perm_thr, df));
  const TTable tt = device_ttable(ctx, df);
  prep_timer.reset();
  ScanOutputs so(ctx, G, m, expected_candidates(prm, m));
  const int2* tiles = nullptr;  // cis: banded tile list (NT of the kernel that runs)
  int n_tiles = 0;
  if (!simt) cis_tile_list(ctx, prm, m, grouped ? LmmGroupEpi::kTileN : 128, tiles, n_tiles);
  std::unique_ptr<StageScope> scan_timer(new StageScope(ctx, EQTL_STAGE_SCAN));
  if (m > 0 && grouped) {
    Rotated& Rt = ctx->rot;
    LmmGroupEpiParams ep{};
    ep.G = G;
    ep.m = m;
    ep.n_acc = nops;
    ep.unscale = unscale.p;
    ep.rss_null = ws.rss.p;
    ep.snp_ok = ok.p;
    ep.win = win;
    ep.df = static_cast<float>(df);
    ep.t_cand = static_cast<float>(t_cand * (1.0 - 1e-3));
    ep.tt = tt;
    const __half* bh[2] = {Rt.gt_hi.p, Rt.gt2_hi.p};
    const __half* bl[2] = {Rt.gt_lo.p, Rt.gt2_lo.p};
    std::vector<int> bsel(nops, 0), prod(nops, 7);
    bsel[1] = 1;  // gg reads Gt^2
    const bool bf16 = ctx->precision == EQTL_PREC_SPLIT_BF16;
    std::vector<const __half*> opb(2 * static_cast<size_t>(nops));
    if (bf16) {
      // split-BF16: both sides re-split into BF16 hi + lo
      gene_ops_bf16(ctx, oph.data(), oph.data() + nops, nops, G, Rt.k_pad, opb.data());
      rot_bf16(ctx, Rt);
      bh[0] = Rt.bgt_hi.p;
      bh[1] = Rt.bgt2_hi.p;
      bl[0] = Rt.bgt_lo.p;
      bl[1] = Rt.bgt2_lo.p;
    }
    const __half* const* ops = bf16 ? opb.data() : oph.data();
    so.run([&](GeneOut out) {
      ep.out = out;
      launch_tile_n<LmmGroupEpi::kTileN, 4>(ctx, bf16, ep, ops, ops + nops, G, bh, bl, Rt.m, Rt.k_pad, bsel.data(),
                                            prod.data(), tiles, n_tiles, 1, nops);
    });
  } else if (m > 0) {
    const __half* ah[4] = {oph[0], oph[1], oph[2], nops > 3 ? oph[3] : oph[2]};
    const __half* al[4] = {oph[nops + 0], oph[nops + 1], oph[nops + 2], nops > 3 ? oph[nops + 3] : oph[nops + 2]};
    auto fill = [&](auto& ep) {
      ep.G = G;
      ep.m = m;
      ep.unscale = unscale.p;
      ep.ainv = ws.ainv.p;
      ep.rss_null = ws.rss.p;
      ep.snp_ok = ok.p;
      ep.win = win;
      ep.df = static_cast<float>(df);
      ep.t_cand = static_cast<float>(t_cand * (1.0 - 1e-3));
      ep.tt = tt;
    };
    auto run = [&](auto ep, auto pc) {
      constexpr int P = decltype(pc)::value;
      fill(ep);
      ep.snp_alpha = ctx->rot.alpha.p;
      so.run([&](GeneOut out) {
        ep.out = out;
        if constexpr (std::is_same_v<std::decay_t<decltype(ep)>, LmmLrEpiParams<P>>) lmm_launch_lr<P>(ctx, ep, ah, al, G, ctx->rot);
        else lmm_launch<P>(ctx, ep, ah, al, G, simt, tiles, n_tiles, ctx->rot);
      });
    };
    using P1 = std::integral_constant<int, 1>;
    using P2 = std::integral_constant<int, 2>;
    if (lr && p == 1) run(LmmLrEpiParams<1>{}, P1{});
    else if (lr) run(LmmLrEpiParams<2>{}, P2{});
    else if (raw && p == 1) run(LmmRawEpiParams<1>{}, P1{});
    else if (raw) run(LmmRawEpiParams<2>{}, P2{});
    else if (p == 1) run(LmmEpiParams<1>{}, P1{});
    else run(LmmEpiParams<2>{}, P2{});
  }
  scan_timer.reset();
  HostTrace tr("scan_trans_lmm");
  std::vector<int2> todo, deferred, tiny;
  so.collect(genes, todo, deferred, &tiny);
  tr.mark("collect (waits for the scan)");

  // ---- FP64 refinement: rotate raw dosages of the SNPs involved
  StageScope refine_timer(ctx, EQTL_STAGE_REFINE);
  if (delta_out) {
    ws.delta.download(delta_out, G, st);
    EQTL_CUDA(cudaStreamSynchronize(st));
  }
  std::vector<eqtl_pair> refined = lmm_refine_pairs(ctx, p, df, todo);
  tr.mark("refine pairs");
  add_deferred_acat(genes, refined, deferred);
  tr.mark("deferred ACAT");
  const std::vector<double> tiny_p =
      raw ? lmm_tiny_p(ctx, p, df, tiny, ws.lmm_uv.p, static_cast<int64_t>(p + 1) * n) : lmm_tiny_p(ctx, p, df, tiny);
  tr.mark("tiny-|t| pairs");
  add_acat_terms(genes, tiny, tiny_p);
  tr.mark("tiny ACAT terms");
  finish_scan(prm, genes, refined, pairs, cands);
  tr.mark("finish");
  if (tr.on)
    std::fprintf(stderr, "[eqtl trace] scan_trans_lmm counts: candidates %zu deferred %zu tiny %zu\n", todo.size(),
                 deferred.size(), tiny.size());
}

void scan_trans_lmm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X, double* delta_out,
                    eqtl_gene_result* genes, std::vector<eqtl_pair>& pairs, std::vector<eqtl_pair>& cands) {
  scan_trans_lmm_impl(ctx, prm, Y, X, delta_out, genes, pairs, cands, false);
}

void scan_trans_lmm_simt(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                         double* delta_out, eqtl_gene_result* genes, std::vector<eqtl_pair>& pairs,
                         std::vector<eqtl_pair>& cands) {
  scan_trans_lmm_impl(ctx, prm, Y, X, delta_out, genes, pairs, cands, true);
}

// FP64 tests of explicit (column of Y, kept SNP) pairs with the resident
// eigenbasis: the full null fit per column (Q'Y, REML delta, GLS), then the
// refinement arithmetic of the scan; a SNP that fails the subset gate gets
// p = NaN (it is never tested in the reference).
void test_pairs_lmm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X,
                    const std::vector<int2>& todo, eqtl_pair* out, double* delta_out) {
  Geno& g = ctx->geno;
  Workspace& ws = ctx->ws;
  EQTL_CHECK(g.m_all > 0, EQTL_E_STATE, "test_pairs: no genotypes loaded");
  const int n = prm->n, G = prm->n_genes, p = prm->p;
  EQTL_CHECK(n == g.n, EQTL_E_ARG, "test_pairs: n differs from the loaded genotypes");
  EQTL_CHECK(G > 0, EQTL_E_ARG, "test_pairs: no columns");
  for (const int2& q : todo)
    EQTL_CHECK(q.x >= 0 && q.x < G && q.y >= 0 && q.y < g.m, EQTL_E_ARG, "test_pairs: pair index out of range");
  const double df = static_cast<double>(n - p - 1);
  const PhenoDev& ph = resolve_pheno(ctx, prm, Y, X);
  lmm_prep(ctx, ph, prm->y_rotated != 0);
  lmm_gate(ctx);
  std::vector<uint8_t> ok(static_cast<size_t>(g.m));
  ws.ok.download(ok.data(), static_cast<size_t>(g.m), ctx->stream);
  const std::vector<eqtl_pair> refined = lmm_refine_pairs(ctx, p, df, todo);
  for (size_t i = 0; i < todo.size(); ++i) {
    out[i] = refined[i];
    if (!ok[todo[i].y]) out[i].p = std::numeric_limits<double>::quiet_NaN();
  }
  if (delta_out) {
    ws.delta.download(delta_out, G, ctx->stream);
    EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
  }
}


// ================================================================ NB GLM
// The NB-GLM score test (src/model_glm.cpp:13-132) on the LMM scan's
// machinery: the null fit of every gene on the device (glm_null_kernel), the
// gene-side operands w, w o x_k (or w o (X U)_k, U U' = (X'WX)^-1, for
// p > 2) and r against the unrotated centred dosages gc and gc^2, the
// score-test epilogues (LmmEpi<P, true>, GlmGroupEpi), and the FP64
// refinement of every candidate from the exact dosages (glm_refine_kernel).
namespace dev {

constexpr int kGlmThreads = 256;

// Null NB2 fit of one gene per block (nb_irls + prep_glm_nb, src/model_glm.cpp:
// 28-96): from beta = 0, mu = max(y, 0.1), phi = 1, IRLS at fixed phi (at most
// 50 rounds, until max |beta change| < 1e-6; w = m^2 / (m + phi m^2),
// z = log m + (y - m) / m, m = max(mu, 1e-8)), then phi by moments
// (sum ((y - m)^2 - m) / m^2 / max(1, n - p), at least 1e-8), until phi moves
// by less than 1e-6 max(1, phi) (at most 10 rounds). The sums of X'WX and X'Wz
// are warp dot products over the samples (warp w takes items w, w + 8, ...);
// thread 0 factorises and solves. Outputs per gene: W = m / (1 + phi m),
// R = (y - mu) / (1 + phi mu), (X'WX)^-1, phi, sum R, ok (every X'WX
// factorised) and counts (every y a non-negative integer within 1e-8).
// MU and R double as the fit's mu and z.
__global__ void __launch_bounds__(kGlmThreads)
    glm_null_kernel(const double* __restrict__ Y, const double* __restrict__ X, int n, int p, int G, double* MU,
                    double* W, double* R, double* phi_out, double* ainv_out, double* rsum_out, uint8_t* ok_out,
                    uint8_t* counts_out) {
  const int g = blockIdx.x;
  if (g >= G) return;
  __shared__ double A[kMaxPLmm * kMaxPLmm];
  __shared__ double rhs[kMaxPLmm], beta[kMaxPLmm], sol[kMaxPLmm];
  __shared__ double red[kGlmThreads / 32];
  __shared__ double s_phi, s_diff;
  __shared__ int s_fail;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int nw = kGlmThreads / 32;
  const double* y = Y + static_cast<int64_t>(g) * n;
  double* mu = MU + static_cast<int64_t>(g) * n;
  double* w = W + static_cast<int64_t>(g) * n;
  double* z = R + static_cast<int64_t>(g) * n;
  auto block_sum = [&](double v) -> double {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();  // red[] of the previous sum has been read
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0;
    for (int k = 0; k < nw; ++k) t += red[k];
    return t;
  };
  // X'WX (lower triangle, items 0 .. p(p+1)/2 - 1) and, with rhs, X'Wz
  const int n_tri = p * (p + 1) / 2;
  auto weighted_sums = [&](bool with_rhs) {
    const int items = n_tri + (with_rhs ? p : 0);
    for (int item = warp; item < items; item += nw) {
      int a = 0, b = 0;
      const bool is_rhs = item >= n_tri;
      if (is_rhs) {
        a = item - n_tri;
      } else {
        while ((a + 1) * (a + 2) / 2 <= item) ++a;
        b = item - a * (a + 1) / 2;
      }
      const double* xa = X + static_cast<int64_t>(a) * n;
      const double* xb = X + static_cast<int64_t>(b) * n;
      double acc = 0;
      for (int i = lane; i < n; i += 32) acc += xa[i] * w[i] * (is_rhs ? z[i] : xb[i]);
      for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) {
        if (is_rhs) {
          rhs[a] = acc;
        } else {
          A[a * p + b] = acc;
          A[b * p + a] = acc;
        }
      }
    }
  };
  // thread 0: lower Cholesky factor of A in place; false if A is not
  // positive definite
  auto cholesky = [&]() -> bool {
    for (int j = 0; j < p; ++j) {
      double d = A[j * p + j];
      for (int k = 0; k < j; ++k) d -= A[j * p + k] * A[j * p + k];
      if (!(d > 0)) return false;
      d = sqrt(d);
      A[j * p + j] = d;
      for (int i = j + 1; i < p; ++i) {
        double v = A[i * p + j];
        for (int k = 0; k < j; ++k) v -= A[i * p + k] * A[j * p + k];
        A[i * p + j] = v / d;
      }
    }
    return true;
  };
  // thread 0: sol = (L L')^-1 v with the factor in A's lower triangle
  auto solve = [&](const double* v) {
    for (int i = 0; i < p; ++i) {
      double t = v[i];
      for (int k = 0; k < i; ++k) t -= A[i * p + k] * sol[k];
      sol[i] = t / A[i * p + i];
    }
    for (int i = p - 1; i >= 0; --i) {
      double t = sol[i];
      for (int k = i + 1; k < p; ++k) t -= A[k * p + i] * sol[k];
      sol[i] = t / A[i * p + i];
    }
  };

  double bad = 0;
  for (int i = tid; i < n; i += kGlmThreads) {
    const double v = y[i];
    if (isfinite(v) && (v < 0 || fabs(v - floor(v)) > 1e-8)) bad = 1;
    mu[i] = fmax(v, 0.1);
  }
  const double n_bad = block_sum(bad);
  if (tid < p) beta[tid] = 0.0;
  if (tid == 0) {
    s_phi = 1.0;
    s_fail = 0;
  }
  __syncthreads();
  const int df = n - p > 1 ? n - p : 1;
  for (int outer = 0; outer < 10; ++outer) {
    for (int it = 0; it < 50; ++it) {
      const double phi = s_phi;
      for (int i = tid; i < n; i += kGlmThreads) {
        const double m = fmax(mu[i], 1e-8);
        const double var = m + phi * m * m;
        w[i] = (m * m) / fmax(var, 1e-12);
        z[i] = log(m) + (y[i] - m) / m;
      }
      __syncthreads();
      weighted_sums(true);
      __syncthreads();
      if (tid == 0) {
        if (!cholesky()) {
          s_fail = 1;
        } else {
          solve(rhs);
          double diff = 0;
          for (int k = 0; k < p; ++k) {
            diff = fmax(diff, fabs(sol[k] - beta[k]));
            beta[k] = sol[k];
          }
          s_diff = diff;
        }
      }
      __syncthreads();
      if (s_fail) break;
      for (int i = tid; i < n; i += kGlmThreads) {
        double e = 0;
        for (int k = 0; k < p; ++k) e += X[static_cast<int64_t>(k) * n + i] * beta[k];
        mu[i] = exp(e);
      }
      __syncthreads();
      if (s_diff < 1e-6) break;
    }
    if (s_fail) break;
    double part = 0;
    for (int i = tid; i < n; i += kGlmThreads) {
      const double m = fmax(mu[i], 1e-8);
      part += ((y[i] - m) * (y[i] - m) - m) / (m * m);
    }
    const double phi_new = fmax(1e-8, block_sum(part) / df);
    const double phi = s_phi;
    __syncthreads();
    if (tid == 0) s_phi = phi_new;
    __syncthreads();
    if (fabs(phi_new - phi) < 1e-6 * fmax(1.0, phi)) break;
  }
  // the fitted null's weights, residuals and (X'WX)^-1
  const double phi = s_phi;
  double rpart = 0;
  for (int i = tid; i < n; i += kGlmThreads) {
    const double m = fmax(mu[i], 1e-8);
    w[i] = m / (1.0 + phi * m);
    const double r = (y[i] - mu[i]) / (1.0 + phi * mu[i]);
    z[i] = r;
    rpart += r;
  }
  const double rs = block_sum(rpart);
  weighted_sums(false);
  __syncthreads();
  if (tid == 0) {
    const bool fact = cholesky();
    double* ai = ainv_out + static_cast<int64_t>(g) * p * p;
    for (int c = 0; c < p; ++c) {
      for (int k = 0; k < p; ++k) rhs[k] = k == c ? 1.0 : 0.0;
      if (fact) solve(rhs);
      for (int k = 0; k < p; ++k) ai[k * p + c] = fact ? sol[k] : 0.0;
    }
    phi_out[g] = phi;
    rsum_out[g] = rs;
    ok_out[g] = (!s_fail && fact) ? 1 : 0;
    counts_out[g] = n_bad == 0 ? 1 : 0;
  }
}

// Gene-side operands of the GLM scan in the LMM kernels' layout (see
// lmm_gene_ops_kernel / lmm_gene_ops_orth_kernel): order [NUM, a_0 ..
// a_{p-1}, gg] = [r, w x_k, w] for p <= 2, [NUM, gg, a~_0 ..] = [r, w,
// w (X U)_k] for the grouped scan, U the lower Cholesky factor of
// (X'WX)^-1; each scaled to a power of two and split into FP16 hi + lo.
__global__ void glm_gene_ops_kernel(const double* __restrict__ W, const double* __restrict__ Rr,
                                    const double* __restrict__ X, const double* __restrict__ ainv, int n, int p, int G,
                                    int k_pad, float s1, float s2, int grouped, __half* const* hi, __half* const* lo,
                                    float* unscale) {
  const int g = blockIdx.x;
  if (g >= G) return;
  const int nops = p + 2;
  __shared__ double mx[kMaxPLmm + 2][8];
  __shared__ double sc[kMaxPLmm + 2];
  __shared__ double U[kMaxPLmm * kMaxPLmm];
  if (grouped && threadIdx.x == 0) {
    const double* A = ainv + static_cast<int64_t>(g) * p * p;
    for (int j = 0; j < p; ++j) {
      double d = A[j * p + j];
      for (int k = 0; k < j; ++k) d -= U[j * p + k] * U[j * p + k];
      d = d > 0 ? sqrt(d) : 0.0;
      U[j * p + j] = d;
      for (int i = j + 1; i < p; ++i) {
        double v = A[i * p + j];
        for (int k = 0; k < j; ++k) v -= U[i * p + k] * U[j * p + k];
        U[i * p + j] = d > 0 ? v / d : 0.0;
      }
      for (int i = 0; i < j; ++i) U[i * p + j] = 0.0;
    }
  }
  __syncthreads();
  const double* wg = W + static_cast<int64_t>(g) * n;
  const double* rg = Rr + static_cast<int64_t>(g) * n;
  const int gg_op = grouped ? 1 : nops - 1;
  auto value = [&](int op, int i) -> double {
    if (i >= n) return 0.0;
    if (op == 0) return rg[i];
    if (op == gg_op) return wg[i];
    if (!grouped) return wg[i] * X[static_cast<int64_t>(op - 1) * n + i];
    const int k = op - 2;
    double v = 0;
    for (int l = k; l < p; ++l) v += X[static_cast<int64_t>(l) * n + i] * U[l * p + k];
    return wg[i] * v;
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int op = 0; op < nops; ++op) {
    double m = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(value(op, i)));
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) mx[op][warp] = m;
  }
  __syncthreads();
  if (threadIdx.x < nops) {
    double m = 0;
    for (int w = 0; w < (blockDim.x >> 5); ++w) m = fmax(m, mx[threadIdx.x][w]);
    int e = 0;
    if (m > 0) e = 10 - static_cast<int>(floor(log2(m)));
    sc[threadIdx.x] = ldexp(1.0, e);
    const double side = static_cast<int>(threadIdx.x) == gg_op ? s2 : s1;
    unscale[static_cast<int64_t>(g) * nops + threadIdx.x] = static_cast<float>(1.0 / (ldexp(1.0, e) * side));
  }
  __syncthreads();
  for (int op = 0; op < nops; ++op) {
    const double sv = sc[op];
    for (int i = threadIdx.x; i < k_pad; i += blockDim.x) {
      const double v = value(op, i) * sv;
      const __half h = __double2half(v);
      hi[op][static_cast<int64_t>(g) * k_pad + i] = h;
      lo[op][static_cast<int64_t>(g) * k_pad + i] = __double2half(v - static_cast<double>(__half2float(h)));
    }
  }
}

// SNP-side operands of the GLM scan: gc * s1 and gc^2 * s2 from the centred
// dosage operand (gc_hi + gc_lo = (dosage - mean) * inv_gc^-1), FP16 hi + lo.
__global__ void glm_snp_ops_kernel(const __half* __restrict__ gc_hi, const __half* __restrict__ gc_lo, int64_t elems,
                                   double inv_gc, float s1, float s2, __half* gh, __half* gl, __half* g2h,
                                   __half* g2l) {
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < elems;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v = (static_cast<double>(__half2float(gc_hi[e])) + static_cast<double>(__half2float(gc_lo[e]))) *
                     inv_gc;
    const double a = v * s1, b = v * v * s2;
    const __half ah = __double2half(a), bh = __double2half(b);
    gh[e] = ah;
    gl[e] = __double2half(a - static_cast<double>(__half2float(ah)));
    g2h[e] = bh;
    g2l[e] = __double2half(b - static_cast<double>(__half2float(bh)));
  }
}

// FP32 imputation mean of every kept SNP (zero past m), and FP32 sum r
__global__ void glm_means_kernel(const int64_t* __restrict__ kept, int64_t m, const double* __restrict__ mu,
                                 int64_t padded, float* mean_f, const double* __restrict__ rsum, int G, float* rsum_f) {
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < padded;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    mean_f[r] = r < m ? static_cast<float>(mu[kept[r]]) : 0.0f;
    if (r < G) rsum_f[r] = static_cast<float>(rsum[r]);
  }
}

// One warp per (gene, kept SNP) pair: the score test in FP64 from the exact
// mean-imputed dosages g, as test_glm_nb computes it: U = g'r, g'Wg,
// X'Wg, and the dosage variance (mean of squares - squared mean).
__global__ void glm_refine_kernel(GenoRows src, const int32_t* __restrict__ col, int n,
                                  const int64_t* __restrict__ kept, const double* __restrict__ mu_imp,
                                  const double* __restrict__ W, const double* __restrict__ Rr,
                                  const double* __restrict__ X, int p, const double* __restrict__ ainv,
                                  const int2* __restrict__ pairs, int n_pairs, eqtl_pair* out) {
  const int lane = threadIdx.x & 31;
  const int wid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (wid >= n_pairs) return;
  const int g = pairs[wid].x;
  const int64_t r = pairs[wid].y;
  const int64_t s = kept[r];
  const double mus = mu_imp[s];
  const double* wg = W + static_cast<int64_t>(g) * n;
  const double* rg = Rr + static_cast<int64_t>(g) * n;
  double U = 0, gwg = 0, sd = 0, sd2 = 0, xw[kMaxPLmm];
#pragma unroll
  for (int k = 0; k < kMaxPLmm; ++k) xw[k] = 0;
  for (int i = lane; i < n; i += 32) {
    double d = src.dosage(s, col[i]);
    if (isnan(d)) d = mus;
    const double wd = wg[i] * d;
    U += d * rg[i];
    gwg += wd * d;
    sd += d;
    sd2 += d * d;
#pragma unroll
    for (int k = 0; k < kMaxPLmm; ++k)
      if (k < p) xw[k] += X[static_cast<int64_t>(k) * n + i] * wd;
  }
  for (int o = 16; o; o >>= 1) {
    U += __shfl_xor_sync(0xffffffffu, U, o);
    gwg += __shfl_xor_sync(0xffffffffu, gwg, o);
    sd += __shfl_xor_sync(0xffffffffu, sd, o);
    sd2 += __shfl_xor_sync(0xffffffffu, sd2, o);
#pragma unroll
    for (int k = 0; k < kMaxPLmm; ++k)
      if (k < p) xw[k] += __shfl_xor_sync(0xffffffffu, xw[k], o);
  }
  if (lane) return;
  const double* A = ainv + static_cast<int64_t>(g) * p * p;
  double xAx = 0;
  for (int a = 0; a < p; ++a) {
    double t = 0;
    for (int b = 0; b < p; ++b) t += A[a * p + b] * xw[b];
    xAx += xw[a] * t;
  }
  const double mean = sd / n;
  eqtl_pair q;
  q.snp = r;
  q.gene = g;
  q.reserved = 0;
  glm_stats_fp64(U, gwg, xAx, sd2 / n - mean * mean, q);
  out[wid] = q;
}

}  // namespace dev

static std::vector<eqtl_pair> glm_refine_pairs(eqtl_ctx* ctx, int p, const std::vector<int2>& todo) {
  Geno& g = ctx->geno;
  Workspace& ws = ctx->ws;
  cudaStream_t st = ctx->stream;
  std::vector<eqtl_pair> refined(todo.size());
  if (todo.empty()) return refined;
  ws.ref_pairs.upload(todo.data(), todo.size(), st);
  ws.refined.alloc(todo.size());
  const int n_pairs = static_cast<int>(todo.size());
  ++ctx->launches;
  glm_refine_kernel<<<static_cast<unsigned>((n_pairs + 7) / 8), 256, 0, st>>>(
      g.rows(), g.col.p, g.n, g.kept.p, g.mu.p, ws.glm_w.p, ws.glm_r.p, ctx->pheno.X.p, p, ws.ainv.p,
      ws.ref_pairs.p, n_pairs, ws.refined.p);
  EQTL_CUDA(cudaGetLastError());
  ws.refined.download(refined.data(), refined.size(), st);
  EQTL_CUDA(cudaStreamSynchronize(st));
  // a gene whose null fit failed tests nothing (p = NaN, test_glm_nb)
  std::vector<uint8_t> ok(ctx->pheno.G);
  ws.glm_ok.download(ok.data(), ok.size(), st);
  EQTL_CUDA(cudaStreamSynchronize(st));
  for (eqtl_pair& q : refined)
    if (!ok[q.gene]) q.p = std::numeric_limits<double>::quiet_NaN();
  return refined;
}

void scan_glm(eqtl_ctx* ctx, const eqtl_scan_params* prm, const double* Y, const double* X, double* phi_out,
              uint8_t* converged_out, eqtl_gene_result* genes, std::vector<eqtl_pair>& pairs,
              std::vector<eqtl_pair>& cands) {
  Geno& g = ctx->geno;
  Workspace& ws = ctx->ws;
  const int n = prm->n, G = prm->n_genes, p = prm->p;
  EQTL_CHECK(g.m_all > 0, EQTL_E_STATE, "scan_glm: no genotypes loaded");
  EQTL_CHECK(!g.subset, EQTL_E_UNSUPPORTED, "scan_glm: the NB-GLM scan takes every analysis sample");
  EQTL_CHECK(n == g.n, EQTL_E_ARG, "scan_glm: n differs from the loaded genotypes");
  EQTL_CHECK(G > 0, EQTL_E_ARG, "scan_glm: no genes");
  EQTL_CHECK(g.m < (int64_t(1) << 30), EQTL_E_UNSUPPORTED, "scan_glm: more than 2^30 kept SNPs");
  EQTL_CHECK(p >= 1 && p <= kMaxPLmm, EQTL_E_UNSUPPORTED,
             "the GLM scan handles 1 to 32 covariate columns (intercept included)");
  EQTL_CHECK(ctx->precision == EQTL_PREC_SPLIT_F16, EQTL_E_UNSUPPORTED, "the GLM scan runs split-FP16");
  const bool grouped = p > 2;
  cudaStream_t st = ctx->stream;
  const PhenoDev& ph = resolve_pheno(ctx, prm, Y, X);
  std::unique_ptr<StageScope> prep_timer(new StageScope(ctx, EQTL_STAGE_PREP));
  // ---- null fits
  const size_t gn = static_cast<size_t>(G) * n;
  ws.glm_mu.alloc(gn);
  ws.glm_w.alloc(gn);
  ws.glm_r.alloc(gn);
  ws.glm_phi.alloc(G);
  ws.glm_rsum.alloc(G);
  ws.glm_ok.alloc(G);
  ws.glm_counts.alloc(G);
  ws.ainv.alloc(static_cast<size_t>(G) * p * p);
  ++ctx->launches;
  glm_null_kernel<<<G, kGlmThreads, 0, st>>>(ph.Y.p, ph.X.p, n, p, G, ws.glm_mu.p, ws.glm_w.p, ws.glm_r.p,
                                             ws.glm_phi.p, ws.ainv.p, ws.glm_rsum.p, ws.glm_ok.p, ws.glm_counts.p);
  EQTL_CUDA(cudaGetLastError());
  {
    std::vector<uint8_t> counts(G), ok(G);
    ws.glm_counts.download(counts.data(), G, st);
    ws.glm_ok.download(ok.data(), G, st);
    if (phi_out) ws.glm_phi.download(phi_out, G, st);
    EQTL_CUDA(cudaStreamSynchronize(st));
    for (int j = 0; j < G; ++j)
      EQTL_CHECK(counts[j], EQTL_E_ARG, "glm (NB) requires non-negative integer counts (column " + std::to_string(j) + ")");
    if (converged_out) std::copy(ok.begin(), ok.end(), converged_out);
  }
  // ---- SNP-side operands (unrotated), means and gene-side operands
  Rotated& S = ctx->glm_ops;
  const int k_pad = g.k_pad;
  const int64_t m = g.m;
  float s1, s2;
  output_scales(n, s1, s2);
  if (!(S.m == m && S.k_pad == k_pad && S.gt_hi.p)) {
    const size_t elems = static_cast<size_t>(m) * k_pad;
    S.gt_hi.alloc(elems);
    S.gt_lo.alloc(elems);
    S.gt2_hi.alloc(elems);
    S.gt2_lo.alloc(elems);
    if (elems) {
      ++ctx->launches;
      glm_snp_ops_kernel<<<static_cast<unsigned>(std::min<int64_t>((elems + 255) / 256, 148 * 64)), 256, 0, st>>>(
          g.gc_hi.p, g.gc_lo.p, static_cast<int64_t>(elems), 1.0 / kGcScale, s1, s2, S.gt_hi.p, S.gt_lo.p,
          S.gt2_hi.p, S.gt2_lo.p);
      EQTL_CUDA(cudaGetLastError());
    }
    S.m = m;
    S.k_pad = k_pad;
  }
  const int64_t padded = ((m + 255) / 256 + 1) * 256;
  ws.snp_mean.alloc(static_cast<size_t>(std::max<int64_t>(padded, G)));
  ws.glm_rsum_f.alloc(G);
  ++ctx->launches;
  glm_means_kernel<<<static_cast<unsigned>(std::min<int64_t>((std::max<int64_t>(padded, G) + 255) / 256, 4096)), 256,
                     0, st>>>(g.kept.p, m, g.mu.p, std::max<int64_t>(padded, G), ws.snp_mean.p, ws.glm_rsum.p, G,
                              ws.glm_rsum_f.p);
  EQTL_CUDA(cudaGetLastError());
  const int nops = p + 2;
  std::vector<__half*> oph(2 * nops);
  for (int k = 0; k < nops; ++k) {
    ws.ops_hi[k].alloc(static_cast<size_t>(G) * k_pad);
    ws.ops_lo[k].alloc(static_cast<size_t>(G) * k_pad);
    oph[k] = ws.ops_hi[k].p;
    oph[nops + k] = ws.ops_lo[k].p;
  }
  ws.ops_ptr.upload(oph.data(), oph.size(), st);
  ws.unscale.alloc(static_cast<size_t>(G) * nops);
  ++ctx->launches;
  glm_gene_ops_kernel<<<G, 256, 0, st>>>(ws.glm_w.p, ws.glm_r.p, ph.X.p, ws.ainv.p, n, p, G, k_pad, s1, s2,
                                         grouped ? 1 : 0, ws.ops_ptr.p, ws.ops_ptr.p + nops, ws.unscale.p);
  EQTL_CUDA(cudaGetLastError());
  lmm_gate(ctx);
  const Windows win =
      upload_windows(ctx, prm, m, prm->exclude_cis == 2 ? kWinInclude : prm->exclude_cis ? kWinExclude : kWinNone);
  double z_cand = z_critical(prm->pthr);
  if (prm->perm_thr > 0) z_cand = std::min(z_cand, z_critical(prm->perm_thr));
  const TTable tt = device_ttable(ctx, 0.0, true);
  prep_timer.reset();
  // ---- scan
  ScanOutputs so(ctx, G, m, expected_candidates(prm, m));
  const int2* tiles = nullptr;
  int n_tiles = 0;
  cis_tile_list(ctx, prm, m, grouped ? GlmGroupEpi::kTileN : 128, tiles, n_tiles);
  std::unique_ptr<StageScope> scan_timer(new StageScope(ctx, EQTL_STAGE_SCAN));
  if (m > 0 && grouped) {
    GlmGroupEpiParams ep{};
    ep.G = G;
    ep.m = m;
    ep.n_acc = nops;
    ep.unscale = ws.unscale.p;
    ep.snp_ok = ws.ok.p;
    ep.win = win;
    ep.t_cand = static_cast<float>(z_cand * (1.0 - 1e-3));
    ep.tt = tt;
    ep.snp_mean = ws.snp_mean.p;
    ep.rsum = ws.glm_rsum_f.p;
    ep.gene_ok = ws.glm_ok.p;
    const __half* bh[2] = {S.gt_hi.p, S.gt2_hi.p};
    const __half* bl[2] = {S.gt_lo.p, S.gt2_lo.p};
    std::vector<int> bsel(nops, 0), prod(nops, 7);
    bsel[1] = 1;  // gg reads gc^2
    so.run([&](GeneOut out) {
      ep.out = out;
      launch_tile_n<GlmGroupEpi::kTileN, 4>(ctx, false, ep, oph.data(), oph.data() + nops, G, bh, bl, S.m, S.k_pad,
                                            bsel.data(), prod.data(), tiles, n_tiles, 1, nops);
    });
  } else if (m > 0) {
    const __half* ah[4] = {oph[0], oph[1], oph[2], nops > 3 ? oph[3] : oph[2]};
    const __half* al[4] = {oph[nops + 0], oph[nops + 1], oph[nops + 2], nops > 3 ? oph[nops + 3] : oph[nops + 2]};
    auto fill = [&](auto& ep) {
      ep.G = G;
      ep.m = m;
      ep.unscale = ws.unscale.p;
      ep.ainv = ws.ainv.p;
      ep.snp_ok = ws.ok.p;
      ep.win = win;
      ep.t_cand = static_cast<float>(z_cand * (1.0 - 1e-3));
      ep.tt = tt;
      ep.snp_mean = ws.snp_mean.p;
      ep.rsum = ws.glm_rsum_f.p;
      ep.gene_ok = ws.glm_ok.p;
    };
    if (p == 1) {
      GlmEpiParams<1> ep{};
      fill(ep);
      so.run([&](GeneOut out) {
        ep.out = out;
        lmm_launch<1>(ctx, ep, ah, al, G, false, tiles, n_tiles, S);
      });
    } else {
      GlmEpiParams<2> ep{};
      fill(ep);
      so.run([&](GeneOut out) {
        ep.out = out;
        lmm_launch<2>(ctx, ep, ah, al, G, false, tiles, n_tiles, S);
      });
    }
  }
  scan_timer.reset();
  std::vector<int2> todo, deferred;
  so.collect(genes, todo, deferred);
  // ---- FP64 refinement of the candidates, deferred and tiny-|z| pairs
  StageScope refine_timer(ctx, EQTL_STAGE_REFINE);
  const std::vector<eqtl_pair> refined = glm_refine_pairs(ctx, p, todo);
  add_deferred_acat(genes, refined, deferred);
  finish_scan(prm, genes, refined, pairs, cands);
}

}  // namespace eqtl
