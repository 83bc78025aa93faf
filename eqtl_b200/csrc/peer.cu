// PEER variational factor analysis of the fission subcommand on the device
// (peer_factors, src/fission.cpp:104-275), in FP64.
//
// Model Y ~ X W' + noise with Y [n, G] (genes centred, NaN -> 0), X [n, K]
// factors, W [G, K] loadings, ARD precisions Alpha [K] (Gamma(0.001, 0.1))
// and per-gene noise precisions Eps [G] (Gamma(0.1, 10)). One iteration,
// in the reference's order:
//   W      XtY = X'Y (DGEMM); per gene d (peer_w_kernel, one block):
//          M_d = diag(Alpha) + Eps_d XE2S, cov_d = M_d^-1 (Cholesky),
//          w_d = Eps_d cov_d XtY[:, d], E2_d = cov_d + w_d w_d';
//          W_E2S = sum_d E2_d, W_Xprec = sum_d Eps_d E2_d (peer_reduce_kernel,
//          a fixed summation order)
//   Alpha  (0.001 + G/2) / (0.1 + W_E2S_kk / 2)
//   X      Xcov = (W_Xprec + I)^-1; X = Y (Eps o W) Xcov (two DGEMMs);
//          XE2S = n Xcov + X'X
//   Eps    (0.1 + n/2) / max(10 + (b1 - 2 b2 + b3) / 2, 1e-10) with
//          b1_d = sum_i (y_id^2 + 0.01), b2_d = XtY[:, d] . w_d and
//          b3_d = sum(XE2S o E2_d) (the reference's stale copies of Alpha
//          and XE2S at the W step make its covariance equal to cov_d)
//   stop   when the mean squared residual of Y - X W' moves by less than
//          1e-8 or the caller's tolerance.
// The starting X and W are the caller's (the reference draws them from
// std::normal_distribution on std::mt19937(seed + 1)).
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "internal.hpp"

namespace eqtl {
namespace {

constexpr int kPeerThreads = 128;
constexpr int kPeerMaxK = 96;
constexpr double kAlphaA = 0.001, kAlphaB = 0.1, kEpsA = 0.1, kEpsB = 10.0;

__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0;
  for (int k = 0; k < static_cast<int>(blockDim.x >> 5); ++k) t += red[k];
  return t;
}

// Lower Cholesky factor of the K x K matrix A in place (all threads of the
// block), then Inv = A^-1 column by column (thread c solves column c).
// Returns false (to every thread) if A is not positive definite.
__device__ bool block_chol_inverse(double* A, double* Inv, int K, int* fail) {
  if (threadIdx.x == 0) *fail = 0;
  __syncthreads();
  for (int j = 0; j < K; ++j) {
    if (threadIdx.x == 0) {
      const double d = A[j * K + j];
      if (!(d > 0)) *fail = 1;
      A[j * K + j] = d > 0 ? sqrt(d) : 1.0;
    }
    __syncthreads();
    const double djj = A[j * K + j];
    for (int i = j + 1 + threadIdx.x; i < K; i += blockDim.x) A[i * K + j] /= djj;
    __syncthreads();
    // trailing update of the lower triangle: A[i][c] -= A[i][j] A[c][j], j < c <= i
    const int rem = K - j - 1;
    for (int e = threadIdx.x; e < rem * rem; e += blockDim.x) {
      const int i = j + 1 + e / rem, c = j + 1 + e % rem;
      if (c <= i) A[i * K + c] -= A[i * K + j] * A[c * K + j];
    }
    __syncthreads();
  }
  for (int c = threadIdx.x; c < K; c += blockDim.x) {
    // forward L y = e_c into column c of Inv, then back L' x = y in place
    for (int i = 0; i < K; ++i) {
      double t = i == c ? 1.0 : 0.0;
      for (int l = 0; l < i; ++l) t -= A[i * K + l] * Inv[l * K + c];
      Inv[i * K + c] = t / A[i * K + i];
    }
    for (int i = K - 1; i >= 0; --i) {
      double t = Inv[i * K + c];
      for (int l = i + 1; l < K; ++l) t -= A[l * K + i] * Inv[l * K + c];
      Inv[i * K + c] = t / A[i * K + i];
    }
  }
  __syncthreads();
  return *fail == 0;
}

// genes centred over their non-NaN values (NaN -> 0); b1 = sum_i (y^2 + 0.01)
__global__ void peer_center_kernel(const double* __restrict__ Y_in, int n, double* Y, double* b1) {
  __shared__ double red[kPeerThreads / 32];
  const int g = blockIdx.x;
  const double* y = Y_in + static_cast<int64_t>(g) * n;
  double s = 0, c = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    if (!isnan(y[i])) {
      s += y[i];
      c += 1;
    }
  s = block_sum(s, red);
  c = block_sum(c, red);
  const double mean = c > 0 ? s / c : 0.0;
  double e = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = isnan(y[i]) ? 0.0 : y[i] - mean;
    Y[static_cast<int64_t>(g) * n + i] = v;
    e += v * v + 0.01;
  }
  e = block_sum(e, red);
  if (threadIdx.x == 0) b1[g] = e;
}

// W step for one gene per block: w_d, E2_d = cov_d + w_d w_d', b2_d.
__global__ void __launch_bounds__(kPeerThreads)
    peer_w_kernel(const double* __restrict__ XtY, const double* __restrict__ XE2S, const double* __restrict__ Alpha,
                  const double* __restrict__ Eps, int K, int G, double* W, double* E2, double* b2, int* fail_out) {
  extern __shared__ double peer_smem[];
  double* M = peer_smem;          // K*K
  double* Inv = M + K * K;        // K*K
  double* rhs = Inv + K * K;      // K
  double* w = rhs + K;            // K
  __shared__ int fail;
  const int d = blockIdx.x;
  const double eps = Eps[d];
  for (int e = threadIdx.x; e < K * K; e += blockDim.x) {
    const int r = e / K, c = e % K;
    M[e] = eps * XE2S[e] + (r == c ? Alpha[r] : 0.0);
  }
  for (int k = threadIdx.x; k < K; k += blockDim.x) rhs[k] = XtY[static_cast<int64_t>(d) * K + k];
  __syncthreads();
  if (!block_chol_inverse(M, Inv, K, &fail) && threadIdx.x == 0) atomicExch(fail_out, 1);
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    double t = 0;
    for (int l = 0; l < K; ++l) t += Inv[k * K + l] * rhs[l];
    w[k] = t * eps;
  }
  __syncthreads();
  double* e2 = E2 + static_cast<int64_t>(d) * K * K;
  for (int e = threadIdx.x; e < K * K; e += blockDim.x) e2[e] = Inv[e] + w[e / K] * w[e % K];
  for (int k = threadIdx.x; k < K; k += blockDim.x) W[d + static_cast<int64_t>(k) * G] = w[k];
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < K; ++k) t += rhs[k] * w[k];
    b2[d] = t;
  }
}

// W_E2S[e] = sum_d E2_d[e], W_Xprec[e] = sum_d Eps_d E2_d[e], one block per e
__global__ void peer_reduce_kernel(const double* __restrict__ E2, const double* __restrict__ Eps, int KK, int G,
                                   double* W_E2S, double* W_Xprec) {
  __shared__ double red[kPeerThreads / 32];
  const int e = blockIdx.x;
  double s = 0, t = 0;
  for (int d = threadIdx.x; d < G; d += blockDim.x) {
    const double v = E2[static_cast<int64_t>(d) * KK + e];
    s += v;
    t += Eps[d] * v;
  }
  s = block_sum(s, red);
  t = block_sum(t, red);
  if (threadIdx.x == 0) {
    W_E2S[e] = s;
    W_Xprec[e] = t;
  }
}

// Alpha from W_E2S, Xcov = (W_Xprec + I)^-1 (one block)
__global__ void peer_alpha_xcov_kernel(const double* __restrict__ W_E2S, const double* __restrict__ W_Xprec, int K,
                                       int G, double* Alpha, double* Xcov, int* fail_out) {
  extern __shared__ double peer_smem[];
  double* M = peer_smem;
  __shared__ int fail;
  for (int k = threadIdx.x; k < K; k += blockDim.x) Alpha[k] = (kAlphaA + 0.5 * G) / (kAlphaB + 0.5 * W_E2S[k * K + k]);
  for (int e = threadIdx.x; e < K * K; e += blockDim.x) M[e] = W_Xprec[e] + (e / K == e % K ? 1.0 : 0.0);
  __syncthreads();
  if (!block_chol_inverse(M, Xcov, K, &fail) && threadIdx.x == 0) atomicExch(fail_out, 1);
}

// epsW[d + k G] = Eps_d W[d + k G]
__global__ void peer_epsw_kernel(const double* __restrict__ W, const double* __restrict__ Eps, int G, int K,
                                 double* epsW) {
  const int64_t total = static_cast<int64_t>(G) * K;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x)
    epsW[e] = Eps[e % G] * W[e];
}

// XE2S += n Xcov (after XE2S = X'X)
__global__ void peer_xe2s_kernel(const double* __restrict__ Xcov, int KK, double n, double* XE2S) {
  for (int e = threadIdx.x; e < KK; e += blockDim.x) XE2S[e] += n * Xcov[e];
}

// b3_d = sum(XE2S o E2_d) and the Eps update, one warp per gene
__global__ void peer_eps_kernel(const double* __restrict__ XE2S, const double* __restrict__ E2,
                                const double* __restrict__ b1, const double* __restrict__ b2, int KK, int G, int n,
                                double* Eps) {
  const int lane = threadIdx.x & 31;
  const int d = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (d >= G) return;
  const double* e2 = E2 + static_cast<int64_t>(d) * KK;
  double t = 0;
  for (int e = lane; e < KK; e += 32) t += XE2S[e] * e2[e];
  for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (lane == 0) {
    const double b = fmax(kEpsB + 0.5 * (b1[d] - 2.0 * b2[d] + t), 1e-10);
    Eps[d] = (kEpsA + 0.5 * n) / b;
  }
}

// sum of squares of R in fixed-order per-block partial sums
__global__ void peer_sumsq_kernel(const double* __restrict__ R, int64_t total, double* part) {
  __shared__ double red[kPeerThreads / 32];
  double s = 0;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x)
    s += R[e] * R[e];
  s = block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void fill_kernel(double* p, int64_t count, double v) {
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < count;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x)
    p[e] = v;
}

cublasHandle_t peer_blas(eqtl_ctx* ctx) {
  if (!ctx->cublas) {
    cublasHandle_t h;
    EQTL_CHECK(cublasCreate(&h) == CUBLAS_STATUS_SUCCESS, EQTL_E_CUDA, "cublasCreate failed");
    cublasSetStream(h, ctx->stream);
    ctx->cublas = h;
  }
  return static_cast<cublasHandle_t>(ctx->cublas);
}

#define PEER_BLAS(call) EQTL_CHECK((call) == CUBLAS_STATUS_SUCCESS, EQTL_E_CUDA, #call " failed")

}  // namespace

int peer_factors(eqtl_ctx* ctx, const double* Y_host, int n, int G, int K, int max_iter, double tol,
                 const double* X0, const double* W0, double* X_out) {
  EQTL_CHECK(n > 0 && G > 0 && K >= 1, EQTL_E_ARG, "peer: bad sizes");
  EQTL_CHECK(K < n && K < G, EQTL_E_ARG, "peer: k must be < min(n_samples, n_genes)");
  EQTL_CHECK(K <= kPeerMaxK, EQTL_E_UNSUPPORTED, "peer: at most 96 factors on the device");
  EQTL_CHECK(max_iter >= 1, EQTL_E_ARG, "peer: max_iter must be >= 1");
  cudaStream_t st = ctx->stream;
  cublasHandle_t h = peer_blas(ctx);
  const int KK = K * K;
  const int64_t nG = static_cast<int64_t>(n) * G;
  DevBuf<double> Yraw, Y, R, XtY, E2, W, epsW, X, T1, XE2S, W_E2S, W_Xprec, Xcov, Alpha, Eps, b1, b2, part;
  DevBuf<int> fail;
  Yraw.upload(Y_host, static_cast<size_t>(nG), st);
  Y.alloc(static_cast<size_t>(nG));
  R.alloc(static_cast<size_t>(nG));
  XtY.alloc(static_cast<size_t>(K) * G);
  E2.alloc(static_cast<size_t>(G) * KK);
  W.upload(W0, static_cast<size_t>(G) * K, st);
  epsW.alloc(static_cast<size_t>(G) * K);
  X.upload(X0, static_cast<size_t>(n) * K, st);
  T1.alloc(static_cast<size_t>(n) * K);
  XE2S.alloc(KK);
  W_E2S.alloc(KK);
  W_Xprec.alloc(KK);
  Xcov.alloc(KK);
  Alpha.alloc(K);
  Eps.alloc(G);
  b1.alloc(G);
  b2.alloc(G);
  const int sum_blocks = 296;
  part.alloc(sum_blocks);
  fail.alloc(1);
  fail.zero(st);
  const double one = 1.0, zero = 0.0, mone = -1.0;
  ctx->launches += 3;
  peer_center_kernel<<<G, kPeerThreads, 0, st>>>(Yraw.p, n, Y.p, b1.p);
  fill_kernel<<<(G + 255) / 256, 256, 0, st>>>(Eps.p, G, kEpsA / kEpsB);
  fill_kernel<<<1, 128, 0, st>>>(Alpha.p, K, (kAlphaA + 0.5 * G) / kAlphaB);  // from W_E2S = 0
  EQTL_CUDA(cudaGetLastError());
  // XE2S = n I + X'X
  {
    std::vector<double> I(static_cast<size_t>(KK), 0.0);
    for (int k = 0; k < K; ++k) I[static_cast<size_t>(k) * K + k] = 1.0;
    Xcov.upload(I.data(), I.size(), st);  // Xcov = I, so XE2S += n Xcov gives n I
  }
  PEER_BLAS(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, K, K, n, &one, X.p, n, X.p, n, &zero, XE2S.p, K));
  ++ctx->launches;
  peer_xe2s_kernel<<<1, 128, 0, st>>>(Xcov.p, KK, static_cast<double>(n), XE2S.p);
  const int w_smem = static_cast<int>((2 * KK + 2 * K) * sizeof(double));
  const int a_smem = static_cast<int>(KK * sizeof(double));
  EQTL_CUDA(cudaFuncSetAttribute(peer_w_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, w_smem));
  EQTL_CUDA(cudaFuncSetAttribute(peer_alpha_xcov_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, a_smem));
  double last = std::numeric_limits<double>::max();
  int it = 0;
  std::vector<double> parts(sum_blocks);
  for (it = 1; it <= max_iter; ++it) {
    // W
    PEER_BLAS(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, K, G, n, &one, X.p, n, Y.p, n, &zero, XtY.p, K));
    ctx->launches += 2;
    peer_w_kernel<<<G, kPeerThreads, w_smem, st>>>(XtY.p, XE2S.p, Alpha.p, Eps.p, K, G, W.p, E2.p, b2.p, fail.p);
    peer_reduce_kernel<<<KK, kPeerThreads, 0, st>>>(E2.p, Eps.p, KK, G, W_E2S.p, W_Xprec.p);
    // Alpha, X
    ctx->launches += 2;
    peer_alpha_xcov_kernel<<<1, kPeerThreads, a_smem, st>>>(W_E2S.p, W_Xprec.p, K, G, Alpha.p, Xcov.p, fail.p);
    peer_epsw_kernel<<<static_cast<unsigned>(std::min<int64_t>((static_cast<int64_t>(G) * K + 255) / 256, 1184)),
                       256, 0, st>>>(W.p, Eps.p, G, K, epsW.p);
    PEER_BLAS(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, K, G, &one, Y.p, n, epsW.p, G, &zero, T1.p, n));
    PEER_BLAS(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, K, K, &one, T1.p, n, Xcov.p, K, &zero, X.p, n));
    PEER_BLAS(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, K, K, n, &one, X.p, n, X.p, n, &zero, XE2S.p, K));
    ctx->launches += 2;
    peer_xe2s_kernel<<<1, 128, 0, st>>>(Xcov.p, KK, static_cast<double>(n), XE2S.p);
    // Eps
    peer_eps_kernel<<<(G + 7) / 8, 256, 0, st>>>(XE2S.p, E2.p, b1.p, b2.p, KK, G, n, Eps.p);
    EQTL_CUDA(cudaGetLastError());
    // mean squared residual of Y - X W'
    EQTL_CUDA(cudaMemcpyAsync(R.p, Y.p, sizeof(double) * nG, cudaMemcpyDeviceToDevice, st));
    PEER_BLAS(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, n, G, K, &mone, X.p, n, W.p, G, &one, R.p, n));
    ++ctx->launches;
    peer_sumsq_kernel<<<sum_blocks, kPeerThreads, 0, st>>>(R.p, nG, part.p);
    EQTL_CUDA(cudaGetLastError());
    part.download(parts.data(), sum_blocks, st);
    EQTL_CUDA(cudaStreamSynchronize(st));
    double ss = 0;
    for (double v : parts) ss += v;
    const double res = ss / static_cast<double>(nG);
    if (std::fabs(last - res) < 1e-8 || std::fabs(last - res) < tol) break;
    last = res;
  }
  if (it > max_iter) it = max_iter;
  int failed = 0;
  fail.download(&failed, 1, st);
  X.download(X_out, static_cast<size_t>(n) * K, st);
  EQTL_CUDA(cudaStreamSynchronize(st));
  EQTL_CHECK(!failed, EQTL_E_INTERNAL, "peer: a precision matrix was not positive definite");
  return it;
}

}  // namespace eqtl
