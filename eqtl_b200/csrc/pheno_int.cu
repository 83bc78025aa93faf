// --pheno-norm int on the device: the rank-based inverse normal transform of
// every phenotype column (inverse_normal_transform, src/util.cpp:177-206,
// with qnorm_inv :132-171).
//
// Per column: the finite values are ranked (ties share the average of their
// 1-based positions), and value i becomes qnorm_inv((rank_i - 1/2) / nf),
// nf = number of finite values; values that are not finite stay as they are,
// and a column with at most one finite value is left unchanged. All columns
// are sorted at once by a segmented radix sort (keys: the values, with every
// value that is not finite mapped to +inf so that the finite ones lead each
// segment; items: the sample index); one thread per sorted entry then finds
// its tie group by binary search in the sorted segment and writes the
// transformed value back at the sample's position.
#include <cub/device/device_segmented_radix_sort.cuh>

#include "internal.hpp"
#include "stats64.hpp"

namespace eqtl {
namespace {

__global__ void int_keys_kernel(const double* __restrict__ Y, int64_t total, int n, double* keys, int* idx) {
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v = Y[e];
    keys[e] = isfinite(v) ? v : __longlong_as_double(0x7ff0000000000000LL);  // +inf
    idx[e] = static_cast<int>(e % n);
  }
}

__global__ void int_offsets_kernel(int G, int n, int* off) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g <= G; g += gridDim.x * blockDim.x) off[g] = g * n;
}

// first position in sorted[0, len) whose value is not below v / above v
__device__ __forceinline__ int lower_pos(const double* s, int len, double v) {
  int lo = 0, hi = len;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (s[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}
__device__ __forceinline__ int upper_pos(const double* s, int len, double v) {
  int lo = 0, hi = len;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (s[mid] <= v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void int_apply_kernel(const double* __restrict__ sorted, const int* __restrict__ idx, int n,
                                 int64_t total, double* Y) {
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t g = e / n;
    const int k = static_cast<int>(e - g * n);
    const double* seg = sorted + g * n;
    const double v = seg[k];
    if (v == inf) continue;  // not finite: unchanged
    const int nf = lower_pos(seg, n, inf);
    if (nf <= 1) continue;
    const int first = lower_pos(seg, nf, v), last = upper_pos(seg, nf, v);
    const double rank = 0.5 * static_cast<double>(first + 1 + last);
    Y[g * n + idx[e]] = normal_quantile((rank - 0.5) / static_cast<double>(nf));
  }
}

}  // namespace

void pheno_int(eqtl_ctx* ctx, double* Y_host, int n, int G) {
  EQTL_CHECK(n > 0 && G > 0, EQTL_E_ARG, "pheno_int: bad sizes");
  EQTL_CHECK(static_cast<int64_t>(n) * G < (int64_t(1) << 31), EQTL_E_UNSUPPORTED,
             "pheno_int: more than 2^31 values in one call");
  cudaStream_t st = ctx->stream;
  const int64_t total = static_cast<int64_t>(n) * G;
  DevBuf<double> y, keys, keys_out;
  DevBuf<int> idx, idx_out, off;
  y.upload(Y_host, static_cast<size_t>(total), st);
  keys.alloc(static_cast<size_t>(total));
  keys_out.alloc(static_cast<size_t>(total));
  idx.alloc(static_cast<size_t>(total));
  idx_out.alloc(static_cast<size_t>(total));
  off.alloc(static_cast<size_t>(G) + 1);
  const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((total + 255) / 256, 148 * 32));
  ctx->launches += 2;
  int_keys_kernel<<<blocks, 256, 0, st>>>(y.p, total, n, keys.p, idx.p);
  int_offsets_kernel<<<static_cast<unsigned>((G + 256) / 256), 256, 0, st>>>(G, n, off.p);
  EQTL_CUDA(cudaGetLastError());
  size_t temp_bytes = 0;
  EQTL_CUDA(cub::DeviceSegmentedRadixSort::SortPairs(nullptr, temp_bytes, keys.p, keys_out.p, idx.p, idx_out.p,
                                                     static_cast<int>(total), G, off.p, off.p + 1, 0, 64, st));
  DevBuf<uint8_t> temp;
  temp.alloc(temp_bytes);
  EQTL_CUDA(cub::DeviceSegmentedRadixSort::SortPairs(temp.p, temp_bytes, keys.p, keys_out.p, idx.p, idx_out.p,
                                                     static_cast<int>(total), G, off.p, off.p + 1, 0, 64, st));
  ++ctx->launches;
  int_apply_kernel<<<blocks, 256, 0, st>>>(keys_out.p, idx_out.p, n, total, y.p);
  EQTL_CUDA(cudaGetLastError());
  y.download(Y_host, static_cast<size_t>(total), st);
  EQTL_CUDA(cudaStreamSynchronize(st));
}

}  // namespace eqtl
