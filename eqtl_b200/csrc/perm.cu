// Permuted null phenotypes drawn on the device: the throughput mode of the
// gene-level permutations.
//
// The reference draws permutation b of a gene with std::mt19937 seeded by
// (seed or 1) + 9973 b + fnv1a(gene) and std::shuffle
// (include/eqtl/scan_cis.hpp:102-147, src/scan_perm.cpp:80-132); the host
// program reproduces those draws exactly (host/perm.cpp). This mode draws
// each permutation on the device instead, from a counter-based generator,
// so that no permuted column is built on the host or crosses PCIe: column
// c = g * B + b gets the keys
//     key_i = (philox(seed, gene_key[g]; b, i) << 32) | i,   i < n
// and the permutation is the order of the keys (a segmented radix sort of
// all columns at once). The 32 random bits make every order equally likely
// up to ties, which the index bits break (a tie among n keys has
// probability about n^2 / 2^33). The permuted column is then
//     LM   base_g[perm(i)]
//     LMM  xb0_g[i] + base_g[perm(i)] / sqrt(max(dinv_g[i], 1e-12))
// as the host builds it from the same base vectors.
//
// Philox4x32-10 follows the published algorithm (Salmon, Moraes, Dror and
// Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011): ten rounds
// of two 32x32 -> 64-bit multiplies with the constants 0xD2511F53 and
// 0xCD9E8D57, the key bumped by the Weyl increments 0x9E3779B9 and
// 0xBB67AE85 between rounds.
#include <cub/device/device_segmented_radix_sort.cuh>

#include <algorithm>

#include "internal.hpp"

namespace eqtl {
namespace {

struct U4 {
  uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// keys of every column: one Philox call gives the random words of four
// consecutive samples
__global__ void perm_keys_kernel(int n, int B, int64_t cols, uint64_t seed, const uint64_t* __restrict__ gene_key,
                                 unsigned long long* keys) {
  const int64_t quads = (static_cast<int64_t>(n) + 3) / 4;
  const int64_t total = cols * quads;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t c = e / quads;
    const int q = static_cast<int>(e - c * quads);
    const int64_t g = c / B;
    const uint32_t b = static_cast<uint32_t>(c - g * B);
    const uint64_t gk = gene_key[g];
    const U4 r = philox4x32_10(U4{b, static_cast<uint32_t>(q), static_cast<uint32_t>(gk),
                                  static_cast<uint32_t>(gk >> 32)},
                               static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
    const uint32_t rw[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int i = 4 * q + t;
      if (i < n) keys[c * n + i] = (static_cast<unsigned long long>(rw[t]) << 32) | static_cast<uint32_t>(i);
    }
  }
}

__global__ void perm_offsets_kernel(int64_t cols, int n, int* off) {
  for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c <= cols;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x)
    off[c] = static_cast<int>(c * n);
}

// the permuted columns from the sorted keys
__global__ void perm_gather_kernel(int n, int B, int64_t cols, const unsigned long long* __restrict__ sorted,
                                   const double* __restrict__ base, const double* __restrict__ xb0,
                                   const double* __restrict__ dinv, double* Y) {
  const int64_t total = cols * n;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t c = e / n;
    const int i = static_cast<int>(e - c * n);
    const int64_t g = c / B;
    const int src = static_cast<int>(sorted[e] & 0xFFFFFFFFull);
    const double v = base[g * n + src];
    Y[e] = xb0 ? xb0[g * n + i] + v / sqrt(fmax(dinv[g * n + i], 1e-12)) : v;
  }
}

}  // namespace

void pheno_permute(eqtl_ctx* ctx, const double* base, const double* xb0, const double* dinv,
                   const uint64_t* gene_key, int n, int G, int B, uint64_t seed, const double* X, int p,
                   double* Y_out) {
  EQTL_CHECK(n > 1 && G > 0 && B > 0 && p > 0, EQTL_E_ARG, "pheno_permute: bad sizes");
  EQTL_CHECK((xb0 == nullptr) == (dinv == nullptr), EQTL_E_ARG, "pheno_permute: give both xb0 and dinv, or neither");
  const int64_t cols = static_cast<int64_t>(G) * B;
  const int64_t total = cols * n;
  EQTL_CHECK(cols < (int64_t(1) << 31) && total < (int64_t(1) << 31), EQTL_E_UNSUPPORTED,
             "pheno_permute: more than 2^31 permuted values in one call");
  cudaStream_t st = ctx->stream;
  Workspace& ws = ctx->ws;
  const size_t gn = static_cast<size_t>(G) * n;
  ws.perm_base.upload(base, gn, st);
  if (xb0) {
    ws.perm_xb0.upload(xb0, gn, st);
    ws.perm_dinv.upload(dinv, gn, st);
  }
  ws.perm_gkey.upload(gene_key, static_cast<size_t>(G), st);
  ws.perm_keys.alloc(static_cast<size_t>(total));
  ws.perm_sorted.alloc(static_cast<size_t>(total));
  ws.perm_off.alloc(static_cast<size_t>(cols) + 1);
  PhenoDev& P = ctx->pheno;
  P.Y.alloc(static_cast<size_t>(total));
  P.X.upload(X, static_cast<size_t>(n) * p, st);
  P.X_h.assign(X, X + static_cast<size_t>(n) * p);
  P.n = n;
  P.G = static_cast<int>(cols);
  P.p = p;
  const int64_t quads = cols * ((n + 3) / 4);
  const unsigned grid = static_cast<unsigned>(std::min<int64_t>((quads + 255) / 256, int64_t(ctx->sm_count) * 16));
  const unsigned ogrid = static_cast<unsigned>(std::min<int64_t>((cols + 256) / 256, int64_t(ctx->sm_count) * 16));
  ctx->launches += 2;
  perm_keys_kernel<<<grid, 256, 0, st>>>(n, B, cols, seed, ws.perm_gkey.p, ws.perm_keys.p);
  perm_offsets_kernel<<<ogrid, 256, 0, st>>>(cols, n, ws.perm_off.p);
  EQTL_CUDA(cudaGetLastError());
  // the random word is bits 32..63; the radix sort is stable, so equal words
  // keep the index order of bits 0..31
  size_t temp_bytes = 0;
  EQTL_CUDA(cub::DeviceSegmentedRadixSort::SortKeys(nullptr, temp_bytes, ws.perm_keys.p, ws.perm_sorted.p,
                                                    static_cast<int>(total), static_cast<int>(cols), ws.perm_off.p,
                                                    ws.perm_off.p + 1, 32, 64, st));
  ws.perm_temp.alloc(temp_bytes);
  EQTL_CUDA(cub::DeviceSegmentedRadixSort::SortKeys(ws.perm_temp.p, temp_bytes, ws.perm_keys.p, ws.perm_sorted.p,
                                                    static_cast<int>(total), static_cast<int>(cols), ws.perm_off.p,
                                                    ws.perm_off.p + 1, 32, 64, st));
  ++ctx->launches;
  const unsigned ggrid = static_cast<unsigned>(std::min<int64_t>((total + 255) / 256, int64_t(ctx->sm_count) * 16));
  perm_gather_kernel<<<ggrid, 256, 0, st>>>(n, B, cols, ws.perm_sorted.p, ws.perm_base.p,
                                            xb0 ? ws.perm_xb0.p : nullptr, xb0 ? ws.perm_dinv.p : nullptr, P.Y.p);
  EQTL_CUDA(cudaGetLastError());
  if (Y_out) P.Y.download(Y_out, static_cast<size_t>(total), st);
  EQTL_CUDA(cudaStreamSynchronize(st));
}

}  // namespace eqtl
