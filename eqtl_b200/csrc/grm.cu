// K2: GCTA-standardised GRM on the tensor cores.
//
// Restates compute_grm_from (src/grm.cpp:113-224) for the loaded genotypes:
//   per SNP   mu = mean of the imputed dosages, p = mu/2, skipped unless
//             p in [1e-8, 1-1e-8] and sd = sqrt(2p(1-p)) >= 1e-12 (:153-158);
//             z = (g - mu) / sd, 0 at missing calls (mean-imputed) (:159);
//   GRM       A = sum_s z_s z_s'  (tcgen05, FP16 hi/lo, split-K with FP64
//             accumulation of the FP32 partials across K ranges);
//   counts    J = M M' with M the 0/1 missing mask: exact in FP16 with FP32
//             accumulation (< 2^24 SNPs); sub_miss_i = J_ii and
//             N_ij = m - J_ii - J_jj + J_ij, N_ii = m - J_ii (:162-221);
//   divide    K_ij = A_ij / N_ij (0 if N_ij <= 0).
#include <algorithm>
#include <mutex>
#include <string>

#include "internal.hpp"
#include "scan_host.hpp"

namespace eqtl {
namespace dev {

__device__ __forceinline__ int bed_code_g(const uint8_t* row, int col) {
  const uint32_t b = __ldg(row + (col >> 2));
  const uint32_t pair = (b >> ((col & 3) * 2)) & 3u;
  return static_cast<int>(static_cast<int8_t>((0x0001FF02u >> (pair * 8)) & 0xFFu));
}

// per kept SNP: GRM usability, mean and 1/sd
__global__ void grm_snp_kernel(const int64_t* __restrict__ kept, int64_t m, int n, const double* __restrict__ mu,
                               const int32_t* __restrict__ n_miss, const double* __restrict__ s1, uint8_t* use,
                               double* mean, double* inv_sd) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const int64_t s = kept[r];
  const double mean_v = (s1[s] + n_miss[s] * mu[s]) / n;
  const double p = mean_v / 2.0;
  bool ok = !(p < 1e-8 || p > 1.0 - 1e-8);
  const double sd = sqrt(2.0 * p * (1.0 - p));
  if (sd < 1e-12) ok = false;
  use[r] = ok ? 1 : 0;
  mean[r] = mean_v;
  inv_sd[r] = ok ? 1.0 / sd : 0.0;
}

// GRM operands Z[i, r] (FP16 hi/lo) and the missing mask M[i, r] for every
// kept SNP r (rows = analysis samples, columns = SNPs, m_pad columns). SNPs
// that the GRM does not use (use[r] = 0) and the padding columns are zero in
// all three, so they add nothing to the sums or the missing-pair counts.
// A block covers 64 SNPs x kTrS samples: the packed rows (the whole row, or
// with the identity sample map just the bytes of these samples) are staged in
// shared memory with 16-byte loads, each SNP's three code values are formed
// once with the arithmetic of one element ((code - mean) * inv_sd in FP64,
// rounded to FP32, split into FP16 hi + lo), and each lane writes 8 SNPs of one
// sample per step with 16-byte stores (128 contiguous bytes per output row).
constexpr int kTrSnps = 64;
constexpr int kTrS = 1024;

__global__ void __launch_bounds__(256)
    grm_operands_kernel(const uint8_t* __restrict__ bed, int64_t bps, const int32_t* __restrict__ col,
                        int identity, int n, const int64_t* __restrict__ kept, int64_t m, int64_t m_pad,
                        const uint8_t* __restrict__ use, const double* __restrict__ mean,
                        const double* __restrict__ inv_sd, int stride, __half* zh, __half* zl, __half* mk) {
  extern __shared__ __align__(16) uint8_t tr_smem[];
  uint64_t* lut = reinterpret_cast<uint64_t*>(tr_smem);           // [64][4]: zh | zl << 16 | mk << 32
  int* skew = reinterpret_cast<int*>(lut + kTrSnps * 4);            // [64]
  uint8_t* rows = tr_smem + kTrSnps * 4 * sizeof(uint64_t) + kTrSnps * sizeof(int);  // [64][stride]
  const int64_t r0 = static_cast<int64_t>(blockIdx.x) * kTrSnps;
  const int i0 = blockIdx.y * kTrS;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // bytes staged per row: the samples' window (identity map) or the whole row
  const int64_t b0 = identity ? (i0 >> 2) : 0;
  const int64_t nbytes = identity ? (bps - b0 < kTrS / 4 ? bps - b0 : kTrS / 4) : bps;
  // per-SNP code values
  if (threadIdx.x < kTrSnps * 4) {
    const int rr = threadIdx.x >> 2, code = threadIdx.x & 3;
    const int64_t r = r0 + rr;
    uint64_t e = 0;  // unused SNPs and padding columns: z 0, no mask
    if (r < m && use[r]) {
      if (code == 1) {
        e = static_cast<uint64_t>(__half_as_ushort(__float2half_rn(1.0f))) << 32;  // missing: z 0, mask 1
      } else {
        const int c = code == 0 ? 2 : (code == 2 ? 1 : 0);
        const float z = static_cast<float>((static_cast<double>(c) - mean[r]) * inv_sd[r]);
        const __half h = __float2half_rn(z);
        const __half l = __float2half_rn(z - __half2float(h));
        e = static_cast<uint64_t>(__half_as_ushort(h)) | (static_cast<uint64_t>(__half_as_ushort(l)) << 16);
      }
    }
    lut[rr * 4 + code] = e;
  }
  // stage the packed rows: warp w takes rows w, w + 8, ...
  for (int rr = warp; rr < kTrSnps; rr += 8) {
    const int64_t r = r0 + rr;
    if (r >= m) continue;
    const int64_t off0 = __ldg(kept + r) * bps + b0;
    const int64_t a0 = off0 & ~int64_t(15);
    const int sk = static_cast<int>(off0 - a0);
    const int nvec = static_cast<int>((sk + nbytes + 15) / 16);
    const uint4* src = reinterpret_cast<const uint4*>(bed + a0);
    // 4-byte stores: the row stride is an odd number of words, so the 8 rows
    // a lane reads and the lanes' row groups spread over the banks
    uint32_t* dst = reinterpret_cast<uint32_t*>(rows + rr * stride);
    for (int v = lane; v < nvec; v += 32) {
      const uint4 x = __ldg(src + v);
      dst[4 * v] = x.x;
      dst[4 * v + 1] = x.y;
      dst[4 * v + 2] = x.z;
      dst[4 * v + 3] = x.w;
    }
    if (lane == 0) skew[rr] = sk;
  }
  __syncthreads();
  // lane: SNP group q = lane % 8 (8 SNPs), sample i = base + lane / 8
  const int q = lane & 7;
  for (int ib = i0 + warp * 4; ib < i0 + kTrS; ib += 32) {
    const int i = ib + (lane >> 3);
    if (i >= n) continue;
    const int c = identity ? i : __ldg(col + i);
    const int64_t byte = (c >> 2) - b0;
    const int sh = (c & 3) * 2;
    uint32_t hw[4], lw[4], mw[4];
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      uint64_t e[2];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int rr = q * 8 + j + t;
        e[t] = 0;
        if (r0 + rr < m) {
          const uint32_t code = (static_cast<uint32_t>(rows[rr * stride + skew[rr] + byte]) >> sh) & 3u;
          e[t] = lut[rr * 4 + code];
        }
      }
      hw[j / 2] = static_cast<uint32_t>(e[0] & 0xFFFFu) | (static_cast<uint32_t>(e[1] & 0xFFFFu) << 16);
      lw[j / 2] = static_cast<uint32_t>((e[0] >> 16) & 0xFFFFu) | (static_cast<uint32_t>((e[1] >> 16) & 0xFFFFu) << 16);
      mw[j / 2] = static_cast<uint32_t>((e[0] >> 32) & 0xFFFFu) | (static_cast<uint32_t>((e[1] >> 32) & 0xFFFFu) << 16);
    }
    const int64_t o = static_cast<int64_t>(i) * m_pad + r0 + q * 8;
    *reinterpret_cast<uint4*>(zh + o) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    *reinterpret_cast<uint4*>(zl + o) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    *reinterpret_cast<uint4*>(mk + o) = make_uint4(mw[0], mw[1], mw[2], mw[3]);
  }
}

// The same operands from FP32 dosage rows: z = (d - mean) * inv_sd in FP64,
// rounded to FP32 and split into FP16 hi + lo; z 0 and mask 1 at a missing
// call. Block: 64 SNPs x 32 samples; warp w takes SNPs r0 + 8w .. r0 + 8w + 7
// of sample i = 32 * blockIdx.y + lane, so each dosage row is read 32
// consecutive samples at a time, and writes them with one 16-byte store per
// operand.
__global__ void __launch_bounds__(256)
    grm_operands_dense_kernel(GenoRows src, const int32_t* __restrict__ col, int n, const int64_t* __restrict__ kept,
                              int64_t m, int64_t m_pad, const uint8_t* __restrict__ use,
                              const double* __restrict__ mean, const double* __restrict__ inv_sd, __half* zh,
                              __half* zl, __half* mk) {
  const int i = blockIdx.y * 32 + (threadIdx.x & 31);
  if (i >= n) return;
  const int64_t rb = static_cast<int64_t>(blockIdx.x) * kTrSnps + (threadIdx.x >> 5) * 8;
  const int c = __ldg(col + i);
  uint32_t hw[4], lw[4], mw[4];
#pragma unroll
  for (int j = 0; j < 8; j += 2) {
    uint32_t h2[2] = {0, 0}, l2[2] = {0, 0}, m2[2] = {0, 0};
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int64_t r = rb + j + t;
      if (r < m && use[r]) {
        const double d = src.dosage(__ldg(kept + r), c);
        if (isnan(d)) {
          m2[t] = __half_as_ushort(__float2half_rn(1.0f));
        } else {
          const float z = static_cast<float>((d - mean[r]) * inv_sd[r]);
          const __half h = __float2half_rn(z);
          const __half l = __float2half_rn(z - __half2float(h));
          h2[t] = __half_as_ushort(h);
          l2[t] = __half_as_ushort(l);
        }
      }
    }
    hw[j / 2] = h2[0] | (h2[1] << 16);
    lw[j / 2] = l2[0] | (l2[1] << 16);
    mw[j / 2] = m2[0] | (m2[1] << 16);
  }
  const int64_t o = static_cast<int64_t>(i) * m_pad + rb;
  *reinterpret_cast<uint4*>(zh + o) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
  *reinterpret_cast<uint4*>(zl + o) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
  *reinterpret_cast<uint4*>(mk + o) = make_uint4(mw[0], mw[1], mw[2], mw[3]);
}

// *m_used = number of SNPs with use[r] set
__global__ void grm_count_kernel(const uint8_t* __restrict__ use, int64_t m, unsigned long long* m_used) {
  unsigned long long c = 0;
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < m;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x)
    c += use[r];
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(m_used, c);
}

struct GrmEpiParams {
  int n;
  double* A;  // [n, n] FP64 sums (atomic)
  int* J;     // [n, n] joint-missing counts (atomic, exact integers)
};

struct GrmEpi {
  static constexpr bool kGrouped = false;
  using Params = GrmEpiParams;
  const Params& P;
  int row = 0;
  int64_t col0 = 0;
  static constexpr int kSmemBytes = 0;
  __device__ GrmEpi(const Params& p, const TileShape&, uint8_t*) : P(p) {}
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
      const int64_t cc = col0 + c + j;
      if (cc >= P.n) break;
      const int64_t idx = static_cast<int64_t>(row) * P.n + cc;
      atomicAdd(P.A + idx, static_cast<double>(v[0][j]));
      if (v[1][j] != 0.0f) atomicAdd(P.J + idx, __float2int_rn(v[1][j]));
    }
  }
  __device__ void end_tile() {}
  __device__ void finish() {}
};

// The same sums over a work item made of K sub-ranges: each sub-range's
// FP32 tensor-core sums (256 SNPs, so the accumulation's drift stays near
// 1e-6) are added into per-thread FP32 registers (round to nearest, so
// across sub-ranges the error is a random walk), and the work item's total
// goes to the FP64 sums with one atomic per element. The joint-missing
// counts are exact integers in every sub-range and are added where
// non-zero. Tiles of 128 x 128: two 16-column chunks per thread.
struct GrmSubEpi {
  static constexpr bool kGrouped = false;
  static constexpr bool kChunkIdx = true;
  static constexpr int kMaxChunks = 2;
  static constexpr int kSmemBytes = 0;
  using Params = GrmEpiParams;
  const Params& P;
  int row = 0;
  int64_t col0 = 0;
  int cbase[kMaxChunks];
  float acc[kMaxChunks][16];
  __device__ GrmSubEpi(const Params& p, const TileShape&, uint8_t*) : P(p) {}
  __device__ void init(int, int) {}
  __device__ void begin_tile(int r, int64_t c0) {
    row = r;
    col0 = c0;
#pragma unroll
    for (int ci = 0; ci < kMaxChunks; ++ci) {
      cbase[ci] = -1;
#pragma unroll
      for (int j = 0; j < 16; ++j) acc[ci][j] = 0.0f;
    }
  }
  template <int NACC>
  __device__ void chunk_at(int ci, int c, const float (&v)[NACC][16]) {
    cbase[ci] = c;
#pragma unroll
    for (int j = 0; j < 16; ++j) acc[ci][j] += v[0][j];
    if (row >= P.n) return;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int64_t cc = col0 + c + j;
      if (cc < P.n && v[1][j] != 0.0f) atomicAdd(P.J + static_cast<int64_t>(row) * P.n + cc, __float2int_rn(v[1][j]));
    }
  }
  __device__ void end_tile() {
    if (row >= P.n) return;
#pragma unroll
    for (int ci = 0; ci < kMaxChunks; ++ci) {
      if (cbase[ci] < 0) continue;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int64_t cc = col0 + cbase[ci] + j;
        if (cc < P.n) atomicAdd(P.A + static_cast<int64_t>(row) * P.n + cc, static_cast<double>(acc[ci][j]));
      }
    }
  }
  __device__ void finish() {}
};

__global__ void grm_finalize_kernel(int n, const unsigned long long* __restrict__ m_used_p,
                                    const double* __restrict__ A, const int* __restrict__ J, double* K,
                                    int32_t* Npk) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= static_cast<int64_t>(n) * n) return;
  const int64_t m_used = static_cast<int64_t>(*m_used_p);
  const int i = static_cast<int>(e / n), j = static_cast<int>(e - static_cast<int64_t>(i) * n);
  // the sums exist for i >= j (lower triangle); K is their mirror image above
  const int64_t lo_e = static_cast<int64_t>(i >= j ? i : j) * n + (i >= j ? j : i);
  const int64_t mi = static_cast<int64_t>(J[static_cast<int64_t>(i) * n + i]);
  const int64_t mj = static_cast<int64_t>(J[static_cast<int64_t>(j) * n + j]);
  int64_t sub;
  if (i == j) sub = m_used - mi;
  else sub = m_used - mi - mj + static_cast<int64_t>(J[lo_e]);
  K[e] = sub > 0 ? A[lo_e] / static_cast<double>(sub) : 0.0;
  if (j <= i) Npk[static_cast<int64_t>(i) * (i + 1) / 2 + j] = static_cast<int32_t>(sub);
}

}  // namespace dev

template <>
struct EpiOf<dev::GrmEpiParams> {
  using type = dev::GrmEpi;
};
// the sub-range form of the same sums (its own parameter type, so that the
// launcher picks its epilogue)
struct GrmSubParams : dev::GrmEpiParams {};
template <>
struct EpiOf<GrmSubParams> {
  using type = dev::GrmSubEpi;
};

// K chunks (of 64 SNPs) summed in one FP32 tensor-core accumulator before
// the FP64 sum across ranges.
constexpr int kGrmChunksPerRange = 8;
constexpr int kGrmChunksPerSub = 4;

// Computes the GRM of the loaded genotypes. K: device [n, n] (row-major ==
// column-major, symmetric). Returns the number of SNPs used.
int64_t grm_compute(eqtl_ctx* ctx, DevBuf<double>& K, DevBuf<int32_t>& Npk) {
  using namespace dev;
  Geno& g = ctx->geno;
  EQTL_CHECK(g.m_all > 0, EQTL_E_STATE, "grm: no genotypes loaded");
  EQTL_CHECK(!g.subset, EQTL_E_STATE, "grm: the GRM covers every analysis sample; restore the full sample view first");
  cudaStream_t st = ctx->stream;
  const int n = g.n;
  const int64_t m = g.m;
  EQTL_CHECK(m > 0, EQTL_E_ARG, "no SNPs for GRM");
  StageScope timer(ctx, EQTL_STAGE_GRM);
  Workspace& ws = ctx->ws;
  DevBuf<uint8_t>& use = ws.grm_use;
  DevBuf<double>& mean = ws.grm_mean;
  DevBuf<double>& inv_sd = ws.grm_isd;
  use.alloc(std::max<int64_t>(m, 1));
  mean.alloc(std::max<int64_t>(m, 1));
  inv_sd.alloc(std::max<int64_t>(m, 1));
  if (m > 0) {
    ++ctx->launches;
    grm_snp_kernel<<<static_cast<unsigned>((m + 255) / 256), 256, 0, st>>>(g.kept.p, m, n, g.mu.p, g.n_miss.p, g.s1.p,
                                                                           use.p, mean.p, inv_sd.p);
    EQTL_CUDA(cudaGetLastError());
  }
  // every kept SNP is a column; the ones the GRM does not use are zero
  const int64_t m_pad = ((m + 63) / 64) * 64;
  DevBuf<unsigned long long>& cnt = ws.grm_count;
  cnt.alloc(1);
  cnt.zero(st);
  if (m > 0) {
    ++ctx->launches;
    grm_count_kernel<<<static_cast<unsigned>(std::min<int64_t>((m + 255) / 256, 1184)), 256, 0, st>>>(use.p, m,
                                                                                                      cnt.p);
    EQTL_CUDA(cudaGetLastError());
  }
  DevBuf<__half>& zh = ws.grm_zh;
  DevBuf<__half>& zl = ws.grm_zl;
  DevBuf<__half>& mk = ws.grm_mk;
  const size_t elems = static_cast<size_t>(n) * m_pad;
  zh.alloc(elems);
  zl.alloc(elems);
  mk.alloc(elems);
  if (g.dense) {
    dim3 grid(static_cast<unsigned>(m_pad / kTrSnps), static_cast<unsigned>((n + 31) / 32));
    ++ctx->launches;
    grm_operands_dense_kernel<<<grid, 256, 0, st>>>(g.rows(), g.col.p, n, g.kept.p, m, m_pad, use.p, mean.p,
                                                    inv_sd.p, zh.p, zl.p, mk.p);
    EQTL_CUDA(cudaGetLastError());
  } else {
    const int64_t nbytes = g.col_identity ? std::min<int64_t>(kTrS / 4, g.bytes_per_snp) : g.bytes_per_snp;
    int stride = static_cast<int>(((nbytes + 30 + 3) / 4) * 4);
    if ((stride / 4) % 2 == 0) stride += 4;  // an odd number of words
    const int smem = kTrSnps * 4 * static_cast<int>(sizeof(uint64_t)) + kTrSnps * static_cast<int>(sizeof(int)) +
                     kTrSnps * stride;
    EQTL_CHECK(smem <= 200 * 1024, EQTL_E_UNSUPPORTED,
               "grm: more than ~12,000 samples in the file with a non-identity sample map");
    EQTL_CUDA(cudaFuncSetAttribute(grm_operands_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    dim3 grid(static_cast<unsigned>(m_pad / kTrSnps), static_cast<unsigned>((n + kTrS - 1) / kTrS));
    ++ctx->launches;
    grm_operands_kernel<<<grid, 256, smem, st>>>(g.bed.p, g.bytes_per_snp, g.col.p, g.col_identity ? 1 : 0, n,
                                                 g.kept.p, m, m_pad, use.p, mean.p, inv_sd.p, stride, zh.p, zl.p,
                                                 mk.p);
    EQTL_CUDA(cudaGetLastError());
  }
  DevBuf<double>& A = ws.grm_A;
  DevBuf<int>& J = ws.grm_J;
  A.alloc(static_cast<size_t>(n) * n);
  J.alloc(static_cast<size_t>(n) * n);
  A.zero(st);
  J.zero(st);
  GrmSubParams ep{};
  ep.n = n;
  ep.A = A.p;
  ep.J = J.p;
  const __half* ah[2] = {zh.p, mk.p};
  const __half* al[2] = {zl.p, mk.p};
  const __half* bh[2] = {zh.p, mk.p};
  const __half* bl[2] = {zl.p, mk.p};
  const int bsel[2] = {0, 1}, prod[2] = {7, 1};
  // K is symmetric: only the tiles of 128 x 128 on or below the diagonal
  std::vector<int2> lower;
  for (int tb = 0; tb < (n + 127) / 128; ++tb)
    for (int ta = tb; ta < (n + 127) / 128; ++ta) lower.push_back(make_int2(ta, tb));
  ws.grm_tiles.upload(lower.data(), lower.size(), st);
  const int tiles = static_cast<int>(lower.size());
  // The tensor cores' FP32 accumulation drifts with the number of K steps
  // summed into one accumulator (about 2.6e-7 of the running sum per step,
  // the same sign for the large positive sums of K's diagonal and of
  // related pairs), so the accumulators restart every kGrmChunksPerSub
  // chunks of 64 SNPs and the epilogue sums the sub-ranges (GrmSubEpi);
  // the K ranges of a tile (enough of them for every SM) meet in FP64.
  const int ksplit = std::max(1, (4 * sm_count(ctx) + tiles - 1) / tiles);
  // the GRM operands are FP16 regardless of the scan precision
  launch_tile_n<128, 2>(ctx, false, ep, ah, al, n, bh, bl, n, static_cast<int>(m_pad), bsel, prod, ws.grm_tiles.p,
                        tiles, ksplit, 2, kGrmChunksPerSub);
  K.alloc(static_cast<size_t>(n) * n);
  Npk.alloc(static_cast<size_t>(n) * (n + 1) / 2);
  const int64_t tot = static_cast<int64_t>(n) * n;
  ++ctx->launches;
  grm_finalize_kernel<<<static_cast<unsigned>((tot + 255) / 256), 256, 0, st>>>(n, cnt.p, A.p, J.p, K.p, Npk.p);
  EQTL_CUDA(cudaGetLastError());
  unsigned long long mu_n = 0;
  cnt.download(&mu_n, 1, st);
  EQTL_CUDA(cudaStreamSynchronize(st));
  EQTL_CHECK(mu_n > 0, EQTL_E_ARG, "no SNPs for GRM");
  return static_cast<int64_t>(mu_n);
}

}  // namespace eqtl

// ===================================================== allocation-free GRM
// The same GRM from caller-owned device buffers, with every piece of scratch
// (FP16 operands of one pass, FP64/int accumulators, per-SNP statistics) in
// one file-scope device array sized for n <= kNaMaxN samples. SNP rows go
// through in passes of kNaChunk; each pass is one tile launch whose K extent
// is the pass, accumulating into A and J with the split-K atomics of the
// regular path, so the result equals the regular path's up to the FP64
// summation order of A.
namespace eqtl {
namespace dev {

constexpr int kNaMaxN = EQTL_GRM_NOALLOC_MAX_N;
constexpr int kNaChunk = EQTL_GRM_NOALLOC_CHUNK;
constexpr size_t na_align(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kNaOpBytes = na_align(sizeof(__half) * kNaMaxN * kNaChunk);
constexpr size_t kNaABytes = na_align(sizeof(double) * kNaMaxN * kNaMaxN);
constexpr size_t kNaJBytes = na_align(sizeof(int) * kNaMaxN * kNaMaxN);
constexpr size_t kNaSnpBytes = na_align(sizeof(double) * kNaChunk);
constexpr size_t kNaUseBytes = na_align(kNaChunk);
// layout: zh | zl | mk | A | J | mean | inv_sd | use | counters
constexpr size_t kNaOffZh = 0;
constexpr size_t kNaOffZl = kNaOffZh + kNaOpBytes;
constexpr size_t kNaOffMk = kNaOffZl + kNaOpBytes;
constexpr size_t kNaOffA = kNaOffMk + kNaOpBytes;
constexpr size_t kNaOffJ = kNaOffA + kNaABytes;
constexpr size_t kNaOffMean = kNaOffJ + kNaJBytes;
constexpr size_t kNaOffIsd = kNaOffMean + kNaSnpBytes;
constexpr size_t kNaOffUse = kNaOffIsd + kNaSnpBytes;
constexpr size_t kNaOffCnt = kNaOffUse + kNaUseBytes;  // [0] SNPs used, [1] bad sample columns
constexpr size_t kNaOffTiles = kNaOffCnt + 64;          // lower-triangle tile list (int2)
constexpr int kNaMaxTiles = ((kNaMaxN + 127) / 128) * ((kNaMaxN + 255) / 256);
constexpr size_t kNaScratchBytes = kNaOffCnt + 256;
static_assert(64 + sizeof(int2) * kNaMaxTiles <= 256, "tile list inside the counter block");
static_assert(kNaScratchBytes == EQTL_GRM_NOALLOC_SCRATCH_BYTES, "header scratch size");

static __device__ __align__(256) uint8_t grm_na_scratch[kNaScratchBytes];

// Sample columns must address the .bed row: 0 <= col < 4 * bytes_per_snp.
__global__ void grm_na_check_cols_kernel(const int32_t* __restrict__ col, int n, int64_t bps,
                                         unsigned long long* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const int32_t c = col[i];
    if (c < 0 || static_cast<int64_t>(c) >= 4 * bps) atomicAdd(bad, 1ull);
  }
}

// One warp per SNP row of the pass: the decode filter of bed_stats_kernel
// (geno.cu) followed by the GRM usability of grm_snp_kernel, in the same
// FP64 expressions.
__global__ void grm_na_stats_kernel(const uint8_t* __restrict__ bed, int64_t bps, const int32_t* __restrict__ col,
                                    int n, int64_t r0, int nr, int miss_hand, double max_miss, double maf_min,
                                    uint8_t* use, double* mean, double* inv_sd, unsigned long long* m_used) {
  const int lane = threadIdx.x & 31;
  const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= kNaChunk) return;
  if (r >= nr) {
    if (lane == 0) {
      use[r] = 0;
      mean[r] = 0.0;
      inv_sd[r] = 0.0;
    }
    return;
  }
  const uint8_t* row = bed + (r0 + r) * bps;
  int nm = 0, a = 0;
  for (int i = lane; i < n; i += 32) {
    const int c = bed_code_g(row, __ldg(col + i));
    if (c < 0)
      ++nm;
    else
      a += c;
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    nm += __shfl_xor_sync(0xffffffffu, nm, o);
    a += __shfl_xor_sync(0xffffffffu, a, o);
  }
  if (lane) return;
  const int n_ok = n - nm;
  bool keep = n_ok > 0;
  const double sum = static_cast<double>(a);
  double m_imp = 0.0, f = 0.0;
  if (n_ok > 0) {
    m_imp = sum / n_ok;
    f = (sum / static_cast<double>(n_ok)) / 2.0;
  }
  const double miss_frac = static_cast<double>(nm) / static_cast<double>(n);
  if (miss_frac > max_miss + 1e-15) keep = false;
  if (miss_hand == EQTL_MISS_FILTER && nm > 0) keep = false;
  if (f < 0) f = 0;
  if (f > 1) f = 1;
  if (f < 1e-12 || f > 1.0 - 1e-12) keep = false;
  if (maf_min > 0.0 && (f < maf_min || f > 1.0 - maf_min)) keep = false;
  const double mean_v = (static_cast<double>(a) + nm * m_imp) / n;
  const double p = mean_v / 2.0;
  bool ok = keep && !(p < 1e-8 || p > 1.0 - 1e-8);
  const double sd = sqrt(2.0 * p * (1.0 - p));
  if (sd < 1e-12) ok = false;
  use[r] = ok ? 1 : 0;
  mean[r] = mean_v;
  inv_sd[r] = ok ? 1.0 / sd : 0.0;
  if (ok) atomicAdd(m_used, 1ull);
}

// Zt[i, c] of the pass (row stride kNaChunk), zero for unused columns:
// 32 x 32 tiles through shared memory, so that both the .bed reads and the
// operand writes coalesce.
__global__ void grm_na_transpose_kernel(const uint8_t* __restrict__ bed, int64_t bps, const int32_t* __restrict__ col,
                                        int n, int64_t r0, const uint8_t* __restrict__ use,
                                        const double* __restrict__ mean, const double* __restrict__ inv_sd,
                                        __half* zh, __half* zl, __half* mk) {
  __shared__ float tz[32][33];
  __shared__ float tm[32][33];
  const int c0 = blockIdx.x * 32;
  const int i0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  const int i = i0 + tx;
  const int ci = i < n ? __ldg(col + i) : 0;
  for (int r = ty; r < 32; r += 8) {
    const int c = c0 + r;
    float z = 0.0f, mm = 0.0f;
    if (i < n && use[c]) {
      const int code = bed_code_g(bed + (r0 + c) * bps, ci);
      if (code < 0) {
        mm = 1.0f;
      } else {
        z = static_cast<float>((static_cast<double>(code) - mean[c]) * inv_sd[c]);
      }
    }
    tz[r][tx] = z;
    tm[r][tx] = mm;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int ii = i0 + r;
    const int c = c0 + tx;
    if (ii < n) {
      const float z = tz[tx][r];
      const __half h = __float2half_rn(z);
      const __half l = __float2half_rn(z - __half2float(h));
      zh[static_cast<int64_t>(ii) * kNaChunk + c] = h;
      zl[static_cast<int64_t>(ii) * kNaChunk + c] = l;
      mk[static_cast<int64_t>(ii) * kNaChunk + c] = __float2half_rn(tm[tx][r]);
    }
  }
}

__global__ void grm_na_finalize_kernel(int n, const unsigned long long* __restrict__ m_used,
                                       const double* __restrict__ A, const int* __restrict__ J, double* K,
                                       int32_t* Npk) {
  const int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= static_cast<int64_t>(n) * n) return;
  const int64_t mu = static_cast<int64_t>(*m_used);
  const int i = static_cast<int>(e / n), j = static_cast<int>(e - static_cast<int64_t>(i) * n);
  // only the tiles holding the lower triangle are summed; K above the
  // diagonal is their mirror image, so K is exactly symmetric
  const int64_t lo_e = static_cast<int64_t>(i >= j ? i : j) * n + (i >= j ? j : i);
  const int64_t mi = static_cast<int64_t>(J[static_cast<int64_t>(i) * n + i]);
  const int64_t mj = static_cast<int64_t>(J[static_cast<int64_t>(j) * n + j]);
  int64_t sub;
  if (i == j)
    sub = mu - mi;
  else
    sub = mu - mi - mj + static_cast<int64_t>(J[lo_e]);
  K[e] = sub > 0 ? A[lo_e] / static_cast<double>(sub) : 0.0;
  if (Npk && j <= i) Npk[static_cast<int64_t>(i) * (i + 1) / 2 + j] = static_cast<int32_t>(sub);
}

}  // namespace dev

namespace {
constexpr int kNaMaxDevices = 64;
std::mutex g_na_mu;
uint8_t* g_na_addr[kNaMaxDevices] = {};
}  // namespace

// Device address of the scratch array on the current device, resolved once
// per device (cudaGetSymbolAddress).
static uint8_t* grm_na_scratch_addr(int device) {
  EQTL_CHECK(device >= 0 && device < kNaMaxDevices, EQTL_E_ARG, "eqtl_grm_noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_addr[device]) {
    void* p = nullptr;
    EQTL_CUDA(cudaGetSymbolAddress(&p, dev::grm_na_scratch));
    g_na_addr[device] = static_cast<uint8_t*>(p);
  }
  return g_na_addr[device];
}

// Called by eqtl_open with the context's device current: resolves the
// scratch array's device address and loads every kernel of the allocation-
// free GRM, so that with lazy module loading the array and the kernel images
// are set up while the caller can still allocate, not in its first call.
void grm_noalloc_prepare(eqtl_ctx* ctx) {
  using namespace dev;
  grm_na_scratch_addr(ctx->device);
  cudaFuncAttributes fa;
  EQTL_CUDA(cudaFuncGetAttributes(&fa, grm_na_check_cols_kernel));
  EQTL_CUDA(cudaFuncGetAttributes(&fa, grm_na_stats_kernel));
  EQTL_CUDA(cudaFuncGetAttributes(&fa, grm_na_transpose_kernel));
  EQTL_CUDA(cudaFuncGetAttributes(&fa, grm_na_finalize_kernel));
  EQTL_CUDA(cudaFuncGetAttributes(&fa, tile_kernel<256, 2, 0u, GrmEpi>));
}

int64_t grm_noalloc(eqtl_ctx* ctx, const uint8_t* bed, int64_t m, int64_t bps, const int32_t* col, int n,
                    int miss_hand, double max_miss, double maf_min, double* K, int32_t* Npk) {
  using namespace dev;
  EQTL_CHECK(bed && col && K, EQTL_E_ARG, "eqtl_grm_noalloc: null input or output");
  EQTL_CHECK(n > 0 && m > 0 && bps > 0, EQTL_E_ARG, "eqtl_grm_noalloc: bad sizes");
  EQTL_CHECK(n <= kNaMaxN, EQTL_E_UNSUPPORTED,
             "eqtl_grm_noalloc: n = " + std::to_string(n) + " exceeds the static scratch limit of " +
                 std::to_string(kNaMaxN) + " samples (use eqtl_grm)");
  EQTL_CHECK(miss_hand == EQTL_MISS_FILTER || miss_hand == EQTL_MISS_IMPUTE, EQTL_E_ARG,
             "eqtl_grm_noalloc: miss_hand");
  uint8_t* s = grm_na_scratch_addr(ctx->device);
  __half* zh = reinterpret_cast<__half*>(s + kNaOffZh);
  __half* zl = reinterpret_cast<__half*>(s + kNaOffZl);
  __half* mk = reinterpret_cast<__half*>(s + kNaOffMk);
  double* A = reinterpret_cast<double*>(s + kNaOffA);
  int* J = reinterpret_cast<int*>(s + kNaOffJ);
  double* mean = reinterpret_cast<double*>(s + kNaOffMean);
  double* isd = reinterpret_cast<double*>(s + kNaOffIsd);
  uint8_t* use = s + kNaOffUse;
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(s + kNaOffCnt);
  int2* tile_list = reinterpret_cast<int2*>(s + kNaOffTiles);
  cudaStream_t st = ctx->stream;
  // accumulators and counters start at zero on every call
  EQTL_CUDA(cudaMemsetAsync(A, 0, sizeof(double) * n * n, st));
  EQTL_CUDA(cudaMemsetAsync(J, 0, sizeof(int) * n * n, st));
  EQTL_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), st));
  ++ctx->launches;
  grm_na_check_cols_kernel<<<(n + 255) / 256, 256, 0, st>>>(col, n, bps, cnt + 1);
  EQTL_CUDA(cudaGetLastError());
  unsigned long long bad = 0;
  EQTL_CUDA(cudaMemcpyAsync(&bad, cnt + 1, sizeof(bad), cudaMemcpyDeviceToHost, st));
  EQTL_CUDA(cudaStreamSynchronize(st));
  EQTL_CHECK(bad == 0, EQTL_E_ARG, "eqtl_grm_noalloc: sample_col outside the .bed row");
  GrmEpiParams ep{n, A, J};
  const __half* ah[2] = {zh, mk};
  const __half* al[2] = {zl, mk};
  const int bsel[2] = {0, 1}, prod[2] = {7, 1};
  // the tiles of 128 rows x 256 columns that hold some element with row >=
  // column, as in grm_compute; the list lives in the scratch array
  int2 lower[kNaMaxTiles];
  int tiles = 0;
  for (int tb = 0; tb < (n + 255) / 256; ++tb)
    for (int ta = 0; ta < (n + 127) / 128; ++ta)
      if (128 * ta + 127 >= 256 * tb) lower[tiles++] = make_int2(ta, tb);
  EQTL_CUDA(cudaMemcpyAsync(tile_list, lower, sizeof(int2) * tiles, cudaMemcpyHostToDevice, st));
  const int ksplit = std::max({1, (4 * sm_count(ctx) + tiles - 1) / tiles,
                               (kNaChunk / 64 + kGrmChunksPerRange - 1) / kGrmChunksPerRange});
  for (int64_t r0 = 0; r0 < m; r0 += kNaChunk) {
    const int nr = static_cast<int>(std::min<int64_t>(kNaChunk, m - r0));
    ctx->launches += 2;
    grm_na_stats_kernel<<<kNaChunk / 8, 256, 0, st>>>(bed, bps, col, n, r0, nr, miss_hand, max_miss, maf_min, use,
                                                       mean, isd, cnt);
    EQTL_CUDA(cudaGetLastError());
    grm_na_transpose_kernel<<<dim3(kNaChunk / 32, (n + 31) / 32), dim3(32, 8), 0, st>>>(bed, bps, col, n, r0, use,
                                                                                        mean, isd, zh, zl, mk);
    EQTL_CUDA(cudaGetLastError());
    launch_tile_n<256, 2>(ctx, false, ep, ah, al, n, ah, al, n, kNaChunk, bsel, prod, tile_list, tiles, ksplit);
  }
  unsigned long long used = 0;
  EQTL_CUDA(cudaMemcpyAsync(&used, cnt, sizeof(used), cudaMemcpyDeviceToHost, st));
  EQTL_CUDA(cudaStreamSynchronize(st));
  EQTL_CHECK(used > 0, EQTL_E_ARG, "no SNPs for GRM");
  const int64_t tot = static_cast<int64_t>(n) * n;
  ++ctx->launches;
  grm_na_finalize_kernel<<<static_cast<unsigned>((tot + 255) / 256), 256, 0, st>>>(n, cnt, A, J, K, Npk);
  EQTL_CUDA(cudaGetLastError());
  EQTL_CUDA(cudaStreamSynchronize(st));
  return static_cast<int64_t>(used);
}

}  // namespace eqtl
