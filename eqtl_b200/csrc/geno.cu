// K1: PLINK .bed decode on the device.
//
// Restates PlinkBed::decode_row (src/plink_bed.cpp:263-320): 2-bit code of
// sample i at byte col/4, bits 2*(col%4); 00 -> 2 A1 alleles, 10 -> 1,
// 11 -> 0, 01 -> missing (LUT :221-224). Per SNP: missing count, A1 sum,
// mean-imputation value mu = sum / n_ok, allele frequency af = mu / 2 and
// the filters (max missing fraction, --miss-hand filter, af in
// (1e-12, 1-1e-12), MAF gate) in the same FP64 expressions, so keep flags
// and af are bit-identical. Kept SNPs are then expanded once into the
// centred FP16 hi/lo operand every tensor-core contraction reads:
//     gc[s, i] = (dosage[s, i] - mu_s) * 64,   missing -> 0,
// (centring leaves every statistic unchanged because the covariates always
// contain an intercept; it removes the mean from the split).
//
// The same decode serves FP32 dosage rows (a VCF's FORMAT/DS values, or GT
// counts, per sample; src/vcf_session.cpp:193-258): a value that is not
// finite is a missing call, every other value is used as it is.
#include <cuda_bf16.h>

#include <algorithm>

#include "internal.hpp"

namespace eqtl {
namespace {

// Per-SNP statistics and filters, one warp per row. With 2-bit rows the sums
// are integers (exact in FP64 in any order); with FP32 dosage rows they are
// FP64 sums of the dosages.
__global__ void bed_stats_kernel(GenoRows src, int64_t m, const int32_t* __restrict__ col, int n, int miss_hand,
                                 double max_miss, double maf_min, int32_t* n_miss, double* s1, double* s2,
                                 uint8_t* pass, double* af, double* mu) {
  const int lane = threadIdx.x & 31;
  const int64_t snp = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (snp >= m) return;
  int nm = 0;
  double a = 0.0, b = 0.0;
  for (int i = lane; i < n; i += 32) {
    const double d = src.dosage(snp, __ldg(col + i));
    if (isnan(d)) {
      ++nm;
    } else {
      a += d;
      b += d * d;
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    nm += __shfl_xor_sync(0xffffffffu, nm, o);
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane) return;
  const int n_ok = n - nm;
  bool keep = n_ok > 0;
  const double sum = a;
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
  n_miss[snp] = nm;
  s1[snp] = a;
  s2[snp] = b;
  pass[snp] = keep ? 1 : 0;
  af[snp] = f;
  mu[snp] = m_imp;
}

template <class T>
__device__ __forceinline__ T to16(double v);
template <>
__device__ __forceinline__ __half to16<__half>(double v) {
  return __double2half(v);
}
template <>
__device__ __forceinline__ __nv_bfloat16 to16<__nv_bfloat16>(double v) {
  return __double2bfloat16(v);
}
__device__ __forceinline__ double from16(__half h) { return static_cast<double>(__half2float(h)); }
__device__ __forceinline__ double from16(__nv_bfloat16 h) { return static_cast<double>(__bfloat162float(h)); }

// One thread per (sample, kept SNP): the general expansion (FP32 dosage rows,
// or 2-bit rows too long to stage).
template <class T>
__global__ void bed_expand_kernel(GenoRows src, const int32_t* __restrict__ col, int n, int k_pad,
                                  const int64_t* __restrict__ kept, int64_t m_kept, const double* __restrict__ mu,
                                  float scale, T* hi, T* lo) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= k_pad) return;
  const int c_col = k < n ? __ldg(col + k) : 0;
  for (int64_t r = blockIdx.y; r < m_kept; r += gridDim.y) {
    const int64_t s = __ldg(kept + r);
    double v = 0.0;
    if (k < n) {
      const double d = src.dosage(s, c_col);
      v = isnan(d) ? 0.0 : (d - __ldg(mu + s));
    }
    v *= static_cast<double>(scale);
    const T h = to16<T>(v);
    const T l = to16<T>(v - from16(h));
    hi[r * k_pad + k] = h;
    lo[r * k_pad + k] = l;
  }
}

// One warp per kept SNP row, for rows of at most kExpandMaxStage staged
// bytes. The packed row goes to shared memory with 16-byte loads, starting at
// the 16-byte boundary at or below the row start (the device copy of the .bed
// carries kBedPad bytes of padding, so the last row's over-read stays inside
// the buffer); the four values a 2-bit code can take are formed once per row
// with bed_expand_kernel's FP64 arithmetic, so the output bits are the same;
// each lane then writes 8 consecutive samples of hi and of lo per step with
// 16-byte stores (512 contiguous bytes per warp store).
constexpr int kExpandWarps = 8;
constexpr int64_t kBedPad = 32;
constexpr int kExpandMaxStage = 12288;

__device__ __forceinline__ uint16_t bits16(__half h) { return __half_as_ushort(h); }
__device__ __forceinline__ uint16_t bits16(__nv_bfloat16 h) { return __bfloat16_as_ushort(h); }

// With the identity sample map (analysis sample k = file column k), samples
// are decoded two at a time: a 16-entry table per row, indexed by the two
// 2-bit codes, holds the packed hi and lo words of the pair (8 bytes; the
// 128-byte table covers the 32 banks once, so the lookups do not conflict).
template <class T>
__global__ void __launch_bounds__(32 * kExpandWarps, 4)
    bed_expand_warp_kernel(const uint8_t* __restrict__ bed, int64_t bps, int stage_bytes,
                           const int32_t* __restrict__ col, int identity, int n, int k_pad,
                           const int64_t* __restrict__ kept, int64_t m_kept, const double* __restrict__ mu,
                           float scale, T* hi, T* lo) {
  extern __shared__ __align__(16) uint8_t expand_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint2* pair_lut = reinterpret_cast<uint2*>(expand_smem) + warp * 16;
  uint8_t* row_s = expand_smem + kExpandWarps * 16 * sizeof(uint2) + warp * stage_bytes;
  const int64_t nwarps = static_cast<int64_t>(gridDim.x) * kExpandWarps;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * kExpandWarps + warp; r < m_kept; r += nwarps) {
    const int64_t s = __ldg(kept + r);
    const int64_t off0 = s * bps;
    const int64_t a0 = off0 & ~int64_t(15);
    const int skew = static_cast<int>(off0 - a0);
    const int nvec = static_cast<int>((skew + bps + 15) / 16);
    const uint4* src = reinterpret_cast<const uint4*>(bed + a0);
    uint4* dst = reinterpret_cast<uint4*>(row_s);
    __syncwarp();  // the previous row's bytes are no longer read
    for (int v = lane; v < nvec; v += 32) dst[v] = __ldg(src + v);
    // values of the 2-bit codes 00, 01, 10, 11 (A1 count 2, missing, 1, 0)
    uint32_t word = 0;
    if (lane < 4) {
      const int c = lane == 0 ? 2 : (lane == 1 ? -1 : (lane == 2 ? 1 : 0));
      double v = c < 0 ? 0.0 : (static_cast<double>(c) - __ldg(mu + s));
      v *= static_cast<double>(scale);
      const T h = to16<T>(v);
      const T l = to16<T>(v - from16(h));
      word = static_cast<uint32_t>(bits16(h)) | (static_cast<uint32_t>(bits16(l)) << 16);
    }
    const uint32_t w0 = __shfl_sync(0xffffffffu, word, 0), w1 = __shfl_sync(0xffffffffu, word, 1);
    const uint32_t w2 = __shfl_sync(0xffffffffu, word, 2), w3 = __shfl_sync(0xffffffffu, word, 3);
    if (lane < 16) {  // entry (code of the first sample) | (code of the second) << 2
      const int ca = lane & 3, cb = lane >> 2;
      const uint32_t wa = ca == 0 ? w0 : (ca == 1 ? w1 : (ca == 2 ? w2 : w3));
      const uint32_t wb = cb == 0 ? w0 : (cb == 1 ? w1 : (cb == 2 ? w2 : w3));
      pair_lut[lane] = make_uint2((wa & 0xFFFFu) | (wb << 16), (wa >> 16) | (wb & 0xFFFF0000u));
    }
    __syncwarp();  // the staged row and the table are visible to every lane
    for (int k0 = lane * 8; k0 < k_pad; k0 += 256) {
      if (identity && k0 + 8 <= n) {  // samples k0 .. k0+7: bytes k0/4 and k0/4 + 1
        const uint32_t b = static_cast<uint32_t>(row_s[skew + (k0 >> 2)]) |
                           (static_cast<uint32_t>(row_s[skew + (k0 >> 2) + 1]) << 8);
        const uint2 e0 = pair_lut[b & 15u], e1 = pair_lut[(b >> 4) & 15u];
        const uint2 e2 = pair_lut[(b >> 8) & 15u], e3 = pair_lut[(b >> 12) & 15u];
        const int64_t o = r * k_pad + k0;
        *reinterpret_cast<uint4*>(hi + o) = make_uint4(e0.x, e1.x, e2.x, e3.x);
        *reinterpret_cast<uint4*>(lo + o) = make_uint4(e0.y, e1.y, e2.y, e3.y);
        continue;
      }
      uint32_t hw[4], lw[4];
#pragma unroll
      for (int j = 0; j < 8; j += 2) {
        uint32_t pv[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int k = k0 + j + q;
          uint32_t v = 0;  // padding samples: +0 in hi and lo
          if (k < n) {
            const int c = __ldg(col + k);
            const uint32_t code = (static_cast<uint32_t>(row_s[skew + (c >> 2)]) >> ((c & 3) * 2)) & 3u;
            v = code == 0 ? w0 : (code == 1 ? w1 : (code == 2 ? w2 : w3));
          }
          pv[q] = v;
        }
        hw[j / 2] = (pv[0] & 0xFFFFu) | (pv[1] << 16);
        lw[j / 2] = (pv[0] >> 16) | (pv[1] & 0xFFFF0000u);
      }
      const int64_t o = r * k_pad + k0;
      *reinterpret_cast<uint4*>(hi + o) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
      *reinterpret_cast<uint4*>(lo + o) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
  }
}

// The exact SNP operand of the LMM scan, one warp per kept SNP of 2-bit
// rows. With n_ok calls present summing to S and c = n_ok / gcd(S, n_ok),
// the imputed mean S / n_ok times c is an integer, so every value of
// c * dosage is exact in FP16 while c <= 2048 (always when n_ok <= 2048).
// Rows with a mean above 1 are stored as c * (2 - dosage), which keeps the
// missing-call value M = c * mean (or c * (2 - mean)) at most c. Column n
// (the first padding sample, n < k_pad) holds M, against which the gene-side
// operands hold minus their own sum, so that the contraction of a gene-side
// vector v with the row is v . (dosage - mean) / alpha, alpha = +-1 / c.
// SNPs that are not exact are counted in *inexact.
__global__ void raw_operand_kernel(const uint8_t* __restrict__ bed, int64_t bps, const int32_t* __restrict__ col,
                                   int n, int n_full, int k_pad, const int64_t* __restrict__ kept,
                                   int64_t m_kept, const int32_t* __restrict__ n_miss, const double* __restrict__ s1,
                                   __half* raw, float* alpha, unsigned long long* inexact) {
  const int lane = threadIdx.x & 31;
  const int64_t r = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= m_kept) return;
  const int64_t s = __ldg(kept + r);
  // the imputation mean S / n_ok is over every analysis sample (n_full), also
  // when the view (n samples) is a subset of them
  const long long n_ok = n_full - __ldg(n_miss + s);
  const long long S = llrint(__ldg(s1 + s));
  long long a = S, b = n_ok;  // gcd(S, n_ok)
  while (b) {
    const long long t = a % b;
    a = b;
    b = t;
  }
  const long long c = a > 0 ? n_ok / a : 1;
  const bool flip = S > n_ok;
  if (lane == 0) {
    alpha[r] = static_cast<float>((flip ? -1.0 : 1.0) / static_cast<double>(c));
    if (c > 2048) atomicAdd(inexact, 1ull);
  }
  // values of the codes 00, 01, 10, 11 (A1 count 2, missing, 1, 0)
  const float cv = static_cast<float>(c);
  const uint32_t vm = __half_as_ushort(__float2half_rn(static_cast<float>(a > 0 ? (flip ? 2 * c - S / a : S / a)
                                                                                 : 0)));
  const uint32_t v0 = __half_as_ushort(__float2half_rn(flip ? 0.0f : 2.0f * cv));
  const uint32_t v2 = __half_as_ushort(__float2half_rn(cv));
  const uint32_t v3 = __half_as_ushort(__float2half_rn(flip ? 2.0f * cv : 0.0f));
  const uint8_t* row = bed + s * bps;
  for (int k0 = lane * 8; k0 < k_pad; k0 += 256) {
    uint32_t w[4];
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      uint32_t h[2];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int k = k0 + j + t;
        uint32_t v = 0;  // padding samples
        if (k < n) {
          const int cc = __ldg(col + k);
          const uint32_t code = (static_cast<uint32_t>(__ldg(row + (cc >> 2))) >> ((cc & 3) * 2)) & 3u;
          v = code == 0 ? v0 : (code == 1 ? vm : (code == 2 ? v2 : v3));
        } else if (k == n) {
          v = vm;
        }
        h[t] = v;
      }
      w[j / 2] = h[0] | (h[1] << 16);
    }
    *reinterpret_cast<uint4*>(raw + r * k_pad + k0) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

__global__ void bed_dosage_kernel(GenoRows src, const int32_t* __restrict__ col, int n,
                                  const int64_t* __restrict__ kept, int64_t lo, int64_t hi,
                                  const double* __restrict__ mu, double* out) {
  const int64_t total = (hi - lo) * n;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = e / n;
    const int i = static_cast<int>(e - r * n);
    const int64_t s = kept[lo + r];
    const double d = src.dosage(s, col[i]);
    out[e] = isnan(d) ? mu[s] : d;
  }
}

__global__ void bed_dosage_rows_kernel(GenoRows src, const int32_t* __restrict__ col, int n,
                                       const int64_t* __restrict__ kept, const int64_t* __restrict__ rows,
                                       int64_t k, const double* __restrict__ mu, double* out) {
  const int64_t total = k * n;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = e / n;
    const int i = static_cast<int>(e - r * n);
    const int64_t s = kept[rows[r]];
    const double d = src.dosage(s, col[i]);
    out[e] = isnan(d) ? mu[s] : d;
  }
}

}  // namespace

namespace {

void check_samples(const int32_t* sample_col, int n, int n_file, int miss_hand) {
  for (int i = 0; i < n; ++i)
    EQTL_CHECK(sample_col[i] >= 0 && sample_col[i] < n_file, EQTL_E_ARG, "geno_load: sample_col out of range");
  EQTL_CHECK(miss_hand == EQTL_MISS_FILTER || miss_hand == EQTL_MISS_IMPUTE, EQTL_E_ARG, "geno_load: miss_hand");
}

// Shared part of both loads, after the rows are on the device: per-SNP
// statistics and filters, the kept list, and the centred FP16 hi/lo operand.
void geno_decode(eqtl_ctx* ctx, const int32_t* sample_col, int miss_hand, double max_miss, double maf_min) {
  Geno& g = ctx->geno;
  cudaStream_t st = ctx->stream;
  const int64_t m = g.m_all;
  const int n = g.n;
  ctx->rot.m = 0;  // rotated genotypes belong to the previous genotypes
  ctx->rot.raw_m = -1;
  ctx->glm_ops.m = 0;
  g.k_pad = ((n + 63) / 64) * 64;
  g.col.upload(sample_col, n, st);
  g.col_identity = true;
  for (int i = 0; i < n; ++i) g.col_identity = g.col_identity && sample_col[i] == i;
  g.n_miss.alloc(m);
  g.s1.alloc(m);
  g.s2.alloc(m);
  g.pass.alloc(m);
  g.af.alloc(m);
  g.mu.alloc(m);
  const GenoRows src = g.rows();
  StageScope timer(ctx, EQTL_STAGE_DECODE);
  if (m > 0) {
    ++ctx->launches;
    const int per_block = 8;
    bed_stats_kernel<<<static_cast<unsigned>((m + per_block - 1) / per_block), 32 * per_block, 0, st>>>(
        src, m, g.col.p, n, miss_hand, max_miss, maf_min, g.n_miss.p, g.s1.p, g.s2.p, g.pass.p, g.af.p, g.mu.p);
    EQTL_CUDA(cudaGetLastError());
  }
  std::vector<uint8_t> pass(m);
  g.mu_h.resize(m);
  g.af_h.resize(m);
  g.n_miss_h.resize(m);
  g.pass.download(pass.data(), m, st);
  g.mu.download(g.mu_h.data(), m, st);
  g.af.download(g.af_h.data(), m, st);
  g.n_miss.download(g.n_miss_h.data(), m, st);
  EQTL_CUDA(cudaStreamSynchronize(st));
  g.kept_h.clear();
  for (int64_t s = 0; s < m; ++s)
    if (pass[s]) g.kept_h.push_back(s);
  g.m = static_cast<int64_t>(g.kept_h.size());
  g.kept.upload(g.kept_h.data(), g.kept_h.size(), st);
  g.n_full = n;
  g.col_full_h.assign(sample_col, sample_col + n);
  g.subset = false;
  geno_expand(ctx);
}

}  // namespace

// The centred FP16 (or BF16) hi/lo operand of the kept SNPs over the current
// sample view (g.col, g.n), missing calls at the imputation mean.
void geno_expand(eqtl_ctx* ctx) {
  Geno& g = ctx->geno;
  cudaStream_t st = ctx->stream;
  const int n = g.n;
  const GenoRows src = g.rows();
  const size_t elems = static_cast<size_t>(g.m) * g.k_pad;
  g.gc_hi.alloc(elems);
  g.gc_lo.alloc(elems);
  const int64_t bytes_per_snp = g.bytes_per_snp;
  const int stage = static_cast<int>(((bytes_per_snp + 30) / 16) * 16);
  if (g.m > 0 && !g.dense && stage <= kExpandMaxStage) {
    const int smem = stage * kExpandWarps + kExpandWarps * 16 * static_cast<int>(sizeof(uint2));
    const int identity = g.col_identity ? 1 : 0;
    const unsigned blocks = static_cast<unsigned>(
        std::min<int64_t>((g.m + kExpandWarps - 1) / kExpandWarps, static_cast<int64_t>(ctx->sm_count) * 16));
    ++ctx->launches;
    if (ctx->precision == EQTL_PREC_SPLIT_BF16) {
      auto kern = bed_expand_warp_kernel<__nv_bfloat16>;
      EQTL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      kern<<<blocks, 32 * kExpandWarps, smem, st>>>(g.bed.p, bytes_per_snp, stage, g.col.p, identity, n, g.k_pad,
                                                    g.kept.p, g.m, g.mu.p, kGcScale,
                                                    reinterpret_cast<__nv_bfloat16*>(g.gc_hi.p),
                                                    reinterpret_cast<__nv_bfloat16*>(g.gc_lo.p));
    } else {
      auto kern = bed_expand_warp_kernel<__half>;
      EQTL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      kern<<<blocks, 32 * kExpandWarps, smem, st>>>(g.bed.p, bytes_per_snp, stage, g.col.p, identity, n, g.k_pad,
                                                    g.kept.p, g.m, g.mu.p, kGcScale, g.gc_hi.p, g.gc_lo.p);
    }
    EQTL_CUDA(cudaGetLastError());
  } else if (g.m > 0) {
    // FP32 dosage rows, or 2-bit rows too long to stage (more than ~49,000
    // samples in the file)
    dim3 grid((g.k_pad + 255) / 256, static_cast<unsigned>(g.m < 65535 ? g.m : 65535));
    ++ctx->launches;
    if (ctx->precision == EQTL_PREC_SPLIT_BF16) {
      bed_expand_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(
          src, g.col.p, n, g.k_pad, g.kept.p, g.m, g.mu.p, kGcScale, reinterpret_cast<__nv_bfloat16*>(g.gc_hi.p),
          reinterpret_cast<__nv_bfloat16*>(g.gc_lo.p));
    } else {
      bed_expand_kernel<__half><<<grid, 256, 0, st>>>(src, g.col.p, n, g.k_pad, g.kept.p, g.m, g.mu.p, kGcScale,
                                                       g.gc_hi.p, g.gc_lo.p);
    }
    EQTL_CUDA(cudaGetLastError());
  }
  EQTL_CUDA(cudaStreamSynchronize(st));
}

namespace {
// Per kept SNP, one warp: sums of the imputed dosage and of its square over
// the view's samples (the gate of a per-gene sample subset).
__global__ void view_sums_kernel(GenoRows src, const int32_t* __restrict__ col, int n,
                                 const int64_t* __restrict__ kept, int64_t m, const double* __restrict__ mu,
                                 double* vs1, double* vs2) {
  const int lane = threadIdx.x & 31;
  const int64_t r = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= m) return;
  const int64_t s = kept[r];
  const double mus = mu[s];
  double a = 0.0, b = 0.0;
  for (int i = lane; i < n; i += 32) {
    const double d0 = src.dosage(s, __ldg(col + i));
    const double d = isnan(d0) ? mus : d0;
    a += d;
    b += d * d;
  }
  for (int o = 16; o; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    vs1[s] = a;
    vs2[s] = b;
  }
}
}  // namespace

void geno_subset(eqtl_ctx* ctx, const int32_t* idx, int n_sub) {
  Geno& g = ctx->geno;
  EQTL_CHECK(g.m_all > 0 && g.n_full > 0, EQTL_E_STATE, "geno_subset: no genotypes loaded");
  cudaStream_t st = ctx->stream;
  std::vector<int32_t> col;
  if (idx) {
    EQTL_CHECK(n_sub >= 1 && n_sub <= g.n_full, EQTL_E_ARG, "geno_subset: bad subset size");
    col.resize(n_sub);
    for (int i = 0; i < n_sub; ++i) {
      EQTL_CHECK(idx[i] >= 0 && idx[i] < g.n_full && (i == 0 || idx[i] > idx[i - 1]), EQTL_E_ARG,
                 "geno_subset: indices must be increasing analysis-sample positions");
      col[i] = g.col_full_h[idx[i]];
    }
  } else {
    col = g.col_full_h;
  }
  const int n = static_cast<int>(col.size());
  ctx->rot.m = 0;  // operands of the previous view
  ctx->rot.raw_m = -1;
  ctx->glm_ops.m = 0;
  g.n = n;
  g.k_pad = ((n + 63) / 64) * 64;
  g.col.upload(col.data(), col.size(), st);
  g.col_identity = true;
  for (int i = 0; i < n; ++i) g.col_identity = g.col_identity && col[i] == i;
  g.subset = idx != nullptr;
  if (g.subset) {
    g.vs1.alloc(static_cast<size_t>(g.m_all));
    g.vs2.alloc(static_cast<size_t>(g.m_all));
    g.vzero.alloc(static_cast<size_t>(g.m_all));
    g.vzero.zero(st);
    if (g.m > 0) {
      ++ctx->launches;
      view_sums_kernel<<<static_cast<unsigned>((g.m + 7) / 8), 256, 0, st>>>(g.rows(), g.col.p, n, g.kept.p, g.m,
                                                                           g.mu.p, g.vs1.p, g.vs2.p);
      EQTL_CUDA(cudaGetLastError());
    }
  }
  geno_expand(ctx);
}

void geno_load(eqtl_ctx* ctx, const uint8_t* rows, int64_t m, int64_t bytes_per_snp, int n_file,
               const int32_t* sample_col, int n, int miss_hand, double max_miss, double maf_min) {
  EQTL_CHECK(m >= 0 && n > 0 && n_file > 0, EQTL_E_ARG, "geno_load: bad sizes");
  EQTL_CHECK(bytes_per_snp == (n_file + 3) / 4, EQTL_E_ARG, "geno_load: bytes_per_snp != ceil(n_file/4)");
  check_samples(sample_col, n, n_file, miss_hand);
  Geno& g = ctx->geno;
  cudaStream_t st = ctx->stream;
  g.m_all = m;
  g.n = n;
  g.n_file = n_file;
  g.bytes_per_snp = bytes_per_snp;
  g.dense = false;
  // kBedPad bytes past the last row: bed_expand_warp_kernel stages rows in
  // 16-byte vectors from the boundary at or below each row start
  g.bed.alloc(static_cast<size_t>(m * bytes_per_snp + kBedPad));
  if (m > 0)
    EQTL_CUDA(cudaMemcpyAsync(g.bed.p, rows, static_cast<size_t>(m * bytes_per_snp), cudaMemcpyHostToDevice, st));
  geno_decode(ctx, sample_col, miss_hand, max_miss, maf_min);
}

void geno_load_dosage(eqtl_ctx* ctx, const float* ds, int64_t m, int n_file, const int32_t* sample_col, int n,
                      int miss_hand, double max_miss, double maf_min) {
  EQTL_CHECK(m >= 0 && n > 0 && n_file > 0, EQTL_E_ARG, "geno_load_dosage: bad sizes");
  check_samples(sample_col, n, n_file, miss_hand);
  Geno& g = ctx->geno;
  g.m_all = m;
  g.n = n;
  g.n_file = n_file;
  g.bytes_per_snp = (n_file + 3) / 4;
  g.dense = true;
  g.ds.upload(ds, static_cast<size_t>(m) * n_file, ctx->stream);
  geno_decode(ctx, sample_col, miss_hand, max_miss, maf_min);
}

// Builds the exact SNP operand of the LMM scan for the loaded 2-bit rows
// (raw_operand_kernel) once per genotype load; returns whether every kept SNP
// is exact (false for FP32 dosage rows, which it does not build, and when
// n leaves no padding sample column).
bool geno_raw_operand(eqtl_ctx* ctx) {
  Geno& g = ctx->geno;
  Rotated& R = ctx->rot;
  if (R.raw_m == g.m && R.raw.p) return R.raw_exact;
  R.raw_exact = false;
  if (g.dense || g.n >= g.k_pad) return false;
  cudaStream_t st = ctx->stream;
  const int64_t m = g.m;
  R.raw.alloc(std::max<size_t>(1, static_cast<size_t>(m) * g.k_pad));
  // the scan epilogues read alpha 16 SNPs at a time, up to the end of the
  // last tile
  R.alpha.alloc(static_cast<size_t>(((m + 255) / 256 + 1) * 256));
  EQTL_CUDA(cudaMemsetAsync(R.alpha.p, 0, sizeof(float) * R.alpha.n, st));
  DevBuf<unsigned long long>& cnt = ctx->ws.raw_inexact;
  cnt.alloc(1);
  cnt.zero(st);
  if (m > 0) {
    ++ctx->launches;
    const int per_block = 8;
    raw_operand_kernel<<<static_cast<unsigned>((m + per_block - 1) / per_block), 32 * per_block, 0, st>>>(
        g.bed.p, g.bytes_per_snp, g.col.p, g.n, g.n_full, g.k_pad, g.kept.p, m, g.n_miss.p, g.s1.p, R.raw.p,
        R.alpha.p, cnt.p);
    EQTL_CUDA(cudaGetLastError());
  }
  unsigned long long bad = 0;
  cnt.download(&bad, 1, st);
  EQTL_CUDA(cudaStreamSynchronize(st));
  R.raw_m = m;
  R.raw_exact = bad == 0;
  return R.raw_exact;
}

void geno_dosage(eqtl_ctx* ctx, int64_t lo, int64_t hi, double* out_host) {
  Geno& g = ctx->geno;
  EQTL_CHECK(lo >= 0 && hi <= g.m && lo <= hi, EQTL_E_ARG, "geno_dosage: range outside kept SNPs");
  if (hi == lo) return;
  DevBuf<double> d;
  d.alloc(static_cast<size_t>(hi - lo) * g.n);
  ++ctx->launches;
  bed_dosage_kernel<<<1184, 256, 0, ctx->stream>>>(g.rows(), g.col.p, g.n, g.kept.p, lo, hi, g.mu.p, d.p);
  EQTL_CUDA(cudaGetLastError());
  d.download(out_host, d.n, ctx->stream);
  EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
}

void geno_dosage_rows(eqtl_ctx* ctx, const int64_t* rows, int64_t k, double* out_host) {
  Geno& g = ctx->geno;
  for (int64_t r = 0; r < k; ++r)
    EQTL_CHECK(rows[r] >= 0 && rows[r] < g.m, EQTL_E_ARG, "geno_dosage_rows: index outside the kept SNPs");
  if (k == 0) return;
  DevBuf<int64_t> d_rows;
  DevBuf<double> d;
  d_rows.upload(rows, k, ctx->stream);
  d.alloc(static_cast<size_t>(k) * g.n);
  ++ctx->launches;
  bed_dosage_rows_kernel<<<1184, 256, 0, ctx->stream>>>(g.rows(), g.col.p, g.n, g.kept.p, d_rows.p, k, g.mu.p,
                                                        d.p);
  EQTL_CUDA(cudaGetLastError());
  d.download(out_host, d.n, ctx->stream);
  EQTL_CUDA(cudaStreamSynchronize(ctx->stream));
}

}  // namespace eqtl
