// Plain FP32 CUDA-core form of the LMM scan contraction: the comparator the
// tensor-core kernel is measured against. Same method and epilogue functor,
// FP32 operands (each FP16 hi/lo pair summed once into an FP32 copy before the
// scan), FP32 fused multiply-adds on the CUDA cores instead of tcgen05.mma.
//
// A register-blocked SGEMM form: a CTA of 256 threads computes a tile of 64
// gene rows x 128 SNP columns for all NACC accumulators; K goes through
// shared memory in chunks of 16 (double-buffered, the next chunk's global
// loads in flight while the current one is used). Each thread keeps
// NACC x 4 genes x 8 SNPs accumulators in registers and per K step reads
// NACC + 4 float4 from shared memory for 32 NACC FMAs. After the K loop the
// accumulators go through shared memory so that each thread hands 16
// contiguous SNP columns of one gene at a time to the epilogue functor.
//
// The accumulator pattern is the LMM scan's: accumulator 0 (gg) reads the
// second SNP-side operand (Gt^2), every other one the first (Gt).
#pragma once
#include "tile_gemm.cuh"

namespace eqtl {
namespace dev {

constexpr int kSimtBM = 64;    // gene rows per CTA
constexpr int kSimtBN = 128;   // SNP columns per CTA
constexpr int kSimtBK = 16;    // K per shared-memory chunk
constexpr int kSimtAPad = kSimtBM + 4;
constexpr int kSimtBPad = kSimtBN + 4;
constexpr int kSimtThreads = 256;

template <int NACC>
struct SimtCfg {
  static constexpr int A_FLOATS = NACC * kSimtBK * kSimtAPad;
  static constexpr int B_FLOATS = 2 * kSimtBK * kSimtBPad;
  static constexpr int STAGE_FLOATS = A_FLOATS + B_FLOATS;
  static constexpr int C_FLOATS = NACC * kSimtBM * (kSimtBN + 1);
  static constexpr int SMEM_BYTES =
      4 * (2 * STAGE_FLOATS > C_FLOATS ? 2 * STAGE_FLOATS : C_FLOATS);
};

// a32[j]: gene-side operand of accumulator j [rows_a, k_pad] FP32; b0, b1:
// SNP-side operands [rows_b, k_pad] FP32 (k_pad a multiple of 16).
template <int NACC, class Epi>
__global__ void __launch_bounds__(kSimtThreads, 1)
    simt_tile_kernel(const float* const* __restrict__ a32, int rows_a, const float* __restrict__ b0,
                     const float* __restrict__ b1, int64_t rows_b, int k_pad, const TileShape sh,
                     const __grid_constant__ typename Epi::Params ep) {
  using C = SimtCfg<NACC>;
  extern __shared__ float4 simt_smem4[];
  float* smem = reinterpret_cast<float*>(simt_smem4);
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int ga = blockIdx.y * kSimtBM;
  const int64_t sb0 = static_cast<int64_t>(blockIdx.x) * kSimtBN;
  // global -> shared staging: A: one float4 per thread and accumulator
  // (row tid / 4, k (tid % 4) * 4); B: two float4 per operand (rows tid / 4
  // and tid / 4 + 64)
  const int lrow = tid >> 2, lk = (tid & 3) * 4;
  const float* ap[NACC];
#pragma unroll
  for (int j = 0; j < NACC; ++j)
    ap[j] = ga + lrow < rows_a ? a32[j] + static_cast<int64_t>(ga + lrow) * k_pad + lk : nullptr;
  const float* bp[2][2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int64_t r = sb0 + lrow + 64 * h;
    bp[0][h] = r < rows_b ? b0 + r * k_pad + lk : nullptr;
    bp[1][h] = r < rows_b ? b1 + r * k_pad + lk : nullptr;
  }
  float4 ra[NACC], rb[2][2];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int j = 0; j < NACC; ++j)
      ra[j] = ap[j] ? __ldg(reinterpret_cast<const float4*>(ap[j] + k0)) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h)
        rb[q][h] = bp[q][h] ? __ldg(reinterpret_cast<const float4*>(bp[q][h] + k0)) : make_float4(0.f, 0.f, 0.f, 0.f);
  };
  auto stash = [&](int buf) {
    float* sa = smem + buf * C::STAGE_FLOATS;
    float* sbm = sa + C::A_FLOATS;
#pragma unroll
    for (int j = 0; j < NACC; ++j) {
      float* d = sa + j * kSimtBK * kSimtAPad + lrow;
      d[(lk + 0) * kSimtAPad] = ra[j].x;
      d[(lk + 1) * kSimtAPad] = ra[j].y;
      d[(lk + 2) * kSimtAPad] = ra[j].z;
      d[(lk + 3) * kSimtAPad] = ra[j].w;
    }
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float* d = sbm + q * kSimtBK * kSimtBPad + lrow + 64 * h;
        d[(lk + 0) * kSimtBPad] = rb[q][h].x;
        d[(lk + 1) * kSimtBPad] = rb[q][h].y;
        d[(lk + 2) * kSimtBPad] = rb[q][h].z;
        d[(lk + 3) * kSimtBPad] = rb[q][h].w;
      }
  };
  float acc[NACC][4][8];
#pragma unroll
  for (int j = 0; j < NACC; ++j)
#pragma unroll
    for (int g = 0; g < 4; ++g)
#pragma unroll
      for (int s = 0; s < 8; ++s) acc[j][g][s] = 0.0f;
  const int nk = k_pad / kSimtBK;
  fetch(0);
  stash(0);
  __syncthreads();
  for (int kc = 0; kc < nk; ++kc) {
    const int buf = kc & 1;
    if (kc + 1 < nk) fetch((kc + 1) * kSimtBK);
    const float* sa = smem + buf * C::STAGE_FLOATS;
    const float* sbm = sa + C::A_FLOATS;
#pragma unroll
    for (int k = 0; k < kSimtBK; ++k) {
      float4 av[NACC];
#pragma unroll
      for (int j = 0; j < NACC; ++j)
        av[j] = *reinterpret_cast<const float4*>(sa + (j * kSimtBK + k) * kSimtAPad + ty * 4);
      float bv[2][8];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const float4 lo = *reinterpret_cast<const float4*>(sbm + (q * kSimtBK + k) * kSimtBPad + tx * 4);
        const float4 hi = *reinterpret_cast<const float4*>(sbm + (q * kSimtBK + k) * kSimtBPad + 64 + tx * 4);
        bv[q][0] = lo.x; bv[q][1] = lo.y; bv[q][2] = lo.z; bv[q][3] = lo.w;
        bv[q][4] = hi.x; bv[q][5] = hi.y; bv[q][6] = hi.z; bv[q][7] = hi.w;
      }
#pragma unroll
      for (int j = 0; j < NACC; ++j) {
        const float a4[4] = {av[j].x, av[j].y, av[j].z, av[j].w};
        const int q = j == 0 ? 1 : 0;
#pragma unroll
        for (int g = 0; g < 4; ++g)
#pragma unroll
          for (int s = 0; s < 8; ++s) acc[j][g][s] = fmaf(a4[g], bv[q][s], acc[j][g][s]);
      }
    }
    if (kc + 1 < nk) stash(buf ^ 1);
    __syncthreads();
  }
  // accumulators -> shared memory [j][gene][snp], then 16 contiguous SNPs of
  // one gene per epilogue call
  float* cs = smem;
#pragma unroll
  for (int j = 0; j < NACC; ++j)
#pragma unroll
    for (int g = 0; g < 4; ++g)
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        const int col = s < 4 ? tx * 4 + s : 64 + tx * 4 + (s - 4);
        cs[(j * kSimtBM + ty * 4 + g) * (kSimtBN + 1) + col] = acc[j][g][s];
      }
  __syncthreads();
  Epi epi(ep, sh, nullptr);
  epi.init(tid, kSimtThreads);
  const int erow = tid >> 2, ecol = (tid & 3) * 32;
  epi.begin_tile(ga + erow, sb0);
#pragma unroll 1
  for (int c = ecol; c < ecol + 32; c += 16) {
    float v[NACC][16];
#pragma unroll
    for (int j = 0; j < NACC; ++j)
#pragma unroll
      for (int i = 0; i < 16; ++i) v[j][i] = cs[(j * kSimtBM + erow) * (kSimtBN + 1) + c + i];
    epi.template chunk<NACC>(c, v);
  }
  epi.end_tile();
  epi.finish();
}

// hi + lo of an FP16 pair operand into one FP32 copy
__global__ void sum_split_kernel(const __half* __restrict__ hi, const __half* __restrict__ lo, int64_t count,
                                 float* out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = __half2float(hi[i]) + __half2float(lo[i]);
}

}  // namespace dev
}  // namespace eqtl
