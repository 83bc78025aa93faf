// Plain FP32 CUDA-core form of the tile contraction: the comparator the
// tensor-core kernel is measured against. Same operands (each hi/lo FP16
// pair is summed once into an exact FP32 value), same epilogue functor, FP32
// fused multiply-adds on the CUDA cores instead of tcgen05.mma.
//
// Block = 128 threads = 128 gene rows x 16 SNP columns; K is staged through
// shared memory in chunks of 16: the gene-side rows transposed so every
// thread reads its own row conflict-free, the SNP-side rows as broadcasts.
#pragma once
#include "tile_gemm.cuh"

namespace eqtl {
namespace dev {

constexpr int kSimtK = 16;
constexpr int kSimtN = 16;

template <int NACC, class Epi>
__global__ void __launch_bounds__(128) simt_tile_kernel(const __half* const* __restrict__ a_hi,
                                                        const __half* const* __restrict__ a_lo, int rows_a,
                                                        const __half* const* __restrict__ b_hi,
                                                        const __half* const* __restrict__ b_lo, int64_t rows_b,
                                                        int k_pad, int4 bsel, const TileShape sh,
                                                        const __grid_constant__ typename Epi::Params ep) {
  __shared__ float sa[NACC][kSimtK][129];
  __shared__ float sb[2][kSimtN][kSimtK + 1];
  const int tid = threadIdx.x;
  const int ga = blockIdx.y * 128;
  const int64_t sb0 = static_cast<int64_t>(blockIdx.x) * kSimtN;
  const int bs[4] = {bsel.x, bsel.y, bsel.z, bsel.w};
  float acc[NACC][kSimtN];
#pragma unroll
  for (int j = 0; j < NACC; ++j)
#pragma unroll
    for (int c = 0; c < kSimtN; ++c) acc[j][c] = 0.0f;
  for (int k0 = 0; k0 < k_pad; k0 += kSimtK) {
    // gene-side rows: 128 rows x 32 k per accumulator
    for (int j = 0; j < NACC; ++j) {
      for (int e = tid; e < 128 * kSimtK; e += 128) {
        const int r = e / kSimtK, k = e % kSimtK;
        float v = 0.0f;
        if (ga + r < rows_a) {
          const int64_t idx = static_cast<int64_t>(ga + r) * k_pad + k0 + k;
          v = __half2float(a_hi[j][idx]) + __half2float(a_lo[j][idx]);
        }
        sa[j][k][r] = v;
      }
    }
    for (int q = 0; q < 2; ++q) {
      for (int e = tid; e < kSimtN * kSimtK; e += 128) {
        const int r = e / kSimtK, k = e % kSimtK;
        float v = 0.0f;
        if (sb0 + r < rows_b && b_hi[q]) {
          const int64_t idx = (sb0 + r) * k_pad + k0 + k;
          v = __half2float(b_hi[q][idx]) + __half2float(b_lo[q][idx]);
        }
        sb[q][r][k] = v;
      }
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < kSimtK; ++k) {
      float av[NACC];
#pragma unroll
      for (int j = 0; j < NACC; ++j) av[j] = sa[j][k][tid];
#pragma unroll
      for (int c = 0; c < kSimtN; ++c) {
        const float b0 = sb[0][c][k], b1 = sb[1][c][k];
#pragma unroll
        for (int j = 0; j < NACC; ++j) acc[j][c] = fmaf(av[j], bs[j] ? b1 : b0, acc[j][c]);
      }
    }
    __syncthreads();
  }
  Epi epi(ep, sh, nullptr);
  epi.init(tid, 128);
  epi.begin_tile(ga + tid, sb0);
  epi.template chunk<NACC>(0, acc);
  epi.end_tile();
  epi.finish();
}

}  // namespace dev
}  // namespace eqtl
