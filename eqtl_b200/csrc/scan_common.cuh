// Pieces shared by the scan epilogues: per-gene / per-SNP window logic
// (include/eqtl/scan_common.hpp:58-69), the per-gene reduction state
// (n_tested, ACAT tan sum, best key) and candidate compaction.
#pragma once
#include "tdist.cuh"
#include "tile_gemm.cuh"

namespace eqtl {
namespace dev {

enum WinMode : int { kWinNone = 0, kWinExclude = 1, kWinInclude = 2 };

// high bit of a candidate's SNP field: its ACAT term is added on the host
constexpr uint32_t kCandDeferred = 0x80000000u;
constexpr uint32_t kCandTiny = 0x40000000u;  // deferred for 0 < |t| < tiny_t (kept SNP indices < 2^30)

struct GeneOut {
  double* acat_sum;            // [G] sum of tan((1/2 - p) pi)
  int* acat_used;              // [G]
  int* n_tested;               // [G]
  unsigned long long* best;    // [G] best_key (min)
  int2* cand;                  // (gene, kept snp | kCandDeferred) with |t| >= t_cand or a deferred ACAT term
  unsigned int* cand_count;
  unsigned int cand_cap;
};

struct Windows {
  int mode;
  const int32_t* gene_chrom;
  const int64_t* gene_lo;
  const int64_t* gene_hi;
  const int32_t* snp_chrom;
  const int64_t* snp_pos;
  // per block of 16 kept SNPs (b = s / 16, covering the padded tiles): the
  // block's chromosome (-1 where it mixes chromosomes or lies past the last
  // SNP) and its smallest and largest position
  const int32_t* blk_chrom;
  const int64_t* blk_lo;
  const int64_t* blk_hi;
};

// Per-thread (= per gene row) running state inside one tile.
struct GeneAcc {
  double acat = 0.0;
  int used = 0;
  int tested = 0;
  unsigned long long best = ~0ull;
  // FP32 sum of the ACAT terms of the current chunk of add_screen pairs, and
  // its best key and SNP (end_chunk folds them into acat and best)
  float chunk_acat = 0.0f;
  float chunk_key = -1.0f;
  uint32_t chunk_snp = 0;
  int chrom = -1;
  int64_t lo = 0, hi = -1;

  __device__ __forceinline__ void reset() {
    acat = 0.0;
    used = 0;
    tested = 0;
    best = ~0ull;
    chunk_acat = 0.0f;
    chunk_key = -1.0f;
  }
  __device__ __forceinline__ void load_window(const Windows& w, int g) {
    if (w.mode != kWinNone) {
      chrom = w.gene_chrom[g];
      lo = w.gene_lo[g];
      hi = w.gene_hi[g];
    }
  }
  // true if no SNP of the 16-SNP block starting at s0 (a multiple of 16) can
  // lie in this gene's window: a gene without one, or a block on another
  // chromosome or wholly before or after it
  __device__ __forceinline__ bool chunk_clear(const Windows& w, int64_t s0) const {
    if (chrom < 0) return true;
    const int64_t b = s0 >> 4;
    const int32_t c = __ldg(w.blk_chrom + b);
    return c >= 0 && (c != chrom || __ldg(w.blk_hi + b) < lo || __ldg(w.blk_lo + b) > hi);
  }
  // true if the (gene, snp) pair is part of this scope
  __device__ __forceinline__ bool in_scope(const Windows& w, int64_t s) const {
    if (w.mode == kWinNone) return true;
    const bool inwin = chrom >= 0 && __ldg(w.snp_chrom + s) == chrom && __ldg(w.snp_pos + s) >= lo &&
                       __ldg(w.snp_pos + s) <= hi;
    return w.mode == kWinExclude ? !inwin : inwin;
  }
  // Update for one (gene, SNP) pair; `valid` masks pairs outside the scan
  // (SNP gate, window, padding). Kept as predicated branches: the
  // select form `acat += u ? term : 0.0` produced zero sums on sm_100a.
  __device__ __forceinline__ void add_masked(const TailOut& o, int64_t s, bool valid) {
    if (valid) {
      ++tested;
      if (o.use_acat) {
        acat += o.term;
        ++used;
      }
      const unsigned long long k = best_key(o.neglog10p, static_cast<uint32_t>(s));
      best = k < best ? k : best;
    }
  }
  // The same for the epilogues' ACAT screen (best SNP keyed on the screen's
  // key, t^2 in the scans). Pairs come in chunks of up to 16 SNPs; the terms
  // of a chunk are summed in FP32 (the error is ~1e-6 of the chunk's largest
  // term, below the screen's own) and added to the FP64 total by end_chunk.
  // A chunk's pairs come in increasing SNP order, so its best is the first
  // pair with the largest key (strict >), and the 64-bit key that breaks ties
  // by SNP index across chunks is formed once per chunk.
  __device__ __forceinline__ void add_screen(const ScreenOut& o, int64_t s, bool valid) {
    if (valid) {
      ++tested;
      if (o.use_acat) {
        chunk_acat += o.term;
        ++used;
      }
      if (o.key > chunk_key) {
        chunk_key = o.key;
        chunk_snp = static_cast<uint32_t>(s);
      }
    }
  }
  __device__ __forceinline__ void end_chunk() {
    acat += static_cast<double>(chunk_acat);
    chunk_acat = 0.0f;
    if (chunk_key >= 0.0f) {
      const unsigned long long k = best_key(chunk_key, chunk_snp);
      best = k < best ? k : best;
      chunk_key = -1.0f;
    }
  }
  __device__ __forceinline__ void add(const TailOut& o, int64_t s) {
    ++tested;
    if (o.use_acat) {
      acat += o.term;  // 0 for deferred terms
      ++used;
    }
    const unsigned long long k = best_key(o.neglog10p, static_cast<uint32_t>(s));
    best = k < best ? k : best;
  }
  __device__ __forceinline__ void flush(const GeneOut& out, int g) const {
    if (tested == 0) return;
    atomicAdd(out.acat_sum + g, acat);
    atomicAdd(out.acat_used + g, used);
    atomicAdd(out.n_tested + g, tested);
    atomicMin(out.best + g, best);
  }
};

__device__ __forceinline__ void named_barrier_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// 16 per-SNP flag bytes starting at a multiple of 16 (arrays padded to 16).
__device__ __forceinline__ void load_flags16(const uint8_t* p, uint32_t (&w)[4]) {
  const uint4 v = *reinterpret_cast<const uint4*>(p);
  w[0] = v.x;
  w[1] = v.y;
  w[2] = v.z;
  w[3] = v.w;
}
__device__ __forceinline__ bool flag16(const uint32_t (&w)[4], int j) { return (w[j >> 2] >> (8 * (j & 3))) & 0xFFu; }

// 16 floats starting at a multiple of 16 of an array padded past its last
// tile (four 16-byte loads).
__device__ __forceinline__ void load16(const float* p, float (&v)[16]) {
  const float4* p4 = reinterpret_cast<const float4*>(p);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float4 x = __ldg(p4 + q);
    v[4 * q] = x.x;
    v[4 * q + 1] = x.y;
    v[4 * q + 2] = x.z;
    v[4 * q + 3] = x.w;
  }
}

__device__ __forceinline__ void emit_candidate(const GeneOut& out, int g, int64_t s, bool deferred, bool tiny) {
  const unsigned int idx = atomicAdd(out.cand_count, 1u);
  if (idx < out.cand_cap)
    out.cand[idx] = make_int2(g, static_cast<int>(static_cast<uint32_t>(s) | (deferred ? kCandDeferred : 0u) |
                                                  (tiny ? kCandTiny : 0u)));
}

// The ACAT screen of one gene's 16 pairs s0 .. s0 + 15 with the per-interval
// cubics (acat_screen_u's lt_u branch, T.lt_u set), for epilogues whose u =
// t^2 is never NaN (a pair outside the scan, or with p = 1, has u = 0). With
// u_tiny > 0:
//   tiny      0 < u < u_tiny         deferred   tiny or u >= u_defer
//   ACAT      u_tiny <= u < u_defer  candidate  u >= min(u_cand, u_defer) or tiny
// The counts, the FP32 term sum and the chunk's best go into acc without
// per-pair flag structs; candidates are emitted as they are found.
__device__ __forceinline__ void screen16_cubic(const TTable& tt, const float (&u)[16], const bool (&valid)[16],
                                               float u_cand, const GeneOut& out, int gene, int64_t s0,
                                               GeneAcc& acc) {
  const float uc = fminf(u_cand, tt.u_defer);
  const float cmax = static_cast<float>(tt.na) - 1e-3f, tmax = static_cast<float>(tt.nq) - 1e-3f;
  float sum = 0.0f, bkey = -1.0f;
  int ntest = 0, nused = 0, bj = 0;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const float uj = u[j];
    const bool central = uj <= tt.uq0;
    const float x = fminf(central ? uj * tt.dqc_inv : (uj - tt.uq0) * tt.dq_inv, central ? cmax : tmax);
    const int i = static_cast<int>(x);
    const float f = x - static_cast<float>(i);
    const float4 a = (central ? tt.c1q : tt.ltq)[i];
    const float y = fmaf(fmaf(fmaf(a.w, f, a.z), f, a.y), f, a.x);
    const float term = central ? y * rsqrtf(uj) : y;
    const bool lo = uj < tt.u_tiny;
    const bool use = !lo && uj < tt.u_defer;
    sum += use ? term : 0.0f;
    nused += use ? 1 : 0;
    ntest += valid[j] ? 1 : 0;
    const float key = valid[j] ? uj : -1.0f;
    bj = key > bkey ? j : bj;
    bkey = fmaxf(key, bkey);
    if (uj >= uc || (lo && uj > 0.0f)) emit_candidate(out, gene, s0 + j, lo || uj >= tt.u_defer, lo);
  }
  acc.tested += ntest;
  acc.used += nused;
  acc.chunk_acat += sum;
  if (bkey >= 0.0f && bkey > acc.chunk_key) {
    acc.chunk_key = bkey;
    acc.chunk_snp = static_cast<uint32_t>(s0 + bj);
  }
  acc.end_chunk();
}

}  // namespace dev
}  // namespace eqtl
