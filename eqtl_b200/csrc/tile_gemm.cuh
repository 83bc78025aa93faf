// Persistent, warp-specialised tcgen05 tile kernel shared by every scan
// contraction. It computes, for a tile of 128 gene-side rows (M) and NT
// SNP-side rows (N), up to NACC FP32 accumulators
//
//     acc[j][g, s] = sum_k  A_j[g, k] * B_{bsel[j]}[s, k]
//
// where every operand is held as an FP16 (or BF16) hi/lo pair and the
// product is formed as hi*hi + hi*lo + lo*hi (the lo*lo term is below FP32
// rounding). Both operands are K-major in global memory (row = gene or SNP,
// K = sample index, zero-padded to a multiple of 64).
//
// Roles (64 + 32 * kEpiWarps threads):
//   warp 0      TMA producer: one elected lane streams 64-wide K chunks of
//               (A_hi, A_lo, B_hi, B_lo) into a STAGES-deep smem ring.
//   warp 1      TMEM owner + MMA issuer: one elected lane issues
//               tcgen05.mma (M=128, N=NT, K=16) into TMEM accumulators and
//               releases ring slots with tcgen05.commit.
//   warps 2..    epilogue (kEpiWarps): each thread owns one accumulator row
//               (TMEM lane; warp w may only read lane quarter w % 4, so the
//               warps come in groups of four that split the columns), reads
//               16-column chunks with tcgen05.ld and hands them to the
//               scan-specific Epi functor, which never writes the M x N
//               matrix to HBM.
// TMEM is used as a ring of NT-column slots: the MMAs of the next tile start
// in whichever slots the epilogue has already read, so the epilogue of tile
// i overlaps the MMAs of tile i+1 (fully when 2 * NACC <= slots, for its
// first accumulators otherwise).
// A tile may need more accumulators than TMEM holds at once (the LMM with p
// covariates needs p + 2): they then run in groups of NACC, one after the
// other on the same CTA, and a grouped epilogue (Epi::kGrouped) receives each
// accumulator of each group and keeps its per-pair state across the groups.
#pragma once
#include <type_traits>

#include "sm100.cuh"

namespace eqtl {
namespace dev {

// Two-phase epilogues (Epi::kTwoPhase): the first Epi::kPhase1 accumulators
// of a unit are read for every chunk first (pre_chunk) and their TMEM slots
// released at once; the remaining ones follow (post_chunk). The next unit's
// MMAs then need to wait only for the short first phase.
template <class E, class = void>
struct IsTwoPhase : std::false_type {};
template <class E>
struct IsTwoPhase<E, std::void_t<decltype(E::kTwoPhase)>> : std::bool_constant<E::kTwoPhase> {};
// Epilogues that keep per-chunk state in registers (E::kChunkIdx): their
// chunks come from a fully unrolled loop with the chunk index known at
// compile time (chunk_at).
template <class E, class = void>
struct HasChunkIdx : std::false_type {};
template <class E>
struct HasChunkIdx<E, std::void_t<decltype(E::kChunkIdx)>> : std::bool_constant<E::kChunkIdx> {};

constexpr int kMaxAcc = 34;  // accumulators of one tile over all its groups (LMM: p + 2, p <= 32)
constexpr int kEpiWarps = 16;
constexpr int kTileThreads = 64 + 32 * kEpiWarps;
constexpr int kTileM = 128;
constexpr int kChunkK = 64;  // 16-bit elements per K chunk (one 128-byte swizzle row)

struct alignas(64) TileMaps {
  CUtensorMap a[2 * kMaxAcc];  // gene-side operand of accumulator j: [2j] hi, [2j+1] lo
  CUtensorMap b[4];            // SNP-side operand pairs: [0] hi, [1] lo, [2] hi, [3] lo
};

struct TileShape {
  int rows_a;             // valid gene-side rows
  int rows_b;             // valid SNP-side rows
  int kchunks;            // K / 64
  int n_acc;              // accumulators per tile (NACC, or more in groups of NACC)
  int n_groups;           // ceil(n_acc / NACC): TMEM holds one group at a time
  int bsel[kMaxAcc];      // SNP-side pair used by accumulator j (0 or 1)
  int prod[kMaxAcc];      // 1 = hi*hi, 2 = hi*lo, 4 = lo*hi (a lo part no product reads is not loaded)
  int tiles_a;            // ceil(rows_a / 128)
  int tiles_b;            // ceil(rows_b / NT)
  int n_tiles;            // work items: (tiles_a * tiles_b or the tile-list length) * ksplit
  int ksplit;             // K ranges per output tile (split-K); 1 = whole K
  int group_a;            // gene-side tiles per raster group (L2 residency of the A operands)
  int kc_per_split;       // K chunks per range
  int kc_sub;             // K chunks per sub-range (0: the whole range). Each sub-range starts its
                          // accumulators afresh and goes through the epilogue on its own, which
                          // sums the sub-ranges of a work item itself (single-group epilogues)
  int kc_beg[kMaxAcc];    // K-chunk range [kc_beg, kc_end) of accumulator j; kc_end 0: the work item's
  int kc_end[kMaxAcc];    // range (an accumulator with its own range needs ksplit 1, no sub-ranges)
  const int2* tile_list;  // optional explicit (tile_a, tile_b) list (banded scans); null = dense
  uint32_t* status;       // device status word (DevStatus)
};

// Where a SNP-side lo part goes (BL):
//   kBLoStage  in the same ring stage as A hi, A lo and B hi (four parts);
//   kBLoNone   nowhere: no product reads one (exact SNP operands), so a
//              stage holds three parts and more stages fit.
constexpr int kBLoStage = 0, kBLoNone = 1;

template <int NT, int NACC, int BL = kBLoStage>
struct TileCfg {
  static constexpr int A_BYTES = kTileM * kChunkK * 2;
  static constexpr int B_BYTES = NT * kChunkK * 2;
  static constexpr int STAGE_BYTES = 2 * A_BYTES + (BL == kBLoStage ? 2 : 1) * B_BYTES;
  static constexpr int STAGES = (196608 / STAGE_BYTES) < 2 ? 2 : (196608 / STAGE_BYTES > 6 ? 6 : 196608 / STAGE_BYTES);
  // TMEM is split into NSLOTS slots of NT columns; accumulator j of work
  // unit u lives in slot (u * NACC + j) % NSLOTS, so the next unit's first
  // accumulators can start in free slots while the epilogue still reads.
  static constexpr int NSLOTS = (512 / NT) > 8 ? 8 : 512 / NT;
  static constexpr uint32_t COLS_USED = NSLOTS * NT;
  static constexpr uint32_t TMEM_COLS = COLS_USED <= 32 ? 32 : COLS_USED <= 64 ? 64 : COLS_USED <= 128 ? 128
                                        : COLS_USED <= 256 ? 256 : 512;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 512;
  static_assert(NACC >= 1 && NACC <= kMaxAcc, "NACC");
  static_assert(NT % 16 == 0 && NT >= 16 && NT <= 256, "NT");
  static_assert(NACC <= NSLOTS, "TMEM slots");
  static_assert(STAGES * STAGE_BYTES + 1024 + 512 <= 232448, "smem");
};

// Work item t -> output tile (ta, tb) and its K-chunk range [k0, k1).
__device__ __forceinline__ void tile_coords(const TileShape& sh, int t, int& ta, int& tb, int& k0, int& k1) {
  int ks = 0;
  if (sh.tile_list) {
    ks = t % sh.ksplit;
    const int2 c = sh.tile_list[t / sh.ksplit];
    ta = c.x;
    tb = c.y;
  } else {
    // Raster: groups of group_a gene-side tiles sweep every SNP-side tile, so
    // the A operands of one group stay resident in L2 while B streams.
    ks = t % sh.ksplit;
    const int r = t / sh.ksplit;
    const int ga = sh.group_a;
    const int full = (sh.tiles_a / ga) * ga;
    const int in_full = full * sh.tiles_b;
    if (r < in_full) {
      const int grp = r / (ga * sh.tiles_b);
      const int q = r - grp * ga * sh.tiles_b;
      tb = q / ga;
      ta = grp * ga + (q - tb * ga);
    } else {
      const int rem = sh.tiles_a - full;
      const int q = r - in_full;
      tb = q / rem;
      ta = full + (q - tb * rem);
    }
  }
  k0 = ks * sh.kc_per_split;
  k1 = min(sh.kchunks, k0 + sh.kc_per_split);
}

template <int NT, int NACC, uint32_t AB_FMT, class Epi, int BL = kBLoStage>
__global__ void __launch_bounds__(kTileThreads, 1)
    tile_kernel(const __grid_constant__ TileMaps maps, const TileShape sh,
                const __grid_constant__ typename Epi::Params ep) {
  using C = TileCfg<NT, NACC, BL>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::STAGES * C::STAGE_BYTES);
  uint64_t* empty = full + C::STAGES;
  uint64_t* sfull = empty + C::STAGES;    // [NSLOTS] MMA -> epilogue: a unit's accumulators are complete
  uint64_t* sempty = sfull + C::NSLOTS;   // [NSLOTS] epilogue -> MMA: the slot has been read
  uint64_t* drain = sempty + C::NSLOTS;   // [1]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile uint32_t* abort_flag = tmem_slot + 1;
  uint8_t* epi_smem = smem + C::STAGES * C::STAGE_BYTES + 512;  // Epi::kSmemBytes of epilogue scratch

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int k = 0; k < C::NSLOTS; ++k) {
      mbar_init(&sfull[k], 1);
      mbar_init(&sempty[k], 32 * kEpiWarps);
    }
    mbar_init(drain, 1);
    *abort_flag = 0u;
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    for (int j = 0; j < 2 * sh.n_acc; ++j) tma_prefetch_map(&maps.a[j]);
    for (int j = 0; j < 4; ++j) tma_prefetch_map(&maps.b[j]);
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, C::TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  uint32_t* status = sh.status;

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (elect_one()) {
      int stage = 0;
      uint32_t phase = 0;
      uint32_t issued_phase[6] = {0, 0, 0, 0, 0, 0};
      bool issued[6] = {false, false, false, false, false, false};
      bool ok = true;
      for (int t = blockIdx.x; t < sh.n_tiles && ok; t += gridDim.x) {
        int ta, tb, k0, k1;
        tile_coords(sh, t, ta, tb, k0, k1);
        const int ra = ta * kTileM, rb = tb * NT;
        const int ksub = sh.kc_sub > 0 ? sh.kc_sub : k1 - k0;
        for (int q0 = k0; q0 < k1 && ok; q0 += ksub)
        for (int j = 0; j < sh.n_acc && ok; ++j) {
          const bool own = sh.kc_end[j] > 0;
          const int qa = own ? sh.kc_beg[j] : q0, qb = own ? sh.kc_end[j] : min(k1, q0 + ksub);
          const int bp = sh.bsel[j];
          // only the lo parts some product of this accumulator reads are loaded
          const bool a_lo = (sh.prod[j] & 4) != 0, b_lo = BL == kBLoStage && (sh.prod[j] & 2) != 0;
          const uint32_t bytes = static_cast<uint32_t>(C::A_BYTES + C::B_BYTES + (a_lo ? C::A_BYTES : 0) +
                                                       (b_lo ? C::B_BYTES : 0));
          for (int kc = qa; kc < qb; ++kc) {
            if (!mbar_wait(&empty[stage], phase ^ 1u, status, abort_flag, kDevTimeoutEmpty)) {
              ok = false;
              break;
            }
            uint8_t* sb = smem + stage * C::STAGE_BYTES;
            mbar_arrive_expect_tx(&full[stage], bytes);
            tma_load_2d(sb, &maps.a[2 * j], &full[stage], kc * kChunkK, ra);
            if (a_lo) tma_load_2d(sb + C::A_BYTES, &maps.a[2 * j + 1], &full[stage], kc * kChunkK, ra);
            tma_load_2d(sb + 2 * C::A_BYTES, &maps.b[2 * bp], &full[stage], kc * kChunkK, rb);
            if (b_lo)
              tma_load_2d(sb + 2 * C::A_BYTES + C::B_BYTES, &maps.b[2 * bp + 1], &full[stage], kc * kChunkK, rb);
            issued[stage] = true;
            issued_phase[stage] = phase;
            if (++stage == C::STAGES) {
              stage = 0;
              phase ^= 1u;
            }
          }
        }
      }
      // Drain: every load issued into a ring slot must land before the CTA
      // may exit (bounded; normally already complete).
      for (int s = 0; s < C::STAGES; ++s) {
        if (!issued[s]) continue;
        const long long t0 = clock64();
        while (!mbar_test(&full[s], issued_phase[s])) {
          if (clock64() - t0 > kWaitCycles) {
            set_status(status, kDevTimeoutDrain);
            break;
          }
        }
      }
    }
  } else if (warp == 1) {
    // ---------------------------------------------------------- MMA issuer
    if (elect_one()) {
      constexpr uint32_t idesc = idesc_f16(kTileM, NT, AB_FMT);
      int stage = 0;
      uint32_t phase = 0;
      uint32_t eph = 0;   // bit k: parity of slot k's next release
      int slot0 = 0;      // ring slot of the current unit's first accumulator
      bool ok = true;
      for (int t = blockIdx.x; t < sh.n_tiles && ok; t += gridDim.x) {
        int ta, tb, k0, k1;
        tile_coords(sh, t, ta, tb, k0, k1);
        const int ksub = sh.kc_sub > 0 ? sh.kc_sub : k1 - k0;
        for (int q0 = k0; q0 < k1 && ok; q0 += ksub)
        for (int grp = 0; grp < sh.n_groups && ok; ++grp, slot0 = (slot0 + NACC) % C::NSLOTS) {
          const int j0 = grp * NACC;
          const int nv = min(NACC, sh.n_acc - j0);
          int last = 0;
          for (int jj = 0; jj < nv && ok; ++jj) {
            const int slot = (slot0 + jj) % C::NSLOTS;
            last = slot;
            if (!mbar_wait(&sempty[slot], ((eph >> slot) & 1u) ^ 1u, status, abort_flag, kDevTimeoutAccEmpty)) {
              ok = false;
              break;
            }
            eph ^= 1u << slot;
            tc_fence_after();
            const uint32_t d = tmem_base + static_cast<uint32_t>(slot * NT);
            const int pm = sh.prod[j0 + jj];
            const bool own = sh.kc_end[j0 + jj] > 0;
            const int qa = own ? sh.kc_beg[j0 + jj] : q0, qb = own ? sh.kc_end[j0 + jj] : min(k1, q0 + ksub);
            for (int kc = qa; kc < qb; ++kc) {
              if (!mbar_wait(&full[stage], phase, status, abort_flag, kDevTimeoutFull)) {
                ok = false;
                break;
              }
              tc_fence_after();
              const uint32_t sbase = smem_u32(smem + stage * C::STAGE_BYTES);
              const uint32_t sa0 = sbase, sa1 = sbase + C::A_BYTES;
              const uint32_t sb0 = sbase + 2 * C::A_BYTES, sb1 = sb0 + C::B_BYTES;
#pragma unroll
              for (int k = 0; k < kChunkK / 16; ++k) {
                const uint32_t off = static_cast<uint32_t>(k * 32);
                // the first product of a (sub-)range starts the accumulator;
                // every later one adds
                uint32_t accum = (kc > qa || k > 0) ? 1u : 0u;
                if (pm & 1) {
                  umma_f16(d, smem_desc_sw128(sa0 + off), smem_desc_sw128(sb0 + off), idesc, accum);
                  accum = 1u;
                }
                if (BL == kBLoStage && (pm & 2)) {
                  umma_f16(d, smem_desc_sw128(sa0 + off), smem_desc_sw128(sb1 + off), idesc, accum);
                  accum = 1u;
                }
                if (pm & 4) {
                  umma_f16(d, smem_desc_sw128(sa1 + off), smem_desc_sw128(sb0 + off), idesc, accum);
                }
              }
              umma_commit(&empty[stage]);
              if (++stage == C::STAGES) {
                stage = 0;
                phase ^= 1u;
              }
            }
          }
          if (!ok) break;
          umma_commit(&sfull[last]);  // completes when every MMA issued so far has
        }
      }
      // Drain: all issued MMAs complete before TMEM is released (bounded).
      umma_commit(drain);
      const long long t0 = clock64();
      while (!mbar_test(drain, 0u)) {
        if (clock64() - t0 > kWaitCycles) {
          set_status(status, kDevTimeoutDrain);
          break;
        }
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int quarter = warp & 3;  // TMEM lane quarter this warp may access
    const int row = quarter * 32 + lane;
    constexpr int kSub = kEpiWarps / 4;  // warps sharing a lane quarter
    const int sub = (warp - 2) >> 2;     // this warp's share of the columns
    Epi epi(ep, sh, Epi::kSmemBytes ? epi_smem : nullptr);
    epi.init(threadIdx.x - 64, 32 * kEpiWarps);
    asm volatile("bar.sync 1, %0;" ::"r"(32 * kEpiWarps) : "memory");
    uint32_t fph = 0;   // bit k: parity of slot k's next completion
    int slot0 = 0;      // ring slot of the current unit's first accumulator
    const uint32_t lanes = tmem_base + (static_cast<uint32_t>(quarter * 32) << 16);
    for (int t = blockIdx.x; t < sh.n_tiles; t += gridDim.x) {
      int ta, tb, k0, k1;
      tile_coords(sh, t, ta, tb, k0, k1);
      epi.begin_tile(ta * kTileM + row, tb * NT);
      bool eok = true;
      const int ksub = sh.kc_sub > 0 ? sh.kc_sub : k1 - k0;
      for (int q0 = k0; q0 < k1 && eok; q0 += ksub)
      for (int grp = 0; grp < sh.n_groups; ++grp, slot0 = (slot0 + NACC) % C::NSLOTS) {
        const int j0 = grp * NACC;
        const int nv = min(NACC, sh.n_acc - j0);
        const int last = (slot0 + nv - 1) % C::NSLOTS;
        if (!mbar_wait(&sfull[last], (fph >> last) & 1u, status, abort_flag, kDevTimeoutAccFull)) {
          eok = false;
          break;
        }
        fph ^= 1u << last;
        tc_fence_after();
        auto col = [&](int jj) { return lanes + static_cast<uint32_t>(((slot0 + jj) % C::NSLOTS) * NT); };
        if constexpr (Epi::kGrouped) {
#pragma unroll 1
          for (int c = 16 * sub; c < NT; c += 16 * kSub) {
#pragma unroll 1
            for (int jj = 0; jj < nv; ++jj) {
              float v[16];
              tmem_ld16(col(jj) + static_cast<uint32_t>(c), v);
              tmem_wait_ld();
              epi.acc_chunk(j0 + jj, c, v);
            }
            if (grp == sh.n_groups - 1) epi.finish_chunk(c);
          }
        } else if constexpr (IsTwoPhase<Epi>::value) {
          constexpr int N1 = Epi::kPhase1;
          static_assert(N1 >= 1 && N1 < NACC, "two-phase epilogue: phase sizes");
          // every warp owns exactly NCH chunks; ci tells the epilogue which
          constexpr int NCH = NT / (16 * kSub);
          static_assert(NT % (16 * kSub) == 0 && NCH <= Epi::kMaxChunks, "two-phase epilogue: chunks per warp");
#pragma unroll 1
          for (int ci = 0; ci < NCH; ++ci) {
            const int c = 16 * sub + 16 * kSub * ci;
            float v[N1][16];
#pragma unroll
            for (int jj = 0; jj < N1; ++jj) tmem_ld16(col(jj) + static_cast<uint32_t>(c), v[jj]);
            tmem_wait_ld();
            epi.template pre_chunk<N1>(ci, c, v);
          }
          tc_fence_before();
          for (int jj = 0; jj < N1; ++jj) mbar_arrive(&sempty[(slot0 + jj) % C::NSLOTS]);
#pragma unroll 1
          for (int ci = 0; ci < NCH; ++ci) {
            const int c = 16 * sub + 16 * kSub * ci;
            float v[NACC - N1][16];
#pragma unroll
            for (int jj = 0; jj < NACC - N1; ++jj) tmem_ld16(col(N1 + jj) + static_cast<uint32_t>(c), v[jj]);
            tmem_wait_ld();
            epi.template post_chunk<NACC - N1>(ci, c, v);
          }
          tc_fence_before();
          for (int jj = N1; jj < nv; ++jj) mbar_arrive(&sempty[(slot0 + jj) % C::NSLOTS]);
          continue;  // slots released above
        } else if constexpr (HasChunkIdx<Epi>::value) {
          constexpr int NCH = NT / (16 * kSub);
          static_assert(NT % (16 * kSub) == 0 && NCH <= Epi::kMaxChunks, "indexed epilogue: chunks per warp");
#pragma unroll
          for (int ci = 0; ci < NCH; ++ci) {
            const int c = 16 * sub + 16 * kSub * ci;
            float v[NACC][16];
#pragma unroll
            for (int jj = 0; jj < NACC; ++jj) tmem_ld16(col(jj) + static_cast<uint32_t>(c), v[jj]);
            tmem_wait_ld();
            epi.template chunk_at<NACC>(ci, c, v);
          }
        } else {
#pragma unroll 1
          for (int c = 16 * sub; c < NT; c += 16 * kSub) {
            float v[NACC][16];
#pragma unroll
            for (int jj = 0; jj < NACC; ++jj) tmem_ld16(col(jj) + static_cast<uint32_t>(c), v[jj]);
            tmem_wait_ld();
            epi.template chunk<NACC>(c, v);
          }
        }
        tc_fence_before();
        for (int jj = 0; jj < nv; ++jj) mbar_arrive(&sempty[(slot0 + jj) % C::NSLOTS]);
      }
      if (!eok) break;
      epi.end_tile();
    }
    epi.finish();
  }

  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, C::TMEM_COLS);
  }
}

}  // namespace dev
}  // namespace eqtl
