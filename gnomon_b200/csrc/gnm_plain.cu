// gnm_plain.cu — plain (FP32 weights, CUDA-core) scoring path for sm_100a.
//
// Replaces the reference GPU engine's unpack_plink -> zero -> scatter ->
// 3x SGEMM -> combine chain (score/cuda_backend.rs:62-218, 2067-2333) for small
// score counts with one fused accumulate kernel per score column:
//
//   * the weights of every 3 consecutive variant rows are folded once per plan
//     (gnm_plain_tables) into a 64-entry table: entry (ca, cb, cc) is the exact
//     sum T_a[ca] + T_b[cb] + T_c[cc] with T = {0, -missing correction,
//     dosage_weight, 2*dosage_weight} (prepare.rs:197-208 folding; code 00
//     contributes 0), put on the stage's int32 fixed-point grid, so decode,
//     effect-allele flip and the missing-call rule become ONE lookup per
//     person per 3 variants; ten group tables, the membership word and the
//     grid step make one 2576-byte stage table;
//   * packed .bed rows are TMA-staged (cp.async.bulk.tensor into this CTA
//     only) in [30 rows x TILE bytes] stages with their stage table (a 1D bulk
//     copy on the same mbarrier), three buffers deep; TILE is 512, 1024 or
//     2048 bytes of every row (2048, 4096 or 8192 people), the autotuner's
//     choice;
//   * each thread owns one 32-bit word column = 16 people; per 3 rows it
//     transposes the 2-bit codes into per-person 6-bit indices (one byte each,
//     pre-scaled by 4) with shift/mask ops and turns each byte into a
//     shared-memory address with one integer dot product (__dp4a); two
//     groups' lookups go into a person's sum with one three-input add;
//   * warps run the stages independently: a warp waits only for the stage's
//     TMA; it releases the buffer either through a shared counter whose last
//     arriver issues the TMA of the stage three ahead, or (producer-warp
//     kernels) by arriving on a release mbarrier that a producer warp waits on
//     before it issues that TMA — no CTA-wide barrier per stage;
//   * missing calls (code 01) are counted with SWAR bit tricks on the raw row
//     words (x & ~(x>>1) & member_mask, three rows summed with one add);
//   * a stage's ten lookups per person add up exactly in int32 and reach FP64
//     once per stage (sum x grid step); variant splits write FP64 partials
//     that gnm_finalize reduces in a fixed order (deterministic) and gathers
//     through output_idx_to_fam_idx, adding the FP64 baseline
//     (pipeline.rs:1739-1775).
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "gnm_device.cuh"
#include "gnm_internal.h"

namespace gnm {

// Shared-memory layout of one plain CTA (dynamic smem, offsets in bytes) for
// a people tile of TILE bytes of every row (TILE / 4 threads, 4 * TILE people).
template <uint32_t TILE>
struct PlainSmem {
  static constexpr uint32_t kStages = 3;
  static constexpr uint32_t kThreads = TILE / 4;
  static constexpr uint32_t kWarps = kThreads / 32;
  static constexpr uint32_t kBoxes = TILE / kPlainBoxBytes;                  // TMA boxes per stage
  static constexpr uint32_t kStageBytes = kPlainRows * TILE;                 // 30720 at 1 KB
  static constexpr uint32_t kBoxBytes = kPlainRows * kPlainBoxBytes;         // 7680
  static constexpr uint32_t kTabStride = 3072;   // one stage table, padded to 1 KB in total
  static constexpr uint32_t kTabOff = 0;
  static constexpr uint32_t kTileOff = kTabOff + kStages * kTabStride;      // 9216
  static constexpr uint32_t kBarOff = kTileOff + kStages * kStageBytes;     // 3 mbarriers
  static constexpr uint32_t kRelOff = kBarOff + 8 * kStages;                // 3 release counters
  static constexpr uint32_t kLastOff = kRelOff + 4 * kStages;               // 3 last-issued stages
  static constexpr uint32_t kEmptyOff = kLastOff + 4 * kStages;             // 3 "released" mbarriers
  static constexpr uint32_t kTotal = kEmptyOff + 8 * kStages;
  static_assert(kEmptyOff % 8 == 0, "mbarrier alignment");
  static_assert(TILE % kPlainBoxBytes == 0 && TILE % 128 == 0, "whole boxes and warps");
  static_assert(kPlainRows % 3 == 0 && kPlainRows <= 32, "groups of 3 rows, one ballot");
  static_assert(kPlainGroups % 2 == 0, "groups are scored in pairs");
  static_assert(kTabStride >= kPlainTableBytes && kTabStride % 256 == 0, "table stride");
  static_assert(kTileOff % 1024 == 0, "tile alignment");
  // Each 64-entry group table starts on a 256-byte boundary, so a lookup
  // address is the table address plus the index byte (no carry).
};

// Multipliers for left shifts and adds written as integer multiply-adds: held
// in constant memory, unknown at compile time, they make the compiler issue
// IMAD on the FMA pipe instead of shift / add on the integer ALU pipe, which
// the index transposes, masks and three-input adds already keep busy.
__constant__ uint32_t c_mul[5] = {2u, 4u, 16u, 64u, 1u};

// Byte selectors for the lookup addresses: __dp4a(ix, c_sel[j], table) is
// byte j of ix plus the table address (the other three byte products are
// zero), one integer dot-product instruction on the FMA pipe where a byte
// permute would take the integer ALU pipe.  Held in constant memory so that
// the compiler keeps the dot product.
__constant__ uint32_t c_sel[4] = {0x1u, 0x100u, 0x10000u, 0x1000000u};

__device__ __forceinline__ int32_t lds_s32(uint32_t addr) {
  int32_t v;
  asm volatile("ld.shared.s32 %0, [%1];" : "=r"(v) : "r"(addr));
  return v;
}

// Shared-memory atomic add with acquire-release ordering at CTA scope.
__device__ __forceinline__ uint32_t atom_add_acq_rel(uint32_t addr, uint32_t v) {
  uint32_t old;
  asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], %2;"
               : "=r"(old) : "r"(addr), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ void sts_u32(uint32_t addr, uint32_t v) {
  asm volatile("st.shared.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

// ---- stage tables ------------------------------------------------------------
// Entry index e (6 bits) = bank (bits 0-4) + table row (bit 5).  The row bit
// is lc, the lo bit of row c's code; the bank bits are row a's and row b's
// codes with lc XORed into their lo bits (bits 0-1, 2-3) and the hi bit of row
// c (bit 4).  The two entries that share a bank therefore differ in the lo bit
// of all three codes (code 01 missing / 11 hom-alt), so one of them needs two
// such calls in one person and lanes rarely meet on a bank with different
// addresses.
//
// Entries are int32 fixed-point values on a per-stage grid: q = 2^(E - 27)
// with 2^E the smallest power of two >= the stage's largest |entry|, entry =
// round(exact FP64 sum of the three FP32 terms / q), so |entry| <= 2^27 and
// the ten lookups of a stage add up EXACTLY in int32 (|sum| < 2^31).  The kernel converts each stage's
// integer sums to FP64 once (sum * q).  The only rounding before FP64 is the
// grid itself, <= q/2 per lookup; FP32 running sums lose up to half an ulp of
// the running partial at every add, which over 10^6 variants came near the
// reference's 1e-6 tolerance.  q sits in the stage table's tail (word 1).

__device__ __forceinline__ float table_term(const TableArgs& a, uint64_t row, uint32_t j) {
  if (a.records) return reinterpret_cast<const float*>(a.records + a.row0 + row)[j];
  const uint64_t r = a.row0 + row;
  if (a.member && a.member[r] == 0) return 0.0f;
  const float w = a.w[r];
  return j == 0 ? -a.corr[r] : (j == 1 ? w : 2.0f * w);
}

__device__ __forceinline__ bool table_member(const TableArgs& a, uint64_t row) {
  if (a.records) return a.records[a.row0 + row].w != 0.0f;
  return a.member == nullptr || a.member[a.row0 + row] != 0;
}

// grid.x = stages, block = kPlainGroups groups x 64 entries.
__global__ void __launch_bounds__(kPlainGroups * 64) gnm_plain_tables(TableArgs a) {
  __shared__ float s_max[kPlainGroups * 2];
  const uint64_t stage = blockIdx.x;
  const uint32_t e = threadIdx.x, g = e >> 6, idx = e & 63u;
  const uint32_t lc = (idx >> 5) & 1u;
  const uint32_t code[3] = {(idx & 3u) ^ lc, ((idx >> 2) & 3u) ^ lc, ((idx >> 3) & 2u) | lc};
  const uint64_t row0 = stage * kPlainRows + 3 * g;
  double v = 0.0;
#pragma unroll
  for (int r = 0; r < 3; ++r)
    if (code[r] != 0 && row0 + r < a.num_rows) v += double(table_term(a, row0 + r, code[r] - 1));
  // largest |entry| of the stage (exact FP64 sums rounded up to FP32)
  float m = __double2float_ru(fabs(v));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  if ((e & 31u) == 0) s_max[e >> 5] = m;
  __syncthreads();
  float mx = 0.0f;
#pragma unroll
  for (uint32_t w = 0; w < kPlainGroups * 2; ++w) mx = fmaxf(mx, s_max[w]);
  // grid step: the power of two 2^(E - 27) with 2^E >= max |entry|, so
  // |entry / q| <= 2^27 and values with few significant bits stay exact
  int ex = 0;
  frexpf(mx, &ex);
  const float q = mx > 0.0f ? ldexpf(1.0f, ex - 27) : 1.0f;
  uint8_t* tab = a.tables + stage * kPlainTableBytes;
  reinterpret_cast<int32_t*>(tab)[e] = int32_t(__double2ll_rn(v / double(q)));
  if (e < 32) {
    const uint64_t row = stage * kPlainRows + e;
    const bool mem = e < kPlainRows && row < a.num_rows && table_member(a, row);
    const uint32_t bits = __ballot_sync(0xFFFFFFFFu, mem);
    if (e < 4)
      reinterpret_cast<uint32_t*>(tab + kPlainGroups * 256)[e] =
          e == 0 ? bits : (e == 1 ? __float_as_uint(q) : 0u);
  }
}

// ---- accumulate --------------------------------------------------------------

// Copies of one stage: the tile's first `boxes` row boxes (the ones that hold
// row bytes) and the stage table, on the buffer's mbarrier.
template <uint32_t TILE>
__device__ __forceinline__ void plain_issue_stage(const CUtensorMap* map, const uint8_t* tables,
                                                  uint32_t smem_base, uint32_t buf,
                                                  int32_t tile_x, int32_t row0, uint64_t stage,
                                                  uint32_t boxes) {
  using L = PlainSmem<TILE>;
  const uint32_t bar = smem_base + L::kBarOff + 8 * buf;
  mbar_arrive_expect_tx(bar, boxes * L::kBoxBytes + kPlainTableBytes);
  const uint32_t tile = smem_base + L::kTileOff + buf * L::kStageBytes;
  for (uint32_t b = 0; b < boxes; ++b)
    tma_load_2d(tile + b * L::kBoxBytes, map, tile_x + int32_t(b * kPlainBoxBytes), row0, bar);
  bulk_load(smem_base + L::kTabOff + buf * L::kTabStride, tables + stage * kPlainTableBytes,
            kPlainTableBytes, bar);
}

template <uint32_t TILE, bool WS>
struct PlainShape {
  static constexpr uint32_t kThreads = TILE / 4 + (WS ? 32u : 0u);
  static constexpr uint32_t kMinBlocks = TILE >= 2048 ? 1u : 2048u / TILE;
};

// One CTA per (people tile, variant split).  The grid is 1D: the first
// (tiles - 1) * splits CTAs cover the full tiles, `splits` each, and the last
// tile (often only partly populated by people) has its own stages-per-split
// field; the host gives it the same split count as the others, because a
// CTA's time per stage is set by each warp's dependency chains, not by how
// many of its warps hold people.  block = TILE / 4 scoring threads, plus (WS) one
// producer warp that issues every stage's copies once the scoring warps have
// released its buffer (they arrive on an mbarrier and never wait for one
// another); without it the scoring warp that releases a buffer last issues
// the refill.
template <uint32_t TILE, bool WS>
__global__ void __launch_bounds__(PlainShape<TILE, WS>::kThreads, PlainShape<TILE, WS>::kMinBlocks)
    gnm_plain_accumulate(const __grid_constant__ CUtensorMap map, PlainArgs a) {
  using L = PlainSmem<TILE>;
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t sbase = smem_u32(smem);
  const uint32_t tid = threadIdx.x, lane = tid & 31u;
  const bool producer = WS && tid >= L::kThreads;
  const uint32_t full_ctas = (a.tiles - 1) * a.splits;
  uint32_t tile, split, sps;
  if (blockIdx.x < full_ctas) {
    tile = blockIdx.x / a.splits;
    split = blockIdx.x % a.splits;
    sps = a.stages_per_split;
  } else {
    tile = a.tiles - 1;
    split = blockIdx.x - full_ctas;
    sps = a.last_stages_per_split;
  }

  const uint64_t rows_per_split = uint64_t(sps) * kPlainRows;
  const uint64_t r_begin = uint64_t(split) * rows_per_split;
  if (r_begin >= a.num_rows) return;
  // table addresses are formed by byte replacement: the window must be aligned
  if ((sbase & 255u) != 0u) {
    if (tid == 0) atomicOr(a.err, kErrShape);
    return;
  }
  const uint64_t r_end = min(a.num_rows, r_begin + rows_per_split);
  const uint32_t nstages = uint32_t((r_end - r_begin + kPlainRows - 1) / kPlainRows);
  const uint64_t stage0 = r_begin / kPlainRows;   // block stage of this split's stage 0
  const int32_t tile_x = int32_t(tile * TILE);
  // The last tile may hold fewer row bytes than TILE: only its populated
  // warps score (the others skip the stage loop and release nothing) and
  // only its populated boxes are copied, so a partly filled tile costs in
  // proportion to its bytes.
  const uint64_t used = min(uint64_t(TILE), a.bytes_per_row - uint64_t(tile) * TILE);
  const uint32_t active_warps = uint32_t((used + 127) / 128);
  const uint32_t boxes = uint32_t((used + kPlainBoxBytes - 1) / kPlainBoxBytes);
  const uint32_t bar0 = sbase + L::kBarOff;
  const uint32_t rel0 = sbase + L::kRelOff;
  const uint32_t empty0 = sbase + L::kEmptyOff;
  uint32_t* last_issued = reinterpret_cast<uint32_t*>(smem + L::kLastOff);

  if (tid == 0) {
    prefetch_tmap(&map);
    for (uint32_t b = 0; b < L::kStages; ++b) {
      mbar_init(bar0 + 8 * b, 1);
      if (WS) mbar_init(empty0 + 8 * b, active_warps);
      sts_u32(rel0 + 4 * b, 0u);
      last_issued[b] = 0xFFFFFFFFu;
    }
    fence_mbar_init();
  }
  __syncthreads();
  if (WS && producer) {
    // ---- producer warp: every stage's copies, each once its buffer is free
    bool ok = true;
    if (lane == 0) {
      for (uint32_t st = 0; st < nstages; ++st) {
        const uint32_t buf = st % L::kStages;
        if (st >= L::kStages) {
          // the scoring warps released stage st - 3 of this buffer
          if (!mbar_wait_bounded(empty0 + 8 * buf, ((st / L::kStages) - 1) & 1u)) {
            atomicOr(a.err, kErrTmaTimeout);
            ok = false;
            break;
          }
          fence_proxy_async_smem();
        }
        last_issued[buf] = st;
        plain_issue_stage<TILE>(&map, a.tables, sbase, buf, tile_x,
                                int32_t(r_begin + uint64_t(st) * kPlainRows), stage0 + st, boxes);
      }
    }
    // every warp of the CTA meets here (the scoring warps at the end of their loop)
    if (__syncthreads_or(!__shfl_sync(0xFFFFFFFFu, ok ? 1 : 0, 0))) {
      if (lane == 0)   // drain each buffer's last issued copy (bounded)
        for (uint32_t b = 0; b < L::kStages; ++b)
          if (last_issued[b] != 0xFFFFFFFFu)
            mbar_wait_bounded(bar0 + 8 * b, (last_issued[b] / L::kStages) & 1u);
    }
    return;
  }
  if (!WS && tid == 0) {
    for (uint32_t s = 0; s < L::kStages && s < nstages; ++s) {
      last_issued[s] = s;
      plain_issue_stage<TILE>(&map, a.tables, sbase, s, tile_x,
                              int32_t(r_begin + s * kPlainRows), stage0 + s, boxes);
    }
  }

  // int32 fixed-point sums of the current stage: iacc[4j + q] is person
  // 4j + q of this thread's 16 (exact: <= 10 lookups of |entry| <= 2^27 + 1).
  int32_t iacc[16];
  double acc64[16];
  uint32_t cnt[16];
  uint32_t by[4] = {0u, 0u, 0u, 0u};   // byte counters: byte j = person 4j+q
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    acc64[i] = 0.0;
    cnt[i] = 0u;
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) iacc[i] = 0;

  // Each thread reads word column `tid` of the TILE-byte stage row; the stage
  // is stored as TILE / 256 TMA boxes of [kPlainRows rows][256 bytes].
  const uint32_t word_off = (tid / (kPlainBoxBytes / 4)) * L::kBoxBytes +
                            (tid % (kPlainBoxBytes / 4)) * 4;
  // warps whose 128 bytes all lie past the row's last byte only hold padding
  const bool warp_active = (tid >> 5) < active_warps;

  bool failed = false;
  for (uint32_t st = 0; st < (warp_active ? nstages : 0u); ++st) {
    const uint32_t buf = st % L::kStages;
    const uint32_t parity = (st / L::kStages) & 1u;
    if (!mbar_wait_bounded(bar0 + 8 * buf, parity)) {
      if (lane == 0) atomicOr(a.err, kErrTmaTimeout);
      failed = true;
      break;
    }

    // Row words are ordinary loads from the shared array (the compiler may
    // hoist the next group's rows above this group's lookups; the mbarrier
    // wait above clobbers memory, so none moves above it); table lookups go
    // through 32-bit shared addresses.
    const uint8_t* tbase = smem + L::kTileOff + buf * L::kStageBytes + word_off;
    const uint32_t lbase = sbase + L::kTabOff + buf * L::kTabStride;
    const uint64_t members = *reinterpret_cast<const uint32_t*>(
        smem + L::kTabOff + buf * L::kTabStride + kPlainGroups * 256);
    // the stage's grid step, read before the buffer is released
    const float stage_q = *reinterpret_cast<const float*>(
        smem + L::kTabOff + buf * L::kTabStride + kPlainGroups * 256 + 4);

    uint32_t ev = 0, od = 0;             // nibble counters (people 2j / 2j+1)
    // Row words of group g -> four index words; returns the group's missing
    // calls (code 01 of member rows) summed into 2-bit fields.
    auto index = [&](uint32_t g, uint32_t (&ix)[4], uint32_t ma, uint32_t mb,
                     uint32_t mc) -> uint32_t {
      const uint32_t xa = *reinterpret_cast<const uint32_t*>(tbase + (3 * g + 0) * kPlainBoxBytes);
      const uint32_t xb = *reinterpret_cast<const uint32_t*>(tbase + (3 * g + 1) * kPlainBoxBytes);
      const uint32_t xc = *reinterpret_cast<const uint32_t*>(tbase + (3 * g + 2) * kPlainBoxBytes);
      // rows a and b get row c's lo bits XORed into their lo bits; row c
      // enters with its code bits swapped (see the table layout above)
      const uint32_t ya = xa ^ (xc & 0x55555555u);
      const uint32_t yb = xb ^ (xc & 0x55555555u);
      const uint32_t xs = ((xc >> 1) & 0x55555555u) | ((xc * c_mul[0]) & 0xAAAAAAAAu);
      const uint32_t E = (ya & 0x33333333u) | ((yb * c_mul[1]) & 0xCCCCCCCCu);
      const uint32_t O = ((ya >> 2) & 0x33333333u) | (yb & 0xCCCCCCCCu);
      // byte j of ix[q] is person 4j + q's 6-bit index, pre-scaled by 4
      ix[0] = ((E * c_mul[1]) & 0x3C3C3C3Cu) | ((xs * c_mul[3]) & 0xC0C0C0C0u);
      ix[1] = ((O * c_mul[1]) & 0x3C3C3C3Cu) | ((xs * c_mul[2]) & 0xC0C0C0C0u);
      ix[2] = ((E >> 2) & 0x3C3C3C3Cu) | ((xs * c_mul[1]) & 0xC0C0C0C0u);
      ix[3] = ((O >> 2) & 0x3C3C3C3Cu) | (xs & 0xC0C0C0C0u);
      return (xa & ~(xa >> 1) & ma) + (xb & ~(xb >> 1) & mb) + (xc & ~(xc >> 1) & mc);
    };
    // Groups g and g + 1 together: each person's two lookups go into its
    // stage sum with one three-input add.  Nibble counters take four groups
    // (<= 12 calls) before they are flushed to the byte counters.
    auto pair = [&](uint32_t g, uint32_t m0, uint32_t m1, uint32_t m2, uint32_t m3,
                    uint32_t m4, uint32_t m5) {
      uint32_t i0[4], i1[4];
      const uint32_t c0 = index(g, i0, m0, m1, m2);
      const uint32_t c1 = index(g + 1, i1, m3, m4, m5);
      const uint32_t l0 = lbase + g * 256, l1 = l0 + 256;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          iacc[4 * j + q] = int32_t(uint32_t(iacc[4 * j + q]) +
                                    uint32_t(lds_s32(__dp4a(i0[q], c_sel[j], l0))) +
                                    uint32_t(lds_s32(__dp4a(i1[q], c_sel[j], l1))));
      }
      ev = (c0 & 0x33333333u) + (c1 & 0x33333333u) + ev;
      od = ((c0 >> 2) & 0x33333333u) + ((c1 >> 2) & 0x33333333u) + od;
      if ((g / 2) % 2 == 1 || g + 2 == kPlainGroups) {
        by[0] += ev & 0x0F0F0F0Fu;
        by[2] += (ev >> 4) & 0x0F0F0F0Fu;
        by[1] += od & 0x0F0F0F0Fu;
        by[3] += (od >> 4) & 0x0F0F0F0Fu;
        ev = 0u;
        od = 0u;
      }
    };
    if (!warp_active) {
      // padding-only warp: nothing to score
    } else if (members == (uint64_t(1) << kPlainRows) - 1) {
      // every row of the stage is a member of this score (the common case)
#pragma unroll
      for (uint32_t g = 0; g < kPlainGroups; g += 2)
        pair(g, 0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u);
    } else {
#pragma unroll
      for (uint32_t g = 0; g < kPlainGroups; g += 2) {
        uint32_t m[6];
#pragma unroll
        for (uint32_t r = 0; r < 6; ++r)
          m[r] = (0u - uint32_t((members >> (3 * g + r)) & 1u)) & 0x55555555u;
        pair(g, m[0], m[1], m[2], m[3], m[4], m[5]);
      }
    }

    // Release the buffer.  __syncwarp orders this warp's reads before lane
    // 0's release-add; the warp that completes the count acquires every
    // warp's release, so all reads of the buffer are done before it hands the
    // buffer to the async proxy for the stage three ahead.
    __syncwarp();
    if (WS) {
      if (lane == 0) mbar_arrive(empty0 + 8 * buf);
    } else if (lane == 0) {
      const uint32_t old = atom_add_acq_rel(rel0 + 4 * buf, 1u);
      if (old == active_warps - 1) {
        sts_u32(rel0 + 4 * buf, 0u);
        const uint32_t nxt = st + L::kStages;
        if (nxt < nstages) {
          last_issued[buf] = nxt;
          fence_proxy_async_smem();
          plain_issue_stage<TILE>(&map, a.tables, sbase, buf, tile_x,
                                  int32_t(r_begin + uint64_t(nxt) * kPlainRows), stage0 + nxt,
                                  boxes);
        }
      }
    }

    // The stage's exact integer sums go to FP64 with the stage's grid step;
    // byte counters span eight stages (<= 240 calls per byte) before they
    // are flushed to 32-bit counts.
    {
      const double q = double(stage_q);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        acc64[i] = fma(double(iacc[i]), q, acc64[i]);
        iacc[i] = 0;
      }
      if ((st & 7u) == 7u || st + 1 == nstages) {
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
#pragma unroll
          for (int j = 0; j < 4; ++j) cnt[4 * j + q4] += (by[q4] >> (8 * j)) & 0xFFu;
          by[q4] = 0u;
        }
      }
    }
  }

  // A warp that gave up on a TMA wait leaves stages other warps may still
  // wait for (bounded).  Once every warp is here, drain each buffer's last
  // issued copy (bounded) so no TMA is in flight when the CTA exits.
  if (__syncthreads_or(failed)) {
    if (!WS && tid == 0) {   // (WS: the producer warp drains)
      for (uint32_t b = 0; b < L::kStages; ++b)
        if (last_issued[b] != 0xFFFFFFFFu)
          mbar_wait_bounded(bar0 + 8 * b, (last_issued[b] / L::kStages) & 1u);
    }
    return;
  }

  // FP64 partials for this (split, person) accumulate across calls; the first
  // launch after a reset writes them (every split of every tile has a CTA, so
  // every slot it covers is written).  Warps that only held padding added
  // nothing: their slots (people past the row) stay as they are.
  if (!warp_active) return;
  const uint64_t person0 = uint64_t(tile) * (TILE * 4) + uint64_t(tid) * 16;
  double* ps = a.part_sum + uint64_t(split) * a.part_stride + person0;
  uint32_t* pc = a.part_cnt + uint64_t(split) * a.part_stride + person0;
  if (a.store) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      ps[i] = acc64[i];
      pc[i] = cnt[i];
    }
  } else {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      ps[i] += acc64[i];
      pc[i] += cnt[i];
    }
  }
}

// out[o*K + k] = init + sum over splits of part[s][fam(o)], init = baseline[k]
// (fresh run).  One launch per score column k.  A CTA takes 32 people; warp g
// sums splits g, g + 8, g + 16, ... of each (a lane per person, so every
// load is 32 consecutive people of one split) into eight independent
// accumulators, so eight loads are in flight per thread; the accumulators,
// then the eight warps' sums (lane o of warp 0, g = 0..7), are added in a
// fixed order, so results are deterministic.
constexpr uint32_t kFinWarps = 8;
constexpr uint32_t kFinLanes = 8;   // independent accumulators per thread
__global__ void __launch_bounds__(32 * kFinWarps) gnm_finalize(FinalizeArgs a) {
  __shared__ double s_sum[kFinWarps][32];
  __shared__ uint32_t s_cnt[kFinWarps][32];
  const uint32_t lane = threadIdx.x & 31u, g = threadIdx.x >> 5;
  const uint64_t o = uint64_t(blockIdx.x) * 32 + lane;
  double s = 0.0;
  uint32_t c = 0;
  if (o < a.num_people) {
    const uint64_t f = a.out_to_fam ? a.out_to_fam[o] : o;
    double acc[kFinLanes];
#pragma unroll
    for (uint32_t u = 0; u < kFinLanes; ++u) acc[u] = 0.0;
    constexpr uint32_t kStep = kFinWarps * kFinLanes;
    uint32_t sp0 = g;
    for (; sp0 + (kFinLanes - 1) * kFinWarps < a.num_splits; sp0 += kStep) {
#pragma unroll
      for (uint32_t u = 0; u < kFinLanes; ++u) {
        const uint64_t at = uint64_t(sp0 + u * kFinWarps) * a.part_stride + f;
        acc[u] += a.part_sum[at];
        c += a.part_cnt[at];
      }
    }
#pragma unroll
    for (uint32_t u = 0; u < kFinLanes; ++u) {   // the last, partial round
      const uint32_t sp = sp0 + u * kFinWarps;
      if (sp < a.num_splits) {
        const uint64_t at = uint64_t(sp) * a.part_stride + f;
        acc[u] += a.part_sum[at];
        c += a.part_cnt[at];
      }
    }
#pragma unroll
    for (uint32_t u = 0; u < kFinLanes; ++u) s += acc[u];
  }
  s_sum[g][lane] = s;
  s_cnt[g][lane] = c;
  __syncthreads();
  if (g != 0 || o >= a.num_people) return;
  double t = a.baseline[a.k];
  uint32_t n = 0;
#pragma unroll
  for (uint32_t w = 0; w < kFinWarps; ++w) {
    t += s_sum[w][lane];
    n += s_cnt[w][lane];
  }
  a.sums[o * a.K + a.k] = t;
  a.counts[o * a.K + a.k] = n;
}

__global__ void gnm_decode(const uint8_t* rows, uint64_t pitch, uint64_t nv, uint64_t np,
                           int8_t* out, uint64_t out_pitch) {
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t v = blockIdx.y + uint64_t(blockIdx.z) * gridDim.y;
  if (i >= np || v >= nv) return;
  const uint32_t code = (rows[v * pitch + (i >> 2)] >> (2 * (i & 3))) & 3u;
  // batch.rs:489-503: d = hi*(lo+1), code 01 -> missing
  const int8_t d = code == 1u ? int8_t(-1) : int8_t((code >> 1) * ((code & 1u) + 1u));
  out[v * out_pitch + i] = d;
}

// One thread per 32-bit word of a row (16 people).  Same generator as the
// CPU oracle: key = mix64(seed) ^ v*C1 ^ i*C2, x = mix64(key), with i the
// cohort-wide person index i0 + local column (a person shard fills its own
// column slice of the cohort).
__global__ void gnm_synth_fill(uint8_t* rows, uint64_t pitch, uint64_t v0, uint64_t nv,
                               uint64_t i0, uint64_t np, const uint32_t* thr, uint64_t seed) {
  const uint64_t words = pitch / 4;
  const uint64_t w = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t j = blockIdx.y + uint64_t(blockIdx.z) * gridDim.y;
  if (w >= words || j >= nv) return;
  const uint32_t tm = thr[3 * j], t0 = thr[3 * j + 1], t1 = thr[3 * j + 2];
  const uint64_t v = v0 + j;
  const uint64_t sk = mix64(seed) ^ (v * 0xD1B54A32D192ED03ull);
  uint32_t word = 0;
#pragma unroll 4
  for (uint32_t q = 0; q < 16; ++q) {
    const uint64_t i = w * 16 + q;
    if (i < np) {
      const uint64_t x = mix64(sk ^ ((i0 + i) * 0x8CB92BA72F3D8DD7ull));
      const uint32_t um = uint32_t(x), ug = uint32_t(x >> 32);
      const uint32_t code = um < tm ? 1u : (ug < t0 ? 0u : (ug < t1 ? 2u : 3u));
      word |= code << (2 * q);
    }
  }
  reinterpret_cast<uint32_t*>(rows + j * pitch)[w] = word;
}

// Packed rows stored back to back (stride bpv, as in a .bed file) -> rows of
// `pitch` bytes (a multiple of 16, as TMA needs), zero padded.  One thread
// per 4-byte output word; byte loads keep unaligned source rows legal and
// are coalesced across the warp.
__global__ void gnm_repitch(const uint8_t* src, uint64_t bpv, uint64_t nrows, uint8_t* dst,
                            uint64_t pitch) {
  const uint64_t words = pitch / 4;
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nrows * words) return;
  const uint64_t r = i / words, c = (i % words) * 4;
  const uint8_t* s = src + r * bpv;
  uint32_t v = 0;
#pragma unroll
  for (uint32_t j = 0; j < 4; ++j)
    if (c + j < bpv) v |= uint32_t(s[c + j]) << (8 * j);
  reinterpret_cast<uint32_t*>(dst + r * pitch)[c / 4] = v;
}

// Watchdog self-test: one warp waits on an mbarrier that nothing ever arrives
// on, with the kernels' bounded-wait helper and a caller-chosen limit.  The
// wait expires, the kernel records the timeout in the error word the way the
// scoring kernels do and returns; the context stays usable.
__global__ void gnm_watchdog_probe(uint64_t limit_ns, uint32_t* err, uint64_t* waited_ns) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t b = smem_u32(&bar);
  if (threadIdx.x == 0) {
    mbar_init(b, 1);
    fence_mbar_init();
  }
  __syncthreads();
  const uint64_t t0 = global_timer_ns();
  const bool ok = mbar_wait_timed(b, 0, limit_ns);   // phase 0 never completes
  if (threadIdx.x == 0) {
    if (!ok) atomicOr(err, kErrTmaTimeout);
    *waited_ns = global_timer_ns() - t0;
  }
}

// ---- host launchers --------------------------------------------------------

cudaError_t launch_repitch(const uint8_t* src, uint64_t bpv, uint64_t nrows, uint8_t* dst,
                           uint64_t pitch, cudaStream_t s) {
  if (nrows == 0) return cudaSuccess;
  const uint64_t n = nrows * (pitch / 4);
  gnm_repitch<<<uint32_t((n + 255) / 256), 256, 0, s>>>(src, bpv, nrows, dst, pitch);
  return cudaGetLastError();
}

cudaError_t launch_watchdog_probe(uint64_t limit_ns, uint32_t* err, uint64_t* waited_ns,
                                  cudaStream_t s) {
  gnm_watchdog_probe<<<1, 32, 0, s>>>(limit_ns, err, waited_ns);
  return cudaGetLastError();
}

cudaError_t launch_plain_tables(const TableArgs& a, cudaStream_t s) {
  const uint64_t stages = (a.num_rows + kPlainRows - 1) / kPlainRows;
  if (stages == 0) return cudaSuccess;
  if (stages > 0x7FFFFFFFull) return cudaErrorInvalidValue;
  gnm_plain_tables<<<uint32_t(stages), kPlainGroups * 64, 0, s>>>(a);
  return cudaGetLastError();
}

template <uint32_t TILE, bool WS>
static cudaError_t launch_plain_tile(const CUtensorMap& map, const PlainArgs& a, uint32_t grid,
                                     cudaStream_t s) {
  using L = PlainSmem<TILE>;
  const cudaError_t e = raise_smem_limit(
      reinterpret_cast<const void*>(gnm_plain_accumulate<TILE, WS>), int(L::kTotal));
  if (e != cudaSuccess) return e;
  gnm_plain_accumulate<TILE, WS><<<grid, PlainShape<TILE, WS>::kThreads, L::kTotal, s>>>(map, a);
  return cudaGetLastError();
}

uint32_t plain_grid(const PlainArgs& a) {
  const uint64_t stages = (a.num_rows + kPlainRows - 1) / kPlainRows;
  const uint64_t last = (stages + a.last_stages_per_split - 1) / a.last_stages_per_split;
  return uint32_t(uint64_t(a.tiles - 1) * a.splits + last);
}

cudaError_t launch_plain_accumulate(const CUtensorMap& map, const PlainArgs& a, uint32_t kernel,
                                    cudaStream_t s) {
  if (a.tiles == 0 || a.splits == 0 || a.stages_per_split == 0 || a.last_stages_per_split == 0)
    return cudaErrorInvalidValue;
  const uint32_t grid = plain_grid(a);
  switch (kernel) {
    case kPlain512: return launch_plain_tile<512, false>(map, a, grid, s);
    case kPlain512Ws: return launch_plain_tile<512, true>(map, a, grid, s);
    case kPlain1024: return launch_plain_tile<1024, false>(map, a, grid, s);
    case kPlain1024Ws: return launch_plain_tile<1024, true>(map, a, grid, s);
    case kPlain2048Ws: return launch_plain_tile<2048, true>(map, a, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_finalize(const FinalizeArgs& a, cudaStream_t s) {
  const uint32_t blocks = uint32_t((a.num_people + 31) / 32);
  gnm_finalize<<<blocks ? blocks : 1, 32 * kFinWarps, 0, s>>>(a);
  return cudaGetLastError();
}

static dim3 rows_grid(uint64_t x_blocks, uint64_t nv) {
  uint64_t y = nv, z = 1;
  while (y > 65535) {
    z *= 2;
    y = (nv + z - 1) / z;
  }
  return dim3(uint32_t(x_blocks), uint32_t(y), uint32_t(z));
}

cudaError_t launch_decode(const uint8_t* rows, uint64_t pitch, uint64_t nv, uint64_t np,
                          int8_t* out, uint64_t out_pitch, cudaStream_t s) {
  if (nv == 0 || np == 0) return cudaSuccess;
  gnm_decode<<<rows_grid((np + 255) / 256, nv), 256, 0, s>>>(rows, pitch, nv, np, out, out_pitch);
  return cudaGetLastError();
}

cudaError_t launch_synth_fill(uint8_t* rows, uint64_t pitch, uint64_t v0, uint64_t nv,
                              uint64_t i0, uint64_t np, const uint32_t* thr, uint64_t seed,
                              cudaStream_t s) {
  if (nv == 0) return cudaSuccess;
  const uint64_t words = pitch / 4;
  gnm_synth_fill<<<rows_grid((words + 255) / 256, nv), 256, 0, s>>>(rows, pitch, v0, nv, i0, np,
                                                                    thr, seed);
  return cudaGetLastError();
}

}  // namespace gnm
