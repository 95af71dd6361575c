// gnm_tensor.cu — the tcgen05 tensor engine (many score columns) and the
// re-unpacking backward kernel dW = G^T dS, each on BF16 limbs (kind::f16)
// and on 8-bit integer limbs (kind::i8):
//   gnm_tc_accumulate / gnm_t8_accumulate  wide: scores as M, one SM per tile
//   gnm_t8_pairs                           wide, 8-bit, SM pairs (cta_group::2),
//                                          one persistent launch per call
//   gnm_tc_narrow / gnm_t8_narrow          narrow: people as M (<= 64 scores)
//   gnm_tc_backward / gnm_t8_backward      dW = G^T dS, dC on CUDA cores
// The BF16 forms come first below; each 8-bit form states what it changes.
//
// Scoring as a GEMM (the reference does this with three cuBLAS SGEMMs per
// score tile, score/cuda_backend.rs:2196-2233):
//   sum[p,k] = baseline[k] + sum_v W'[k,v] d(p,v) - sum_v C[k,v] m(p,v)
//   miss[p,k] = sum_v member[k,v] m(p,v)
// with d the allele-2 dosage (missing -> 0), m the missing indicator.
//
// Precision (the "hi/mid/lo" split): every weight-like value x of score k is
// written as hi + mid + lo (+ lo2 for dosage weights), each an integer multiple
// of a power-of-two quantum (q, q/2^8, q/2^16, q/2^24 with 2^E = 256 q >= max |x|
// of the score), |integer| <= 256, so every limb is exact in BF16.  Products with
// d in {0,1,2} and m in {0,1} are exact, every partial sum of one limb is an
// integer multiple of its quantum, and below 32768 variants its magnitude stays
// under 2^24 quanta: the FP32 tensor-memory accumulation of each limb is EXACT.
// Accumulators are flushed to FP64 every 16384 variants (the cross-block
// reduction is the only FP64 arithmetic).  The only error left is the limb
// residual: below 2^-33 of the score's largest weight for dosage weights (four
// limbs; with three it was 2^-25, and ~10^5 such residuals per sum reached
// 1e-6 of the score) and 2^-25 for missing corrections (three limbs; they touch
// only the ~1% missing calls).
//
// Kernel shape (one CTA per SM): M = 128 score rows (TMEM lanes), N = 256
// people (TMEM columns), K = 64 variants per stage, two limb planes per pass
// (2 x 256 FP32 accumulator columns fill the 512 TMEM columns), three stages
// of 68 KB in shared memory.  With 256 people per CTA every weight byte
// staged from L2 feeds twice the MMA work of a 128-person tile; the four
// passes (dosage limbs 0-1, dosage limbs 2-3, correction limbs 0-1,
// correction limb 2 + member count) each re-expand the genotypes, which is
// cheap CUDA-core work on separate warps.  Warp 0 issues TMA (weight limb
// planes, 3D map, 128-byte swizzle; packed rows, 2D map), warp 1 owns TMEM
// and issues tcgen05.mma, warps 2-5 expand packed 2-bit genotypes into the
// BF16 K-major operand in shared memory and drain TMEM at block ends.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "gnm_device.cuh"
#include "gnm_plan.h"
#include "gnm_tcgen05.cuh"
#include "gnm_tensor.h"

namespace gnm {

constexpr uint32_t kTcM = 128;        // score rows per tile
constexpr uint32_t kTcN = 256;        // people per tile
constexpr uint32_t kTcK = 64;         // variants per stage
constexpr uint32_t kTcFlush = 256;    // stages per exact FP32 block (16384 variants)
constexpr uint32_t kTcThreads = 192;  // 6 warps
constexpr int kTcPlanes = 2;          // limb planes per pass (2 x 256 TMEM columns)
constexpr int kTcStages = 3;          // pipeline stages (68 KB each)
constexpr uint64_t kNarrowMaxScores = 64;   // up to 4 narrow score tiles

struct TensorPlan {
  uint64_t K_pad = 0, V_pad = 0, P_pad = 0;
  uint32_t ptiles = 0, stiles = 0;
  __nv_bfloat16* d_planes_dos = nullptr;  // [4][K_pad][V_pad] W' limbs
  __nv_bfloat16* d_planes_mis = nullptr;  // [4][K_pad][V_pad] -corr limbs, member
  double* d_part_sum = nullptr;           // wide: [K_pad][P_pad]; narrow: [nsplits][K16][P_pad]
  uint32_t* d_part_cnt = nullptr;
  uint64_t part_elems = 0;                // elements of d_part_sum / d_part_cnt
  uint32_t nsplits = 1;                   // narrow: variant splits (grid z)
  uint64_t nslot = 0;                     // narrow: elements per split slot (K16 * P_pad)
  CUtensorMap map_dos, map_mis;
  int8_t* d_planes8 = nullptr;            // [9][K_pad][V_pad8] 8-bit limbs (dosage, -corr, member)
  double* d_quanta8 = nullptr;            // [9][K_pad] quantum of each 8-bit plane
  uint64_t V_pad8 = 0;
  CUtensorMap map8_2, map8_1;             // boxes of two planes / one plane
  bool i8 = false;                        // wide GEMM on 8-bit limbs (gnm_t8_accumulate)
  bool pair = false;                      // ... over SM pairs (gnm_t8_pairs)
  double* d_part_pass = nullptr;          // SM pairs, passes 1-3: [3][K_pad][P_pad]
  bool pass_valid = false;                // d_part_pass written since the last reset
  bool narrow = false;                    // few scores: gnm_tc_narrow (people as M)
  bool can_narrow = false;                // K <= 64: either kernel can run the plan
  CUtensorMap nmap_dos, nmap_mis;         // narrow boxes: 16 scores x 4 planes
  CUtensorMap nmap8_dos, nmap8_mis;       // narrow 8-bit boxes: 128 variants x 16 scores x 4 / 5 planes
};

struct TcArgs {
  uint64_t num_rows;       // rows of this block
  int32_t a_x0;            // absolute variant index of block row 0 (multiple of 64)
  double* part_sum;
  uint32_t* part_cnt;
  uint64_t P_pad;
  uint32_t* err;
  uint32_t raster;         // 0: blockIdx.x = people tile, 1: blockIdx.x = score tile
  int32_t z0;              // first limb plane of this pass (TMA z coordinate)
};

template <int NP, int ST>
struct TcSmem {
  static constexpr uint32_t kPlane = kTcM * kTcK * 2;   // 16 KB
  static constexpr uint32_t kAStage = NP * kPlane;
  static constexpr uint32_t kB = kTcN * kTcK * 2;       // 32 KB
  static constexpr uint32_t kPk = kTcK * (kTcN / 4);    // 4 KB
  static constexpr uint32_t kAOff = 0;
  static constexpr uint32_t kBOff = kAOff + ST * kAStage;
  static constexpr uint32_t kPkOff = kBOff + ST * kB;
  static constexpr uint32_t kBarOff = kPkOff + ST * kPk;
  static constexpr uint32_t kHolder = kBarOff + 8 * (3 * ST + 2);
  static constexpr uint32_t kTotal = kHolder + 16 + 1024;  // + alignment slack
};

// code -> BF16 byte tables for __byte_perm (pool bytes 0-3: low bytes by
// code, 4-7: high bytes by code).  Dosage: 00->0, 01(missing)->0, 10->1, 11->2.
// Missing indicator: 01 -> 1, else 0.
constexpr uint32_t kDosLo = 0x00800000u, kDosHi = 0x403F0000u;
constexpr uint32_t kMisLo = 0x00008000u, kMisHi = 0x00003F00u;

__device__ __forceinline__ uint32_t bf16_pair(uint32_t y16, uint32_t lo, uint32_t hi) {
  return __byte_perm(lo, hi, y16 * 0x11u + 0x4040u);
}

// MISSING: the B operand is the missing indicator (else the dosage).
// COUNT_LAST: the pass's last plane is the member plane; its products are the
// missing counts (else every plane is a limb of the pass's sum).
template <int NP, int ST, bool MISSING, bool COUNT_LAST>
__global__ void __launch_bounds__(kTcThreads, 1)
    gnm_tc_accumulate(const __grid_constant__ CUtensorMap amap,
                      const __grid_constant__ CUtensorMap pmap, TcArgs a) {
  using L = TcSmem<NP, ST>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sb = smem_u32(smem);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t ptile = a.raster ? blockIdx.y : blockIdx.x;
  const uint32_t stile = a.raster ? blockIdx.x : blockIdx.y;
  const uint32_t nit = uint32_t((a.num_rows + kTcK - 1) / kTcK);
  auto full = [&](uint32_t s) { return sb + L::kBarOff + 8 * s; };
  auto bready = [&](uint32_t s) { return sb + L::kBarOff + 8 * (ST + s); };
  auto empty = [&](uint32_t s) { return sb + L::kBarOff + 8 * (2 * ST + s); };
  const uint32_t accfull = sb + L::kBarOff + 8 * (3 * ST);
  const uint32_t accempty = sb + L::kBarOff + 8 * (3 * ST + 1);
  volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + L::kHolder + 8);
  const uint32_t abort_addr = sb + L::kHolder + 8;

  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < ST; ++s) {
      mbar_init(full(s), 1);
      mbar_init(bready(s), 128);
      mbar_init(empty(s), 1);
    }
    mbar_init(accfull, 1);
    mbar_init(accempty, 128);
    *abort_flag = 0u;
    fence_mbar_init();
    prefetch_tmap(&amap);
    prefetch_tmap(&pmap);
  }
  if (warp == 1) {
    tmem_alloc(sb + L::kHolder, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + L::kHolder);

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST, ph = (it / ST) & 1u;
        if (!mbar_wait_bounded(empty(s), ph ^ 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        mbar_arrive_expect_tx(full(s), L::kAStage + L::kPk);
        tma_load_3d(sb + L::kAOff + s * L::kAStage, &amap, a.a_x0 + int32_t(it * kTcK),
                    int32_t(stile * kTcM), a.z0, full(s));
        tma_load_2d(sb + L::kPkOff + s * L::kPk, &pmap, int32_t(ptile * (kTcN / 4)),
                    int32_t(it * kTcK), full(s));
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_bf16_f32(kTcM, kTcN);
      uint32_t blk = 0;
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST, ph = (it / ST) & 1u;
        const bool first = (it % kTcFlush) == 0;
        if (first && it > 0) {
          if (!mbar_wait_bounded(accempty, (blk - 1) & 1u)) {
            *abort_flag = 1u;
            atomicOr(a.err, kErrMmaTimeout);
            break;
          }
        }
        if (!mbar_wait_bounded(bready(s), ph)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        tc_fence_after();
        const uint32_t a0 = sb + L::kAOff + s * L::kAStage;
        const uint32_t b0 = sb + L::kBOff + s * L::kB;
#pragma unroll
        for (uint32_t kk = 0; kk < kTcK / 16; ++kk) {
          const uint64_t bdesc = desc_kmajor_sw128(b0 + kk * 32);
#pragma unroll
          for (uint32_t j = 0; j < NP; ++j) {
            const uint64_t adesc = desc_kmajor_sw128(a0 + j * L::kPlane + kk * 32);
            tc_mma_f16(tmem + j * kTcN, adesc, bdesc, idesc, (first && kk == 0) ? 0u : 1u);
          }
        }
        tc_commit(empty(s));
        if ((it % kTcFlush) == kTcFlush - 1 || it == nit - 1) {
          tc_commit(accfull);
          ++blk;
        }
      }
    }
  } else {
    // ---------------- genotype expansion + epilogue (warps 2-5) ----------------
    const uint32_t pt = threadIdx.x - 64;      // 0..127
    const uint32_t col = pt & 31;              // byte column: people 4col..4col+3
    const uint32_t vg = pt >> 5;               // variant group: rows 16vg..16vg+15
    const uint32_t quad = warp & 3;            // TMEM lane quadrant of this warp
    uint32_t blk = 0;
    for (uint32_t it = 0; it < nit; ++it) {
      const uint32_t s = it % ST, ph = (it / ST) & 1u;
      if (!mbar_wait_bounded(full(s), ph)) {
        *abort_flag = 1u;
        atomicOr(a.err, kErrTmaTimeout);
        break;
      }
      if (lds_volatile_u32(abort_addr)) break;
      // explicit shared-space accesses: the realigned base is a generic pointer
      const uint32_t pk = sb + L::kPkOff + s * L::kPk;
      const uint32_t bt = sb + L::kBOff + s * L::kB;
#pragma unroll
      for (uint32_t h = 0; h < kTcN / 128; ++h) {
        const uint32_t bc = 32 * h + col;   // byte column: people 4bc..4bc+3
#pragma unroll
        for (uint32_t cc = 0; cc < 2; ++cc) {
          const uint32_t r0 = 16 * vg + 8 * cc;
          uint32_t xl = 0, xh = 0;
#pragma unroll
          for (uint32_t i = 0; i < 4; ++i) {
            xl |= lds_u8(pk + (r0 + i) * (kTcN / 4) + bc) << (8 * i);
            xh |= lds_u8(pk + (r0 + 4 + i) * (kTcN / 4) + bc) << (8 * i);
          }
          const uint32_t c = 2 * vg + cc;  // 16-byte chunk (8 variants) index
#pragma unroll
          for (uint32_t q = 0; q < 4; ++q) {
            const uint32_t yl = (xl >> (2 * q)) & 0x03030303u;
            const uint32_t yh = (xh >> (2 * q)) & 0x03030303u;
            const uint32_t lo = MISSING ? kMisLo : kDosLo, hi = MISSING ? kMisHi : kDosHi;
            uint4 v;
            v.x = bf16_pair(yl & 0xFFFFu, lo, hi);
            v.y = bf16_pair(yl >> 16, lo, hi);
            v.z = bf16_pair(yh & 0xFFFFu, lo, hi);
            v.w = bf16_pair(yh >> 16, lo, hi);
            // operand row of person 128h + 4col + q (conflict-free 16-byte stores)
            const uint32_t n = 128 * h + 32 * q + col;
            sts_u128(bt + (n >> 3) * 1024 + (n & 7) * 128 + ((c ^ (n & 7)) << 4), v);
          }
        }
      }
      fence_proxy_async_smem();
      mbar_arrive(bready(s));

      if ((it % kTcFlush) == kTcFlush - 1 || it == nit - 1) {
        if (!mbar_wait_bounded(accfull, blk & 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        tc_fence_after();
        const uint64_t k = uint64_t(stile) * kTcM + 32 * quad + lane;
        double* ps = a.part_sum + k * a.P_pad + uint64_t(ptile) * kTcN;
        uint32_t* pc = a.part_cnt + k * a.P_pad + uint64_t(ptile) * kTcN;
        const uint32_t lane_base = tmem + ((32 * quad) << 16);
#pragma unroll 1
        for (uint32_t cb = 0; cb < kTcN / 32; ++cb) {
          double acc[32];
#pragma unroll
          for (int i = 0; i < 32; ++i) acc[i] = 0.0;
          // limb planes of this pass's sum (the member plane, when present, is last)
          constexpr uint32_t kSum = COUNT_LAST ? uint32_t(NP) - 1u : uint32_t(NP);
#pragma unroll
          for (uint32_t j = 0; j < kSum; ++j) {
            uint32_t r[32];
            tmem_ld32(lane_base + j * kTcN + 32 * cb, r);
            tmem_ld_wait();
#pragma unroll
            for (int i = 0; i < 32; ++i) acc[i] += double(__uint_as_float(r[i]));
          }
#pragma unroll
          for (int i = 0; i < 32; ++i) ps[32 * cb + i] += acc[i];
          if (COUNT_LAST) {
            uint32_t r[32];
            tmem_ld32(lane_base + (NP - 1) * kTcN + 32 * cb, r);
            tmem_ld_wait();
#pragma unroll
            for (int i = 0; i < 32; ++i) pc[32 * cb + i] += __float2uint_rn(__uint_as_float(r[i]));
          }
        }
        tc_fence_before();
        mbar_arrive(accempty);
        ++blk;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ---- 8-bit integer wide engine ---------------------------------------------------
// The wide GEMM of gnm_tc_accumulate with tcgen05.mma kind::i8: twice the MMA
// rate of BF16 per instruction, signed 8-bit weight limbs against unsigned
// 8-bit genotype operands (dosage 0/1/2 or the missing indicator), S32
// accumulators in tensor memory.  Every dosage weight of score k is split as
// l0 q0 + l1 q1 + l2 q2 + l3 q3 with q0 = max |x| of the score's values / 127,
// q(i+1) = q(i) / 254 and integers |l| <= 127 (each rounding leaves a
// remainder of at most half a quantum, which the next limb covers at 1/254 of
// that quantum), so the residual is below q3 / 2, 2^-31.9 of the score's
// largest value; missing corrections likewise.  (Three correction limbs,
// 2^-23.9, gave 5.4e-7 of the reference's 1e-6 tolerance on the biobank
// workload at full length.)  Products and
// their sums are exact integers in S32 for blocks of up to 2^23 variants; each
// plane's block sum reaches FP64 as int x its quantum at the flush, once per
// block (the flush's partial read-modify-write is one score row per lane, so
// flushing rarely keeps the memory queues free for the expansion).  Nine
// planes: dosage limbs 0-3, -correction limbs 0-3 and the member plane, in
// five passes (two planes fill tensor memory's 2 x 256 S32 columns; the
// member plane runs alone), each re-expanding the genotypes: dosage limbs
// 0-1 and 2-3 against the dosage operand, correction limbs 0-1 and 2-3 and
// the member plane against the missing indicator.  K = 128 variants per
// stage (a 128-byte K-major row), so a stage holds twice the variants of the
// BF16 kernel in the same bytes.
constexpr uint32_t kT8K = 128;       // variants per stage
// stages per flushed block: 2^23 variants, where |limb x dosage| <= 254 per
// variant keeps every S32 sum exact (254 x 2^23 < 2^31); an accumulate call
// shorter than that flushes once, at its end
constexpr uint32_t kT8Flush = (1u << 23) / kT8K;
constexpr int kT8Planes = 9;
constexpr uint32_t kT8Expand = 256;                 // expansion / epilogue threads (8 warps)
constexpr uint32_t kT8Threads = 64 + kT8Expand;     // + TMA warp + MMA warp
constexpr int kT8StagesPair = 4;   // TMA ring depth of two-plane passes (4 x 40 KB + 2 x 32 KB)
constexpr int kT8StagesOne = 6;    // of the one-plane pass (6 x 24 KB + 2 x 32 KB)

// ST: depth of the TMA ring (weight limbs + packed rows of a stage); the
// expanded genotype operand has its own two-deep ring, freed as soon as the
// stage's MMAs complete, so the TMA loads run ST stages ahead while the
// operand takes only two slots.
template <int NP, int ST>
struct T8Smem {
  static constexpr uint32_t kBStages = 2;
  static constexpr uint32_t kPlane = kTcM * kT8K;       // 16 KB
  static constexpr uint32_t kAStage = NP * kPlane;
  static constexpr uint32_t kB = kTcN * kT8K;           // 32 KB
  static constexpr uint32_t kPk = kT8K * (kTcN / 4);    // 8 KB
  static constexpr uint32_t kAOff = 0;
  static constexpr uint32_t kPkOff = kAOff + ST * kAStage;
  static constexpr uint32_t kBOff = kPkOff + ST * kPk;
  static constexpr uint32_t kBarOff = kBOff + kBStages * kB;
  static constexpr uint32_t kHolder = kBarOff + 8 * (2 * ST + 2 * kBStages + 2);
  static constexpr uint32_t kTotal = kHolder + 16 + 1024;  // + alignment slack
  static_assert(kTotal <= 227 * 1024, "shared memory");
  static_assert(kBOff % 1024 == 0 && kPkOff % 1024 == 0, "swizzled operands need 1 KB alignment");
};

struct T8Args {
  uint64_t num_rows;       // rows of this block
  int32_t a_x0;            // absolute variant index of block row 0 (multiple of 128)
  double* part_sum;
  uint32_t* part_cnt;
  uint64_t P_pad;
  uint64_t K_pad;
  const double* quanta;    // [kT8Planes][K_pad] quantum of every plane of every score
  uint32_t* err;
  uint32_t raster;         // 0: blockIdx.x = people tile, 1: blockIdx.x = score tile
  int32_t z0;              // first plane of this pass (TMA z coordinate)
};

// Sixteen 2-bit genotype codes -> sixteen 2-bit operand values in place: the
// allele-2 dosage (00 -> 0, 01 -> 0, 10 -> 1, 11 -> 2: low bit hi & ~lo, high
// bit hi & lo), or the missing indicator (01 -> 1).  Person q's values of
// four rows are then (w >> 2q) & 0x03030303, one per byte.
template <bool MISSING>
__device__ __forceinline__ uint32_t code_fields(uint32_t x) {
  const uint32_t hi = (x >> 1) & 0x55555555u, lo = x & 0x55555555u;
  return MISSING ? (lo & ~hi) : ((hi & ~lo) | ((hi & lo) << 1));
}

template <int NP, int ST, bool MISSING, bool COUNT_LAST>
__global__ void __launch_bounds__(kT8Threads, 1)
    gnm_t8_accumulate(const __grid_constant__ CUtensorMap amap,
                      const __grid_constant__ CUtensorMap pmap, T8Args a) {
  using L = T8Smem<NP, ST>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sb = smem_u32(smem);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t ptile = a.raster ? blockIdx.y : blockIdx.x;
  const uint32_t stile = a.raster ? blockIdx.x : blockIdx.y;
  const uint32_t nit = uint32_t((a.num_rows + kT8K - 1) / kT8K);
  constexpr uint32_t BS = L::kBStages;
  auto full = [&](uint32_t s) { return sb + L::kBarOff + 8 * s; };          // TMA landed
  auto aempty = [&](uint32_t s) { return sb + L::kBarOff + 8 * (ST + s); }; // TMA slot free
  auto bready = [&](uint32_t b) { return sb + L::kBarOff + 8 * (2 * ST + b); };
  auto bempty = [&](uint32_t b) { return sb + L::kBarOff + 8 * (2 * ST + BS + b); };
  const uint32_t accfull = sb + L::kBarOff + 8 * (2 * ST + 2 * BS);
  const uint32_t accempty = sb + L::kBarOff + 8 * (2 * ST + 2 * BS + 1);
  volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + L::kHolder + 8);
  const uint32_t abort_addr = sb + L::kHolder + 8;

  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < ST; ++s) {
      mbar_init(full(s), 1);
      mbar_init(aempty(s), 1);
    }
    for (uint32_t b = 0; b < BS; ++b) {
      mbar_init(bready(b), kT8Expand);
      mbar_init(bempty(b), 1);
    }
    mbar_init(accfull, 1);
    mbar_init(accempty, kT8Expand);
    *abort_flag = 0u;
    fence_mbar_init();
    prefetch_tmap(&amap);
    prefetch_tmap(&pmap);
  }
  if (warp == 1) {
    tmem_alloc(sb + L::kHolder, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + L::kHolder);

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST, ph = (it / ST) & 1u;
        if (!mbar_wait_bounded(aempty(s), ph ^ 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        mbar_arrive_expect_tx(full(s), L::kAStage + L::kPk);
        tma_load_3d(sb + L::kAOff + s * L::kAStage, &amap, a.a_x0 + int32_t(it * kT8K),
                    int32_t(stile * kTcM), a.z0, full(s));
        tma_load_2d(sb + L::kPkOff + s * L::kPk, &pmap, int32_t(ptile * (kTcN / 4)),
                    int32_t(it * kT8K), full(s));
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_s8u8_s32(kTcM, kTcN);
      uint32_t blk = 0;
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST;
        const uint32_t bsl = it % BS, bph = (it / BS) & 1u;
        const bool first = (it % kT8Flush) == 0;
        if (first && it > 0) {
          if (!mbar_wait_bounded(accempty, (blk - 1) & 1u)) {
            *abort_flag = 1u;
            atomicOr(a.err, kErrMmaTimeout);
            break;
          }
        }
        if (!mbar_wait_bounded(bready(bsl), bph)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        tc_fence_after();
        const uint32_t a0 = sb + L::kAOff + s * L::kAStage;
        const uint32_t b0 = sb + L::kBOff + bsl * L::kB;
#pragma unroll
        for (uint32_t kk = 0; kk < kT8K / 32; ++kk) {   // K = 32 bytes per MMA
          const uint64_t bdesc = desc_kmajor_sw128(b0 + kk * 32);
#pragma unroll
          for (uint32_t j = 0; j < NP; ++j) {
            const uint64_t adesc = desc_kmajor_sw128(a0 + j * L::kPlane + kk * 32);
            tc_mma_i8(tmem + j * kTcN, adesc, bdesc, idesc, (first && kk == 0) ? 0u : 1u);
          }
        }
        tc_commit(aempty(s));
        tc_commit(bempty(bsl));
        if ((it % kT8Flush) == kT8Flush - 1 || it == nit - 1) {
          tc_commit(accfull);
          ++blk;
        }
      }
    }
  } else {
    // ---------------- genotype expansion + epilogue (warps 2-9) ----------------
    // warp 2 + 4h + vg: people half h (128 people), 16-variant chunks 2vg and
    // 2vg + 1; at block ends it drains TMEM lane quadrant warp % 4, column
    // blocks of its half
    const uint32_t ew = warp - 2;              // 0..7
    const uint32_t col = lane;                 // byte column: people 4col..4col+3
    const uint32_t vg = ew & 3;
    const uint32_t h = ew >> 2;
    const uint32_t quad = warp & 3;            // TMEM lane quadrant of this warp
    uint32_t blk = 0;
    for (uint32_t it = 0; it < nit; ++it) {
      const uint32_t s = it % ST, ph = (it / ST) & 1u;
      const uint32_t bsl = it % BS, bph = (it / BS) & 1u;
      if (!mbar_wait_bounded(full(s), ph)) {
        *abort_flag = 1u;
        atomicOr(a.err, kErrTmaTimeout);
        break;
      }
      // the operand slot is free once the MMAs of stage it - BS completed
      if (!mbar_wait_bounded(bempty(bsl), bph ^ 1u)) {
        *abort_flag = 1u;
        atomicOr(a.err, kErrMmaTimeout);
        break;
      }
      if (lds_volatile_u32(abort_addr)) break;
      const uint32_t pk = sb + L::kPkOff + s * L::kPk;
      const uint32_t bt = sb + L::kBOff + bsl * L::kB;
      {
        const uint32_t bc = 32 * h + col;   // byte column: people 4bc..4bc+3
#pragma unroll
        for (uint32_t cc = 0; cc < 2; ++cc) {
          const uint32_t c = 2 * vg + cc;   // 16-byte chunk (16 variants) of the operand row
          uint32_t x[4] = {0u, 0u, 0u, 0u};
#pragma unroll
          for (uint32_t i = 0; i < 16; ++i)
            x[i >> 2] |= lds_u8(pk + (16 * c + i) * (kTcN / 4) + bc) << (8 * (i & 3));
#pragma unroll
          for (uint32_t i = 0; i < 4; ++i) x[i] = code_fields<MISSING>(x[i]);
#pragma unroll
          for (uint32_t q = 0; q < 4; ++q) {
            uint4 v;
            v.x = (x[0] >> (2 * q)) & 0x03030303u;
            v.y = (x[1] >> (2 * q)) & 0x03030303u;
            v.z = (x[2] >> (2 * q)) & 0x03030303u;
            v.w = (x[3] >> (2 * q)) & 0x03030303u;
            // operand row of person 128h + 4col + q (conflict-free 16-byte stores)
            const uint32_t n = 128 * h + 32 * q + col;
            sts_u128(bt + (n >> 3) * 1024 + (n & 7) * 128 + ((c ^ (n & 7)) << 4), v);
          }
        }
      }
      fence_proxy_async_smem();
      mbar_arrive(bready(bsl));

      if ((it % kT8Flush) == kT8Flush - 1 || it == nit - 1) {
        if (!mbar_wait_bounded(accfull, blk & 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        tc_fence_after();
        const uint64_t k = uint64_t(stile) * kTcM + 32 * quad + lane;
        double* ps = a.part_sum + k * a.P_pad + uint64_t(ptile) * kTcN;
        uint32_t* pc = a.part_cnt + k * a.P_pad + uint64_t(ptile) * kTcN;
        const uint32_t lane_base = tmem + ((32 * quad) << 16);
        constexpr uint32_t kSum = COUNT_LAST ? uint32_t(NP) - 1u : uint32_t(NP);
        double qv[NP];
#pragma unroll
        for (uint32_t j = 0; j < uint32_t(NP); ++j) qv[j] = a.quanta[(a.z0 + j) * a.K_pad + k];
#pragma unroll 1
        for (uint32_t cb = h * (kTcN / 64); cb < (h + 1) * (kTcN / 64); ++cb) {
          if constexpr (kSum > 0) {
            double acc[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) acc[i] = 0.0;
#pragma unroll
            for (uint32_t j = 0; j < kSum; ++j) {
              uint32_t r[32];
              tmem_ld32(lane_base + j * kTcN + 32 * cb, r);
              tmem_ld_wait();
#pragma unroll
              for (int i = 0; i < 32; ++i) acc[i] = fma(double(int32_t(r[i])), qv[j], acc[i]);
            }
#pragma unroll
            for (int i = 0; i < 32; ++i) ps[32 * cb + i] += acc[i];
          }
          if (COUNT_LAST) {
            uint32_t r[32];
            tmem_ld32(lane_base + (NP - 1) * kTcN + 32 * cb, r);
            tmem_ld_wait();
#pragma unroll
            for (int i = 0; i < 32; ++i) pc[32 * cb + i] += r[i];
          }
        }
        tc_fence_before();
        mbar_arrive(accempty);
        ++blk;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ---- 8-bit wide engine on SM pairs ---------------------------------------------
// gnm_t8_accumulate with one tcgen05.mma.cta_group::2 spanning the two CTAs of
// a cluster: M = 256 scores (128 per CTA), N = 256 people (128 per CTA), K =
// 32 variants per instruction.  On one SM the N = 256 operand is read from
// shared memory once per plane and expanded by that SM alone, and the
// stage's shared-memory traffic (weight and genotype TMA writes, operand
// stores, MMA operand reads) takes longer than its MMAs; over a pair each SM
// stores, expands and serves only its 128 people, and each CTA's tensor
// memory still holds its 128 scores x all 256 people per plane.
//
// Roles per CTA: warp 0 issues the CTA's own TMA loads (its 128 scores' limb
// planes, its 128 people's packed rows) onto its own mbarriers; warps 2-9
// expand the CTA's genotypes into its half of the B operand and arrive (one
// lane per warp, after an async-proxy fence) on the even (leader) CTA's
// operand barrier, after the CTA's own TMA for the stage landed, so the
// arrival also vouches for its A half; warp 1 of the leader alone issues the
// MMAs, and its commits arrive on the freeing barriers of both CTAs
// (tcgen05.commit multicast).  Each CTA's epilogue drains its own 128 score
// rows; the leader waits for both epilogues before it overwrites the
// accumulators of the next block.  Every wait is bounded; a cluster barrier
// keeps both CTAs resident until neither can touch the other's shared
// memory, and tensor memory is allocated and released by warp 1 of both CTAs
// together.  The operand ring is four deep: every hand-off between the CTAs
// of a pair (operand ready, slot free) crosses SMs, so the expansion runs
// further ahead of the MMAs than on one SM.  The member plane's pass spans
// two score pairs per cluster (two planes' MMA work, like the other passes).
constexpr int kT8PairStagesPair = 4;  // TMA ring depth, two planes (4 x 36 KB + 4 x 16 KB)

template <int NP, int ST>
struct T8PairSmem {
  static constexpr uint32_t kBStages = 4;
  static constexpr uint32_t kPlane = kTcM * kT8K;         // 16 KB: 128 scores x 128 variants
  static constexpr uint32_t kAStage = NP * kPlane;
  static constexpr uint32_t kB = (kTcN / 2) * kT8K;       // 16 KB: this CTA's 128 people
  static constexpr uint32_t kPkRow = kTcN / 8;            // 32 packed bytes per variant row
  static constexpr uint32_t kPk = kT8K * kPkRow;          // 4 KB
  static constexpr uint32_t kAOff = 0;
  static constexpr uint32_t kPkOff = kAOff + ST * kAStage;
  static constexpr uint32_t kBOff = kPkOff + ST * kPk;
  static constexpr uint32_t kBarOff = kBOff + kBStages * kB;
  static constexpr uint32_t kHolder = kBarOff + 8 * (2 * ST + 2 * kBStages + 3);
  static constexpr uint32_t kTotal = kHolder + 16 + 1024;  // + alignment slack
  static_assert(kTotal <= 227 * 1024, "shared memory");
  static_assert(kBOff % 1024 == 0 && kPkOff % 1024 == 0, "swizzled operands need 1 KB alignment");
};

// One persistent launch per accumulate call: each cluster walks the work items
// w = cluster, cluster + clusters, ... of a static list, pass-major: passes
// 0-3 (dosage limbs 0-1 and 2-3, correction limbs 0-1 and 2-3) over every
// (people tile, score pair), then pass 4 (the member plane) over every
// (people tile, two score pairs).  Passes 1-3 add into FP64 partial arrays of
// their own, since a tile's passes may run on different clusters at the same
// time; pass 0 adds into the plan's partials with the other kernels, and the
// first call after a reset writes the pass arrays instead of adding to them.
struct T8PairArgs {
  uint64_t num_rows;       // rows of this block
  int32_t a_x0;            // absolute variant index of block row 0 (multiple of 128)
  double* part_sum;        // pass 0 (and every other kernel): [K_pad][P_pad]
  double* part_pass;       // passes 1-3: [3][K_pad][P_pad]
  uint32_t* part_cnt;
  uint64_t P_pad;
  uint64_t K_pad;
  const double* quanta;    // [kT8Planes][K_pad]
  uint32_t* err;
  uint32_t raster;         // 1: score pairs fastest within a pass
  uint32_t ptiles, spairs, spairs_m;   // people tiles, score pairs, pairs of score pairs
  uint32_t items;          // 4 * ptiles * spairs + ptiles * spairs_m
  uint32_t store;          // the pass arrays are written, not added to
};

struct PairItem {
  uint32_t pass, ptile, spair;   // pass 4: spair = index of the pair of score pairs
};

__device__ __forceinline__ PairItem pair_item(const T8PairArgs& a, uint32_t w) {
  const uint32_t per = a.ptiles * a.spairs;
  PairItem r;
  uint32_t t, sp;
  if (w < 4 * per) {
    r.pass = w / per;
    t = w % per;
    sp = a.spairs;
  } else {
    r.pass = 4;
    t = w - 4 * per;
    sp = a.spairs_m;
  }
  r.ptile = a.raster ? t / sp : t % a.ptiles;
  r.spair = a.raster ? t % sp : t / a.ptiles;
  return r;
}

template <int ST>
__global__ void __launch_bounds__(kT8Threads, 1)
    gnm_t8_pairs(const __grid_constant__ CUtensorMap amap2,
                 const __grid_constant__ CUtensorMap amap1,
                 const __grid_constant__ CUtensorMap pmap, T8PairArgs a) {
  using L = T8PairSmem<2, ST>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sb = smem_u32(smem);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();   // 0: leader (issues the MMAs), 1: peer
  const uint32_t cid = blockIdx.x >> 1, ncl = gridDim.x >> 1;
  // this CTA's first score row of plane j of an item (uniform per CTA)
  auto srow = [&](const PairItem& w, uint32_t j) -> uint32_t {
    return w.pass == 4 ? (2 * (2 * w.spair + j) + rank) * kTcM : (2 * w.spair + rank) * kTcM;
  };
  const uint32_t nit = uint32_t((a.num_rows + kT8K - 1) / kT8K);
  constexpr uint32_t BS = L::kBStages;
  auto full = [&](uint32_t s) { return sb + L::kBarOff + 8 * s; };          // TMA landed
  auto aempty = [&](uint32_t s) { return sb + L::kBarOff + 8 * (ST + s); }; // TMA slot free
  auto bready = [&](uint32_t b) { return sb + L::kBarOff + 8 * (2 * ST + b); };
  auto bempty = [&](uint32_t b) { return sb + L::kBarOff + 8 * (2 * ST + BS + b); };
  const uint32_t accfull = sb + L::kBarOff + 8 * (2 * ST + 2 * BS);
  const uint32_t accempty = sb + L::kBarOff + 8 * (2 * ST + 2 * BS + 1);
  const uint32_t drain = sb + L::kBarOff + 8 * (2 * ST + 2 * BS + 2);
  volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + L::kHolder + 8);
  const uint32_t abort_addr = sb + L::kHolder + 8;

  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < ST; ++s) {
      mbar_init(full(s), 1);
      mbar_init(aempty(s), 1);
    }
    for (uint32_t b = 0; b < BS; ++b) {
      mbar_init(bready(b), 2 * kT8Expand / 32);   // one arrival per expansion warp of both CTAs
      mbar_init(bempty(b), 1);
    }
    mbar_init(accfull, 1);
    mbar_init(accempty, 2 * kT8Expand);
    mbar_init(drain, 1);
    *abort_flag = 0u;
    fence_mbar_init();
    prefetch_tmap(&amap2);
    prefetch_tmap(&amap1);
    prefetch_tmap(&pmap);
  }
  if (warp == 1) {
    tmem_alloc_pair(sb + L::kHolder, 512);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  cluster_sync_all();   // barriers of both CTAs initialised, tensor memory allocated
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + L::kHolder);

  if (warp == 0) {
    // ---------------- TMA producer (each CTA its own halves) ----------------
    if (lane == 0) {
      uint32_t g = 0;   // stages issued so far, over every item
      bool stop = false;
      for (uint32_t wi = cid; wi < a.items && !stop; wi += ncl) {
        const PairItem w = pair_item(a, wi);
        for (uint32_t it = 0; it < nit; ++it, ++g) {
          const uint32_t s = g % ST, ph = (g / ST) & 1u;
          if (!mbar_wait_bounded(aempty(s), ph ^ 1u)) {
            *abort_flag = 1u;
            atomicOr(a.err, kErrMmaTimeout);
            stop = true;
            break;
          }
          if (lds_volatile_u32(abort_addr)) {
            stop = true;
            break;
          }
          mbar_arrive_expect_tx(full(s), L::kAStage + L::kPk);
          const uint32_t a_st = sb + L::kAOff + s * L::kAStage;
          const int32_t x = a.a_x0 + int32_t(it * kT8K);
          if (w.pass == 4) {   // the member plane of two score pairs
            tma_load_3d(a_st, &amap1, x, int32_t(srow(w, 0)), 8, full(s));
            tma_load_3d(a_st + L::kPlane, &amap1, x, int32_t(srow(w, 1)), 8, full(s));
          } else {
            tma_load_3d(a_st, &amap2, x, int32_t(srow(w, 0)), int32_t(2 * w.pass), full(s));
          }
          tma_load_2d(sb + L::kPkOff + s * L::kPk, &pmap,
                      int32_t(w.ptile * (kTcN / 4) + rank * L::kPkRow), int32_t(it * kT8K),
                      full(s));
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (leader CTA only) ----------------
    if (lane == 0 && rank == 0) {
      constexpr uint32_t idesc = idesc_s8u8_s32(2 * kTcM, kTcN);
      uint32_t g = 0, blk = 0;
      bool stop = false;
      for (uint32_t wi = cid; wi < a.items && !stop; wi += ncl) {
        for (uint32_t it = 0; it < nit; ++it, ++g) {
          const uint32_t s = g % ST;
          const uint32_t bsl = g % BS, bph = (g / BS) & 1u;
          const bool first = (it % kT8Flush) == 0;
          if (first && blk > 0) {
            // the epilogues of both CTAs drained the previous block
            if (!mbar_wait_bounded_cluster(accempty, (blk - 1) & 1u)) {
              *abort_flag = 1u;
              atomicOr(a.err, kErrMmaTimeout);
              stop = true;
              break;
            }
          }
          if (!mbar_wait_bounded(bready(bsl), bph)) {
            *abort_flag = 1u;
            atomicOr(a.err, kErrMmaTimeout);
            stop = true;
            break;
          }
          if (lds_volatile_u32(abort_addr)) {
            stop = true;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = sb + L::kAOff + s * L::kAStage;
          const uint32_t b0 = sb + L::kBOff + bsl * L::kB;
#pragma unroll
          for (uint32_t kk = 0; kk < kT8K / 32; ++kk) {   // K = 32 bytes per MMA
            const uint64_t bdesc = desc_kmajor_sw128(b0 + kk * 32);
#pragma unroll
            for (uint32_t j = 0; j < 2; ++j) {
              const uint64_t adesc = desc_kmajor_sw128(a0 + j * L::kPlane + kk * 32);
              tc_mma_i8_pair(tmem + j * kTcN, adesc, bdesc, idesc,
                             (first && kk == 0) ? 0u : 1u);
            }
          }
          tc_commit_pair(aempty(s), 0x3);
          tc_commit_pair(bempty(bsl), 0x3);
          if ((it % kT8Flush) == kT8Flush - 1 || it == nit - 1) {
            tc_commit_pair(accfull, 0x3);
            ++blk;
          }
        }
      }
      // every MMA this thread issued has completed before either CTA moves on
      tc_commit_pair(drain, 0x1);
      if (!mbar_wait_bounded(drain, 0)) atomicOr(a.err, kErrMmaTimeout);
    }
  } else {
    // ---------------- genotype expansion + epilogue (warps 2-9) ----------------
    // warp 2 + e: 16-variant chunk e of the stage for the CTA's 128 people
    // (byte column `lane`: people 4 lane .. 4 lane + 3); at block ends it
    // drains TMEM lane quadrant warp % 4, column blocks of half e / 4
    const uint32_t ew = warp - 2;              // 0..7
    const uint32_t col = lane;
    const uint32_t c = ew;                     // 16-byte chunk (16 variants) of the operand row
    const uint32_t h = ew >> 2;
    const uint32_t quad = warp & 3;
    const uint32_t lead_accempty = mapa_shared(accempty, 0);
    const uint64_t pass_stride = a.K_pad * a.P_pad;
    uint32_t g = 0, blk = 0;
    bool stop = false;
    for (uint32_t wi = cid; wi < a.items && !stop; wi += ncl) {
      const PairItem w = pair_item(a, wi);
      const bool missing = w.pass >= 2;
      for (uint32_t it = 0; it < nit; ++it, ++g) {
        const uint32_t s = g % ST, ph = (g / ST) & 1u;
        const uint32_t bsl = g % BS, bph = (g / BS) & 1u;
        if (!mbar_wait_bounded(full(s), ph)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrTmaTimeout);
          stop = true;
          break;
        }
        // the operand slot is free once the MMAs of stage g - BS completed
        if (!mbar_wait_bounded(bempty(bsl), bph ^ 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          stop = true;
          break;
        }
        if (lds_volatile_u32(abort_addr)) {
          stop = true;
          break;
        }
        const uint32_t pk = sb + L::kPkOff + s * L::kPk;
        const uint32_t bt = sb + L::kBOff + bsl * L::kB;
        {
          uint32_t x[4] = {0u, 0u, 0u, 0u};
#pragma unroll
          for (uint32_t i = 0; i < 16; ++i)
            x[i >> 2] |= lds_u8(pk + (16 * c + i) * L::kPkRow + col) << (8 * (i & 3));
#pragma unroll
          for (uint32_t i = 0; i < 4; ++i)
            x[i] = missing ? code_fields<true>(x[i]) : code_fields<false>(x[i]);
#pragma unroll
          for (uint32_t q = 0; q < 4; ++q) {
            uint4 v;
            v.x = (x[0] >> (2 * q)) & 0x03030303u;
            v.y = (x[1] >> (2 * q)) & 0x03030303u;
            v.z = (x[2] >> (2 * q)) & 0x03030303u;
            v.w = (x[3] >> (2 * q)) & 0x03030303u;
            // operand row of person 4col + q of this CTA's half; the pair's
            // TMEM column is 128 rank + row, the wide kernels' slot order
            const uint32_t n = 32 * q + col;
            sts_u128(bt + (n >> 3) * 1024 + (n & 7) * 128 + ((c ^ (n & 7)) << 4), v);
          }
        }
        // the warp's operand stores, fenced into the tensor core's (async)
        // proxy, are ordered before one arrival on the leader's barrier; its
        // consumer is the MMA, so no cluster-scope release is needed
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive_remote(mapa_shared(bready(bsl), 0));

        if ((it % kT8Flush) == kT8Flush - 1 || it == nit - 1) {
          if (!mbar_wait_bounded(accfull, blk & 1u)) {
            *abort_flag = 1u;
            atomicOr(a.err, kErrMmaTimeout);
            stop = true;
            break;
          }
          tc_fence_after();
          const uint32_t lane_base = tmem + ((32 * quad) << 16);
          if (w.pass == 4) {
#pragma unroll
            for (uint32_t j = 0; j < 2; ++j) {
              if (srow(w, j) >= a.K_pad) continue;
              const uint64_t k = uint64_t(srow(w, j)) + 32 * quad + lane;
              uint32_t* pc = a.part_cnt + k * a.P_pad + uint64_t(w.ptile) * kTcN;
#pragma unroll 1
              for (uint32_t cb = h * (kTcN / 64); cb < (h + 1) * (kTcN / 64); ++cb) {
                uint32_t r[32];
                tmem_ld32(lane_base + j * kTcN + 32 * cb, r);
                tmem_ld_wait();
#pragma unroll
                for (int i = 0; i < 32; ++i) pc[32 * cb + i] += r[i];
              }
            }
          } else if (srow(w, 0) < a.K_pad) {
            const uint64_t k = uint64_t(srow(w, 0)) + 32 * quad + lane;
            double* ps = (w.pass == 0 ? a.part_sum : a.part_pass + (w.pass - 1) * pass_stride) +
                         k * a.P_pad + uint64_t(w.ptile) * kTcN;
            // the pass arrays' first block after a reset is written, not added
            const bool write = w.pass > 0 && a.store && it < kT8Flush;
            const double q0 = a.quanta[(2 * w.pass) * a.K_pad + k];
            const double q1 = a.quanta[(2 * w.pass + 1) * a.K_pad + k];
#pragma unroll 1
            for (uint32_t cb = h * (kTcN / 64); cb < (h + 1) * (kTcN / 64); ++cb) {
              uint32_t r0[32], r1[32];
              tmem_ld32(lane_base + 32 * cb, r0);
              tmem_ld32(lane_base + kTcN + 32 * cb, r1);
              tmem_ld_wait();
              if (write) {
#pragma unroll
                for (int i = 0; i < 32; ++i)
                  ps[32 * cb + i] = fma(double(int32_t(r1[i])), q1, double(int32_t(r0[i])) * q0);
              } else {
#pragma unroll
                for (int i = 0; i < 32; ++i)
                  ps[32 * cb + i] += fma(double(int32_t(r1[i])), q1, double(int32_t(r0[i])) * q0);
              }
            }
          }
          tc_fence_before();
          mbar_arrive_cluster(lead_accempty);
          ++blk;
        }
      }
    }
  }
  tc_fence_before();
  __syncwarp();
  cluster_sync_all();   // no CTA leaves while the other may read or signal its shared memory
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tmem, 512);
  }
}

// 8-bit limb planes [kT8Planes][K_pad][V_pad] and their quanta [kT8Planes][K_pad]
// from the CSR: one thread per variant; the quanta by one thread per score.
__global__ void gnm_t8_quanta(const uint32_t* amax_bits, uint64_t K_pad, double* quanta) {
  const uint64_t k = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= K_pad) return;
  const float am = __uint_as_float(amax_bits[k]);
  double q = am > 0.0f ? double(am) / 127.0 : 1.0;
  for (int l = 0; l < 4; ++l, q /= 254.0) {
    quanta[l * K_pad + k] = q;          // dosage limb l
    quanta[(4 + l) * K_pad + k] = q;    // correction limb l
  }
  quanta[8 * K_pad + k] = 1.0;          // member plane: counts
}

__global__ void gnm_t8_build_planes(const float* w, const float* corr, const uint32_t* cols,
                                    const uint64_t* offs, uint64_t V, const double* quanta,
                                    int8_t* planes, uint64_t K_pad, uint64_t V_pad) {
  const uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= V) return;
  const uint64_t plane = K_pad * V_pad;
  for (uint64_t e = offs[v]; e < offs[v + 1]; ++e) {
    const uint32_t k = cols[e];
    const uint64_t at = uint64_t(k) * V_pad + v;
    const double xs[2] = {double(w[e]), -double(corr[e])};
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      double r = xs[t];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const double q = quanta[l * K_pad + k];
        const double li = fmin(fmax(rint(r / q), -127.0), 127.0);
        r -= li * q;
        planes[(4 * t + l) * plane + at] = int8_t(li);
      }
    }
    planes[8 * plane + at] = 1;
  }
}

// ---- narrow tensor engine (few score columns) ---------------------------------
// For a handful of scores the M = 128 score rows of gnm_tc_accumulate would be
// mostly empty, so the roles turn: M = 128 PEOPLE (TMEM lanes), N = 64 = the
// four limb planes of 16 scores (row n = 16 * plane + score, one 3D TMA box of
// the same limb planes), K = 64 variants per stage.  Each stage runs two MMAs
// per 16-variant slice: the dosage operand against the W' limbs and the
// missing-indicator operand against the -C limbs and the member plane, into
// 2 x 64 accumulator columns, so ONE pass produces sums and missing counts.
// The genotype expansion is the transposing one of gnm_tc_accumulate (operand
// row n = 32 q + col holds person 4 col + q), writing both operands, spread
// over eight warps (one 8-variant chunk per thread): with fewer, each warp's
// chain of dependent byte loads and permutes set the stage time.  Sums of a
// 16384-variant block are exact in FP32 (same limb argument) and are added to
// the FP64 partials of the CTA's variant split in natural person order at
// block ends; gnm_tc_finalize adds the split slots in a fixed order.
constexpr uint32_t kNrM = 128;                // people per CTA
constexpr uint32_t kNrScores = 16;            // scores per CTA
constexpr uint32_t kNrN = 4 * kNrScores;      // accumulator columns per operand
constexpr uint32_t kNrStages = 4;
constexpr uint32_t kNrExpand = 256;           // expansion threads (warps 2-9)
constexpr uint32_t kNrThreads = 64 + kNrExpand;

struct NrSmem {
  static constexpr uint32_t kA = kNrM * kTcK * 2;          // 16 KB per operand
  static constexpr uint32_t kB = kNrN * kTcK * 2;          // 8 KB per limb set
  static constexpr uint32_t kPk = kTcK * (kNrM / 4);       // 2 KB packed rows
  static constexpr uint32_t kADos = 0;
  static constexpr uint32_t kAMis = kADos + kA;
  static constexpr uint32_t kBDos = kAMis + kA;
  static constexpr uint32_t kBMis = kBDos + kB;
  static constexpr uint32_t kPkOff = kBMis + kB;
  static constexpr uint32_t kStage = kPkOff + kPk;          // 50 KB
  static constexpr uint32_t kBarOff = kNrStages * kStage;
  static constexpr uint32_t kHolder = kBarOff + 8 * (3 * kNrStages + 2);
  static constexpr uint32_t kTotal = kHolder + 16 + 1024;   // + alignment slack
};
static_assert(NrSmem::kStage % 1024 == 0 && NrSmem::kBDos % 1024 == 0 &&
                  NrSmem::kBMis % 1024 == 0,
              "operand alignment");

struct NrArgs {
  uint64_t num_rows;          // rows of this block
  int32_t a_x0;               // absolute variant index of block row 0 (multiple of 64)
  uint32_t stages_per_split;  // 64-variant stages per blockIdx.z split
  double* part_sum;           // [split][K_pad][P_pad], natural person order
  uint32_t* part_cnt;
  uint64_t P_pad;
  uint64_t slot_stride;       // K_pad * P_pad
  uint32_t* err;
};

__global__ void __launch_bounds__(kNrThreads, 1)
    gnm_tc_narrow(const __grid_constant__ CUtensorMap dmap,
                  const __grid_constant__ CUtensorMap mmap,
                  const __grid_constant__ CUtensorMap pmap, NrArgs a) {
  using L = NrSmem;
  constexpr uint32_t ST = kNrStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sb = smem_u32(smem);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t ptile = blockIdx.x, stile = blockIdx.y, split = blockIdx.z;
  const uint32_t nall = uint32_t((a.num_rows + kTcK - 1) / kTcK);
  const uint32_t it0 = split * a.stages_per_split;
  const uint32_t nit = it0 < nall ? min(a.stages_per_split, nall - it0) : 0u;
  auto full = [&](uint32_t s) { return sb + L::kBarOff + 8 * s; };
  auto bready = [&](uint32_t s) { return sb + L::kBarOff + 8 * (ST + s); };
  auto empty = [&](uint32_t s) { return sb + L::kBarOff + 8 * (2 * ST + s); };
  const uint32_t accfull = sb + L::kBarOff + 8 * (3 * ST);
  const uint32_t accempty = sb + L::kBarOff + 8 * (3 * ST + 1);
  volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + L::kHolder + 8);
  const uint32_t abort_addr = sb + L::kHolder + 8;
  if (nit == 0) return;   // a split past the block's last stage (uniform per CTA)

  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < ST; ++s) {
      mbar_init(full(s), 1);
      mbar_init(bready(s), kNrExpand);
      mbar_init(empty(s), 1);
    }
    mbar_init(accfull, 1);
    mbar_init(accempty, kNrExpand);
    *abort_flag = 0u;
    fence_mbar_init();
    prefetch_tmap(&dmap);
    prefetch_tmap(&mmap);
    prefetch_tmap(&pmap);
  }
  if (warp == 1) {
    tmem_alloc(sb + L::kHolder, 2 * kNrN);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + L::kHolder);

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST, ph = (it / ST) & 1u;
        if (!mbar_wait_bounded(empty(s), ph ^ 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        const uint32_t st = sb + s * L::kStage;
        mbar_arrive_expect_tx(full(s), 2 * L::kB + L::kPk);
        const int32_t x = a.a_x0 + int32_t((it0 + it) * kTcK);
        tma_load_3d(st + L::kBDos, &dmap, x, int32_t(stile * kNrScores), 0, full(s));
        tma_load_3d(st + L::kBMis, &mmap, x, int32_t(stile * kNrScores), 0, full(s));
        tma_load_2d(st + L::kPkOff, &pmap, int32_t(ptile * (kNrM / 4)),
                    int32_t((it0 + it) * kTcK), full(s));
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_bf16_f32(kNrM, kNrN);
      uint32_t blk = 0;
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST, ph = (it / ST) & 1u;
        const bool first = (it % kTcFlush) == 0;
        if (first && it > 0) {
          if (!mbar_wait_bounded(accempty, (blk - 1) & 1u)) {
            *abort_flag = 1u;
            atomicOr(a.err, kErrMmaTimeout);
            break;
          }
        }
        if (!mbar_wait_bounded(bready(s), ph)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        tc_fence_after();
        const uint32_t st = sb + s * L::kStage;
#pragma unroll
        for (uint32_t kk = 0; kk < kTcK / 16; ++kk) {
          const uint32_t acc = (first && kk == 0) ? 0u : 1u;
          tc_mma_f16(tmem, desc_kmajor_sw128(st + L::kADos + kk * 32),
                     desc_kmajor_sw128(st + L::kBDos + kk * 32), idesc, acc);
          tc_mma_f16(tmem + kNrN, desc_kmajor_sw128(st + L::kAMis + kk * 32),
                     desc_kmajor_sw128(st + L::kBMis + kk * 32), idesc, acc);
        }
        tc_commit(empty(s));
        if ((it % kTcFlush) == kTcFlush - 1 || it == nit - 1) {
          tc_commit(accfull);
          ++blk;
        }
      }
    }
  } else {
    // ---------------- genotype expansion + epilogue (warps 2-9) ----------------
    const uint32_t pt = threadIdx.x - 64;   // 0..255
    const uint32_t col = pt & 31;           // byte column: people 4col..4col+3
    const uint32_t c = pt >> 5;             // 16-byte chunk: variants 8c..8c+7 of the stage
    const uint32_t quad = warp & 3;         // TMEM lane quadrant of this warp
    const uint32_t half = (warp - 2) >> 2;  // epilogue: scores 8 half .. 8 half + 7
    double* ps = a.part_sum + uint64_t(split) * a.slot_stride;
    uint32_t* pc = a.part_cnt + uint64_t(split) * a.slot_stride;
    uint32_t blk = 0;
    for (uint32_t it = 0; it < nit; ++it) {
      const uint32_t s = it % ST, ph = (it / ST) & 1u;
      if (!mbar_wait_bounded(full(s), ph)) {
        *abort_flag = 1u;
        atomicOr(a.err, kErrTmaTimeout);
        break;
      }
      if (lds_volatile_u32(abort_addr)) break;
      // explicit shared-space accesses: the realigned base is a generic pointer
      const uint32_t pk = sb + s * L::kStage + L::kPkOff;
      const uint32_t ad = sb + s * L::kStage + L::kADos;
      const uint32_t am = sb + s * L::kStage + L::kAMis;
      {
        const uint32_t r0 = 8 * c;
        uint32_t xl = 0, xh = 0;
#pragma unroll
        for (uint32_t i = 0; i < 4; ++i) {
          xl |= lds_u8(pk + (r0 + i) * (kNrM / 4) + col) << (8 * i);
          xh |= lds_u8(pk + (r0 + 4 + i) * (kNrM / 4) + col) << (8 * i);
        }
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
          const uint32_t yl = (xl >> (2 * q)) & 0x03030303u;
          const uint32_t yh = (xh >> (2 * q)) & 0x03030303u;
          uint4 vd, vm;
          vd.x = bf16_pair(yl & 0xFFFFu, kDosLo, kDosHi);
          vd.y = bf16_pair(yl >> 16, kDosLo, kDosHi);
          vd.z = bf16_pair(yh & 0xFFFFu, kDosLo, kDosHi);
          vd.w = bf16_pair(yh >> 16, kDosLo, kDosHi);
          vm.x = bf16_pair(yl & 0xFFFFu, kMisLo, kMisHi);
          vm.y = bf16_pair(yl >> 16, kMisLo, kMisHi);
          vm.z = bf16_pair(yh & 0xFFFFu, kMisLo, kMisHi);
          vm.w = bf16_pair(yh >> 16, kMisLo, kMisHi);
          // operand row of person 4col + q (conflict-free 16-byte stores)
          const uint32_t n = 32 * q + col;
          const uint32_t off = (n >> 3) * 1024 + (n & 7) * 128 + ((c ^ (n & 7)) << 4);
          sts_u128(ad + off, vd);
          sts_u128(am + off, vm);
        }
      }
      fence_proxy_async_smem();
      mbar_arrive(bready(s));

      if ((it % kTcFlush) == kTcFlush - 1 || it == nit - 1) {
        if (!mbar_wait_bounded(accfull, blk & 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        tc_fence_after();
        // TMEM lane 32 quad + lane = operand row n -> person 4 (n % 32) + n / 32.
        // Column group g (16 columns): dosage limbs 0-3, -C limbs 0-2, member;
        // this thread reads its 8 scores of every group.
        const uint64_t person = uint64_t(ptile) * kNrM + 4 * lane + quad;
        const uint32_t lane_base = tmem + ((32 * quad) << 16) + 8 * half;
        double acc[8];
        uint32_t cnt[8];
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) acc[k] = 0.0;
#pragma unroll
        for (uint32_t g = 0; g < 8; ++g) {
          uint32_t d[8];
          tmem_ld8(lane_base + 16 * g, d);
          tmem_ld_wait();
#pragma unroll
          for (uint32_t k = 0; k < 8; ++k) {
            if (g < 7) acc[k] += double(__uint_as_float(d[k]));
            else cnt[k] = __float2uint_rn(__uint_as_float(d[k]));
          }
        }
        tc_fence_before();
        mbar_arrive(accempty);
        ++blk;
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) {
          const uint64_t at = (uint64_t(stile) * kNrScores + 8 * half + k) * a.P_pad + person;
          ps[at] += acc[k];
          pc[at] += cnt[k];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * kNrN);
  }
}

// ---- narrow engine on 8-bit limbs -------------------------------------------------
// gnm_tc_narrow with tcgen05.mma kind::i8: M = 128 people, N = 16 scores x
// the 8-bit planes of each operand (row n = 16 * plane + score, one 3D TMA box
// of the wide engine's [9][K_pad][V] limb planes: dosage limbs 0-3, N = 64;
// correction limbs 0-3 and the member plane, N = 80), K = 128 variants per
// stage.  Per 32-variant slice two MMAs, the dosage operand against the
// dosage limbs and the missing indicator against the rest, into 64 + 80 S32
// accumulator columns.  Every operand byte is half the BF16 kernel's, which is what
// bounds that kernel: its stage time is set by shared-memory traffic (TMA
// writes, operand stores, MMA operand reads), not by the MMAs.  The TMA ring
// (limb planes + packed rows) runs ST stages deep beside a two-deep ring of
// expanded operands, as in gnm_t8_accumulate; sums stay exact in S32 for
// blocks of up to 2^23 variants and reach the FP64 partials of the CTA's
// variant split (natural person order) once per block.
constexpr int kT8NrStages = 5;

constexpr uint32_t kT8NrNDos = 4 * kNrScores;   // dosage limbs 0-3
constexpr uint32_t kT8NrNMis = 5 * kNrScores;   // correction limbs 0-3, member plane

struct T8NrSmem {
  static constexpr uint32_t kBStages = 2;
  static constexpr uint32_t kA = kNrM * kT8K;               // 16 KB per operand (people rows)
  static constexpr uint32_t kPkRow = kNrM / 4;              // 32 packed bytes per variant row
  static constexpr uint32_t kPk = kT8K * kPkRow;            // 4 KB
  static constexpr uint32_t kBDos = 0;                      // offsets inside a TMA stage
  static constexpr uint32_t kBMis = kT8NrNDos * kT8K;       // 8 KB
  static constexpr uint32_t kPkIn = kBMis + kT8NrNMis * kT8K;   // + 10 KB
  static constexpr uint32_t kTma = kPkIn + kPk;             // one TMA stage: 22 KB
  static constexpr uint32_t kAOff = kT8NrStages * kTma;     // operand ring
  static constexpr uint32_t kBarOff = kAOff + kBStages * 2 * kA;
  static constexpr uint32_t kHolder = kBarOff + 8 * (2 * kT8NrStages + 2 * kBStages + 2);
  static constexpr uint32_t kTotal = kHolder + 16 + 1024;  // + alignment slack
  static_assert(kTotal <= 227 * 1024, "shared memory");
  static_assert(kTma % 1024 == 0 && kAOff % 1024 == 0 && kBMis % 1024 == 0 && kPkIn % 1024 == 0,
                "operand alignment");
};

__global__ void __launch_bounds__(kNrThreads, 1)
    gnm_t8_narrow(const __grid_constant__ CUtensorMap dmap,
                  const __grid_constant__ CUtensorMap mmap,
                  const __grid_constant__ CUtensorMap pmap, NrArgs a, const double* quanta,
                  uint64_t K_pad) {
  using L = T8NrSmem;
  constexpr uint32_t ST = kT8NrStages;
  constexpr uint32_t BS = L::kBStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sb = smem_u32(smem);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t ptile = blockIdx.x, stile = blockIdx.y, split = blockIdx.z;
  const uint32_t nall = uint32_t((a.num_rows + kT8K - 1) / kT8K);
  const uint32_t it0 = split * a.stages_per_split;
  const uint32_t nit = it0 < nall ? min(a.stages_per_split, nall - it0) : 0u;
  auto full = [&](uint32_t s) { return sb + L::kBarOff + 8 * s; };
  auto tempty = [&](uint32_t s) { return sb + L::kBarOff + 8 * (ST + s); };
  auto bready = [&](uint32_t b) { return sb + L::kBarOff + 8 * (2 * ST + b); };
  auto bempty = [&](uint32_t b) { return sb + L::kBarOff + 8 * (2 * ST + BS + b); };
  const uint32_t accfull = sb + L::kBarOff + 8 * (2 * ST + 2 * BS);
  const uint32_t accempty = sb + L::kBarOff + 8 * (2 * ST + 2 * BS + 1);
  volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + L::kHolder + 8);
  const uint32_t abort_addr = sb + L::kHolder + 8;
  if (nit == 0) return;   // a split past the block's last stage (uniform per CTA)

  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < ST; ++s) {
      mbar_init(full(s), 1);
      mbar_init(tempty(s), 1);
    }
    for (uint32_t b = 0; b < BS; ++b) {
      mbar_init(bready(b), kNrExpand);
      mbar_init(bempty(b), 1);
    }
    mbar_init(accfull, 1);
    mbar_init(accempty, kNrExpand);
    *abort_flag = 0u;
    fence_mbar_init();
    prefetch_tmap(&dmap);
    prefetch_tmap(&mmap);
    prefetch_tmap(&pmap);
  }
  if (warp == 1) {
    tmem_alloc(sb + L::kHolder, 256);   // 64 + 80 columns
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + L::kHolder);

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST, ph = (it / ST) & 1u;
        if (!mbar_wait_bounded(tempty(s), ph ^ 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        const uint32_t st = sb + s * L::kTma;
        mbar_arrive_expect_tx(full(s), L::kTma);
        const int32_t x = a.a_x0 + int32_t((it0 + it) * kT8K);
        tma_load_3d(st + L::kBDos, &dmap, x, int32_t(stile * kNrScores), 0, full(s));
        tma_load_3d(st + L::kBMis, &mmap, x, int32_t(stile * kNrScores), 4, full(s));
        tma_load_2d(st + L::kPkIn, &pmap, int32_t(ptile * L::kPkRow),
                    int32_t((it0 + it) * kT8K), full(s));
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t idesc_d = idesc_s8s8_s32(kNrM, kT8NrNDos);
      constexpr uint32_t idesc_m = idesc_s8s8_s32(kNrM, kT8NrNMis);
      uint32_t blk = 0;
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST;
        const uint32_t bsl = it % BS, bph = (it / BS) & 1u;
        const bool first = (it % kT8Flush) == 0;
        if (first && it > 0) {
          if (!mbar_wait_bounded(accempty, (blk - 1) & 1u)) {
            *abort_flag = 1u;
            atomicOr(a.err, kErrMmaTimeout);
            break;
          }
        }
        if (!mbar_wait_bounded(bready(bsl), bph)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        tc_fence_after();
        const uint32_t st = sb + s * L::kTma;
        const uint32_t ad = sb + L::kAOff + bsl * 2 * L::kA;
        const uint32_t am = ad + L::kA;
#pragma unroll
        for (uint32_t kk = 0; kk < kT8K / 32; ++kk) {   // K = 32 bytes per MMA
          const uint32_t acc = (first && kk == 0) ? 0u : 1u;
          tc_mma_i8(tmem, desc_kmajor_sw128(ad + kk * 32),
                    desc_kmajor_sw128(st + L::kBDos + kk * 32), idesc_d, acc);
          tc_mma_i8(tmem + kT8NrNDos, desc_kmajor_sw128(am + kk * 32),
                    desc_kmajor_sw128(st + L::kBMis + kk * 32), idesc_m, acc);
        }
        tc_commit(tempty(s));
        tc_commit(bempty(bsl));
        if ((it % kT8Flush) == kT8Flush - 1 || it == nit - 1) {
          tc_commit(accfull);
          ++blk;
        }
      }
    }
  } else {
    // ---------------- genotype expansion + epilogue (warps 2-9) ----------------
    // warp 2 + e: 16-variant chunk e of the stage; lane = byte column (people
    // 4 lane .. 4 lane + 3); both operands from the same packed bytes
    const uint32_t c = warp - 2;
    const uint32_t col = lane;
    const uint32_t quad = warp & 3;         // TMEM lane quadrant of this warp
    const uint32_t half = (warp - 2) >> 2;  // epilogue: scores 8 half .. 8 half + 7
    double* ps = a.part_sum + uint64_t(split) * a.slot_stride;
    uint32_t* pc = a.part_cnt + uint64_t(split) * a.slot_stride;
    uint32_t blk = 0;
    for (uint32_t it = 0; it < nit; ++it) {
      const uint32_t s = it % ST, ph = (it / ST) & 1u;
      const uint32_t bsl = it % BS, bph = (it / BS) & 1u;
      if (!mbar_wait_bounded(full(s), ph)) {
        *abort_flag = 1u;
        atomicOr(a.err, kErrTmaTimeout);
        break;
      }
      if (!mbar_wait_bounded(bempty(bsl), bph ^ 1u)) {
        *abort_flag = 1u;
        atomicOr(a.err, kErrMmaTimeout);
        break;
      }
      if (lds_volatile_u32(abort_addr)) break;
      const uint32_t pk = sb + s * L::kTma + L::kPkIn;
      const uint32_t ad = sb + L::kAOff + bsl * 2 * L::kA;
      const uint32_t am = ad + L::kA;
      {
        uint32_t x[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (uint32_t i = 0; i < 16; ++i)
          x[i >> 2] |= lds_u8(pk + (16 * c + i) * L::kPkRow + col) << (8 * (i & 3));
        uint32_t xd[4], xm[4];
#pragma unroll
        for (uint32_t i = 0; i < 4; ++i) {
          xd[i] = code_fields<false>(x[i]);
          xm[i] = code_fields<true>(x[i]);
        }
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
          uint4 vd, vm;
          vd.x = (xd[0] >> (2 * q)) & 0x03030303u;
          vd.y = (xd[1] >> (2 * q)) & 0x03030303u;
          vd.z = (xd[2] >> (2 * q)) & 0x03030303u;
          vd.w = (xd[3] >> (2 * q)) & 0x03030303u;
          vm.x = (xm[0] >> (2 * q)) & 0x03030303u;
          vm.y = (xm[1] >> (2 * q)) & 0x03030303u;
          vm.z = (xm[2] >> (2 * q)) & 0x03030303u;
          vm.w = (xm[3] >> (2 * q)) & 0x03030303u;
          // operand row of person 4col + q (conflict-free 16-byte stores)
          const uint32_t n = 32 * q + col;
          const uint32_t off = (n >> 3) * 1024 + (n & 7) * 128 + ((c ^ (n & 7)) << 4);
          sts_u128(ad + off, vd);
          sts_u128(am + off, vm);
        }
      }
      fence_proxy_async_smem();
      mbar_arrive(bready(bsl));

      if ((it % kT8Flush) == kT8Flush - 1 || it == nit - 1) {
        if (!mbar_wait_bounded(accfull, blk & 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        tc_fence_after();
        // TMEM lane 32 quad + lane = operand row n -> person 4 (n % 32) + n / 32.
        // Column group g (16 columns): dosage limbs 0-3, -C limbs 0-3, member
        // (plane g of the limb planes); this thread reads its 8 scores of
        // every group.
        const uint64_t person = uint64_t(ptile) * kNrM + 4 * lane + quad;
        const uint32_t lane_base = tmem + ((32 * quad) << 16) + 8 * half;
        const uint64_t k0 = uint64_t(stile) * kNrScores + 8 * half;
        double acc[8];
        uint32_t cnt[8];
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) acc[k] = 0.0;
#pragma unroll
        for (uint32_t g = 0; g < 9; ++g) {
          uint32_t d[8];
          tmem_ld8(lane_base + 16 * g, d);
          tmem_ld_wait();
#pragma unroll
          for (uint32_t k = 0; k < 8; ++k) {
            if (g < 8) acc[k] = fma(double(int32_t(d[k])), quanta[g * K_pad + k0 + k], acc[k]);
            else cnt[k] = d[k];
          }
        }
        tc_fence_before();
        mbar_arrive(accempty);
        ++blk;
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) {
          const uint64_t at = (k0 + k) * a.P_pad + person;
          ps[at] += acc[k];
          pc[at] += cnt[k];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

// Limb planes from the CSR: one thread per variant.
// Per-score max(|w|, |corr|) as float bit patterns (non-negative floats order
// like their bits): shared-memory maxima per block, then one global atomic per
// score and block (global atomics only when the scores do not fit).
constexpr uint64_t kAmaxSharedScores = 8192;
__global__ void gnm_tc_amax(const float* w, const float* corr, const uint32_t* cols, uint64_t nnz,
                            uint64_t K_pad, uint32_t* amax_bits) {
  extern __shared__ uint32_t s_max[];
  const bool shared = K_pad <= kAmaxSharedScores;
  if (shared) {
    for (uint64_t k = threadIdx.x; k < K_pad; k += blockDim.x) s_max[k] = 0u;
    __syncthreads();
  }
  for (uint64_t e = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < nnz;
       e += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t m = __float_as_uint(fmaxf(fabsf(w[e]), fabsf(corr[e])));
    if (shared)
      atomicMax(s_max + cols[e], m);
    else
      atomicMax(amax_bits + cols[e], m);
  }
  if (shared) {
    __syncthreads();
    for (uint64_t k = threadIdx.x; k < K_pad; k += blockDim.x)
      if (s_max[k]) atomicMax(amax_bits + k, s_max[k]);
  }
}

__global__ void gnm_tc_build_planes(const float* w, const float* corr, const uint32_t* cols,
                                    const uint64_t* offs, uint64_t V, const uint32_t* amax_bits,
                                    __nv_bfloat16* dos, __nv_bfloat16* mis, uint64_t K_pad,
                                    uint64_t V_pad) {
  const uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= V) return;
  const uint64_t plane = K_pad * V_pad;
  for (uint64_t e = offs[v]; e < offs[v + 1]; ++e) {
    const uint32_t k = cols[e];
    // quantum q = 2^(E-8) with amax = f 2^E, f in [0.5, 1); then q/2^8, q/2^16,
    // q/2^24 (powers of two: the divisions are exact and every residual below
    // is exact in FP32)
    float q = 1.0f;
    const float am = __uint_as_float(amax_bits[k]);
    if (am > 0.0f) {
      int ex = 0;
      frexpf(am, &ex);
      q = ldexpf(1.0f, max(ex - 8, -125));   // q / 2^24 stays a (subnormal) FP32 value
    }
    const float qm = q * (1.0f / 256.0f), ql = q * (1.0f / 65536.0f),
                ql2 = q * (1.0f / 16777216.0f);
    const uint64_t at = uint64_t(k) * V_pad + v;
    const float xs[2] = {w[e], -corr[e]};
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const float x = xs[t];
      const float h = rintf(x / q) * q;
      const float r1 = x - h;
      const float m = rintf(r1 / qm) * qm;
      const float r2 = r1 - m;
      const float l = rintf(r2 / ql) * ql;
      __nv_bfloat16* base = t == 0 ? dos : mis;
      base[at] = __float2bfloat16_rn(h);
      base[plane + at] = __float2bfloat16_rn(m);
      base[2 * plane + at] = __float2bfloat16_rn(l);
      if (t == 0) base[3 * plane + at] = __float2bfloat16_rn(rintf((r2 - l) / ql2) * ql2);
    }
    mis[3 * plane + at] = __float2bfloat16_rn(1.0f);
  }
}

// out[o*K + k] = init[k] + part_sum[k][slot(fam(o))]; slot(f) is the operand
// row of person f: tile (f / 256), row 128*h + 32*(r%4) + (r%128)/4 with
// r = f % 256 and h = r / 128.  `pass` (may be null): the SM-pair kernel's
// partials of passes 1-3, [3][pass_stride], added after part_sum in pass
// order.  The narrow engine's epilogue writes in person order, one slot per
// variant split: those slots are added in split order.
__global__ void gnm_tc_finalize(const double* part_sum, const uint32_t* part_cnt, uint64_t P_pad,
                                const double* init, const uint32_t* out_to_fam, uint64_t P,
                                uint64_t K, uint32_t nslots, uint64_t slot_stride,
                                const double* pass, uint64_t pass_stride, double* sums,
                                uint32_t* counts) {
  const uint64_t x = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (x >= P * K) return;
  const uint64_t o = x / K, k = x % K;
  const uint64_t f = out_to_fam ? out_to_fam[o] : o;
  if (nslots == 0) {   // wide engine: one slot, operand-row order
    const uint64_t r = f % kTcN, h = r / 128, rr = r % 128;
    const uint64_t slot = (f / kTcN) * kTcN + 128 * h + 32 * (rr % 4) + rr / 4;
    double s = part_sum[k * P_pad + slot];
    if (pass)
      for (uint32_t j = 0; j < 3; ++j) s += pass[j * pass_stride + k * P_pad + slot];
    sums[x] = init[k] + s;
    counts[x] = part_cnt[k * P_pad + slot];
    return;
  }
  // narrow engine: natural order, variant-split slots added in split order
  double s = 0.0;
  uint32_t c = 0;
  for (uint32_t z = 0; z < nslots; ++z) {
    s += part_sum[z * slot_stride + k * P_pad + f];
    c += part_cnt[z * slot_stride + k * P_pad + f];
  }
  sums[x] = init[k] + s;
  counts[x] = c;
}

// ---- backward: dW[v,k] = sum_p d(p,v) dS[p,k], dC[v,k] = -sum_{p missing} dS[p,k]
//
// A tcgen05 GEMM with the variants as M: D[v, n] = sum_p A[v, p] B[n, p].  A is
// the allele-2 dosage (missing -> 0) re-expanded from the packed rows into BF16
// by CUDA-core warps; a .bed row is already contiguous along people, so the
// K-major operand row of a variant is its own row, expanded in place (no
// transpose).  B holds dS split into four BF16 limbs per score (row
// n = 16 * limb + score): the hi/mid/lo/lo2 split of the forward planes, each
// limb an integer multiple of its quantum (q, q/2^8, q/2^16, q/2^24 with
// 2^E = 256 q >= max_p |dS[p,k]|) with |integer| <= 256, so products with
// d in {0,1,2} are exact and every partial sum stays exact in FP32 below
// 32768 people, where the accumulators are flushed to FP64.  The only error
// left is the limb residual (< 2^-33 of the score's largest |dS|).
//
// The missing-call term touches ~1% of the calls, so it is not a second GEMM:
// the thread that expands a variant row finds the row's code-01 calls with
// SWAR masks and adds that person's FP32 dS row (staged next to the limbs)
// into FP32 registers, flushed to FP64 every 4096 people (about 41 terms at
// 1% missing: the FP32 rounding stays below 3e-6 of the |dS| it sums, which
// is itself ~1% of the score's sum of |dS|).  Converting every term to FP64
// instead saturated the conversion pipe.
//
// CTA: 128 variants x 16 scores; people in stages of 64 (one 128-byte
// K-major operand row per variant).  Warp 0 issues TMA (packed rows
// [128 x 16 bytes], dS limbs [64 x 64] BF16 with 128-byte swizzle, FP32 dS
// [64 people x 16 scores]), warp 1 owns 64 TMEM columns and issues
// tcgen05.mma (M = 128, N = 64, K = 16), warps 2-9 expand genotypes: two
// threads per variant row (row 32 * (warp % 4) + lane, the TMEM lane the pair
// later drains; people 32 * half ..), each draining 8 of the 16 scores.  With
// one expanding warp per scheduler the chain of dependent permutes and stores
// set the stage time; with two, their latencies overlap.
constexpr uint32_t kBwM = 128;                    // variants per CTA (TMEM lanes)
constexpr uint32_t kBwScores = 16;                // scores per CTA
constexpr uint32_t kBwN = 4 * kBwScores;          // limb rows = accumulator columns
constexpr uint32_t kBwK = 64;                     // people per stage
constexpr uint32_t kBwStages = 6;
constexpr uint32_t kBwFlush = 512;                // stages per exact FP32 block (32768 people)
constexpr uint32_t kBwMissFlush = 64;             // stages per FP32 missing-term sum (4096 people)
constexpr uint32_t kBwExpand = 256;               // expansion threads (warps 2-9)
constexpr uint32_t kBwThreads = 64 + kBwExpand;

struct BwSmem {
  static constexpr uint32_t kA = kBwM * kBwK * 2;           // 16 KB dosage operand
  static constexpr uint32_t kB = kBwN * kBwK * 2;           // 8 KB dS limbs
  static constexpr uint32_t kPk = kBwM * (kBwK / 4);        // 2 KB packed rows
  static constexpr uint32_t kDs = kBwK * kBwScores * 4;     // 4 KB FP32 dS
  static constexpr uint32_t kAOff = 0;
  static constexpr uint32_t kBOff = kAOff + kA;
  static constexpr uint32_t kPkOff = kBOff + kB;
  static constexpr uint32_t kDsOff = kPkOff + kPk;
  static constexpr uint32_t kStage = kDsOff + kDs;           // 30 KB
  static constexpr uint32_t kBarOff = kBwStages * kStage;
  static constexpr uint32_t kHolder = kBarOff + 8 * (3 * kBwStages + 2);
  static constexpr uint32_t kTotal = kHolder + 16 + 1024;    // + alignment slack
  // end of kernel: both halves' FP64 missing sums [2][128][16], over stage 0-1
  static constexpr uint32_t kSwap = 2 * kBwM * kBwScores * 8;
};
static_assert(BwSmem::kStage % 1024 == 0 && BwSmem::kBOff % 1024 == 0, "operand alignment");
static_assert(BwSmem::kSwap <= BwSmem::kBarOff, "swap area");

struct BwArgs {
  uint64_t V, K;
  uint32_t nstages;   // people stages: P_pad / kBwK
  float* gw;
  float* gc;          // may be null
  uint32_t* err;
};

// Two BF16 dosages from two codes held in bytes 0 and 1 of y (bytes 2-3 ignored).
__device__ __forceinline__ uint32_t dos_pair(uint32_t y) {
  return __byte_perm(kDosLo, kDosHi, y * 0x11u + 0x4040u);
}

__global__ void __launch_bounds__(kBwThreads, 1)
    gnm_tc_backward(const __grid_constant__ CUtensorMap rmap,
                    const __grid_constant__ CUtensorMap bmap,
                    const __grid_constant__ CUtensorMap dmap, BwArgs a) {
  using L = BwSmem;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sb = smem_u32(smem);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t vtile = blockIdx.x, stile = blockIdx.y;
  const uint32_t nit = a.nstages;
  constexpr uint32_t ST = kBwStages;
  auto full = [&](uint32_t s) { return sb + L::kBarOff + 8 * s; };
  auto aready = [&](uint32_t s) { return sb + L::kBarOff + 8 * (ST + s); };
  auto empty = [&](uint32_t s) { return sb + L::kBarOff + 8 * (2 * ST + s); };
  const uint32_t accfull = sb + L::kBarOff + 8 * (3 * ST);
  const uint32_t accempty = sb + L::kBarOff + 8 * (3 * ST + 1);
  volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + L::kHolder + 8);
  const uint32_t abort_addr = sb + L::kHolder + 8;

  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < ST; ++s) {
      mbar_init(full(s), 1);
      mbar_init(aready(s), kBwExpand);
      mbar_init(empty(s), 1);
    }
    mbar_init(accfull, 1);
    mbar_init(accempty, kBwExpand);
    *abort_flag = 0u;
    fence_mbar_init();
    prefetch_tmap(&rmap);
    prefetch_tmap(&bmap);
    prefetch_tmap(&dmap);
  }
  if (warp == 1) {
    tmem_alloc(sb + L::kHolder, kBwN);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + L::kHolder);

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST, ph = (it / ST) & 1u;
        if (!mbar_wait_bounded(empty(s), ph ^ 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        const uint32_t st = sb + s * L::kStage;
        mbar_arrive_expect_tx(full(s), L::kB + L::kPk + L::kDs);
        tma_load_2d(st + L::kPkOff, &rmap, int32_t(it * (kBwK / 4)), int32_t(vtile * kBwM),
                    full(s));
        tma_load_2d(st + L::kBOff, &bmap, int32_t(it * kBwK), int32_t(stile * kBwN), full(s));
        tma_load_2d(st + L::kDsOff, &dmap, int32_t(stile * kBwScores), int32_t(it * kBwK),
                    full(s));
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_bf16_f32(kBwM, kBwN);
      uint32_t blk = 0;
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST, ph = (it / ST) & 1u;
        const bool first = (it % kBwFlush) == 0;
        if (first && it > 0) {
          if (!mbar_wait_bounded(accempty, (blk - 1) & 1u)) {
            *abort_flag = 1u;
            atomicOr(a.err, kErrMmaTimeout);
            break;
          }
        }
        if (!mbar_wait_bounded(aready(s), ph)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        tc_fence_after();
        const uint32_t a0 = sb + s * L::kStage + L::kAOff;
        const uint32_t b0 = sb + s * L::kStage + L::kBOff;
#pragma unroll
        for (uint32_t kk = 0; kk < kBwK / 16; ++kk)
          tc_mma_f16(tmem, desc_kmajor_sw128(a0 + kk * 32), desc_kmajor_sw128(b0 + kk * 32), idesc,
                     (first && kk == 0) ? 0u : 1u);
        tc_commit(empty(s));
        if ((it % kBwFlush) == kBwFlush - 1 || it == nit - 1) {
          tc_commit(accfull);
          ++blk;
        }
      }
    }
  } else {
    // ---------------- genotype expansion + epilogue (warps 2-9) ----------------
    const uint32_t quad = warp & 3;
    const uint32_t half = (warp - 2) >> 2;  // people 32 half .. of each stage; scores 8 half ..
    const uint32_t r = 32 * quad + lane;    // variant row of this thread and its TMEM lane
    double gwd[8], gcd[kBwScores];
    float gcf[kBwScores];   // missing term of the last <= kBwMissFlush stages
#pragma unroll
    for (uint32_t k = 0; k < kBwScores; ++k) {
      gcd[k] = 0.0;
      gcf[k] = 0.0f;
    }
#pragma unroll
    for (uint32_t k = 0; k < 8; ++k) gwd[k] = 0.0;
    bool ok = true;
    uint32_t blk = 0;
    for (uint32_t it = 0; it < nit; ++it) {
      const uint32_t s = it % ST, ph = (it / ST) & 1u;
      if (!mbar_wait_bounded(full(s), ph)) {
        *abort_flag = 1u;
        atomicOr(a.err, kErrTmaTimeout);
        ok = false;
        break;
      }
      if (lds_volatile_u32(abort_addr)) {
        ok = false;
        break;
      }
      const uint32_t st = sb + s * L::kStage;
      // words 2 half, 2 half + 1 of the row: people 32 half + 16 w' ..
      // explicit shared-space accesses: the realigned base is a generic pointer
      const uint2 x2 = lds_u64(st + L::kPkOff + r * (kBwK / 4) + 8 * half);
      const uint32_t xw[2] = {x2.x, x2.y};
      const uint32_t arow = st + L::kAOff + (r >> 3) * 1024 + (r & 7) * 128;
#pragma unroll
      for (uint32_t w = 0; w < 2; ++w) {
        // byte j of s_q = code of person 4j + q of the word
        const uint32_t x = xw[w];
        const uint32_t s0 = x & 0x03030303u, s1 = (x >> 2) & 0x03030303u;
        const uint32_t s2 = (x >> 4) & 0x03030303u, s3 = (x >> 6) & 0x03030303u;
#pragma unroll
        for (uint32_t h = 0; h < 2; ++h) {
          // 16-byte chunk c = people 8c..8c+7 of the stage (bytes 2h, 2h+1 of x)
          const uint32_t sa = 0x40u + 0x22u * h, sbb = 0x51u + 0x22u * h;
          uint4 v;
          v.x = dos_pair(__byte_perm(s0, s1, sa));
          v.y = dos_pair(__byte_perm(s2, s3, sa));
          v.z = dos_pair(__byte_perm(s0, s1, sbb));
          v.w = dos_pair(__byte_perm(s2, s3, sbb));
          const uint32_t c = 4 * half + 2 * w + h;
          sts_u128(arow + ((c ^ (r & 7)) << 4), v);
        }
      }
      // missing calls (code 01): add the person's FP32 dS row; bit 2i of m
      // is person 32 half + i
      uint64_t m = (uint64_t(xw[1] & ~(xw[1] >> 1) & 0x55555555u) << 32) |
                   (xw[0] & ~(xw[0] >> 1) & 0x55555555u);
      while (m) {
        const uint32_t b = 63u - __clzll(m);   // highest set bit: one find-leading-one
        m ^= uint64_t(1) << b;
        const uint32_t drow = st + L::kDsOff + (32 * half + b / 2) * (kBwScores * 4);
#pragma unroll
        for (uint32_t q = 0; q < kBwScores / 4; ++q) {
          const uint4 f = lds_u128(drow + 16 * q);
          gcf[4 * q + 0] += __uint_as_float(f.x);
          gcf[4 * q + 1] += __uint_as_float(f.y);
          gcf[4 * q + 2] += __uint_as_float(f.z);
          gcf[4 * q + 3] += __uint_as_float(f.w);
        }
      }
      if ((it % kBwMissFlush) == kBwMissFlush - 1 || it == nit - 1) {
#pragma unroll
        for (uint32_t k = 0; k < kBwScores; ++k) {
          gcd[k] += double(gcf[k]);
          gcf[k] = 0.0f;
        }
      }
      fence_proxy_async_smem();
      mbar_arrive(aready(s));

      if ((it % kBwFlush) == kBwFlush - 1 || it == nit - 1) {
        if (!mbar_wait_bounded(accfull, blk & 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          ok = false;
          break;
        }
        tc_fence_after();
        // columns 16 j + 8 half + k: limb j of score 8 half + k
        const uint32_t lane_base = tmem + ((32 * quad) << 16) + 8 * half;
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j) {
          uint32_t d[8];
          tmem_ld8(lane_base + 16 * j, d);
          tmem_ld_wait();
#pragma unroll
          for (uint32_t k = 0; k < 8; ++k) gwd[k] += double(__uint_as_float(d[k]));
        }
        tc_fence_before();
        mbar_arrive(accempty);
        ++blk;
      }
    }
    // The two halves of a row hold the missing term of different people: add
    // them in a fixed order through shared memory (stage buffers are idle: the
    // last accumulator commit followed every MMA, and every TMA was consumed).
    named_barrier(1, kBwExpand);
    double* swap = reinterpret_cast<double*>(smem);
#pragma unroll
    for (uint32_t k = 0; k < kBwScores; ++k) swap[(half * kBwM + r) * kBwScores + k] = gcd[k];
    named_barrier(1, kBwExpand);
    const uint64_t v = uint64_t(vtile) * kBwM + r;
    if (ok && !lds_volatile_u32(abort_addr) && v < a.V) {
#pragma unroll
      for (uint32_t k = 0; k < 8; ++k) {
        const uint32_t kl = 8 * half + k;
        const uint64_t kk = uint64_t(stile) * kBwScores + kl;
        if (kk < a.K) {
          a.gw[v * a.K + kk] = float(gwd[k]);
          if (a.gc)
            a.gc[v * a.K + kk] =
                float(-(swap[r * kBwScores + kl] + swap[(kBwM + r) * kBwScores + kl]));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, kBwN);
  }
}

// ---- backward on 8-bit limbs -------------------------------------------------------
// gnm_tc_backward with tcgen05.mma kind::i8: A = the allele-2 dosage of 128
// variants (one byte per person, K-major rows expanded in place from the
// packed rows), B = dS split into four signed 8-bit limbs per score (row
// n = 16 * limb + score; q0 = max_p |dS[p,k]| / 127, q(j+1) = q(j) / 254, every
// |limb| <= 127, residual below 2^-31.9 of the score's largest |dS|), S32
// accumulators exact for up to 2^23 people, converted to FP64 with the
// quanta once per call.  K = 128 people per stage (a 128-byte operand row),
// so every operand byte is half the BF16 kernel's.  The sparse missing-call
// term is the BF16 kernel's: the thread that expands a row adds the FP32 dS
// row of each code-01 call, flushed to FP64 every 4096 people.
constexpr uint32_t kBw8K = 128;                      // people per stage
constexpr uint32_t kBw8Stages = 6;
constexpr uint32_t kBw8Flush = (1u << 23) / kBw8K;   // stages per exact S32 block
constexpr uint32_t kBw8MissFlush = 4096 / kBw8K;     // stages per FP32 missing-term sum

struct Bw8Smem {
  static constexpr uint32_t kA = kBwM * kBw8K;               // 16 KB dosage operand
  static constexpr uint32_t kB = kBwN * kBw8K;               // 8 KB dS limbs
  static constexpr uint32_t kPkRow = kBw8K / 4;              // 32 packed bytes per variant
  static constexpr uint32_t kPk = kBwM * kPkRow;             // 4 KB packed rows
  static constexpr uint32_t kDs = kBw8K * kBwScores * 4;     // 8 KB FP32 dS
  static constexpr uint32_t kAOff = 0;
  static constexpr uint32_t kBOff = kAOff + kA;
  static constexpr uint32_t kPkOff = kBOff + kB;
  static constexpr uint32_t kDsOff = kPkOff + kPk;
  static constexpr uint32_t kStage = kDsOff + kDs;            // 36 KB
  static constexpr uint32_t kBarOff = kBw8Stages * kStage;
  static constexpr uint32_t kHolder = kBarOff + 8 * (3 * kBw8Stages + 2);
  static constexpr uint32_t kTotal = kHolder + 16 + 1024;     // + alignment slack
  static constexpr uint32_t kSwap = 2 * kBwM * kBwScores * 8;
  static_assert(kTotal <= 227 * 1024, "shared memory");
};
static_assert(Bw8Smem::kStage % 1024 == 0 && Bw8Smem::kBOff % 1024 == 0, "operand alignment");
static_assert(Bw8Smem::kSwap <= Bw8Smem::kBarOff, "swap area");

__global__ void __launch_bounds__(kBwThreads, 1)
    gnm_t8_backward(const __grid_constant__ CUtensorMap rmap,
                    const __grid_constant__ CUtensorMap bmap,
                    const __grid_constant__ CUtensorMap dmap, BwArgs a, const double* quanta,
                    uint64_t K16) {
  using L = Bw8Smem;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sb = smem_u32(smem);
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t vtile = blockIdx.x, stile = blockIdx.y;
  const uint32_t nit = a.nstages;
  constexpr uint32_t ST = kBw8Stages;
  auto full = [&](uint32_t s) { return sb + L::kBarOff + 8 * s; };
  auto aready = [&](uint32_t s) { return sb + L::kBarOff + 8 * (ST + s); };
  auto empty = [&](uint32_t s) { return sb + L::kBarOff + 8 * (2 * ST + s); };
  const uint32_t accfull = sb + L::kBarOff + 8 * (3 * ST);
  const uint32_t accempty = sb + L::kBarOff + 8 * (3 * ST + 1);
  volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(smem + L::kHolder + 8);
  const uint32_t abort_addr = sb + L::kHolder + 8;

  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < ST; ++s) {
      mbar_init(full(s), 1);
      mbar_init(aready(s), kBwExpand);
      mbar_init(empty(s), 1);
    }
    mbar_init(accfull, 1);
    mbar_init(accempty, kBwExpand);
    *abort_flag = 0u;
    fence_mbar_init();
    prefetch_tmap(&rmap);
    prefetch_tmap(&bmap);
    prefetch_tmap(&dmap);
  }
  if (warp == 1) {
    tmem_alloc(sb + L::kHolder, kBwN);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + L::kHolder);

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST, ph = (it / ST) & 1u;
        if (!mbar_wait_bounded(empty(s), ph ^ 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        const uint32_t st = sb + s * L::kStage;
        mbar_arrive_expect_tx(full(s), L::kB + L::kPk + L::kDs);
        tma_load_2d(st + L::kPkOff, &rmap, int32_t(it * L::kPkRow), int32_t(vtile * kBwM),
                    full(s));
        tma_load_2d(st + L::kBOff, &bmap, int32_t(it * kBw8K), int32_t(stile * kBwN), full(s));
        tma_load_2d(st + L::kDsOff, &dmap, int32_t(stile * kBwScores), int32_t(it * kBw8K),
                    full(s));
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_s8s8_s32(kBwM, kBwN);
      uint32_t blk = 0;
      for (uint32_t it = 0; it < nit; ++it) {
        const uint32_t s = it % ST, ph = (it / ST) & 1u;
        const bool first = (it % kBw8Flush) == 0;
        if (first && it > 0) {
          if (!mbar_wait_bounded(accempty, (blk - 1) & 1u)) {
            *abort_flag = 1u;
            atomicOr(a.err, kErrMmaTimeout);
            break;
          }
        }
        if (!mbar_wait_bounded(aready(s), ph)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          break;
        }
        if (lds_volatile_u32(abort_addr)) break;
        tc_fence_after();
        const uint32_t a0 = sb + s * L::kStage + L::kAOff;
        const uint32_t b0 = sb + s * L::kStage + L::kBOff;
#pragma unroll
        for (uint32_t kk = 0; kk < kBw8K / 32; ++kk)
          tc_mma_i8(tmem, desc_kmajor_sw128(a0 + kk * 32), desc_kmajor_sw128(b0 + kk * 32), idesc,
                    (first && kk == 0) ? 0u : 1u);
        tc_commit(empty(s));
        if ((it % kBw8Flush) == kBw8Flush - 1 || it == nit - 1) {
          tc_commit(accfull);
          ++blk;
        }
      }
    }
  } else {
    // ---------------- genotype expansion + epilogue (warps 2-9) ----------------
    const uint32_t quad = warp & 3;
    const uint32_t half = (warp - 2) >> 2;  // people 64 half .. of each stage; scores 8 half ..
    const uint32_t r = 32 * quad + lane;    // variant row of this thread and its TMEM lane
    double gwd[8], gcd[kBwScores];
    float gcf[kBwScores];   // missing term of the last <= kBw8MissFlush stages
#pragma unroll
    for (uint32_t k = 0; k < kBwScores; ++k) {
      gcd[k] = 0.0;
      gcf[k] = 0.0f;
    }
#pragma unroll
    for (uint32_t k = 0; k < 8; ++k) gwd[k] = 0.0;
    bool ok = true;
    uint32_t blk = 0;
    for (uint32_t it = 0; it < nit; ++it) {
      const uint32_t s = it % ST, ph = (it / ST) & 1u;
      if (!mbar_wait_bounded(full(s), ph)) {
        *abort_flag = 1u;
        atomicOr(a.err, kErrTmaTimeout);
        ok = false;
        break;
      }
      if (lds_volatile_u32(abort_addr)) {
        ok = false;
        break;
      }
      const uint32_t st = sb + s * L::kStage;
      // words 4 half .. 4 half + 3 of the row: people 64 half + 16 w ..
      const uint4 x4 = lds_u128(st + L::kPkOff + r * L::kPkRow + 16 * half);
      const uint32_t xw[4] = {x4.x, x4.y, x4.z, x4.w};
      const uint32_t arow = st + L::kAOff + (r >> 3) * 1024 + (r & 7) * 128;
#pragma unroll
      for (uint32_t w = 0; w < 4; ++w) {
        // byte t of s_q = dosage of person 4t + q of the word; a 4 x 4 byte
        // transpose puts person 4t + i at byte i of word t
        const uint32_t d = code_fields<false>(xw[w]);
        const uint32_t s0 = d & 0x03030303u, s1 = (d >> 2) & 0x03030303u;
        const uint32_t s2 = (d >> 4) & 0x03030303u, s3 = (d >> 6) & 0x03030303u;
        const uint32_t lo01 = __byte_perm(s0, s1, 0x5140u), hi01 = __byte_perm(s0, s1, 0x7362u);
        const uint32_t lo23 = __byte_perm(s2, s3, 0x5140u), hi23 = __byte_perm(s2, s3, 0x7362u);
        uint4 v;
        v.x = __byte_perm(lo01, lo23, 0x5410u);
        v.y = __byte_perm(lo01, lo23, 0x7632u);
        v.z = __byte_perm(hi01, hi23, 0x5410u);
        v.w = __byte_perm(hi01, hi23, 0x7632u);
        const uint32_t c = 4 * half + w;   // 16-byte chunk: people 16c .. 16c + 15
        sts_u128(arow + ((c ^ (r & 7)) << 4), v);
      }
      // missing calls (code 01): add the person's FP32 dS row; bit 2i of m is
      // person i of the word
#pragma unroll
      for (uint32_t w = 0; w < 4; ++w) {
        uint32_t m = xw[w] & ~(xw[w] >> 1) & 0x55555555u;
        while (m) {
          const uint32_t b = 31u - __clz(m);
          m ^= 1u << b;
          const uint32_t drow = st + L::kDsOff + (64 * half + 16 * w + b / 2) * (kBwScores * 4);
#pragma unroll
          for (uint32_t q = 0; q < kBwScores / 4; ++q) {
            const uint4 f = lds_u128(drow + 16 * q);
            gcf[4 * q + 0] += __uint_as_float(f.x);
            gcf[4 * q + 1] += __uint_as_float(f.y);
            gcf[4 * q + 2] += __uint_as_float(f.z);
            gcf[4 * q + 3] += __uint_as_float(f.w);
          }
        }
      }
      if ((it % kBw8MissFlush) == kBw8MissFlush - 1 || it == nit - 1) {
#pragma unroll
        for (uint32_t k = 0; k < kBwScores; ++k) {
          gcd[k] += double(gcf[k]);
          gcf[k] = 0.0f;
        }
      }
      fence_proxy_async_smem();
      mbar_arrive(aready(s));

      if ((it % kBw8Flush) == kBw8Flush - 1 || it == nit - 1) {
        if (!mbar_wait_bounded(accfull, blk & 1u)) {
          *abort_flag = 1u;
          atomicOr(a.err, kErrMmaTimeout);
          ok = false;
          break;
        }
        tc_fence_after();
        // columns 16 j + 8 half + k: limb j of score 8 half + k
        const uint32_t lane_base = tmem + ((32 * quad) << 16) + 8 * half;
        const uint64_t k0 = uint64_t(stile) * kBwScores + 8 * half;
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j) {
          uint32_t d[8];
          tmem_ld8(lane_base + 16 * j, d);
          tmem_ld_wait();
#pragma unroll
          for (uint32_t k = 0; k < 8; ++k)
            gwd[k] = fma(double(int32_t(d[k])), quanta[j * K16 + k0 + k], gwd[k]);
        }
        tc_fence_before();
        mbar_arrive(accempty);
        ++blk;
      }
    }
    // The two halves of a row hold the missing term of different people: add
    // them in a fixed order through shared memory (stage buffers are idle: the
    // last accumulator commit followed every MMA, and every TMA was consumed).
    named_barrier(1, kBwExpand);
    double* swap = reinterpret_cast<double*>(smem);
#pragma unroll
    for (uint32_t k = 0; k < kBwScores; ++k) swap[(half * kBwM + r) * kBwScores + k] = gcd[k];
    named_barrier(1, kBwExpand);
    const uint64_t v = uint64_t(vtile) * kBwM + r;
    if (ok && !lds_volatile_u32(abort_addr) && v < a.V) {
#pragma unroll
      for (uint32_t k = 0; k < 8; ++k) {
        const uint32_t kl = 8 * half + k;
        const uint64_t kk = uint64_t(stile) * kBwScores + kl;
        if (kk < a.K) {
          a.gw[v * a.K + kk] = float(gwd[k]);
          if (a.gc)
            a.gc[v * a.K + kk] =
                float(-(swap[r * kBwScores + kl] + swap[(kBwM + r) * kBwScores + kl]));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, kBwN);
  }
}

// dS [rows][K] -> 8-bit limb rows (tile t = k / 16: rows 64t + 16j + k % 16,
// limb j) of P_pad people each, their quanta [4][K16], and the FP32 copy
// [P_pad][K16] for the missing term; zeros past the last person and score.
__global__ void gnm_bw_build8(const float* g, uint64_t rows, uint64_t K, uint64_t K16,
                              uint64_t P_pad, const uint32_t* amax_bits, int8_t* planes,
                              double* quanta, float* ds) {
  const uint64_t x = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (x >= K16 * P_pad) return;
  const uint64_t p = x % P_pad, k = x / P_pad;
  const bool in = p < rows && k < K;
  const float val = in ? g[p * K + k] : 0.0f;
  ds[p * K16 + k] = val;
  const float am = k < K ? __uint_as_float(amax_bits[k]) : 0.0f;
  double q = am > 0.0f ? double(am) / 127.0 : 1.0;
  const uint64_t row0 = (k / kBwScores) * kBwN + (k % kBwScores);
  double rem = double(val);
#pragma unroll
  for (uint32_t j = 0; j < 4; ++j, q /= 254.0) {
    const double li = fmin(fmax(rint(rem / q), -127.0), 127.0);
    rem -= li * q;
    planes[(row0 + kBwScores * j) * P_pad + p] = int8_t(li);
    if (p == 0) quanta[j * K16 + k] = q;
  }
}

// dS in output order -> fam order (zero for people outside the keep set).
__global__ void gnm_scatter_grad(const float* gs, const uint32_t* out_to_fam, uint64_t P,
                                 uint64_t K, float* gsf) {
  const uint64_t x = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (x >= P * K) return;
  const uint64_t o = x / K, k = x % K;
  gsf[uint64_t(out_to_fam[o]) * K + k] = gs[x];
}

// Per-score max |dS| as float bit patterns (non-negative floats order like
// their bits); thread = (64-person chunk, score), consecutive threads read
// consecutive scores of a row.
__global__ void gnm_bw_amax(const float* g, uint64_t rows, uint64_t K, uint32_t* amax_bits) {
  const uint64_t x = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t k = x % K, p0 = (x / K) * 64;
  if (p0 >= rows) return;
  const uint64_t p1 = p0 + 64 < rows ? p0 + 64 : rows;
  uint32_t m = 0;
  for (uint64_t p = p0; p < p1; ++p) m = max(m, __float_as_uint(fabsf(g[p * K + k])));
  atomicMax(amax_bits + k, m);
}

// dS [rows][K] -> limb rows (tile t = k / 16: rows 64t + 16j + k % 16, limb j)
// of P_pad people each, and the FP32 copy [P_pad][K16] for the missing term;
// zeros past the last person and the last score.
__global__ void gnm_bw_build(const float* g, uint64_t rows, uint64_t K, uint64_t K16,
                             uint64_t P_pad, const uint32_t* amax_bits, __nv_bfloat16* planes,
                             float* ds) {
  const uint64_t x = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (x >= K16 * P_pad) return;
  const uint64_t p = x % P_pad, k = x / P_pad;
  const bool in = p < rows && k < K;
  const float val = in ? g[p * K + k] : 0.0f;
  ds[p * K16 + k] = val;
  // quantum q = 2^(E-8), 2^E > max |dS| of the score (no smaller than 2^-126)
  float q = 1.0f;
  if (k < K) {
    const float am = __uint_as_float(amax_bits[k]);
    if (am > 0.0f) {
      int e = 0;
      frexpf(am, &e);
      q = ldexpf(1.0f, max(e - 8, -126));
    }
  }
  const uint64_t row0 = (k / kBwScores) * kBwN + (k % kBwScores);
  float rem = val;
#pragma unroll
  for (uint32_t j = 0; j < 4; ++j) {
    const float qj = q * ldexpf(1.0f, -8 * int(j));   // power of two: exact division
    const float limb = qj > 0.0f ? rintf(rem / qj) * qj : 0.0f;
    rem -= limb;
    planes[(row0 + kBwScores * j) * P_pad + p] = __float2bfloat16_rn(limb);
  }
}

// ---- host ------------------------------------------------------------------------

template <int NP, int ST, bool MISSING, bool COUNT_LAST>
static cudaError_t launch_tc(const CUtensorMap& amap, const CUtensorMap& pmap, const TcArgs& a,
                             uint32_t ptiles, uint32_t stiles, cudaStream_t s) {
  using L = TcSmem<NP, ST>;
  const cudaError_t e = raise_smem_limit(
      reinterpret_cast<const void*>(gnm_tc_accumulate<NP, ST, MISSING, COUNT_LAST>),
      int(L::kTotal));
  if (e != cudaSuccess) return e;
  const dim3 grid = a.raster ? dim3(stiles, ptiles) : dim3(ptiles, stiles);
  gnm_tc_accumulate<NP, ST, MISSING, COUNT_LAST><<<grid, kTcThreads, L::kTotal, s>>>(amap, pmap,
                                                                                     a);
  return cudaGetLastError();
}

template <int NP, int ST, bool MISSING, bool COUNT_LAST>
static cudaError_t launch_t8(const CUtensorMap& amap, const CUtensorMap& pmap, const T8Args& a,
                             uint32_t ptiles, uint32_t stiles, cudaStream_t s) {
  using L = T8Smem<NP, ST>;
  const cudaError_t e = raise_smem_limit(
      reinterpret_cast<const void*>(gnm_t8_accumulate<NP, ST, MISSING, COUNT_LAST>),
      int(L::kTotal));
  if (e != cudaSuccess) return e;
  const dim3 grid = a.raster ? dim3(stiles, ptiles) : dim3(ptiles, stiles);
  gnm_t8_accumulate<NP, ST, MISSING, COUNT_LAST><<<grid, kT8Threads, L::kTotal, s>>>(amap, pmap,
                                                                                     a);
  return cudaGetLastError();
}

// Persistent clusters of two CTAs along x (CTA 2i + r is rank r of cluster
// i): as many as can be resident at once, at most one per work item.
static uint32_t pair_clusters(int dev, uint32_t items) {
  static std::mutex mu;
  static int cached[64] = {};
  int n = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64) n = cached[dev];
  }
  if (n == 0) {
    using L = T8PairSmem<2, kT8PairStagesPair>;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2);
    cfg.blockDim = dim3(kT8Threads);
    cfg.dynamicSmemBytes = L::kTotal;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaOccupancyMaxActiveClusters(&n, gnm_t8_pairs<kT8PairStagesPair>, &cfg) != cudaSuccess ||
        n <= 0) {
      (void)cudaGetLastError();
      int sms = 0;
      check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
                 "cudaDeviceGetAttribute");
      n = std::max(1, sms / 2);
    }
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64) cached[dev] = n;
  }
  return std::max<uint32_t>(1, std::min<uint32_t>(uint32_t(n), items));
}

static void launch_t8_pairs(const CUtensorMap& amap2, const CUtensorMap& amap1,
                            const CUtensorMap& pmap, const T8PairArgs& a, int dev,
                            cudaStream_t s) {
  using L = T8PairSmem<2, kT8PairStagesPair>;
  const void* fn = reinterpret_cast<const void*>(gnm_t8_pairs<kT8PairStagesPair>);
  check_cuda(raise_smem_limit(fn, int(L::kTotal)), "8-bit pair shared memory");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * pair_clusters(dev, a.items));
  cfg.blockDim = dim3(kT8Threads);
  cfg.dynamicSmemBytes = L::kTotal;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  check_cuda(cudaLaunchKernelEx(&cfg, gnm_t8_pairs<kT8PairStagesPair>, amap2, amap1, pmap, a),
             "8-bit pair launch");
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      fail(GNM_ERR_COMPUTE, "cuTensorMapEncodeTiled is not available from the driver");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 4 limb planes [4][K_pad][V_pad]; a box holds `np` consecutive planes.
static CUtensorMap make_plane_map(const __nv_bfloat16* planes, uint64_t V_pad, uint64_t K_pad,
                                  uint32_t box_scores, uint32_t np) {
  CUtensorMap map;
  cuuint64_t dims[3] = {V_pad, K_pad, 4};
  cuuint64_t strides[2] = {V_pad * 2, K_pad * V_pad * 2};
  cuuint32_t box[3] = {kTcK, box_scores, np};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = tensor_map_encoder()(
      &map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16*>(planes), dims,
      strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(GNM_ERR_COMPUTE, "cuTensorMapEncodeTiled failed for limb planes");
  return map;
}

// 8-bit limb planes [kT8Planes][K_pad][V_pad]; a box holds `rows` scores of `np`
// consecutive planes.
static CUtensorMap make_plane_map8(const int8_t* planes, uint64_t V_pad, uint64_t K_pad,
                                   uint32_t rows, uint32_t np) {
  CUtensorMap map;
  cuuint64_t dims[3] = {V_pad, K_pad, uint64_t(kT8Planes)};
  cuuint64_t strides[2] = {V_pad, K_pad * V_pad};
  cuuint32_t box[3] = {kT8K, rows, np};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = tensor_map_encoder()(
      &map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t*>(planes), dims, strides, box,
      estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(GNM_ERR_COMPUTE, "cuTensorMapEncodeTiled failed for 8-bit planes");
  return map;
}

// Row-major 2D map [rows][cols] (cols innermost; the row stride is cols
// elements, a multiple of 16 bytes).
static CUtensorMap make_2d_map(CUtensorMapDataType type, uint32_t elem_bytes, const void* base,
                               uint64_t cols, uint64_t rows, uint32_t box_cols,
                               uint32_t box_rows, CUtensorMapSwizzle swizzle, const char* what) {
  if ((cols * elem_bytes) % 16 != 0 || reinterpret_cast<uintptr_t>(base) % 16 != 0)
    fail(GNM_ERR_COMPUTE, std::string(what) + ": rows are not 16-byte aligned");
  CUtensorMap map;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * elem_bytes};
  cuuint32_t box[2] = {box_cols, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = tensor_map_encoder()(&map, type, 2, const_cast<void*>(base), dims, strides, box,
                                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(GNM_ERR_COMPUTE, std::string("cuTensorMapEncodeTiled failed for ") + what);
  return map;
}

// Variant splits of the narrow engine: enough CTAs for about four waves, then
// the count whose last wave is fullest (at most 16 splits, one stage each).
static uint32_t narrow_splits(uint64_t base_ctas, uint64_t stages, int sms) {
  uint32_t best = 1;
  double best_score = -1.0;
  for (uint32_t s = 1; s <= 16 && s <= std::max<uint64_t>(1, stages); ++s) {
    const uint64_t ctas = base_ctas * s;
    const uint64_t waves = (ctas + sms - 1) / sms;
    const double tail = double(ctas) / double(waves * uint64_t(sms));
    const double score = tail * std::min(1.0, double(ctas) / (4.0 * sms));
    if (score > best_score + 1e-9) {
      best_score = score;
      best = s;
    }
  }
  return best;
}

void tensor_plan_create(gnm_plan* p, const gnm_prep_view* prep, PhaseTrace* trace) {
  auto mark = [&](const char* what) {
    if (trace) trace->mark(what);
  };
  auto* t = new TensorPlan();
  p->tensor = t;
  t->K_pad = (p->K + kTcM - 1) / kTcM * kTcM;
  t->V_pad = std::max<uint64_t>(kTcK, (p->V + kTcK - 1) / kTcK * kTcK);
  t->ptiles = uint32_t(std::max<uint64_t>(1, (p->fam + kTcN - 1) / kTcN));
  t->stiles = uint32_t(t->K_pad / kTcM);
  t->P_pad = uint64_t(t->ptiles) * kTcN;
  t->can_narrow = p->K <= kNarrowMaxScores;
  t->narrow = t->can_narrow;
  // the wide kernel runs on 8-bit limbs unless a shape says otherwise: 1.4x
  // the BF16 limbs' speed on the batched workload, errors below 2.3e-7 at full
  // length on every workload
  t->i8 = true;
  // SM pairs when the plan fills pairs of 128-score tiles (with one tile the
  // pair's second CTA would hold no scores)
  t->pair = t->stiles >= 2;
  // score tiles fastest: the CTAs (clusters) running at once share a people
  // tile's packed rows (batched workload: 126.8 against 144.6 ms per step on
  // pairs, 159.4 against 165.7 on one SM)
  p->raster = 1;
  if (t->V_pad > (uint64_t(1) << 31)) fail(GNM_ERR_INVALID, "too many variants for the tensor engine");

  const uint64_t plane = t->K_pad * t->V_pad;
  auto alloc = [&](void** ptr, uint64_t bytes, const char* what) {
    *ptr = pool_alloc(p->device, bytes, what);
    p->device_bytes += bytes;
  };
  alloc(reinterpret_cast<void**>(&t->d_planes_dos), 4 * plane * 2, "cudaMalloc(limb planes)");
  alloc(reinterpret_cast<void**>(&t->d_planes_mis), 4 * plane * 2, "cudaMalloc(limb planes)");
  // partials hold either kernel's layout when both can run the plan (the
  // autotuner chooses between them)
  t->part_elems = t->K_pad * t->P_pad;
  if (t->can_narrow) {
    const uint64_t k16 = (p->K + kNrScores - 1) / kNrScores * kNrScores;
    const uint64_t base = ((p->fam + kNrM - 1) / kNrM) * (k16 / kNrScores);
    int sms = 0;
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device),
               "cudaDeviceGetAttribute");
    t->nsplits = narrow_splits(base, t->V_pad / kTcK, std::max(1, sms));
    t->nslot = k16 * t->P_pad;
    t->part_elems = std::max(t->part_elems, uint64_t(t->nsplits) * t->nslot);
  }
  alloc(reinterpret_cast<void**>(&t->d_part_sum), t->part_elems * 8, "cudaMalloc(partials)");
  alloc(reinterpret_cast<void**>(&t->d_part_cnt), t->part_elems * 4, "cudaMalloc(partials)");
  if (t->pair)   // the SM-pair kernel's passes 1-3 (written before being read)
    alloc(reinterpret_cast<void**>(&t->d_part_pass), 3 * t->K_pad * t->P_pad * 8,
          "cudaMalloc(pass partials)");
  check_cuda(cudaMemset(t->d_planes_dos, 0, 4 * plane * 2), "memset planes");
  check_cuda(cudaMemset(t->d_planes_mis, 0, 4 * plane * 2), "memset planes");
  t->V_pad8 = std::max<uint64_t>(kT8K, (p->V + kT8K - 1) / kT8K * kT8K);
  const uint64_t plane8 = t->K_pad * t->V_pad8;
  alloc(reinterpret_cast<void**>(&t->d_planes8), kT8Planes * plane8, "cudaMalloc(8-bit planes)");
  alloc(reinterpret_cast<void**>(&t->d_quanta8), kT8Planes * t->K_pad * 8, "cudaMalloc(quanta)");
  check_cuda(cudaMemset(t->d_planes8, 0, kT8Planes * plane8), "memset planes");
  mark("  tensor: planes alloc");

  const uint64_t nnz = p->V ? prep->sparse_row_offsets[p->V] : 0;
  float *dw = nullptr, *dc = nullptr;
  uint32_t* dq = nullptr;
  uint32_t* dcol = nullptr;
  uint64_t* doff = nullptr;
  dw = static_cast<decltype(dw)>(
      pool_alloc(p->device, std::max<uint64_t>(1, nnz) * 4, "plane build inputs"));
  dc = static_cast<decltype(dc)>(
      pool_alloc(p->device, std::max<uint64_t>(1, nnz) * 4, "plane build inputs"));
  dcol = static_cast<decltype(dcol)>(
      pool_alloc(p->device, std::max<uint64_t>(1, nnz) * 4, "plane build inputs"));
  doff = static_cast<decltype(doff)>(
      pool_alloc(p->device, (p->V + 1) * 8, "plane build inputs"));
  dq = static_cast<uint32_t*>(pool_alloc(p->device, t->K_pad * 4, "plane build inputs"));
  struct Tmp {
    void* a[5];
    ~Tmp() {
      for (void* x : a) pool_free(x);
    }
  } tmp{{dw, dc, dcol, doff, dq}};
  if (nnz) {
    copy_to_device(dw, prep->sparse_weights, nnz * 4, 0);
    copy_to_device(dc, prep->sparse_missing_corrections, nnz * 4, 0);
    copy_to_device(dcol, prep->sparse_score_columns, nnz * 4, 0);
  }
  copy_to_device(doff, prep->sparse_row_offsets, (p->V + 1) * 8, 0);
  mark("  tensor: csr upload");
  // per-score quantum from max |x| over the score's values (on the device)
  check_cuda(cudaMemset(dq, 0, t->K_pad * 4), "memset");
  if (nnz) {
    const uint32_t smem = t->K_pad <= kAmaxSharedScores ? uint32_t(t->K_pad * 4) : 0u;
    const uint64_t blocks = std::min<uint64_t>((nnz + 255) / 256, 4096);
    gnm_tc_amax<<<uint32_t(blocks), 256, smem>>>(dw, dc, dcol, nnz, t->K_pad, dq);
    check_cuda(cudaGetLastError(), "weight maximum launch");
  }
  if (p->V) {
    gnm_tc_build_planes<<<uint32_t((p->V + 255) / 256), 256>>>(
        dw, dc, dcol, doff, p->V, dq, t->d_planes_dos, t->d_planes_mis, t->K_pad, t->V_pad);
    check_cuda(cudaGetLastError(), "plane build launch");
  }
  gnm_t8_quanta<<<uint32_t((t->K_pad + 255) / 256), 256>>>(dq, t->K_pad, t->d_quanta8);
  check_cuda(cudaGetLastError(), "quanta launch");
  if (p->V) {
    gnm_t8_build_planes<<<uint32_t((p->V + 255) / 256), 256>>>(
        dw, dc, dcol, doff, p->V, t->d_quanta8, t->d_planes8, t->K_pad, t->V_pad8);
    check_cuda(cudaGetLastError(), "8-bit plane build launch");
  }
  check_cuda(cudaStreamSynchronize(0), "plane build");
  mark("  tensor: plane build");
  t->map8_2 = make_plane_map8(t->d_planes8, t->V_pad8, t->K_pad, kTcM, 2);
  t->map8_1 = make_plane_map8(t->d_planes8, t->V_pad8, t->K_pad, kTcM, 1);
  t->map_dos = make_plane_map(t->d_planes_dos, t->V_pad, t->K_pad, kTcM, kTcPlanes);
  t->map_mis = make_plane_map(t->d_planes_mis, t->V_pad, t->K_pad, kTcM, kTcPlanes);
  if (t->can_narrow) {
    t->nmap_dos = make_plane_map(t->d_planes_dos, t->V_pad, t->K_pad, kNrScores, 4);
    t->nmap_mis = make_plane_map(t->d_planes_mis, t->V_pad, t->K_pad, kNrScores, 4);
    t->nmap8_dos = make_plane_map8(t->d_planes8, t->V_pad8, t->K_pad, kNrScores, 4);
    t->nmap8_mis = make_plane_map8(t->d_planes8, t->V_pad8, t->K_pad, kNrScores, 5);
  }
}

void tensor_plan_destroy(gnm_plan* p) {
  TensorPlan* t = p->tensor;
  if (!t) return;
  pool_free(t->d_planes_dos);
  pool_free(t->d_planes_mis);
  pool_free(t->d_planes8);
  pool_free(t->d_quanta8);
  pool_free(t->d_part_sum);
  pool_free(t->d_part_cnt);
  pool_free(t->d_part_pass);
  delete t;
  p->tensor = nullptr;
}

bool tensor_can_narrow(const gnm_plan* p) { return p->tensor && p->tensor->can_narrow; }
bool tensor_is_narrow(const gnm_plan* p) { return p->tensor && p->tensor->narrow; }
bool tensor_is_i8(const gnm_plan* p) { return p->tensor && p->tensor->i8; }
void tensor_set_i8(gnm_plan* p, bool i8) { p->tensor->i8 = i8; }
bool tensor_is_pair(const gnm_plan* p) { return p->tensor && p->tensor->pair; }
void tensor_set_pair(gnm_plan* p, bool pair) {
  TensorPlan* t = p->tensor;
  if (pair && !t->d_part_pass) {   // the pass arrays of the SM-pair kernel, on first use
    const uint64_t bytes = 3 * t->K_pad * t->P_pad * 8;
    t->d_part_pass = static_cast<double*>(pool_alloc(p->device, bytes, "pass partials"));
    p->device_bytes += bytes;
    t->pass_valid = false;
  }
  t->pair = pair;
}
void tensor_set_narrow(gnm_plan* p, bool narrow) {
  if (narrow && !tensor_can_narrow(p))
    fail(GNM_ERR_INVALID, "the narrow tensor kernel serves at most 64 scores");
  p->tensor->narrow = narrow;
}

void tensor_reset(gnm_plan* p, cudaStream_t s) {
  TensorPlan* t = p->tensor;
  check_cuda(cudaMemsetAsync(t->d_part_sum, 0, t->part_elems * 8, s), "reset partials");
  check_cuda(cudaMemsetAsync(t->d_part_cnt, 0, t->part_elems * 4, s), "reset partials");
  t->pass_valid = false;   // the next SM-pair accumulate writes its pass arrays
}

void tensor_accumulate(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch, uint64_t v0,
                       uint64_t nv, cudaStream_t s) {
  TensorPlan* t = p->tensor;
  if (v0 % kTcK != 0)
    fail(GNM_ERR_INVALID, "tensor engine blocks must start at a multiple of 64 variants");
  if (t->narrow && t->i8 && v0 % kT8K == 0) {
    const CUtensorMap pmap8 = make_row_map(d_rows, p->bpv, nv, pitch, kNrM / 4, kT8K);
    check_cuda(raise_smem_limit(reinterpret_cast<const void*>(gnm_t8_narrow),
                                int(T8NrSmem::kTotal)),
               "narrow 8-bit shared memory");
    NrArgs a;
    a.num_rows = nv;
    a.a_x0 = int32_t(v0);
    const uint32_t nall = uint32_t((nv + kT8K - 1) / kT8K);
    a.stages_per_split = (nall + t->nsplits - 1) / t->nsplits;
    a.part_sum = t->d_part_sum;
    a.part_cnt = t->d_part_cnt;
    a.P_pad = t->P_pad;
    a.slot_stride = t->nslot;
    a.err = p->d_err;
    const dim3 grid(uint32_t((p->fam + kNrM - 1) / kNrM),
                    uint32_t((p->K + kNrScores - 1) / kNrScores), t->nsplits);
    gnm_t8_narrow<<<grid, kNrThreads, T8NrSmem::kTotal, s>>>(t->nmap8_dos, t->nmap8_mis, pmap8,
                                                             a, t->d_quanta8, t->K_pad);
    check_cuda(cudaGetLastError(), "narrow 8-bit tensor launch");
    p->launches += 1;
    return;
  }
  if (t->narrow) {
    const CUtensorMap pmap = make_row_map(d_rows, p->bpv, nv, pitch, kNrM / 4, kTcK);
    check_cuda(raise_smem_limit(reinterpret_cast<const void*>(gnm_tc_narrow), int(NrSmem::kTotal)),
               "narrow shared memory");
    NrArgs a;
    a.num_rows = nv;
    a.a_x0 = int32_t(v0);
    const uint32_t nall = uint32_t((nv + kTcK - 1) / kTcK);
    a.stages_per_split = (nall + t->nsplits - 1) / t->nsplits;
    a.part_sum = t->d_part_sum;
    a.part_cnt = t->d_part_cnt;
    a.P_pad = t->P_pad;
    a.slot_stride = t->nslot;
    a.err = p->d_err;
    const dim3 grid(uint32_t((p->fam + kNrM - 1) / kNrM),
                    uint32_t((p->K + kNrScores - 1) / kNrScores), t->nsplits);
    gnm_tc_narrow<<<grid, kNrThreads, NrSmem::kTotal, s>>>(t->nmap_dos, t->nmap_mis, pmap, a);
    check_cuda(cudaGetLastError(), "narrow tensor launch");
    p->launches += 1;
    return;
  }
  if (t->i8 && v0 % kT8K == 0) {
    // dosage limbs 0-1 and 2-3, correction limbs 0-1 and 2-3, then the counts
    const CUtensorMap pmap8 = make_row_map(d_rows, p->bpv, nv, pitch, kTcN / 4, kT8K);
    T8Args b;
    b.num_rows = nv;
    b.a_x0 = int32_t(v0);
    b.part_sum = t->d_part_sum;
    b.part_cnt = t->d_part_cnt;
    b.P_pad = t->P_pad;
    b.K_pad = t->K_pad;
    b.quanta = t->d_quanta8;
    b.err = p->d_err;
    b.raster = p->raster;
    if (b.raster && t->ptiles > 65535u) b.raster = 0;  // grid.y limit
    if (t->pair) {
      // SM pairs, one persistent launch: each CTA loads its 128 people's
      // packed bytes (32 per row)
      const CUtensorMap pmap_half = make_row_map(d_rows, p->bpv, nv, pitch, kTcN / 8, kT8K);
      T8PairArgs c;
      c.num_rows = nv;
      c.a_x0 = int32_t(v0);
      c.part_sum = t->d_part_sum;
      c.part_pass = t->d_part_pass;
      c.part_cnt = t->d_part_cnt;
      c.P_pad = t->P_pad;
      c.K_pad = t->K_pad;
      c.quanta = t->d_quanta8;
      c.err = p->d_err;
      c.raster = p->raster;
      c.ptiles = t->ptiles;
      c.spairs = (t->stiles + 1) / 2;
      c.spairs_m = (c.spairs + 1) / 2;
      c.items = 4 * c.ptiles * c.spairs + c.ptiles * c.spairs_m;
      c.store = t->pass_valid ? 0u : 1u;
      launch_t8_pairs(t->map8_2, t->map8_1, pmap_half, c, p->device, s);
      t->pass_valid = true;
      p->launches += 1;
      return;
    }
    for (int32_t z : {0, 2}) {
      b.z0 = z;
      check_cuda((launch_t8<2, kT8StagesPair, false, false>(t->map8_2, pmap8, b, t->ptiles,
                                                        t->stiles, s)),
                 "8-bit tensor dosage launch");
    }
    for (int32_t z : {4, 6}) {
      b.z0 = z;
      check_cuda((launch_t8<2, kT8StagesPair, true, false>(t->map8_2, pmap8, b, t->ptiles,
                                                       t->stiles, s)),
                 "8-bit tensor missing launch");
    }
    b.z0 = 8;
    check_cuda((launch_t8<1, kT8StagesOne, true, true>(t->map8_1, pmap8, b, t->ptiles, t->stiles,
                                                    s)),
               "8-bit tensor count launch");
    p->launches += 5;
    return;
  }
  const CUtensorMap pmap = make_row_map(d_rows, p->bpv, nv, pitch, kTcN / 4, kTcK);
  TcArgs a;
  a.num_rows = nv;
  a.a_x0 = int32_t(v0);
  a.part_sum = t->d_part_sum;
  a.part_cnt = t->d_part_cnt;
  a.P_pad = t->P_pad;
  a.err = p->d_err;
  a.raster = p->raster;
  if (a.raster && t->ptiles > 65535u) a.raster = 0;  // grid.y limit
  // dosage limbs 0-1 and 2-3, then correction limbs 0-1 and (limb 2, count)
  a.z0 = 0;
  check_cuda((launch_tc<kTcPlanes, kTcStages, false, false>(t->map_dos, pmap, a, t->ptiles,
                                                            t->stiles, s)),
             "tensor dosage launch");
  a.z0 = 2;
  check_cuda((launch_tc<kTcPlanes, kTcStages, false, false>(t->map_dos, pmap, a, t->ptiles,
                                                            t->stiles, s)),
             "tensor dosage launch");
  a.z0 = 0;
  check_cuda((launch_tc<kTcPlanes, kTcStages, true, false>(t->map_mis, pmap, a, t->ptiles,
                                                           t->stiles, s)),
             "tensor missing launch");
  a.z0 = 2;
  check_cuda((launch_tc<kTcPlanes, kTcStages, true, true>(t->map_mis, pmap, a, t->ptiles,
                                                          t->stiles, s)),
             "tensor missing launch");
  p->launches += 4;
}

void tensor_finalize(gnm_plan* p, double* d_sums, uint32_t* d_counts, bool add_baseline,
                     cudaStream_t s) {
  TensorPlan* t = p->tensor;
  const uint64_t n = p->P * p->K;
  if (n == 0) return;
  gnm_tc_finalize<<<uint32_t((n + 255) / 256), 256, 0, s>>>(
      t->d_part_sum, t->d_part_cnt, t->P_pad, add_baseline ? p->d_baseline : p->d_zero_base,
      p->d_out_to_fam, p->P, p->K, t->narrow ? t->nsplits : 0u, t->nslot,
      t->pass_valid ? t->d_part_pass : nullptr, t->K_pad * t->P_pad, d_sums, d_counts);
  check_cuda(cudaGetLastError(), "tensor finalize launch");
  p->launches += 1;
}

// dS limbs in 8 bits (gnm_t8_backward): buffers [limb rows][P_pad] int8,
// [P_pad][K16] FP32 dS, [4][K16] FP64 quanta, [K16] maxima, re-derived on
// every call.
static void backward_dw8(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch, const float* gsf,
                         float* d_grad_w, float* d_grad_corr, cudaStream_t s) {
  const uint64_t K16 = (p->K + kBwScores - 1) / kBwScores * kBwScores;
  const uint64_t P_pad = std::max<uint64_t>(kBw8K, (p->fam + kBw8K - 1) / kBw8K * kBw8K);
  const uint64_t limb_rows = K16 / kBwScores * kBwN;
  const uint64_t planes_bytes = (limb_rows * P_pad + 255) / 256 * 256;
  const uint64_t ds_bytes = (P_pad * K16 * 4 + 255) / 256 * 256;
  const uint64_t q_bytes = 4 * K16 * 8;
  const uint64_t need = planes_bytes + ds_bytes + q_bytes + K16 * 4;
  if (p->bw_bytes < need) {
    check_cuda(cudaStreamSynchronize(s), "backward buffer resize");
    pool_free(p->d_bw);
    p->d_bw = nullptr;
    p->device_bytes -= p->bw_bytes;
    p->bw_bytes = 0;
    p->d_bw = static_cast<uint8_t*>(pool_alloc(p->device, need, "backward dS limbs"));
    p->bw_bytes = need;
    p->device_bytes += need;
  }
  auto* planes = reinterpret_cast<int8_t*>(p->d_bw);
  auto* ds = reinterpret_cast<float*>(p->d_bw + planes_bytes);
  auto* quanta = reinterpret_cast<double*>(p->d_bw + planes_bytes + ds_bytes);
  auto* amax = reinterpret_cast<uint32_t*>(p->d_bw + planes_bytes + ds_bytes + q_bytes);
  check_cuda(cudaMemsetAsync(amax, 0, K16 * 4, s), "memset");
  const uint64_t na = (p->fam + 63) / 64 * p->K;
  if (na) {
    gnm_bw_amax<<<uint32_t((na + 255) / 256), 256, 0, s>>>(gsf, p->fam, p->K, amax);
    check_cuda(cudaGetLastError(), "gradient maximum launch");
    p->launches += 1;
  }
  const uint64_t nb = K16 * P_pad;
  gnm_bw_build8<<<uint32_t((nb + 255) / 256), 256, 0, s>>>(gsf, p->fam, p->K, K16, P_pad, amax,
                                                           planes, quanta, ds);
  check_cuda(cudaGetLastError(), "gradient limb launch");
  p->launches += 1;

  const CUtensorMap rmap = make_row_map(d_rows, p->bpv, p->V, pitch, Bw8Smem::kPkRow, kBwM);
  const CUtensorMap bmap =
      make_2d_map(CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, planes, P_pad, limb_rows, kBw8K, kBwN,
                  CU_TENSOR_MAP_SWIZZLE_128B, "gradient limbs");
  const CUtensorMap dmap = make_2d_map(CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, ds, K16, P_pad,
                                       kBwScores, kBw8K, CU_TENSOR_MAP_SWIZZLE_NONE, "gradient");
  check_cuda(raise_smem_limit(reinterpret_cast<const void*>(gnm_t8_backward), int(Bw8Smem::kTotal)),
             "backward shared memory");
  BwArgs a;
  a.V = p->V;
  a.K = p->K;
  a.nstages = uint32_t(P_pad / kBw8K);
  a.gw = d_grad_w;
  a.gc = d_grad_corr;
  a.err = p->d_err;
  const dim3 grid(uint32_t((p->V + kBwM - 1) / kBwM), uint32_t(K16 / kBwScores));
  gnm_t8_backward<<<grid, kBwThreads, Bw8Smem::kTotal, s>>>(rmap, bmap, dmap, a, quanta, K16);
  check_cuda(cudaGetLastError(), "backward launch");
  p->launches += 1;
}

void backward_dw(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch, const float* d_grad_s,
                 float* d_grad_w, float* d_grad_corr, cudaStream_t s) {
  if (!d_rows || !d_grad_s || !d_grad_w) fail(GNM_ERR_INVALID, "NULL buffer");
  if (pitch < p->bpv) fail(GNM_ERR_INVALID, "pitch smaller than bytes per variant");
  if (pitch % 16 != 0 || reinterpret_cast<uintptr_t>(d_rows) % 16 != 0)
    fail(GNM_ERR_INVALID, "packed rows must be 16-byte aligned with a pitch multiple of 16");
  if (p->V == 0) return;
  const float* gsf = d_grad_s;
  if (p->d_out_to_fam || p->P != p->fam) {
    // dS rows in .bed person order: zero for people outside the keep set
    if (!p->d_grad_fam) {
      p->d_grad_fam = static_cast<float*>(
          pool_alloc(p->device, std::max<uint64_t>(1, p->fam * p->K) * 4, "fam-order gradient"));
      p->device_bytes += p->fam * p->K * 4;
    }
    check_cuda(cudaMemsetAsync(p->d_grad_fam, 0, p->fam * p->K * 4, s), "memset");
    const uint64_t n = p->P * p->K;
    if (n) {
      gnm_scatter_grad<<<uint32_t((n + 255) / 256), 256, 0, s>>>(
          d_grad_s, p->d_out_to_fam, p->P, p->K, p->d_grad_fam);
      check_cuda(cudaGetLastError(), "gradient scatter launch");
      p->launches += 1;
    }
    gsf = p->d_grad_fam;
  }
  if (p->bw_limb_bits == 8) {
    backward_dw8(p, d_rows, pitch, gsf, d_grad_w, d_grad_corr, s);
    return;
  }
  // dS limb rows and the FP32 copy, re-derived on every call
  const uint64_t K16 = (p->K + kBwScores - 1) / kBwScores * kBwScores;
  const uint64_t P_pad = std::max<uint64_t>(kBwK, (p->fam + kBwK - 1) / kBwK * kBwK);
  const uint64_t limb_rows = K16 / kBwScores * kBwN;
  const uint64_t planes_bytes = (limb_rows * P_pad * 2 + 255) / 256 * 256;
  const uint64_t ds_bytes = (P_pad * K16 * 4 + 255) / 256 * 256;
  const uint64_t need = planes_bytes + ds_bytes + K16 * 4;
  if (p->bw_bytes < need) {
    check_cuda(cudaStreamSynchronize(s), "backward buffer resize");
    pool_free(p->d_bw);
    p->d_bw = nullptr;
    p->device_bytes -= p->bw_bytes;
    p->bw_bytes = 0;
    p->d_bw = static_cast<uint8_t*>(pool_alloc(p->device, need, "backward dS limbs"));
    p->bw_bytes = need;
    p->device_bytes += need;
  }
  auto* planes = reinterpret_cast<__nv_bfloat16*>(p->d_bw);
  auto* ds = reinterpret_cast<float*>(p->d_bw + planes_bytes);
  auto* amax = reinterpret_cast<uint32_t*>(p->d_bw + planes_bytes + ds_bytes);
  check_cuda(cudaMemsetAsync(amax, 0, K16 * 4, s), "memset");
  const uint64_t na = (p->fam + 63) / 64 * p->K;
  if (na) {
    gnm_bw_amax<<<uint32_t((na + 255) / 256), 256, 0, s>>>(gsf, p->fam, p->K, amax);
    check_cuda(cudaGetLastError(), "gradient maximum launch");
    p->launches += 1;
  }
  const uint64_t nb = K16 * P_pad;
  gnm_bw_build<<<uint32_t((nb + 255) / 256), 256, 0, s>>>(gsf, p->fam, p->K, K16, P_pad, amax,
                                                          planes, ds);
  check_cuda(cudaGetLastError(), "gradient limb launch");
  p->launches += 1;

  const CUtensorMap rmap = make_row_map(d_rows, p->bpv, p->V, pitch, kBwK / 4, kBwM);
  const CUtensorMap bmap =
      make_2d_map(CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, planes, P_pad, limb_rows, kBwK, kBwN,
                  CU_TENSOR_MAP_SWIZZLE_128B, "gradient limbs");
  const CUtensorMap dmap = make_2d_map(CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, ds, K16, P_pad,
                                       kBwScores, kBwK, CU_TENSOR_MAP_SWIZZLE_NONE, "gradient");
  check_cuda(raise_smem_limit(reinterpret_cast<const void*>(gnm_tc_backward), int(BwSmem::kTotal)),
             "backward shared memory");
  BwArgs a;
  a.V = p->V;
  a.K = p->K;
  a.nstages = uint32_t(P_pad / kBwK);
  a.gw = d_grad_w;
  a.gc = d_grad_corr;
  a.err = p->d_err;
  const dim3 grid(uint32_t((p->V + kBwM - 1) / kBwM), uint32_t(K16 / kBwScores));
  gnm_tc_backward<<<grid, kBwThreads, BwSmem::kTotal, s>>>(rmap, bmap, dmap, a);
  check_cuda(cudaGetLastError(), "backward launch");
  p->launches += 1;
}

}  // namespace gnm
