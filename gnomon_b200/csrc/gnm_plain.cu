// gnm_plain.cu — plain (FP32 CUDA-core) scoring path for sm_100a.
//
// Replaces the reference GPU engine's unpack_plink -> zero -> scatter ->
// 3x SGEMM -> combine chain (score/cuda_backend.rs:62-218, 2067-2333) for small
// score counts with ONE fused kernel per score column:
//
//   * packed .bed rows are TMA-staged (cp.async.bulk.tensor, no multicast)
//     into shared memory in [48 rows x 1024 bytes] stages, double-buffered;
//   * each thread owns one 32-bit word column = 16 people; every 3 variant
//     rows it transposes the 2-bit codes into per-person 6-bit indices (one
//     byte each, pre-scaled by 4) with a handful of shift/mask ops;
//   * a 64-entry FP32 table per 3-variant group, built in shared memory from
//     {-missing_correction, dosage_weight, 2*dosage_weight} (prepare.rs:197-208
//     folding, code 00 contributes 0), turns 3 genotypes into ONE lookup:
//     decode, effect-allele flip and the missing-call rule are all folded in;
//   * missing calls (code 01) are counted with SWAR bit tricks on the raw row
//     words (x & ~(x>>1) & member_mask, three rows summed with one add);
//   * FP32 partial sums cover one 48-variant stage and are flushed to FP64
//     registers; variant splits write FP64 partials that gnm_finalize reduces
//     in a fixed order (deterministic) and gathers through
//     output_idx_to_fam_idx, adding the FP64 baseline (pipeline.rs:1739-1775).
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "gnm_device.cuh"
#include "gnm_internal.h"

namespace gnm {

// Shared-memory layout of one plain CTA (dynamic smem, offsets in bytes).
struct PlainSmem {
  static constexpr uint32_t kStageBytes = kPlainRows * kPlainTileBytes;      // 49152
  static constexpr uint32_t kBoxBytes = kPlainRows * kPlainBoxBytes;         // 12288
  static constexpr uint32_t kRecBytes = kPlainRows * 16;                     // 768
  static constexpr uint32_t kLutBytes = (kPlainRows / 3) * 64 * 4;           // 4096
  static constexpr uint32_t kStages = 2;
  static constexpr uint32_t kTileOff = 0;
  static constexpr uint32_t kRecOff = kTileOff + kStages * kStageBytes;
  static constexpr uint32_t kLutOff = kRecOff + kStages * kRecBytes;
  static constexpr uint32_t kBarOff = kLutOff + kStages * kLutBytes;
  static constexpr uint32_t kTotal = kBarOff + 64;
};

// Two FP32 additions in one instruction (sm_100 packed f32x2): acc += {lo, hi}.
__device__ __forceinline__ uint64_t add_f32x2(uint64_t acc, float lo, float hi) {
  uint64_t r;
  asm("{\n\t.reg .b64 t;\n\tmov.b64 t, {%2, %3};\n\tadd.rn.f32x2 %0, %1, t;\n\t}"
      : "=l"(r)
      : "l"(acc), "f"(lo), "f"(hi));
  return r;
}

__device__ __forceinline__ void unpack_f32x2(uint64_t v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

__device__ __forceinline__ void plain_issue_stage(const CUtensorMap* map, const float4* recs,
                                                  uint32_t smem_base, uint32_t buf,
                                                  int32_t tile_x, int32_t row0,
                                                  uint64_t rec_row0) {
  const uint32_t bar = smem_base + PlainSmem::kBarOff + 8 * buf;
  mbar_arrive_expect_tx(bar, PlainSmem::kStageBytes + PlainSmem::kRecBytes);
  const uint32_t tile = smem_base + PlainSmem::kTileOff + buf * PlainSmem::kStageBytes;
#pragma unroll
  for (uint32_t b = 0; b < kPlainTileBytes / kPlainBoxBytes; ++b)
    tma_load_2d(tile + b * PlainSmem::kBoxBytes, map, tile_x + int32_t(b * kPlainBoxBytes), row0,
                bar);
  bulk_load(smem_base + PlainSmem::kRecOff + buf * PlainSmem::kRecBytes, recs + rec_row0,
            PlainSmem::kRecBytes, bar);
}

// grid = (people tiles, variant splits); block = kPlainThreads.
__global__ void __launch_bounds__(kPlainThreads, 2)
    gnm_plain_accumulate(const __grid_constant__ CUtensorMap map, PlainArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t sbase = smem_u32(smem);
  const uint32_t tid = threadIdx.x;
  const uint32_t tile = blockIdx.x;
  const uint32_t split = blockIdx.y;

  const uint64_t rows_per_split = uint64_t(a.stages_per_split) * kPlainRows;
  const uint64_t r_begin = uint64_t(split) * rows_per_split;
  if (r_begin >= a.num_rows) return;
  const uint64_t r_end = min(a.num_rows, r_begin + rows_per_split);
  const uint32_t nstages = uint32_t((r_end - r_begin + kPlainRows - 1) / kPlainRows);
  const int32_t tile_x = int32_t(tile * kPlainTileBytes);

  if (tid == 0) {
    prefetch_tmap(&map);
    mbar_init(sbase + PlainSmem::kBarOff, 1);
    mbar_init(sbase + PlainSmem::kBarOff + 8, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0) {
    for (uint32_t s = 0; s < 2 && s < nstages; ++s)
      plain_issue_stage(&map, a.records, sbase, s, tile_x, int32_t(r_begin + s * kPlainRows),
                        a.record_row0 + r_begin + s * kPlainRows);
  }

  // FP32 sums as packed pairs for add.rn.f32x2: accp[2q] holds people
  // (q, 4+q), accp[2q+1] people (8+q, 12+q) of this thread's 16.
  uint64_t accp[8];
  double acc64[16];
  uint32_t cnt[16];
  uint32_t by[4] = {0u, 0u, 0u, 0u};   // byte counters: byte j = person 4j+q
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    acc64[i] = 0.0;
    cnt[i] = 0u;
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) accp[i] = 0ull;

  // Each thread reads word column `tid` of the 1024-byte stage row; the stage
  // is stored as 4 TMA boxes of [48 rows][256 bytes].
  const uint32_t word_off = (tid / (kPlainBoxBytes / 4)) * PlainSmem::kBoxBytes +
                            (tid % (kPlainBoxBytes / 4)) * 4;
  // warps whose 128 bytes all lie past the row's last byte only hold padding
  const bool warp_active =
      uint64_t(tile) * kPlainTileBytes + uint64_t(tid & ~31u) * 4 < a.bytes_per_row;

  for (uint32_t st = 0; st < nstages; ++st) {
    const uint32_t buf = st & 1u;
    const uint32_t parity = (st >> 1) & 1u;
    const bool ok = mbar_wait_bounded(sbase + PlainSmem::kBarOff + 8 * buf, parity);

    // Build the 16 group tables of this stage: 1024 entries, 4 per thread.
    // Entry index e (6 bits): code of row a in bits 0-1, row b in bits 2-3,
    // row c with its two bits swapped (hi in bit 4, lo in bit 5) so that the
    // rarely-set lo bit of row c selects the shared-memory row of the table
    // and lanes collide on banks less often.  The sum of the three FP32 terms
    // is exact in FP64 and rounded to FP32 once.
    {
      const uint64_t row0 = r_begin + uint64_t(st) * kPlainRows;
      const float* rec = reinterpret_cast<const float*>(smem + PlainSmem::kRecOff +
                                                        buf * PlainSmem::kRecBytes);
      float* lut = reinterpret_cast<float*>(smem + PlainSmem::kLutOff + buf * PlainSmem::kLutBytes);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint32_t e = tid * 4 + q;          // 0..1023
        const uint32_t g = e >> 6, idx = e & 63;  // group, index
        const uint32_t code[3] = {idx & 3u, (idx >> 2) & 3u,
                                  ((idx >> 3) & 2u) | ((idx >> 5) & 1u)};
        double v = 0.0;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const uint32_t row = 3 * g + r;
          if (code[r] != 0 && row0 + row < r_end) v += double(rec[row * 4 + (code[r] - 1)]);
        }
        lut[e] = float(v);
      }
      // Membership bitmap of the stage's 48 rows (rows past the split end are
      // not members): two ballots replace 48 per-row mask loads.
      if (tid < 64) {
        const uint32_t r = tid;
        const bool m = r < kPlainRows && row0 + r < r_end && rec[r * 4 + 3] != 0.0f;
        const uint32_t bits = __ballot_sync(0xFFFFFFFFu, m);
        if ((tid & 31) == 0)
          reinterpret_cast<uint32_t*>(smem + PlainSmem::kBarOff + 16)[2 * buf + (tid >> 5)] = bits;
      }
    }
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(a.err, kErrTmaTimeout);
      // Drain the other in-flight stage (bounded) before leaving.
      if (st + 1 < nstages) mbar_wait_bounded(sbase + PlainSmem::kBarOff + 8 * (buf ^ 1u),
                                              ((st + 1) >> 1) & 1u);
      return;
    }

    const uint8_t* tbase = smem + PlainSmem::kTileOff + buf * PlainSmem::kStageBytes + word_off;
    const uint8_t* lbase = smem + PlainSmem::kLutOff + buf * PlainSmem::kLutBytes;
    const uint32_t* mbits = reinterpret_cast<const uint32_t*>(smem + PlainSmem::kBarOff + 16);
    const uint64_t members = uint64_t(mbits[2 * buf]) | (uint64_t(mbits[2 * buf + 1]) << 32);

    uint32_t ev = 0, od = 0;             // nibble counters (people 2j / 2j+1)
    auto group = [&](uint32_t g, uint32_t ma, uint32_t mb, uint32_t mc) {
      const uint32_t xa = *reinterpret_cast<const uint32_t*>(tbase + (3 * g + 0) * kPlainBoxBytes);
      const uint32_t xb = *reinterpret_cast<const uint32_t*>(tbase + (3 * g + 1) * kPlainBoxBytes);
      const uint32_t xc = *reinterpret_cast<const uint32_t*>(tbase + (3 * g + 2) * kPlainBoxBytes);
      // ---- per-person 6-bit indices (x4) ------------------------------
      // row c enters with its code bits swapped (see the table layout above)
      const uint32_t xs = ((xc >> 1) & 0x55555555u) | ((xc << 1) & 0xAAAAAAAAu);
      const uint32_t E = (xa & 0x33333333u) | ((xb << 2) & 0xCCCCCCCCu);
      const uint32_t O = ((xa >> 2) & 0x33333333u) | (xb & 0xCCCCCCCCu);
      uint32_t ix[4];
      ix[0] = ((E << 2) & 0x3C3C3C3Cu) | ((xs << 6) & 0xC0C0C0C0u);
      ix[1] = ((O << 2) & 0x3C3C3C3Cu) | ((xs << 4) & 0xC0C0C0C0u);
      ix[2] = ((E >> 2) & 0x3C3C3C3Cu) | ((xs << 2) & 0xC0C0C0C0u);
      ix[3] = ((O >> 2) & 0x3C3C3C3Cu) | (xs & 0xC0C0C0C0u);
      const uint8_t* lg = lbase + g * 256;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
          v[j] = *reinterpret_cast<const float*>(lg + __byte_perm(ix[q], 0u, 0x4440u + j));
        accp[2 * q] = add_f32x2(accp[2 * q], v[0], v[1]);
        accp[2 * q + 1] = add_f32x2(accp[2 * q + 1], v[2], v[3]);
      }
      // ---- missing counts (code 01 of member rows) ---------------------
      const uint32_t c3 = (xa & ~(xa >> 1) & ma) + (xb & ~(xb >> 1) & mb) + (xc & ~(xc >> 1) & mc);
      ev += c3 & 0x33333333u;
      od += (c3 >> 2) & 0x33333333u;
      if ((g % 5) == 4 || g == kPlainRows / 3 - 1) {
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
      for (uint32_t g = 0; g < kPlainRows / 3; ++g) group(g, 0x55555555u, 0x55555555u, 0x55555555u);
    } else {
#pragma unroll
      for (uint32_t g = 0; g < kPlainRows / 3; ++g) {
        const uint32_t ma = (0u - uint32_t((members >> (3 * g + 0)) & 1u)) & 0x55555555u;
        const uint32_t mb = (0u - uint32_t((members >> (3 * g + 1)) & 1u)) & 0x55555555u;
        const uint32_t mc = (0u - uint32_t((members >> (3 * g + 2)) & 1u)) & 0x55555555u;
        group(g, ma, mb, mc);
      }
    }
    // FP32 sums and byte counters span two stages (96 variants, <= 96 calls
    // per byte counter) before they are flushed to FP64 / 32-bit counts.
    if ((st & 1u) || st + 1 == nstages) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int j = 0; j < 4; ++j) cnt[4 * j + q] += (by[q] >> (8 * j)) & 0xFFu;
        by[q] = 0u;
        float lo, hi;
        unpack_f32x2(accp[2 * q], lo, hi);
        acc64[q] += double(lo);
        acc64[4 + q] += double(hi);
        unpack_f32x2(accp[2 * q + 1], lo, hi);
        acc64[8 + q] += double(lo);
        acc64[12 + q] += double(hi);
        accp[2 * q] = 0ull;
        accp[2 * q + 1] = 0ull;
      }
    }

    __syncthreads();  // every thread is done with stage buffer `buf`
    if (tid == 0 && st + 2 < nstages) {
      fence_proxy_async_smem();
      plain_issue_stage(&map, a.records, sbase, buf, tile_x,
                        int32_t(r_begin + (st + 2) * kPlainRows),
                        a.record_row0 + r_begin + (st + 2) * kPlainRows);
    }
  }

  // FP64 partials for this (split, person) accumulate across calls.
  const uint64_t person0 = uint64_t(tile) * (kPlainTileBytes * 4) + uint64_t(tid) * 16;
  double* ps = a.part_sum + uint64_t(split) * a.part_stride + person0;
  uint32_t* pc = a.part_cnt + uint64_t(split) * a.part_stride + person0;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    ps[i] += acc64[i];
    pc[i] += cnt[i];
  }
}

// out[o*K + k] = init + sum_s part[s][fam(o)] in split order.  One launch per
// score column k (partials of column k).  init = baseline[k] (fresh run).
__global__ void gnm_finalize(FinalizeArgs a) {
  const uint64_t o = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (o >= a.num_people) return;
  const uint64_t f = a.out_to_fam ? a.out_to_fam[o] : o;
  double s = a.baseline[a.k];
  uint32_t c = 0;
  for (uint32_t sp = 0; sp < a.num_splits; ++sp) {
    s += a.part_sum[uint64_t(sp) * a.part_stride + f];
    c += a.part_cnt[uint64_t(sp) * a.part_stride + f];
  }
  a.sums[o * a.K + a.k] = s;
  a.counts[o * a.K + a.k] = c;
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
// CPU oracle: key = mix64(seed) ^ v*C1 ^ i*C2, x = mix64(key).
__global__ void gnm_synth_fill(uint8_t* rows, uint64_t pitch, uint64_t v0, uint64_t nv,
                               uint64_t np, const uint32_t* thr, uint64_t seed) {
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
      const uint64_t x = mix64(sk ^ (i * 0x8CB92BA72F3D8DD7ull));
      const uint32_t um = uint32_t(x), ug = uint32_t(x >> 32);
      const uint32_t code = um < tm ? 1u : (ug < t0 ? 0u : (ug < t1 ? 2u : 3u));
      word |= code << (2 * q);
    }
  }
  reinterpret_cast<uint32_t*>(rows + j * pitch)[w] = word;
}

// ---- host launchers --------------------------------------------------------

cudaError_t launch_plain_accumulate(const CUtensorMap& map, const PlainArgs& a, uint32_t tiles,
                                    uint32_t splits, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(gnm_plain_accumulate,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(PlainSmem::kTotal));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  gnm_plain_accumulate<<<dim3(tiles, splits), kPlainThreads, PlainSmem::kTotal, s>>>(map, a);
  return cudaGetLastError();
}

uint32_t plain_smem_bytes() { return PlainSmem::kTotal; }

cudaError_t launch_finalize(const FinalizeArgs& a, cudaStream_t s) {
  const uint32_t blocks = uint32_t((a.num_people + 255) / 256);
  gnm_finalize<<<blocks ? blocks : 1, 256, 0, s>>>(a);
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
                              uint64_t np, const uint32_t* thr, uint64_t seed, cudaStream_t s) {
  if (nv == 0) return cudaSuccess;
  const uint64_t words = pitch / 4;
  gnm_synth_fill<<<rows_grid((words + 255) / 256, nv), 256, 0, s>>>(rows, pitch, v0, nv, np, thr,
                                                                    seed);
  return cudaGetLastError();
}

}  // namespace gnm
