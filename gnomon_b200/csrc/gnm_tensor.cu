// gnm_tensor.cu — split-BF16 tcgen05 engine (many score columns) and the
// re-unpacking backward kernel dW = G^T dS.
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

struct TensorPlan {
  uint64_t K_pad = 0, V_pad = 0, P_pad = 0;
  uint32_t ptiles = 0, stiles = 0;
  __nv_bfloat16* d_planes_dos = nullptr;  // [4][K_pad][V_pad] W' limbs
  __nv_bfloat16* d_planes_mis = nullptr;  // [4][K_pad][V_pad] -corr limbs, member
  double* d_part_sum = nullptr;           // [K_pad][P_pad]
  uint32_t* d_part_cnt = nullptr;         // [K_pad][P_pad]
  CUtensorMap map_dos, map_mis;
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
        if (*abort_flag) break;
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
        if (*abort_flag) break;
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
      if (*abort_flag) break;
      const uint8_t* pk = smem + L::kPkOff + s * L::kPk;
      uint8_t* bt = smem + L::kBOff + s * L::kB;
#pragma unroll
      for (uint32_t h = 0; h < kTcN / 128; ++h) {
        const uint32_t bc = 32 * h + col;   // byte column: people 4bc..4bc+3
#pragma unroll
        for (uint32_t cc = 0; cc < 2; ++cc) {
          const uint32_t r0 = 16 * vg + 8 * cc;
          uint32_t xl = 0, xh = 0;
#pragma unroll
          for (uint32_t i = 0; i < 4; ++i) {
            xl |= uint32_t(pk[(r0 + i) * (kTcN / 4) + bc]) << (8 * i);
            xh |= uint32_t(pk[(r0 + 4 + i) * (kTcN / 4) + bc]) << (8 * i);
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
            *reinterpret_cast<uint4*>(bt + (n >> 3) * 1024 + (n & 7) * 128 +
                                      ((c ^ (n & 7)) << 4)) = v;
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

// Limb planes from the CSR: one thread per variant.
__global__ void gnm_tc_build_planes(const float* w, const float* corr, const uint32_t* cols,
                                    const uint64_t* offs, uint64_t V, const float* qhi,
                                    __nv_bfloat16* dos, __nv_bfloat16* mis, uint64_t K_pad,
                                    uint64_t V_pad) {
  const uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= V) return;
  const uint64_t plane = K_pad * V_pad;
  for (uint64_t e = offs[v]; e < offs[v + 1]; ++e) {
    const uint32_t k = cols[e];
    // quanta q, q/2^8, q/2^16, q/2^24 (powers of two: the divisions are exact and
    // every residual below is exact in FP32)
    const float q = qhi[k], qm = q * (1.0f / 256.0f), ql = q * (1.0f / 65536.0f),
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
// r = f % 256 and h = r / 128.
__global__ void gnm_tc_finalize(const double* part_sum, const uint32_t* part_cnt, uint64_t P_pad,
                                const double* init, const uint32_t* out_to_fam, uint64_t P,
                                uint64_t K, double* sums, uint32_t* counts) {
  const uint64_t x = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (x >= P * K) return;
  const uint64_t o = x / K, k = x % K;
  const uint64_t f = out_to_fam ? out_to_fam[o] : o;
  const uint64_t r = f % kTcN, h = r / 128, rr = r % 128;
  const uint64_t slot = (f / kTcN) * kTcN + 128 * h + 32 * (rr % 4) + rr / 4;
  sums[x] = init[k] + part_sum[k * P_pad + slot];
  counts[x] = part_cnt[k * P_pad + slot];
}

// ---- backward: dW[v,k] = sum_p d(p,v) dS[p,k], dC[v,k] = -sum_{p missing} dS[p,k]
// One thread per variant row, 16 score columns per CTA column block.  dS comes
// in .bed (fam) person order, [fam][K] (scattered from output order when a keep
// subset is used); 512-person chunks of the block's 16 columns are staged in
// shared memory and read as broadcasts, genotypes come straight from the
// packed row as 16-byte vectors (64 people), and the 16 products per person
// are two-wide FMAs (fma.rn.f32x2).  FP32 sums per chunk, FP64 across chunks.
constexpr uint32_t kBwThreads = 128;
constexpr uint32_t kBwChunk = 512;

__device__ __forceinline__ uint64_t fma_f32x2(float d, uint64_t g, uint64_t acc) {
  uint64_t r;
  asm("{\n\t.reg .b64 dd;\n\tmov.b64 dd, {%1, %1};\n\tfma.rn.f32x2 %0, dd, %2, %3;\n\t}"
      : "=l"(r)
      : "f"(d), "l"(g), "l"(acc));
  return r;
}
__device__ __forceinline__ uint64_t sub_f32x2(uint64_t acc, uint64_t g) {
  uint64_t r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(acc), "l"(g));
  return r;
}

// dS in output order -> fam order (zero for people outside the keep set).
__global__ void gnm_scatter_grad(const float* gs, const uint32_t* out_to_fam, uint64_t P,
                                 uint64_t K, float* gsf) {
  const uint64_t x = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (x >= P * K) return;
  const uint64_t o = x / K, k = x % K;
  gsf[uint64_t(out_to_fam[o]) * K + k] = gs[x];
}

__global__ void __launch_bounds__(kBwThreads)
    gnm_backward_kernel(const uint8_t* rows, uint64_t pitch, uint64_t bpv, uint64_t V,
                        const float* gsf, uint64_t fam, uint32_t K, float* gw, float* gc) {
  __shared__ __align__(16) float g_s[kBwChunk * 16];
  const uint32_t t = threadIdx.x;
  const uint64_t v = uint64_t(blockIdx.x) * kBwThreads + t;
  const uint32_t k0 = blockIdx.y * 16;
  const uint8_t* row = rows + (v < V ? v : 0) * pitch;
  uint64_t aw[8], ac[8];
  double dw[16];
#pragma unroll
  for (int j = 0; j < 8; ++j) aw[j] = ac[j] = 0ull;
#pragma unroll
  for (int j = 0; j < 16; ++j) dw[j] = 0.0;
  for (uint64_t p0 = 0; p0 < fam; p0 += kBwChunk) {
    const uint32_t np = uint32_t(fam - p0 < kBwChunk ? fam - p0 : kBwChunk);
    __syncthreads();
    for (uint32_t i = t; i < kBwChunk * 16; i += kBwThreads) {
      const uint32_t pp = i / 16, kk = i % 16;
      g_s[i] = (pp < np && k0 + kk < K) ? __ldg(gsf + (p0 + pp) * K + k0 + kk) : 0.f;
    }
    __syncthreads();
    if (v < V) {
      for (uint32_t seg = 0; seg < kBwChunk / 64; ++seg) {
        const uint64_t b0 = p0 / 4 + seg * 16;  // 16 bytes = 64 people
        if (b0 >= bpv) break;
        const uint4 x4 = *reinterpret_cast<const uint4*>(row + b0);
        const uint32_t xw[4] = {x4.x, x4.y, x4.z, x4.w};
#pragma unroll
        for (int wi = 0; wi < 4; ++wi) {
          const uint32_t x = xw[wi];
          if (x == 0u) continue;   // 16 homozygous-reference calls
#pragma unroll 4
          for (int i = 0; i < 16; ++i) {
            const uint32_t c = (x >> (2 * i)) & 3u;
            const uint64_t* gp =
                reinterpret_cast<const uint64_t*>(&g_s[(seg * 64 + wi * 16 + i) * 16]);
            uint64_t g[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) g[j] = gp[j];
            // dosage 0 for codes 00 and 01 (missing): one FMA path for everyone
            const float d = c == 3u ? 2.f : (c == 2u ? 1.f : 0.f);
#pragma unroll
            for (int j = 0; j < 8; ++j) aw[j] = fma_f32x2(d, g[j], aw[j]);
            if (c == 1u) {
#pragma unroll
              for (int j = 0; j < 8; ++j) ac[j] = sub_f32x2(ac[j], g[j]);
            }
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float lo, hi;
      asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(aw[j]));
      dw[2 * j] += double(lo);
      dw[2 * j + 1] += double(hi);
      aw[j] = 0ull;
    }
  }
  if (v < V) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float lo, hi;
      asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(ac[j]));
      const uint32_t k = k0 + 2 * j;
      if (k < K) {
        gw[v * K + k] = float(dw[2 * j]);
        if (gc) gc[v * K + k] = lo;
      }
      if (k + 1 < K) {
        gw[v * K + k + 1] = float(dw[2 * j + 1]);
        if (gc) gc[v * K + k + 1] = hi;
      }
    }
  }
}

// ---- host ------------------------------------------------------------------------

template <int NP, int ST, bool MISSING, bool COUNT_LAST>
static cudaError_t launch_tc(const CUtensorMap& amap, const CUtensorMap& pmap, const TcArgs& a,
                             uint32_t ptiles, uint32_t stiles, cudaStream_t s) {
  using L = TcSmem<NP, ST>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(gnm_tc_accumulate<NP, ST, MISSING, COUNT_LAST>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(L::kTotal));
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const dim3 grid = a.raster ? dim3(stiles, ptiles) : dim3(ptiles, stiles);
  gnm_tc_accumulate<NP, ST, MISSING, COUNT_LAST><<<grid, kTcThreads, L::kTotal, s>>>(amap, pmap,
                                                                                     a);
  return cudaGetLastError();
}

// 4 limb planes [4][K_pad][V_pad]; a box holds `np` consecutive planes.
static CUtensorMap make_plane_map(const __nv_bfloat16* planes, uint64_t V_pad, uint64_t K_pad,
                                  uint32_t np) {
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
  CUtensorMap map;
  cuuint64_t dims[3] = {V_pad, K_pad, 4};
  cuuint64_t strides[2] = {V_pad * 2, K_pad * V_pad * 2};
  cuuint32_t box[3] = {kTcK, kTcM, np};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16*>(planes),
                  dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(GNM_ERR_COMPUTE, "cuTensorMapEncodeTiled failed for limb planes");
  return map;
}

void tensor_plan_create(gnm_plan* p) {
  auto* t = new TensorPlan();
  p->tensor = t;
  t->K_pad = (p->K + kTcM - 1) / kTcM * kTcM;
  t->V_pad = std::max<uint64_t>(kTcK, (p->V + kTcK - 1) / kTcK * kTcK);
  t->ptiles = uint32_t(std::max<uint64_t>(1, (p->fam + kTcN - 1) / kTcN));
  t->stiles = uint32_t(t->K_pad / kTcM);
  t->P_pad = uint64_t(t->ptiles) * kTcN;
  if (t->V_pad > (uint64_t(1) << 31)) fail(GNM_ERR_INVALID, "too many variants for the tensor engine");

  // per-score quantum q = 2^(E-8), 2^E >= max |x| over the score's values
  std::vector<float> amax(t->K_pad, 0.f), qhi(t->K_pad, 1.f);
  for (size_t e = 0; e < p->h_cols.size(); ++e) {
    const uint32_t k = p->h_cols[e];
    amax[k] = std::max(amax[k], std::max(std::fabs(p->h_w[e]), std::fabs(p->h_corr[e])));
  }
  for (uint64_t k = 0; k < t->K_pad; ++k)
    if (amax[k] > 0.f) {
      int ex = 0;
      std::frexp(amax[k], &ex);  // amax = f * 2^ex, f in [0.5, 1)
      qhi[k] = std::ldexp(1.0f, ex - 8);
    }
  const uint64_t plane = t->K_pad * t->V_pad;
  auto alloc = [&](void** ptr, uint64_t bytes, const char* what) {
    *ptr = pool_alloc(p->device, bytes, what);
    p->device_bytes += bytes;
  };
  alloc(reinterpret_cast<void**>(&t->d_planes_dos), 4 * plane * 2, "cudaMalloc(limb planes)");
  alloc(reinterpret_cast<void**>(&t->d_planes_mis), 4 * plane * 2, "cudaMalloc(limb planes)");
  alloc(reinterpret_cast<void**>(&t->d_part_sum), t->K_pad * t->P_pad * 8, "cudaMalloc(partials)");
  alloc(reinterpret_cast<void**>(&t->d_part_cnt), t->K_pad * t->P_pad * 4, "cudaMalloc(partials)");
  check_cuda(cudaMemset(t->d_planes_dos, 0, 4 * plane * 2), "memset planes");
  check_cuda(cudaMemset(t->d_planes_mis, 0, 4 * plane * 2), "memset planes");

  const uint64_t nnz = p->h_cols.size();
  float *dw = nullptr, *dc = nullptr, *dq = nullptr;
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
  dq = static_cast<decltype(dq)>(
      pool_alloc(p->device, t->K_pad * 4, "plane build inputs"));
  struct Tmp {
    void* a[5];
    ~Tmp() {
      for (void* x : a) pool_free(x);
    }
  } tmp{{dw, dc, dcol, doff, dq}};
  if (nnz) {
    check_cuda(cudaMemcpy(dw, p->h_w.data(), nnz * 4, cudaMemcpyHostToDevice), "upload");
    check_cuda(cudaMemcpy(dc, p->h_corr.data(), nnz * 4, cudaMemcpyHostToDevice), "upload");
    check_cuda(cudaMemcpy(dcol, p->h_cols.data(), nnz * 4, cudaMemcpyHostToDevice), "upload");
  }
  check_cuda(cudaMemcpy(doff, p->h_offs.data(), (p->V + 1) * 8, cudaMemcpyHostToDevice), "upload");
  check_cuda(cudaMemcpy(dq, qhi.data(), t->K_pad * 4, cudaMemcpyHostToDevice), "upload");
  if (p->V) {
    gnm_tc_build_planes<<<uint32_t((p->V + 255) / 256), 256>>>(
        dw, dc, dcol, doff, p->V, dq, t->d_planes_dos, t->d_planes_mis, t->K_pad, t->V_pad);
    check_cuda(cudaGetLastError(), "plane build launch");
  }
  check_cuda(cudaStreamSynchronize(0), "plane build");
  t->map_dos = make_plane_map(t->d_planes_dos, t->V_pad, t->K_pad, kTcPlanes);
  t->map_mis = make_plane_map(t->d_planes_mis, t->V_pad, t->K_pad, kTcPlanes);
}

void tensor_plan_destroy(gnm_plan* p) {
  TensorPlan* t = p->tensor;
  if (!t) return;
  pool_free(t->d_planes_dos);
  pool_free(t->d_planes_mis);
  pool_free(t->d_part_sum);
  pool_free(t->d_part_cnt);
  delete t;
  p->tensor = nullptr;
}

void tensor_reset(gnm_plan* p, cudaStream_t s) {
  TensorPlan* t = p->tensor;
  check_cuda(cudaMemsetAsync(t->d_part_sum, 0, t->K_pad * t->P_pad * 8, s), "reset partials");
  check_cuda(cudaMemsetAsync(t->d_part_cnt, 0, t->K_pad * t->P_pad * 4, s), "reset partials");
}

void tensor_accumulate(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch, uint64_t v0,
                       uint64_t nv, cudaStream_t s) {
  TensorPlan* t = p->tensor;
  if (v0 % kTcK != 0)
    fail(GNM_ERR_INVALID, "tensor engine blocks must start at a multiple of 64 variants");
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
      p->d_out_to_fam, p->P, p->K, d_sums, d_counts);
  check_cuda(cudaGetLastError(), "tensor finalize launch");
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
  const dim3 grid(uint32_t((p->V + kBwThreads - 1) / kBwThreads), uint32_t((p->K + 15) / 16));
  gnm_backward_kernel<<<grid, kBwThreads, 0, s>>>(d_rows, pitch, p->bpv, p->V, gsf, p->fam,
                                                  uint32_t(p->K), d_grad_w, d_grad_corr);
  check_cuda(cudaGetLastError(), "backward launch");
  p->launches += 1;
}

}  // namespace gnm
