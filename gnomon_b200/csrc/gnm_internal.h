// gnm_internal.h — shapes, kernel argument blocks and launcher declarations
// shared between the kernels and the C-ABI host layer.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>
#include <vector_types.h>

namespace gnm {

// Error bits written to the plan's device error word.
enum : uint32_t {
  kErrTmaTimeout = 1u,     // a TMA / bulk-copy mbarrier wait expired
  kErrMmaTimeout = 2u,     // a tcgen05 commit barrier wait expired
  kErrShape = 4u           // a kernel saw an impossible launch shape
};

// ---- plain engine shape ----------------------------------------------------
// A plain CTA scores a tile of 512, 1024 or 2048 bytes of every row (2048,
// 4096 or 8192 people) with one thread per 32-bit word column (16 people):
// 128 or 256 threads and 4 or 2 CTAs per SM, or 512 threads plus a producer
// warp and one CTA per SM.
constexpr uint32_t kPlainTileBytes = 1024;
constexpr uint32_t kPlainWideTileBytes = 2048;   // also the partial-slot padding
constexpr uint32_t kPlainBoxBytes = 256;     // TMA box inner extent (max 256 elements)
constexpr uint32_t kPlainRows = 30;          // variant rows per pipeline stage (10 groups of 3)
constexpr uint32_t kPlainGroups = kPlainRows / 3;
// One stage table: 10 group tables of 64 FP32 entries (256 B each) + the
// stage's membership word, padded to a multiple of 16 bytes (bulk copies).
constexpr uint32_t kPlainTableBytes = kPlainGroups * 256 + 16;   // 2576
constexpr uint32_t kRecordPad = 64;          // zero records past the last variant
constexpr uint64_t kTableCacheBytes = uint64_t(4) << 30;  // per-plan stage-table cache budget

// Source of the per-row terms {-corr, w', 2w'} and membership for the stage
// table builder: the plan's records, or raw per-row arrays (no-alloc path).
struct TableArgs {
  const float4* records;   // {-corr, w', 2w', member mask bits} per row, or null
  const float* w;          // raw arrays (used when records is null)
  const float* corr;
  const uint8_t* member;   // null = every row is a member
  uint64_t row0;           // index of table row 0 in the source arrays
  uint64_t num_rows;       // rows covered; tables for ceil(num_rows / kPlainRows) stages
  uint8_t* tables;         // out: [stages][kPlainTableBytes]
};

struct PlainArgs {
  const uint8_t* tables;   // [stages of this block][kPlainTableBytes], stage 0 = block row 0
  uint64_t num_rows;       // rows in this block
  uint64_t bytes_per_row;  // meaningful bytes of a row (ceil(people / 4))
  uint32_t tiles;          // people tiles (the last may be partly populated)
  uint32_t splits;         // variant splits of each full tile (CTAs per full tile)
  uint32_t stages_per_split;        // stages per split of a full tile
  uint32_t last_stages_per_split;   // stages per split of the last tile
  double* part_sum;        // [splits][part_stride] partials of this score
  uint32_t* part_cnt;
  uint64_t part_stride;
  uint32_t* err;
  uint32_t store = 0;      // 1: write the partials (first launch since a reset); 0: add to them
};

struct FinalizeArgs {
  const double* part_sum;
  const uint32_t* part_cnt;
  uint64_t part_stride;
  uint32_t num_splits;
  const double* baseline;   // [K]
  const uint32_t* out_to_fam;
  uint64_t num_people;
  uint64_t K, k;
  double* sums;             // [P][K]
  uint32_t* counts;
};

// Raises `kernel`'s dynamic shared-memory limit to `bytes` on the current
// device, once per (kernel, device): the attribute belongs to one device's
// context, so every GPU a process uses needs its own call (thread-safe).
cudaError_t raise_smem_limit(const void* kernel, int bytes);

cudaError_t launch_plain_tables(const TableArgs& a, cudaStream_t s);
// Plain accumulate kernels: the tile width in bytes, plus 1 for the variant
// with a producer warp (its scoring warps only arrive on a release barrier).
enum : uint32_t {
  kPlain512 = 512,        // 4 warps, 4 CTAs per SM
  kPlain512Ws = 513,      // 4 warps + producer warp, 4 CTAs per SM
  kPlain1024 = 1024,      // 8 warps, 2 CTAs per SM
  kPlain1024Ws = 1025,    // 8 warps + producer warp, 2 CTAs per SM
  kPlain2048Ws = 2049     // 16 warps + producer warp, 1 CTA per SM
};
constexpr uint32_t kPlainKernels[] = {kPlain1024, kPlain512, kPlain512Ws, kPlain1024Ws,
                                      kPlain2048Ws};
constexpr uint32_t kPlainDefaultKernel = kPlain2048Ws;   // fastest on the bandwidth workload
inline uint32_t plain_tile_bytes(uint32_t kernel) { return kernel & ~1u; }
inline uint32_t plain_ctas_per_sm(uint32_t kernel) {
  return plain_tile_bytes(kernel) >= 2048 ? 1u : 2048u / plain_tile_bytes(kernel);
}

// Launches (tiles - 1) * splits + ceil(stages / last_stages_per_split) CTAs of
// the given plain kernel.
cudaError_t launch_plain_accumulate(const CUtensorMap& map, const PlainArgs& a, uint32_t kernel,
                                    cudaStream_t s);
uint32_t plain_grid(const PlainArgs& a);
cudaError_t launch_finalize(const FinalizeArgs& a, cudaStream_t s);
cudaError_t launch_repitch(const uint8_t* src, uint64_t bpv, uint64_t nrows, uint8_t* dst,
                           uint64_t pitch, cudaStream_t s);
cudaError_t launch_watchdog_probe(uint64_t limit_ns, uint32_t* err, uint64_t* waited_ns,
                                  cudaStream_t s);
cudaError_t launch_decode(const uint8_t* rows, uint64_t pitch, uint64_t nv, uint64_t np,
                          int8_t* out, uint64_t out_pitch, cudaStream_t s);
cudaError_t launch_synth_fill(uint8_t* rows, uint64_t pitch, uint64_t v0, uint64_t nv,
                              uint64_t i0, uint64_t np, const uint32_t* thr, uint64_t seed,
                              cudaStream_t s);

}  // namespace gnm
