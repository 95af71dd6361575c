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
constexpr uint32_t kPlainThreads = 256;      // one 32-bit word column (16 people) each
constexpr uint32_t kPlainTileBytes = 1024;   // bytes of a row per CTA (4096 people)
constexpr uint32_t kPlainBoxBytes = 256;     // TMA box inner extent (max 256 elements)
constexpr uint32_t kPlainRows = 48;          // variant rows per pipeline stage (16 groups of 3)
constexpr uint32_t kRecordPad = 64;          // zero records past the last variant

struct PlainArgs {
  const float4* records;   // [V + pad] {-corr, w', 2w', member mask bits} of one score
  uint64_t record_row0;    // absolute variant index of block row 0
  uint64_t num_rows;       // rows in this block
  uint64_t bytes_per_row;  // meaningful bytes of a row (ceil(people / 4))
  uint32_t stages_per_split;
  double* part_sum;        // [splits][part_stride] partials of this score
  uint32_t* part_cnt;
  uint64_t part_stride;
  uint32_t* err;
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

cudaError_t launch_plain_accumulate(const CUtensorMap& map, const PlainArgs& a, uint32_t tiles,
                                    uint32_t splits, cudaStream_t s);
uint32_t plain_smem_bytes();
cudaError_t launch_finalize(const FinalizeArgs& a, cudaStream_t s);
cudaError_t launch_decode(const uint8_t* rows, uint64_t pitch, uint64_t nv, uint64_t np,
                          int8_t* out, uint64_t out_pitch, cudaStream_t s);
cudaError_t launch_synth_fill(uint8_t* rows, uint64_t pitch, uint64_t v0, uint64_t nv,
                              uint64_t np, const uint32_t* thr, uint64_t seed, cudaStream_t s);

}  // namespace gnm
