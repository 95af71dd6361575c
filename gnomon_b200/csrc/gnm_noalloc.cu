// gnm_noalloc.cu — gnm_score_noalloc: the plain scoring kernel with its scratch
// in a file-scope device array, for callers that cannot allocate device memory
// (see include/gnomon_gpu.h).  No cudaMalloc / cudaFree / allocating library
// call is made on this path.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "gnm_plan.h"

namespace gnm {

// Scratch layout (bytes, 256-aligned): a stage-table region (the 3-variant
// lookup tables of one chunk of kNaChunkRows rows; the variants are scored
// chunk by chunk), FP64 partial sums and u32 partial counts for up to
// kNaSplits splits of GNM_NOALLOC_MAX_PEOPLE people, then the baseline (FP64)
// and the watchdog word.
constexpr uint32_t kNaSplits = 16;
constexpr uint64_t kNaTabOff = 0;
constexpr uint64_t kNaTabBytes = (uint64_t(GNM_NOALLOC_MAX_VARIANTS) + kRecordPad) * 16;
// stage tables are built and consumed one chunk of rows at a time
constexpr uint64_t kNaChunkStages = kNaTabBytes / kPlainTableBytes;
constexpr uint64_t kNaChunkRows = kNaChunkStages * kPlainRows;
constexpr uint64_t kNaSumOff = kNaTabOff + kNaTabBytes;
constexpr uint64_t kNaSumBytes = uint64_t(kNaSplits) * GNM_NOALLOC_MAX_PEOPLE * 8;
constexpr uint64_t kNaCntOff = kNaSumOff + kNaSumBytes;
constexpr uint64_t kNaCntBytes = uint64_t(kNaSplits) * GNM_NOALLOC_MAX_PEOPLE * 4;
constexpr uint64_t kNaMiscOff = kNaCntOff + kNaCntBytes;
constexpr uint64_t kNaBytes = kNaMiscOff + 256;
static_assert(kNaBytes == GNM_NOALLOC_SCRATCH_BYTES, "scratch size in the header is stale");
static_assert(GNM_NOALLOC_MAX_PEOPLE % (kPlainTileBytes * 4) == 0, "whole people tiles");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

// Device address of g_noalloc_scratch on the current device.  In host code
// the symbol itself is only a host-side stand-in, never a device address.
static unsigned char* scratch_on_current_device() {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static void* addr[kMaxDevices] = {};
  int dev = -1;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) fail(GNM_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      fail(GNM_ERR_COMPUTE, std::string("cudaGetSymbolAddress(scratch) failed: ") +
                                cudaGetErrorString(e));
    }
    addr[dev] = p;
  }
  return static_cast<unsigned char*>(addr[dev]);
}

// Writes the score's baseline into the scratch and clears the watchdog word.
__global__ void gnm_noalloc_init(double baseline, double* base_out, uint32_t* err) {
  *base_out = baseline;
  *err = 0u;
}

static void score_noalloc(const uint8_t* d_rows, uint64_t pitch, uint64_t V, uint64_t P,
                          const float* d_w, const float* d_corr, const uint8_t* d_member,
                          double baseline, double* d_sums, uint32_t* d_counts, cudaStream_t s) {
  if (V > GNM_NOALLOC_MAX_VARIANTS)
    fail(GNM_ERR_INVALID, "gnm_score_noalloc: num_variants exceeds GNM_NOALLOC_MAX_VARIANTS (" +
                              std::to_string(GNM_NOALLOC_MAX_VARIANTS) + ")");
  if (P > GNM_NOALLOC_MAX_PEOPLE)
    fail(GNM_ERR_INVALID, "gnm_score_noalloc: num_people exceeds GNM_NOALLOC_MAX_PEOPLE (" +
                              std::to_string(GNM_NOALLOC_MAX_PEOPLE) + ")");
  if (V == 0 || P == 0) fail(GNM_ERR_INVALID, "gnm_score_noalloc: empty input");
  if (!d_rows || !d_w || !d_corr || !d_sums || !d_counts)
    fail(GNM_ERR_INVALID, "gnm_score_noalloc: NULL buffer");
  const uint64_t bpv = (P + 3) / 4;
  // the row-map rules, checked before anything is queued on the stream
  if (reinterpret_cast<uintptr_t>(d_rows) % 16 != 0)
    fail(GNM_ERR_INVALID, "gnm_score_noalloc: packed rows must start on a 16-byte boundary");
  if (pitch % 16 != 0)
    fail(GNM_ERR_INVALID, "gnm_score_noalloc: row pitch must be a multiple of 16 bytes");
  if (pitch < bpv) fail(GNM_ERR_INVALID, "gnm_score_noalloc: row pitch is smaller than ceil(people / 4)");
  unsigned char* sc = scratch_on_current_device();
  uint8_t* tables = reinterpret_cast<uint8_t*>(sc + kNaTabOff);
  double* part_sum = reinterpret_cast<double*>(sc + kNaSumOff);
  uint32_t* part_cnt = reinterpret_cast<uint32_t*>(sc + kNaCntOff);
  double* base = reinterpret_cast<double*>(sc + kNaMiscOff);
  uint32_t* err = reinterpret_cast<uint32_t*>(sc + kNaMiscOff + 16);

  // geometry of the plain kernel, splits capped by the scratch
  int dev = 0, sms = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
  const uint32_t tiles = uint32_t((bpv + kPlainTileBytes - 1) / kPlainTileBytes);
  const uint64_t stride = uint64_t(tiles) * kPlainTileBytes * 4;
  // splits per chunk of rows; every chunk adds into the same partial slots
  const uint64_t chunk_rows = V < kNaChunkRows ? V : kNaChunkRows;
  const uint64_t stages = (chunk_rows + kPlainRows - 1) / kPlainRows;
  uint64_t splits = uint64_t(2 * sms) / tiles;
  splits = splits < 1 ? 1 : splits;
  splits = splits > kNaSplits ? kNaSplits : splits;
  splits = splits > stages ? stages : splits;
  const uint32_t sps = uint32_t((stages + splits - 1) / splits);
  const uint32_t grid_splits = uint32_t((stages + sps - 1) / sps);

  // the array keeps the previous call's contents: clear the partials
  check_cuda(cudaMemsetAsync(part_sum, 0, grid_splits * stride * 8, s), "clear scratch");
  check_cuda(cudaMemsetAsync(part_cnt, 0, grid_splits * stride * 4, s), "clear scratch");
  gnm_noalloc_init<<<1, 1, 0, s>>>(baseline, base, err);
  check_cuda(cudaGetLastError(), "init launch");

  for (uint64_t c0 = 0; c0 < V; c0 += kNaChunkRows) {
    const uint64_t nv = V - c0 < kNaChunkRows ? V - c0 : kNaChunkRows;
    TableArgs t{};
    t.w = d_w;
    t.corr = d_corr;
    t.member = d_member;
    t.row0 = c0;
    t.num_rows = nv;
    t.tables = tables;
    check_cuda(launch_plain_tables(t, s), "stage table launch");
    const CUtensorMap map = make_row_map(d_rows + c0 * pitch, bpv, nv, pitch, kPlainBoxBytes,
                                         kPlainRows);
    const uint64_t cst = (nv + kPlainRows - 1) / kPlainRows;
    PlainArgs a;
    a.tables = tables;
    a.num_rows = nv;
    a.bytes_per_row = bpv;
    a.tiles = tiles;
    a.splits = uint32_t((cst + sps - 1) / sps);   // the same split count for every tile
    a.stages_per_split = sps;
    a.last_stages_per_split = sps;
    a.part_sum = part_sum;
    a.part_cnt = part_cnt;
    a.part_stride = stride;
    a.err = err;
    check_cuda(launch_plain_accumulate(map, a, kPlain1024, s), "plain accumulate launch");
  }
  FinalizeArgs f;
  f.part_sum = part_sum;
  f.part_cnt = part_cnt;
  f.part_stride = stride;
  f.num_splits = grid_splits;
  f.baseline = base;
  f.out_to_fam = nullptr;
  f.num_people = P;
  f.K = 1;
  f.k = 0;
  f.sums = d_sums;
  f.counts = d_counts;
  check_cuda(launch_finalize(f, s), "finalize launch");

  uint32_t host_err = 0;
  check_cuda(cudaMemcpyAsync(&host_err, err, 4, cudaMemcpyDeviceToHost, s), "read watchdog");
  check_cuda(cudaStreamSynchronize(s), "stream synchronize");
  if (host_err & kErrTmaTimeout) fail(GNM_ERR_TIMEOUT, "device watchdog: a TMA wait expired");
  if (host_err) fail(GNM_ERR_COMPUTE, "device reported an error");
}

}  // namespace gnm

extern "C" gnm_status gnm_score_noalloc(const uint8_t* d_rows, uint64_t pitch,
                                        uint64_t num_variants, uint64_t num_people,
                                        const float* d_dosage_weight,
                                        const float* d_missing_correction,
                                        const uint8_t* d_member, double baseline,
                                        double* d_sums_out, uint32_t* d_missing_out,
                                        void* stream, gnm_error* err) {
  try {
    gnm::score_noalloc(d_rows, pitch, num_variants, num_people, d_dosage_weight,
                       d_missing_correction, d_member, baseline, d_sums_out, d_missing_out,
                       static_cast<cudaStream_t>(stream));
    if (err) err->message[0] = '\0';
    return GNM_OK;
  } catch (const gnm::Failure& e) {
    if (err) snprintf(err->message, sizeof(err->message), "%s", e.message.c_str());
    return e.status;
  } catch (...) {
    if (err) snprintf(err->message, sizeof(err->message), "internal error");
    return GNM_ERR_COMPUTE;
  }
}
