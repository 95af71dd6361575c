// gnm_plan.h — the plan object behind the C ABI (host side).
#pragma once
#include <chrono>
#include <exception>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gnomon_gpu.h"
#include "gnm_internal.h"

namespace gnm {

struct TensorPlan;  // split-BF16 engine state (gnm_tensor.cu)

// Thrown inside the library only; converted to a gnm_status at the ABI edge.
struct Failure {
  gnm_status status;
  std::string message;
};

[[noreturn]] void fail(gnm_status s, const std::string& msg);
void check_cuda(cudaError_t e, const char* what);

// Scoped current-device switch.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev);
  ~DeviceGuard();
};

// Runs f at the C-ABI edge: a Failure becomes its status and message, any
// other exception GNM_ERR_COMPUTE; nothing is thrown across the ABI.
inline void set_error(gnm_error* err, const std::string& m) {
  if (!err) return;
  std::snprintf(err->message, sizeof(err->message), "%s", m.c_str());
}

template <class F>
gnm_status guarded(gnm_error* err, F&& f) {
  try {
    f();
    if (err) err->message[0] = '\0';
    return GNM_OK;
  } catch (const Failure& e) {
    set_error(err, e.message);
    return e.status;
  } catch (const std::exception& e) {
    set_error(err, std::string("internal error: ") + e.what());
    return GNM_ERR_COMPUTE;
  } catch (...) {
    set_error(err, "internal error");
    return GNM_ERR_COMPUTE;
  }
}

// A CUDA device with this ordinal exists (clears the error of a failed query).
inline bool device_available(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return false;
  }
  return device < n;
}

// The device a call runs on: an ordinal (>= 0, must exist), -1 = the current
// device, GNM_DEVICE_BEST = the visible sm_100 device with the most free
// memory, ties broken by SM count (the reference's ranking of candidate
// devices, score/cuda_backend.rs:894-991, whose tile sizes grow with free
// memory).  Raises GNM_DECLINED when no such device exists.
int resolve_device(int device);

// Device buffers of plans come from the library's per-device memory pool.
void* pool_alloc(int device, uint64_t bytes, const char* what);
void pool_free(void* ptr);

// Optional phase trace of plan creation and gnm_score_run / gnm_score_run_ex
// on stderr (environment variable GNM_TRACE set and not "0"): host wall time
// of each phase, after synchronising the streams it waited on.
struct PhaseTrace {
  bool on = false;
  std::chrono::steady_clock::time_point t0, last;
  PhaseTrace() {
    const char* e = std::getenv("GNM_TRACE");
    on = e && *e && std::strcmp(e, "0") != 0;
    t0 = last = std::chrono::steady_clock::now();
  }
  void mark(const char* phase) {
    if (!on) return;
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "gnm_trace %-22s %9.3f ms  (total %9.3f ms)\n", phase,
                 std::chrono::duration<double, std::milli>(now - last).count(),
                 std::chrono::duration<double, std::milli>(now - t0).count());
    last = now;
  }
};

// Synchronous host -> device copy on stream s; large pageable sources go
// through a pinned ring with threaded host copies.
void copy_to_device(void* dst, const void* src, uint64_t bytes, cudaStream_t s);

// PLINK 2 .pgen decoding (gnm_pgen.cu), for the end-to-end .pgen run.
// alt_counts: ALT alleles per variant (null: every variant read as biallelic);
// alt_ords: the ALT (1-based) each listed row holds (null: ALT 1).
gnm_pgen* pgen_open_impl(const uint8_t* pgen, uint64_t pgen_len, int device,
                         const uint32_t* alt_counts = nullptr);
void pgen_decode_list_impl(gnm_pgen* pg, const uint64_t* list, uint64_t count, uint8_t* d_rows,
                           uint64_t pitch, cudaStream_t s, const uint32_t* alt_ords = nullptr);
void pgen_check_impl(gnm_pgen* pg, cudaStream_t s);
uint64_t pgen_samples(const gnm_pgen* pg);
uint64_t pgen_variants(const gnm_pgen* pg);

CUtensorMap make_row_map(const uint8_t* d_rows, uint64_t bytes_per_row, uint64_t num_rows,
                         uint64_t pitch, uint32_t box_x, uint32_t box_y);

}  // namespace gnm

struct gnm_plan {
  int device = 0;
  gnm_engine engine = GNM_ENGINE_PLAIN;
  uint64_t P = 0, fam = 0, bpv = 0, K = 0, V = 0;
  int num_sms = 0;

  // plain engine
  uint32_t kernel = 1024;      // plain accumulate kernel (gnm_internal.h kPlain*)
  double split_mult = 1.0;     // CTA slots per SM multiplier the split counts are sized for
  uint32_t tiles = 0;          // people tiles of the kernel's width
  uint32_t splits = 0;         // variant splits of each full tile
  uint32_t last_splits = 0;    // variant splits of the last (partly populated) tile
  uint32_t slots = 0;          // partial slots in use: max(splits, last_splits)
  uint32_t valid_slots = 0;    // slots written since the last reset (finalize sums these)
  uint32_t splits_alloc = 0;   // partial slots allocated per score (autotune range)
  uint32_t raster = 0;         // tensor engine CTA order: 0 people-tile fastest, 1 score-tile
  uint64_t part_stride = 0;    // people per partial slot (bpv rounded up to 2048 bytes, x4)
  struct Tuning {              // one autotuner candidate and its best accumulate time
    uint32_t kernel;
    double mult;
    uint32_t splits, last_splits;
    float ms;
  };
  std::vector<Tuning> tuning_log;
  uint64_t rec_stride = 0;     // records per score (V + pad)
  float4* d_records = nullptr; // [K][rec_stride]
  uint8_t* d_tables = nullptr;  // stage tables of every score, [K][tab_stages][kPlainTableBytes]
  uint64_t tab_stages = 0;      // ceil(V / kPlainRows) when d_tables is cached, else 0
  uint8_t* d_tab_scratch = nullptr;  // one score's tables for blocks the cache cannot serve
  uint64_t tab_scratch_stages = 0;
  double* d_part_sum = nullptr;
  uint32_t* d_part_cnt = nullptr;

  // shared
  double* d_baseline = nullptr;    // [K]
  double* d_zero_base = nullptr;   // [K] zeros (resume runs)
  uint32_t* d_out_to_fam = nullptr;
  uint32_t* d_err = nullptr;
  float* d_grad_fam = nullptr;     // backward: dS in .bed person order (keep subsets)
  uint8_t* d_bw = nullptr;         // backward: dS limb rows, FP32 dS, per-score maxima
  uint64_t bw_bytes = 0;
  uint32_t bw_limb_bits = 8;       // backward dS limbs: 8 (gnm_t8_backward) or 16 (BF16)
  std::vector<double> h_baseline;
  uint64_t device_bytes = 0;
  uint64_t launches = 0;


  gnm::TensorPlan* tensor = nullptr;
};
