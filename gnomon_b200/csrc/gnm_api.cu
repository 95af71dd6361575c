// gnm_api.cu — C ABI (include/gnomon_gpu.h) over the sm_100a kernels.
//
// The host side of try_run_cuda (score/cuda_backend.rs:604-1535) rebuilt for
// B200: weights are compiled once per plan into per-variant device records,
// packed rows are streamed from the caller's .bed bytes into HBM (pinned
// double buffer, copy stream overlapped with the compute stream), kernels
// accumulate FP64 partials on the device, and one finalize pass adds the
// baseline and gathers output rows.  No cuBLAS, no NVRTC, no host-side
// per-tile accumulation.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <memory>
#include <chrono>
#include <cstdlib>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <exception>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "gnm_plan.h"
#include "gnm_tensor.h"

// A projection in progress (gnm_project_*): its scores so far.
struct gnm_projector {
  int device = 0;
  uint64_t n = 0, K = 0;
  std::vector<double> acc;   // [n][K] row-major, every block so far
};

namespace gnm {

void fail(gnm_status s, const std::string& msg) { throw Failure{s, msg}; }

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();  // clear sticky-free errors so the context stays usable
    fail(GNM_ERR_COMPUTE, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

DeviceGuard::DeviceGuard(int dev) {
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (dev >= 0 && dev != prev) check_cuda(cudaSetDevice(dev), "cudaSetDevice");
}
DeviceGuard::~DeviceGuard() {
  int cur = -1;
  if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
}

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  if (!fn) fail(GNM_ERR_COMPUTE, "cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

int resolve_device(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    fail(GNM_DECLINED, "no CUDA device available");
  }
  if (device >= 0) {
    if (device >= n) fail(GNM_DECLINED, "no CUDA device with ordinal " + std::to_string(device));
    return device;
  }
  if (device == -1) {
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    return device;
  }
  if (device != GNM_DEVICE_BEST) fail(GNM_ERR_INVALID, "device must be >= 0, -1 or GNM_DEVICE_BEST");
  int prev = -1;
  check_cuda(cudaGetDevice(&prev), "cudaGetDevice");
  int best = -1;
  size_t best_free = 0;
  int best_sms = 0;
  std::string rejected;
  for (int d = 0; d < n; ++d) {
    cudaDeviceProp pr{};
    if (cudaGetDeviceProperties(&pr, d) != cudaSuccess) {
      cudaGetLastError();
      rejected += " " + std::to_string(d) + ": properties query failed;";
      continue;
    }
    if (pr.major != 10 || pr.minor != 0) {   // the kernels are built for sm_100a only
      rejected += " " + std::to_string(d) + ": compute capability " + std::to_string(pr.major) +
                  "." + std::to_string(pr.minor) + ";";
      continue;
    }
    size_t free_b = 0, total_b = 0;
    if (cudaSetDevice(d) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      rejected += " " + std::to_string(d) + ": memory query failed;";
      continue;
    }
    if (best < 0 || free_b > best_free ||
        (free_b == best_free && pr.multiProcessorCount > best_sms)) {
      best = d;
      best_free = free_b;
      best_sms = pr.multiProcessorCount;
    }
  }
  cudaSetDevice(prev);
  if (best < 0) fail(GNM_DECLINED, "no visible device can run this library:" + rejected);
  return best;
}

cudaError_t raise_smem_limit(const void* kernel, int bytes) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static std::vector<std::pair<const void*, int>> done;   // (kernel, device) pairs set
  std::lock_guard<std::mutex> lock(mu);
  for (const auto& d : done)
    if (d.first == kernel && d.second == dev) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.emplace_back(kernel, dev);
  return e;
}

CUtensorMap make_row_map(const uint8_t* d_rows, uint64_t bytes_per_row, uint64_t num_rows,
                         uint64_t pitch, uint32_t box_x, uint32_t box_y) {
  if (reinterpret_cast<uintptr_t>(d_rows) % 16 != 0)
    fail(GNM_ERR_INVALID, "packed rows must start on a 16-byte boundary");
  if (pitch % 16 != 0) fail(GNM_ERR_INVALID, "row pitch must be a multiple of 16 bytes");
  if (bytes_per_row > pitch) fail(GNM_ERR_INVALID, "row pitch is smaller than bytes per row");
  CUtensorMap map;
  cuuint64_t dims[2] = {bytes_per_row, num_rows};
  cuuint64_t strides[1] = {pitch};
  cuuint32_t box[2] = {box_x, box_y};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(d_rows),
                           dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(GNM_ERR_COMPUTE, "cuTensorMapEncodeTiled failed for the row map");
  return map;
}

// Per-device memory pool for every device buffer of the library (plans and
// gnm_score_run's row blocks, staging and outputs).  Freed buffers stay
// reserved in the pool, so the next plan or run on the device allocates
// without mapping memory again (mapping and unmapping a 12.5 GB row block
// costs tens of milliseconds); gnm_release_cached_memory returns the reserve
// to the device.
static cudaMemPool_t run_pool(int dev) {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static cudaMemPool_t pools[kMaxDevices] = {};
  if (dev < 0 || dev >= kMaxDevices) fail(GNM_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    check_cuda(cudaMemPoolCreate(&pools[dev], &props), "cudaMemPoolCreate");
    uint64_t keep = UINT64_MAX;
    check_cuda(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep),
               "cudaMemPoolSetAttribute");
  }
  return pools[dev];
}

// Plan buffers: allocated on the default stream and made visible to every
// stream at once; freed by gnm_plan_destroy after a device synchronize.
void* pool_alloc(int dev, uint64_t bytes, const char* what) {
  void* ptr = nullptr;
  check_cuda(cudaMallocFromPoolAsync(&ptr, std::max<uint64_t>(1, bytes), run_pool(dev), 0), what);
  check_cuda(cudaStreamSynchronize(0), what);
  return ptr;
}

void pool_free(void* ptr) {
  if (ptr) cudaFreeAsync(ptr, 0);
}

template <class T>
static T* dalloc(gnm_plan* p, uint64_t n, const char* what) {
  const uint64_t bytes = std::max<uint64_t>(1, n * sizeof(T));
  void* ptr = pool_alloc(p->device, bytes, what);
  p->device_bytes += bytes;
  return static_cast<T*>(ptr);
}

// ---- validation (prepare.rs:760-790 invariants) ----------------------------
// Runs f(begin, end, chunk) over [0, n) on up to 16 host threads (chunks of at
// least `min_chunk`); f must not throw.
template <class F>
static void parallel_chunks(uint64_t n, uint64_t min_chunk, F f) {
  const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const uint64_t nt =
      std::max<uint64_t>(1, std::min<uint64_t>(hw, n / std::max<uint64_t>(1, min_chunk)));
  if (nt == 1) {
    f(uint64_t(0), n, uint64_t(0));
    return;
  }
  std::vector<std::thread> th;
  for (uint64_t i = 0; i < nt; ++i) th.emplace_back(f, n * i / nt, n * (i + 1) / nt, i);
  for (auto& x : th) x.join();
}

// First failure over parallel chunks (lowest index wins, as a serial scan).
struct ChunkErrors {
  std::vector<uint64_t> at;
  std::vector<const char*> what;
  ChunkErrors() : at(16, UINT64_MAX), what(16, nullptr) {}
  void set(uint64_t chunk, uint64_t index, const char* msg) {
    if (index < at[chunk]) {
      at[chunk] = index;
      what[chunk] = msg;
    }
  }
  void raise() const {
    uint64_t best = UINT64_MAX;
    const char* msg = nullptr;
    for (size_t i = 0; i < at.size(); ++i)
      if (at[i] < best) {
        best = at[i];
        msg = what[i];
      }
    if (msg) fail(GNM_ERR_INVALID, msg);
  }
};

static void validate_prep(const gnm_prep_view* p) {
  if (!p) fail(GNM_ERR_INVALID, "prep is NULL");
  if (p->num_scores == 0) fail(GNM_ERR_INVALID, "num_scores must be > 0");
  if (p->bytes_per_variant != (p->total_people_in_fam + 3) / 4)
    fail(GNM_ERR_INVALID, "bytes_per_variant != ceil(total_people_in_fam / 4)");
  if (p->total_people_in_fam > (uint64_t(1) << 31))
    fail(GNM_ERR_INVALID, "more than 2^31 people per row is not supported");
  if (p->num_variants > 0 && (!p->sparse_row_offsets))
    fail(GNM_ERR_INVALID, "sparse_row_offsets is NULL");
  if (p->num_people > 0 && !p->output_idx_to_fam_idx && p->num_people > p->total_people_in_fam)
    fail(GNM_ERR_INVALID, "num_people exceeds total_people_in_fam with identity mapping");
  const uint64_t* offs = p->sparse_row_offsets;
  const uint64_t V = p->num_variants;
  if (V > 0) {
    if (offs[0] != 0) fail(GNM_ERR_INVALID, "sparse_row_offsets[0] must be 0");
    ChunkErrors mono;
    parallel_chunks(V, 1 << 16, [&](uint64_t b, uint64_t e, uint64_t c) {
      for (uint64_t v = b; v < e; ++v)
        if (offs[v + 1] < offs[v]) {
          mono.set(c, v, "sparse_row_offsets not monotone");
          return;
        }
    });
    mono.raise();
    const uint64_t nnz = offs[V];
    if (nnz && (!p->sparse_weights || !p->sparse_missing_corrections || !p->sparse_score_columns))
      fail(GNM_ERR_INVALID, "CSR arrays are NULL");
    const uint32_t* cols = p->sparse_score_columns;
    ChunkErrors col;
    parallel_chunks(V, 1 << 14, [&](uint64_t b, uint64_t e, uint64_t c) {
      for (uint64_t v = b; v < e; ++v)
        for (uint64_t x = offs[v]; x < offs[v + 1]; ++x) {
          if (cols[x] >= p->num_scores) {
            col.set(c, v, "CSR score column out of range");
            return;
          }
          if (x > offs[v] && cols[x] <= cols[x - 1]) {
            col.set(c, v, "CSR columns must be strictly ascending within a row");
            return;
          }
        }
    });
    col.raise();
  }
  if (p->output_idx_to_fam_idx) {
    ChunkErrors map;
    parallel_chunks(p->num_people, 1 << 16, [&](uint64_t b, uint64_t e, uint64_t c) {
      for (uint64_t o = b; o < e; ++o)
        if (p->output_idx_to_fam_idx[o] >= p->total_people_in_fam) {
          map.set(c, o, "output_idx_to_fam_idx entry out of range");
          return;
        }
    });
    map.raise();
  }
}



// ---- plan --------------------------------------------------------------------
// Launch shape of the plain kernel: people tiles of the kernel's width and
// `splits` variant splits per tile, with tiles x splits about `mult` x the SMs'
// CTA slots (1, 2 or 4 CTAs per SM).  Every tile, the partly filled last one
// included, gets the same split count: a CTA's time per stage is set by the
// dependency chains of each warp's own column, not by how many of its warps
// hold people, so a last-tile CTA with more stages would finish last (giving
// it a quarter as many splits for a quarter-filled tile doubled the kernel
// time on the bandwidth workload).
static void plain_shape_fixed(gnm_plan* p, uint32_t kernel, uint32_t splits) {
  const uint32_t tile_bytes = plain_tile_bytes(kernel);
  const uint64_t stages = std::max<uint64_t>(1, (p->V + kPlainRows - 1) / kPlainRows);
  const uint64_t tiles = std::max<uint64_t>(1, (p->bpv + tile_bytes - 1) / tile_bytes);
  const uint64_t sp = std::min<uint64_t>(std::max<uint32_t>(1, splits), stages);
  p->kernel = kernel;
  p->tiles = uint32_t(tiles);
  p->splits = uint32_t(sp);
  p->last_splits = uint32_t(sp);
  p->slots = uint32_t(sp);
}

// The autotuner's split multipliers (of the SMs' CTA slots).
constexpr double kPlainSplitMults[] = {0.5, 1.0, 2.0, 3.0, 4.0, 6.0, 8.0};
constexpr double kPlainMaxSplitMult = 8.0;

static void plain_shape(gnm_plan* p, uint32_t kernel, double mult) {
  const uint32_t tile_bytes = plain_tile_bytes(kernel);
  const uint64_t tiles = std::max<uint64_t>(1, (p->bpv + tile_bytes - 1) / tile_bytes);
  const double ctas = double(plain_ctas_per_sm(kernel)) * double(p->num_sms) * mult;
  plain_shape_fixed(p, kernel, uint32_t(std::max(1.0, std::floor(ctas / double(tiles)))));
  p->split_mult = mult;
}

static void plain_geometry(gnm_plan* p) {
  // partial slots are padded to whole tiles of the widest kernel, so every
  // kernel's people index stays inside a slot
  p->part_stride = std::max<uint64_t>(1, (p->bpv + kPlainWideTileBytes - 1) / kPlainWideTileBytes) *
                   kPlainWideTileBytes * 4;
  check_cuda(cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, p->device),
             "cudaDeviceGetAttribute");
  plain_shape(p, kPlainDefaultKernel, 1.0);
  // keep partials of all scores within 8 GiB (many score columns still get a
  // full-occupancy grid); allocate room for the autotuner's largest candidate
  // (eight times the CTA slots, any kernel)
  const uint64_t per_split_bytes = p->K * p->part_stride * 12;
  const uint64_t cap = uint64_t(8) << 30;
  uint64_t alloc = p->slots;
  for (uint32_t kn : kPlainKernels) {
    gnm_plan probe = {};
    probe.V = p->V;
    probe.bpv = p->bpv;
    probe.num_sms = p->num_sms;
    plain_shape(&probe, kn, kPlainMaxSplitMult);
    alloc = std::max<uint64_t>(alloc, probe.slots);
  }
  while (alloc > 1 && alloc * per_split_bytes > cap) --alloc;
  p->splits_alloc = uint32_t(alloc);
  // shrink the default grid until its slots fit the allocation
  double mult = 1.0;
  while (p->slots > p->splits_alloc && mult > 1e-3) {
    mult *= 0.5;
    plain_shape(p, kPlainDefaultKernel, mult);
  }
}

static void upload_plain_records(gnm_plan* p, const std::vector<float4>& rec, PhaseTrace& trace);

static void build_plain_records(gnm_plan* p, const gnm_prep_view* prep, PhaseTrace& trace) {
  p->rec_stride = p->V + kRecordPad;
  std::vector<float4> rec(p->K * p->rec_stride);
  const uint32_t member_bits = 0x55555555u;
  float member_f;
  std::memcpy(&member_f, &member_bits, 4);
  // Host threads over disjoint variant ranges: each clears its variants'
  // records in every score row and writes their cells.
  const uint64_t stride = p->rec_stride, V = p->V, K = p->K;
  auto fill = [&](uint64_t v0, uint64_t v1) {
    for (uint64_t k = 0; k < K; ++k)
      std::fill(rec.begin() + k * stride + v0, rec.begin() + k * stride + v1,
                make_float4(0.f, 0.f, 0.f, 0.f));
    for (uint64_t v = v0; v < std::min(v1, V); ++v)
      for (uint64_t e = prep->sparse_row_offsets[v]; e < prep->sparse_row_offsets[v + 1]; ++e) {
        const uint32_t k = prep->sparse_score_columns[e];
        const float w = prep->sparse_weights[e];
        const float c = prep->sparse_missing_corrections[e];
        rec[k * stride + v] = make_float4(-c, w, 2.0f * w, member_f);
      }
  };
  const uint64_t nthreads = std::min<uint64_t>(
      std::max(1u, std::thread::hardware_concurrency()), std::max<uint64_t>(1, stride / 65536));
  if (nthreads <= 1) {
    fill(0, stride);
  } else {
    std::vector<std::thread> pool;
    const uint64_t per = (stride + nthreads - 1) / nthreads;
    for (uint64_t t = 0; t < nthreads; ++t)
      pool.emplace_back(fill, t * per, std::min(stride, (t + 1) * per));
    for (auto& th : pool) th.join();
  }
  trace.mark("  plan: records (host)");
  upload_plain_records(p, rec, trace);
}

// Upload a plain plan's cell records, allocate its partials and build the
// stage tables while they fit the cache.
static void upload_plain_records(gnm_plan* p, const std::vector<float4>& rec, PhaseTrace& trace) {
  p->d_records = dalloc<float4>(p, rec.size(), "cudaMalloc(records)");
  check_cuda(cudaMemcpy(p->d_records, rec.data(), rec.size() * sizeof(float4),
                        cudaMemcpyHostToDevice),
             "upload records");
  trace.mark("  plan: records upload");
  const uint64_t part = p->K * uint64_t(p->splits_alloc) * p->part_stride;
  p->d_part_sum = dalloc<double>(p, part, "cudaMalloc(partial sums)");
  p->d_part_cnt = dalloc<uint32_t>(p, part, "cudaMalloc(partial counts)");
  trace.mark("  plan: partials");

  // Stage tables (the 3-variant lookup tables) of every score, built once on
  // the device while they fit the cache budget; blocks that start on a
  // kPlainRows-variant boundary read them directly.  Otherwise each accumulate call
  // builds the tables of its block into a one-score scratch.
  const uint64_t stages = (p->V + kPlainRows - 1) / kPlainRows;
  if (p->K * stages * kPlainTableBytes <= kTableCacheBytes) {
    p->tab_stages = stages;
    p->d_tables = dalloc<uint8_t>(p, p->K * stages * kPlainTableBytes, "cudaMalloc(stage tables)");
    for (uint64_t k = 0; k < p->K; ++k) {
      TableArgs t{};
      t.records = p->d_records + k * p->rec_stride;
      t.row0 = 0;
      t.num_rows = p->V;
      t.tables = p->d_tables + k * stages * kPlainTableBytes;
      check_cuda(launch_plain_tables(t, 0), "stage table launch");
    }
  }
}

// Stage tables for score k over block rows [v0, v0 + nv): the cached tables
// when the block starts on a stage boundary, else a fresh build into scratch.
static const uint8_t* plain_tables_for(gnm_plan* p, uint64_t k, uint64_t v0, uint64_t nv,
                                       cudaStream_t s) {
  if (p->d_tables && v0 % kPlainRows == 0)
    return p->d_tables + (k * p->tab_stages + v0 / kPlainRows) * kPlainTableBytes;
  const uint64_t stages = (nv + kPlainRows - 1) / kPlainRows;
  if (stages > p->tab_scratch_stages) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    check_cuda(cudaStreamIsCapturing(s, &cs), "cudaStreamIsCapturing");
    if (cs != cudaStreamCaptureStatusNone)
      fail(GNM_ERR_INVALID, "stage-table scratch must grow during stream capture: run one "
                            "uncaptured pass over the same block first, or start blocks on "
                            "a multiple of " + std::to_string(kPlainRows) + " variants");
    check_cuda(cudaStreamSynchronize(s), "stream synchronize");
    if (p->d_tab_scratch) {
      pool_free(p->d_tab_scratch);
      p->device_bytes -= p->tab_scratch_stages * kPlainTableBytes;
      p->d_tab_scratch = nullptr;
      p->tab_scratch_stages = 0;
    }
    p->d_tab_scratch = dalloc<uint8_t>(p, stages * kPlainTableBytes, "cudaMalloc(table scratch)");
    p->tab_scratch_stages = stages;
  }
  TableArgs t{};
  t.records = p->d_records + k * p->rec_stride;
  t.row0 = v0;
  t.num_rows = nv;
  t.tables = p->d_tab_scratch;
  check_cuda(launch_plain_tables(t, s), "stage table launch");
  ++p->launches;
  return p->d_tab_scratch;
}

static gnm_plan* plan_create_impl(const gnm_prep_view* prep, gnm_engine engine, int device,
                                  bool validated = false) {
  PhaseTrace trace;
  if (!validated) validate_prep(prep);
  trace.mark("  plan: validate");
  device = resolve_device(device);
  DeviceGuard g(device);
  auto* p = new gnm_plan();
  try {
    p->device = device;
    p->P = prep->num_people;
    p->fam = prep->total_people_in_fam;
    p->bpv = prep->bytes_per_variant;
    p->K = prep->num_scores;
    p->V = prep->num_variants;
    if (engine == GNM_ENGINE_AUTO) engine = p->K >= kTensorMinScores ? GNM_ENGINE_TENSOR : GNM_ENGINE_PLAIN;
    p->engine = engine;

    // baseline (prepare.rs:644-646), f64 in CSR order
    p->h_baseline.assign(p->K, 0.0);
    const uint64_t nnz = p->V ? prep->sparse_row_offsets[p->V] : 0;
    if (prep->baseline) {
      std::copy(prep->baseline, prep->baseline + p->K, p->h_baseline.begin());
    } else {
      for (uint64_t e = 0; e < nnz; ++e)
        p->h_baseline[prep->sparse_score_columns[e]] += double(prep->sparse_missing_corrections[e]);
    }
    p->d_baseline = dalloc<double>(p, p->K, "cudaMalloc(baseline)");
    check_cuda(cudaMemcpy(p->d_baseline, p->h_baseline.data(), p->K * sizeof(double),
                          cudaMemcpyHostToDevice),
               "upload baseline");
    p->d_zero_base = dalloc<double>(p, p->K, "cudaMalloc(zero baseline)");
    check_cuda(cudaMemset(p->d_zero_base, 0, p->K * sizeof(double)), "memset");
    if (prep->output_idx_to_fam_idx) {
      p->d_out_to_fam = dalloc<uint32_t>(p, p->P, "cudaMalloc(output map)");
      check_cuda(cudaMemcpy(p->d_out_to_fam, prep->output_idx_to_fam_idx, p->P * 4,
                            cudaMemcpyHostToDevice),
                 "upload output map");
    }
    p->d_err = dalloc<uint32_t>(p, 1, "cudaMalloc(error word)");
    check_cuda(cudaMemset(p->d_err, 0, 4), "memset");

    trace.mark("  plan: baseline, maps");
    if (p->engine == GNM_ENGINE_PLAIN) {
      plain_geometry(p);
      trace.mark("  plan: csr copy, geometry");
      build_plain_records(p, prep, trace);
    } else {
      tensor_plan_create(p, prep, &trace);
    }
    trace.mark("  plan: weights, tables");
    // only the default stream: a concurrent run may be streaming rows
    check_cuda(cudaStreamSynchronize(0), "plan upload");
    trace.mark("  plan: device sync");
  } catch (...) {
    gnm_plan_destroy(p);
    throw;
  }
  return p;
}

static void plan_reset_impl(gnm_plan* p, cudaStream_t s) {
  DeviceGuard g(p->device);
  if (p->engine == GNM_ENGINE_PLAIN) {
    // nothing to clear: the next accumulate writes the slots it covers, and
    // finalize sums only slots written since this reset
    p->valid_slots = 0;
  } else {
    tensor_reset(p, s);
  }
  check_cuda(cudaMemsetAsync(p->d_err, 0, 4, s), "reset error word");
  p->launches = 0;
}

static void accumulate_impl(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch, uint64_t v0,
                            uint64_t nv, cudaStream_t s) {
  if (v0 + nv > p->V) fail(GNM_ERR_INVALID, "variant range exceeds num_variants");
  if (nv == 0) return;
  DeviceGuard g(p->device);
  if (p->engine == GNM_ENGINE_TENSOR) {
    tensor_accumulate(p, d_rows, pitch, v0, nv, s);
    return;
  }
  const CUtensorMap map = make_row_map(d_rows, p->bpv, nv, pitch, kPlainBoxBytes, kPlainRows);
  const uint64_t stages = (nv + kPlainRows - 1) / kPlainRows;
  const uint32_t sps = uint32_t((stages + p->splits - 1) / p->splits);
  const uint32_t lsps = uint32_t((stages + p->last_splits - 1) / p->last_splits);
  // Slots this launch covers (every tile gets the same count).  The first
  // launch after a reset writes them; a later one adds, after clearing any
  // slots past those written so far.
  const uint32_t covered = uint32_t((stages + sps - 1) / sps);
  const bool store = p->valid_slots == 0;
  if (!store && covered > p->valid_slots) {
    const uint64_t row = uint64_t(p->splits_alloc) * p->part_stride;
    const uint64_t off = uint64_t(p->valid_slots) * p->part_stride;
    const uint64_t add = uint64_t(covered - p->valid_slots) * p->part_stride;
    check_cuda(cudaMemset2DAsync(p->d_part_sum + off, row * sizeof(double), 0,
                                 add * sizeof(double), p->K, s),
               "clear partials");
    check_cuda(cudaMemset2DAsync(p->d_part_cnt + off, row * sizeof(uint32_t), 0,
                                 add * sizeof(uint32_t), p->K, s),
               "clear partials");
  }
  p->valid_slots = std::max(p->valid_slots, covered);
  for (uint64_t k = 0; k < p->K; ++k) {
    PlainArgs a;
    a.tables = plain_tables_for(p, k, v0, nv, s);
    a.num_rows = nv;
    a.bytes_per_row = p->bpv;
    a.tiles = p->tiles;
    a.splits = uint32_t((stages + sps - 1) / sps);   // non-empty splits of a full tile
    a.stages_per_split = sps;
    a.last_stages_per_split = lsps;
    a.part_sum = p->d_part_sum + k * uint64_t(p->splits_alloc) * p->part_stride;
    a.part_cnt = p->d_part_cnt + k * uint64_t(p->splits_alloc) * p->part_stride;
    a.part_stride = p->part_stride;
    a.err = p->d_err;
    a.store = store ? 1u : 0u;
    check_cuda(launch_plain_accumulate(map, a, p->kernel, s), "plain accumulate launch");
    ++p->launches;
  }
}

static void finalize_impl(gnm_plan* p, double* d_sums, uint32_t* d_counts, bool add_baseline,
                          cudaStream_t s) {
  DeviceGuard g(p->device);
  if (p->engine == GNM_ENGINE_TENSOR) {
    tensor_finalize(p, d_sums, d_counts, add_baseline, s);
    return;
  }
  for (uint64_t k = 0; k < p->K; ++k) {
    FinalizeArgs a;
    a.part_sum = p->d_part_sum + k * uint64_t(p->splits_alloc) * p->part_stride;
    a.part_cnt = p->d_part_cnt + k * uint64_t(p->splits_alloc) * p->part_stride;
    a.part_stride = p->part_stride;
    a.num_splits = p->valid_slots;
    a.baseline = add_baseline ? p->d_baseline : p->d_zero_base;
    a.out_to_fam = p->d_out_to_fam;
    a.num_people = p->P;
    a.K = p->K;
    a.k = k;
    a.sums = d_sums;
    a.counts = d_counts;
    check_cuda(launch_finalize(a, s), "finalize launch");
    ++p->launches;
  }
}

static void sync_impl(gnm_plan* p, cudaStream_t s) {
  DeviceGuard g(p->device);
  check_cuda(cudaStreamSynchronize(s), "stream synchronize");
  uint32_t e = 0;
  check_cuda(cudaMemcpy(&e, p->d_err, 4, cudaMemcpyDeviceToHost), "read error word");
  if (e & kErrTmaTimeout) fail(GNM_ERR_TIMEOUT, "device watchdog: a TMA wait expired");
  if (e & kErrMmaTimeout) fail(GNM_ERR_TIMEOUT, "device watchdog: a tensor-core wait expired");
  if (e) fail(GNM_ERR_COMPUTE, "device reported an error");
}

// ---- autotuner -----------------------------------------------------------------
// Times candidate launch shapes of the plan's accumulate on the caller's
// resident rows and keeps the fastest.  Plain engine: the five accumulate
// kernels (512-byte, 1 KB and 2 KB people tiles with 4, 8 and 16 scoring warps
// and 4, 2 and 1 CTAs per SM, with or without a producer warp; a narrow
// cohort fills every warp of a narrow tile) times the split count (0.5x to 4x
// the SMs' CTA slots: fewer splits write fewer FP64 partials, more splits
// even out the last wave).  A candidate is timed over accumulate + finalize,
// since the finalize reads every split's partials.  Tensor engine
// with more than 64 scores: the CTA raster order (people tiles fastest: CTAs
// in flight share weight-limb tiles in L2; score tiles fastest: they share
// genotype tiles).
static void autotune_impl(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch, uint64_t nv,
                          cudaStream_t s) {
  DeviceGuard g(p->device);
  if (nv == 0 || nv > p->V) fail(GNM_ERR_INVALID, "autotune: variant_count out of range");
  cudaEvent_t e0, e1;
  check_cuda(cudaEventCreate(&e0), "event");
  check_cuda(cudaEventCreate(&e1), "event");
  struct Ev {
    cudaEvent_t a, b;
    ~Ev() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } ev{e0, e1};
  // scratch outputs for the plain engine's finalize
  struct Scratch {
    void* p = nullptr;
    ~Scratch() { pool_free(p); }
  } out;
  const uint64_t PK = std::max<uint64_t>(1, p->P * p->K);
  if (p->engine == GNM_ENGINE_PLAIN) out.p = pool_alloc(p->device, PK * 12, "autotune outputs");
  auto time_once = [&]() {
    plan_reset_impl(p, s);
    check_cuda(cudaEventRecord(e0, s), "event");
    accumulate_impl(p, d_rows, pitch, 0, nv, s);
    if (out.p)
      finalize_impl(p, static_cast<double*>(out.p),
                    reinterpret_cast<uint32_t*>(static_cast<double*>(out.p) + PK), true, s);
    check_cuda(cudaEventRecord(e1, s), "event");
    sync_impl(p, s);
    float ms = 0.f;
    check_cuda(cudaEventElapsedTime(&ms, e0, e1), "event time");
    return ms;
  };
  auto time_best = [&]() {
    time_once();  // warm-up
    return std::min(time_once(), time_once());
  };
  float best_ms = 1e30f;
  if (p->engine == GNM_ENGINE_PLAIN) {
    uint32_t best_kernel = p->kernel;
    double best_mult = p->split_mult;
    p->tuning_log.clear();
    const char* tr = std::getenv("GNM_TRACE");
    const bool trace = tr && std::strcmp(tr, "0") != 0;
    for (uint32_t kn : kPlainKernels) {
      for (double m : kPlainSplitMults) {
        plain_shape(p, kn, m);
        if (p->slots > p->splits_alloc) continue;
        const float ms = time_best();
        p->tuning_log.push_back({kn, m, p->splits, p->last_splits, ms});
        if (trace)
          std::fprintf(stderr, "[gnm autotune] tile %u B%s, %.1fx slots: %u splits (last tile "
                               "%u), %.4f ms\n", plain_tile_bytes(kn),
                       (kn & 1u) ? " + producer warp" : "", m, p->splits, p->last_splits, ms);
        if (ms < best_ms) {
          best_ms = ms;
          best_kernel = kn;
          best_mult = m;
        }
      }
    }
    plain_shape(p, best_kernel, best_mult);
  } else {
    // shape bit 0: raster order of the wide kernel; bit 1: the narrow kernel;
    // bit 2: 8-bit limbs; bit 3: the 8-bit wide kernel over SM pairs
    std::vector<uint32_t> cand = {0u, 1u, 4u, 5u, 12u, 13u};
    if (tensor_can_narrow(p)) cand.insert(cand.begin(), {2u, 6u});
    uint32_t best = (tensor_is_narrow(p) ? 2u : 0u) | (tensor_is_i8(p) ? 4u : 0u) |
                    (tensor_is_pair(p) ? 8u : 0u) | p->raster;
    const char* tr = std::getenv("GNM_TRACE");
    const bool trace = tr && std::strcmp(tr, "0") != 0;
    for (uint32_t c : cand) {
      tensor_set_narrow(p, (c & 2u) != 0);
      tensor_set_i8(p, (c & 4u) != 0);
      tensor_set_pair(p, (c & 8u) != 0);
      p->raster = c & 1u;
      const float ms = time_best();
      if (trace)
        std::fprintf(stderr, "[gnm autotune] tensor %s kernel%s: %.4f ms\n",
                     (c & 2u) ? ((c & 4u) ? "narrow 8-bit (people as M)" : "narrow (people as M)")
                              : ((c & 8u) ? "wide 8-bit on SM pairs (scores as M)"
                                          : ((c & 4u) ? "wide 8-bit (scores as M)"
                                                      : "wide (scores as M)")),
                     (c & 2u) ? "" : ((c & 1u) ? ", score tiles fastest" : ", people tiles fastest"),
                     ms);
      if (ms < best_ms) {
        best_ms = ms;
        best = c;
      }
    }
    tensor_set_narrow(p, (best & 2u) != 0);
    tensor_set_i8(p, (best & 4u) != 0);
    tensor_set_pair(p, (best & 8u) != 0);
    p->raster = best & 1u;
  }
  plan_reset_impl(p, s);
  sync_impl(p, s);
}

// ---- host streaming run ------------------------------------------------------
struct HostRun {
  uint64_t bpv;
  const gnm_prep_view* prep;
  const gnm_bed_view* bed;
  uint64_t pitch;
  uint64_t zero_before;  // rows below this reconciled index are staged as zeros
};

static bool is_pinned(const void* ptr) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost || at.type == cudaMemoryTypeManaged;
}

// Device -> host copy of a result array.  Large copies into pageable memory go
// through a cached pinned ring (two 64 MB chunks): the DMA fills one chunk at
// the link rate while host threads copy the other out (a direct pageable copy
// of the batched workload's 0.6 GB of results ran at ~4 GB/s).
namespace {
std::mutex g_ring_mu;
uint8_t* g_ring[2] = {nullptr, nullptr};
constexpr uint64_t kRingChunk = uint64_t(64) << 20;
}  // namespace

static void release_result_ring() {
  std::lock_guard<std::mutex> lock(g_ring_mu);
  for (auto*& r : g_ring) {
    if (r) cudaFreeHost(r);
    r = nullptr;
  }
}

static void copy_to_host(void* dst, const void* src, uint64_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  if (bytes < 2 * kRingChunk || is_pinned(dst)) {
    check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "D2H results");
    check_cuda(cudaStreamSynchronize(s), "D2H results");
    return;
  }
  std::lock_guard<std::mutex> lock(g_ring_mu);
  for (auto*& r : g_ring)
    if (!r) check_cuda(cudaHostAlloc(&r, kRingChunk, cudaHostAllocDefault), "cudaHostAlloc");
  cudaEvent_t landed[2] = {nullptr, nullptr};
  struct Ev {
    cudaEvent_t* e;
    ~Ev() {
      for (int i = 0; i < 2; ++i)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } ev{landed};
  for (auto& e : landed) check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  const uint64_t n = (bytes + kRingChunk - 1) / kRingChunk;
  auto issue = [&](uint64_t i) {
    const uint64_t off = i * kRingChunk, len = std::min(kRingChunk, bytes - off);
    check_cuda(cudaMemcpyAsync(g_ring[i % 2], static_cast<const uint8_t*>(src) + off, len,
                               cudaMemcpyDeviceToHost, s),
               "D2H results");
    check_cuda(cudaEventRecord(landed[i % 2], s), "event");
  };
  issue(0);
  for (uint64_t i = 0; i < n; ++i) {
    check_cuda(cudaEventSynchronize(landed[i % 2]), "D2H results");
    if (i + 1 < n) issue(i + 1);   // the other chunk was copied out last iteration
    const uint64_t off = i * kRingChunk, len = std::min(kRingChunk, bytes - off);
    const uint8_t* from = g_ring[i % 2];
    uint8_t* to = static_cast<uint8_t*>(dst) + off;
    parallel_chunks(len, uint64_t(4) << 20, [&](uint64_t b, uint64_t e, uint64_t) {
      std::memcpy(to + b, from + b, e - b);
    });
  }
}

// Host -> device copy of a large pageable array (the tensor plan's CSR)
// through the same pinned ring: host threads fill one chunk while the DMA
// sends the other (a direct pageable copy of the batched workload's 1.6 GB
// CSR ran at ~10 GB/s).
void copy_to_device(void* dst, const void* src, uint64_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  if (bytes < 2 * kRingChunk || is_pinned(src)) {
    check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "H2D upload");
    check_cuda(cudaStreamSynchronize(s), "H2D upload");
    return;
  }
  std::lock_guard<std::mutex> lock(g_ring_mu);
  for (auto*& r : g_ring)
    if (!r) check_cuda(cudaHostAlloc(&r, kRingChunk, cudaHostAllocDefault), "cudaHostAlloc");
  cudaEvent_t sent[2] = {nullptr, nullptr};
  struct Ev {
    cudaEvent_t* e;
    ~Ev() {
      for (int i = 0; i < 2; ++i)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } ev{sent};
  for (auto& e : sent) check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  const uint64_t n = (bytes + kRingChunk - 1) / kRingChunk;
  for (uint64_t i = 0; i < n; ++i) {
    const int slot = int(i % 2);
    if (i >= 2) check_cuda(cudaEventSynchronize(sent[slot]), "H2D upload");
    const uint64_t off = i * kRingChunk, len = std::min(kRingChunk, bytes - off);
    const uint8_t* from = static_cast<const uint8_t*>(src) + off;
    uint8_t* to = g_ring[slot];
    parallel_chunks(len, uint64_t(4) << 20, [&](uint64_t b, uint64_t e, uint64_t) {
      std::memcpy(to + b, from + b, e - b);
    });
    check_cuda(cudaMemcpyAsync(static_cast<uint8_t*>(dst) + off, to, len, cudaMemcpyHostToDevice, s),
               "H2D upload");
    check_cuda(cudaEventRecord(sent[slot], s), "event");
  }
  check_cuda(cudaStreamSynchronize(s), "H2D upload");
}

// Copy rows [v0, v0+n) into dst (pitch layout); zero the padding.
static void gather_rows(const HostRun& r, uint64_t v0, uint64_t n, uint8_t* dst) {
  const uint64_t bpv = r.bpv;
  const uint64_t* map = r.prep->required_bim_indices;
  const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const unsigned nt = unsigned(std::min<uint64_t>(hw, std::max<uint64_t>(1, n / 256)));
  std::atomic<int> bad{0};
  auto work = [&](unsigned t) {
    for (uint64_t i = t; i < n; i += nt) {
      uint8_t* d = dst + i * r.pitch;
      if (v0 + i < r.zero_before) {  // already folded into the resume state
        std::memset(d, 0, r.pitch);
        continue;
      }
      const uint64_t row = map ? map[v0 + i] : v0 + i;
      if (r.bed->data) {
        if ((row + 1) * bpv > r.bed->data_len) {
          bad = 1;
          return;
        }
        std::memcpy(d, r.bed->data + row * bpv, bpv);
      } else if (r.bed->read_at(r.bed->user_ctx, row * bpv, d, bpv) != 0) {
        bad = 2;
        return;
      }
      std::memset(d + bpv, 0, r.pitch - bpv);
    }
  };
  if (nt == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) th.emplace_back(work, t);
    for (auto& x : th) x.join();
  }
  if (bad == 1) fail(GNM_ERR_IO, "truncated .bed: a required row lies past the end of the data");
  if (bad == 2) fail(GNM_ERR_PRODUCER, "read_at callback failed");
}

// Streams and pool buffers of one host run.  Whatever way the run ends, the
// streams are drained before the buffers go back to the pool.
struct RunResources {
  int dev = 0;
  cudaStream_t cs = nullptr, xs = nullptr, rs = nullptr;   // compute, copy, repitch
  std::vector<void*> bufs;
  explicit RunResources(int d) : dev(d) {
    check_cuda(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "stream");
    check_cuda(cudaStreamCreateWithFlags(&xs, cudaStreamNonBlocking), "stream");
    check_cuda(cudaStreamCreateWithFlags(&rs, cudaStreamNonBlocking), "stream");
  }
  template <class T>
  T* alloc(uint64_t bytes, const char* what) {
    void* ptr = nullptr;
    check_cuda(cudaMallocFromPoolAsync(&ptr, std::max<uint64_t>(1, bytes), run_pool(dev), cs),
               what);
    bufs.push_back(ptr);
    return static_cast<T*>(ptr);
  }
  void release() {
    for (cudaStream_t st : {cs, xs, rs})
      if (st) cudaStreamSynchronize(st);
    for (void* b : bufs) cudaFreeAsync(b, cs);
    bufs.clear();
    if (cs) cudaStreamSynchronize(cs);
  }
  ~RunResources() {
    release();
    for (cudaStream_t st : {cs, xs, rs})
      if (st) cudaStreamDestroy(st);
  }
};


static void host_run_impl(const gnm_prep_view* prep, const gnm_bed_view* bed,
                          const gnm_resume* resume, const gnm_run_options* opts,
                          double* sums_out, uint32_t* missing_out) {
  if (!bed || (!bed->data && !bed->read_at)) fail(GNM_ERR_INVALID, "bed view has no data source");
  if (!sums_out || !missing_out) fail(GNM_ERR_INVALID, "output buffers are NULL");
  gnm_run_options o{};
  o.engine = GNM_ENGINE_AUTO;
  o.device = -1;
  if (opts) o = *opts;
  PhaseTrace trace;
  validate_prep(prep);
  int device = o.device;
  device = resolve_device(device);
  DeviceGuard g(device);
  const gnm_engine engine =
      o.engine == GNM_ENGINE_AUTO
          ? (prep->num_scores >= kTensorMinScores ? GNM_ENGINE_TENSOR : GNM_ENGINE_PLAIN)
          : o.engine;

  const uint64_t P = prep->num_people, K = prep->num_scores, V = prep->num_variants;
  const uint64_t bpv = prep->bytes_per_variant;
  const uint64_t v_start = resume ? resume->completed_variants : 0;
  if (v_start > V) fail(GNM_ERR_INVALID, "resume.completed_variants exceeds num_variants");
  if (resume && (!resume->sums || !resume->counts))
    fail(GNM_ERR_INVALID, "resume state has NULL buffers");
  const uint64_t pitch = (bpv + 127) / 128 * 128;
  // tensor-engine blocks start on 64-variant boundaries, by default on
  // 128-variant ones (the 8-bit kernels' stage; other blocks fall back to
  // BF16 limbs); rows between the boundary and the resume point are staged
  // as zeros (they contribute nothing)
  constexpr uint64_t kTensorAlign = 128;
  const uint64_t t_align = o.block_variants ? 64 : kTensorAlign;
  const uint64_t v_first = engine == GNM_ENGINE_TENSOR ? v_start - v_start % t_align : v_start;
  HostRun r{bpv, prep, bed, pitch, v_start};

  RunResources res(device);
  cudaStream_t cs = res.cs, xs = res.xs, rs = res.rs;

  // Block size: everything if it fits in ~60% of free memory, else two
  // alternating blocks of block_variants rows.
  size_t free_b = 0, total_b = 0;
  check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
  const uint64_t remaining = V - v_first;
  uint64_t block = o.block_variants ? o.block_variants : remaining;
  const uint64_t cap_rows = std::max<uint64_t>(kPlainRows, uint64_t(0.6 * double(free_b)) / pitch);
  if (!o.block_variants && block > cap_rows) block = std::max<uint64_t>(kPlainRows, cap_rows / 2);
  // The tensor engine's accumulate takes about as long as the copy of the
  // rows (batched workload: 365 ms against ~230 ms), so its rows go in four
  // blocks and each block's accumulate overlaps the next block's copy; the
  // plain engine's accumulate is ~2% of the copy, one block is best there.
  if (!o.block_variants && engine == GNM_ENGINE_TENSOR && remaining >= 4 * kTensorMinBlock)
    block = std::min(block, (remaining + 3) / 4);
  block = std::max<uint64_t>(1, std::min<uint64_t>(block, std::max<uint64_t>(1, remaining)));
  // a caller's block size is kept to the engine's 64-variant granularity (its
  // blocks then may run on BF16 limbs); the default one is a multiple of 128
  if (engine == GNM_ENGINE_TENSOR) block = (block + t_align - 1) / t_align * t_align;
  const int nbuf = remaining > block ? 2 : 1;

  std::vector<uint8_t*> dbuf(nbuf, nullptr);
  for (int i = 0; i < nbuf; ++i) dbuf[i] = res.alloc<uint8_t>(block * pitch, "row block");
  double* d_sums = res.alloc<double>(P * K * sizeof(double), "sums");
  uint32_t* d_cnt = res.alloc<uint32_t>(P * K * sizeof(uint32_t), "counts");

  // Direct path: identity rows from pinned memory, copied in 128 MB chunks
  // with at most two in flight (so other copies, like the plan's weight
  // upload, are not queued behind the whole matrix).  Rows whose length is
  // not the device pitch go back to back into a device staging ring (the
  // link's full rate; a pitched 2D copy runs ~5% slower) and are re-pitched
  // on the device, each chunk's repitch overlapping the next chunk's copy.
  const bool identity = prep->required_bim_indices == nullptr;
  const bool direct = identity && bed->data && is_pinned(bed->data);
  if (direct && V * bpv > bed->data_len)
    fail(GNM_ERR_IO, "truncated .bed: a required row lies past the end of the data");
  const bool repitch = direct && pitch != bpv;
  const uint64_t rpc = std::max<uint64_t>(1, (uint64_t(128) << 20) / std::max<uint64_t>(1, bpv));
  uint8_t* staging[2] = {nullptr, nullptr};
  if (repitch)
    for (int i = 0; i < 2; ++i) staging[i] = res.alloc<uint8_t>(rpc * bpv, "staging");
  const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(block, (uint64_t(128) << 20) / pitch));
  uint8_t* pinned[2] = {nullptr, nullptr};
  struct Pinned {
    uint8_t** p;
    ~Pinned() {
      cudaFreeHost(p[0]);
      cudaFreeHost(p[1]);
    }
  } pin_owner{pinned};
  if (!direct)
    for (int i = 0; i < 2; ++i)
      check_cuda(cudaHostAlloc(&pinned[i], chunk * pitch, cudaHostAllocDefault), "cudaHostAlloc");
  check_cuda(cudaStreamSynchronize(cs), "pool allocations");

  // copied: block rows are in dbuf; consumed: compute done with dbuf;
  // staged: host staging buffer free; landed / repitched: device staging
  // buffer filled / drained
  cudaEvent_t copied[2], consumed[2], staged[2], landed[2], repitched[2];
  struct Events {
    cudaEvent_t* e[5];
    ~Events() {
      for (auto* a : e)
        for (int i = 0; i < 2; ++i)
          if (a[i]) cudaEventDestroy(a[i]);
    }
  } ev_owner{{copied, consumed, staged, landed, repitched}};
  for (auto* a : ev_owner.e) a[0] = a[1] = nullptr;
  for (int i = 0; i < 2; ++i) {
    for (auto* a : ev_owner.e)
      check_cuda(cudaEventCreateWithFlags(&a[i], cudaEventDisableTiming), "event");
    check_cuda(cudaEventRecord(consumed[i], cs), "event");
    check_cuda(cudaEventRecord(staged[i], xs), "event");
    check_cuda(cudaEventRecord(landed[i], xs), "event");
    check_cuda(cudaEventRecord(repitched[i], rs), "event");
  }
  trace.mark("buffers");

  // Rows of block [b0, b0 + nb) into dbuf[slot]; copied[slot] fires when they are in.
  uint64_t stage_idx = 0;
  auto issue_block = [&](uint64_t b0, uint64_t nb, int slot) {
    const uint64_t skip = b0 < v_start ? v_start - b0 : 0;
    if (direct) {
      cudaStream_t ws = repitch ? rs : xs;        // the stream that writes dbuf
      check_cuda(cudaStreamWaitEvent(ws, consumed[slot], 0), "wait");
      if (!repitch) check_cuda(cudaStreamWaitEvent(xs, consumed[slot], 0), "wait");
      if (skip) check_cuda(cudaMemsetAsync(dbuf[slot], 0, skip * pitch, ws), "zero rows");
      const uint64_t step = repitch ? rpc : chunk;
      for (uint64_t c0 = skip; c0 < nb; c0 += step, ++stage_idx) {
        const uint64_t nc = std::min(step, nb - c0);
        const int sb = int(stage_idx & 1);
        check_cuda(cudaEventSynchronize(landed[sb]), "pace copies");   // two chunks in flight
        const uint8_t* src = bed->data + (b0 + c0) * bpv;
        if (repitch) {
          check_cuda(cudaStreamWaitEvent(xs, repitched[sb], 0), "wait");
          check_cuda(cudaMemcpyAsync(staging[sb], src, nc * bpv, cudaMemcpyHostToDevice, xs),
                     "H2D rows");
          check_cuda(cudaEventRecord(landed[sb], xs), "event");
          check_cuda(cudaStreamWaitEvent(rs, landed[sb], 0), "wait");
          check_cuda(launch_repitch(staging[sb], bpv, nc, dbuf[slot] + c0 * pitch, pitch, rs),
                     "repitch launch");
          check_cuda(cudaEventRecord(repitched[sb], rs), "event");
        } else {
          check_cuda(cudaMemcpyAsync(dbuf[slot] + c0 * pitch, src, nc * bpv,
                                     cudaMemcpyHostToDevice, xs),
                     "H2D rows");
          check_cuda(cudaEventRecord(landed[sb], xs), "event");
        }
      }
      check_cuda(cudaEventRecord(copied[slot], repitch ? rs : xs), "event");
    } else {
      check_cuda(cudaStreamWaitEvent(xs, consumed[slot], 0), "wait");
      for (uint64_t c0 = 0; c0 < nb; c0 += chunk, ++stage_idx) {
        const uint64_t nc = std::min(chunk, nb - c0);
        const int ps = int(stage_idx & 1);
        check_cuda(cudaEventSynchronize(staged[ps]), "wait pinned buffer");
        gather_rows(r, b0 + c0, nc, pinned[ps]);
        check_cuda(cudaMemcpyAsync(dbuf[slot] + c0 * pitch, pinned[ps], nc * pitch,
                                   cudaMemcpyHostToDevice, xs),
                   "H2D rows");
        check_cuda(cudaEventRecord(staged[ps], xs), "event");
      }
      check_cuda(cudaEventRecord(copied[slot], xs), "event");
    }
  };

  // The plan (weights -> records / stage tables / limb planes on the device)
  // is built on a helper thread while this thread streams the first block.
  gnm_plan* p = nullptr;
  std::exception_ptr plan_error;
  std::thread planner([&] {
    try {
      DeviceGuard pg(device);
      p = plan_create_impl(prep, engine, device, true);
    } catch (...) {
      plan_error = std::current_exception();
    }
  });
  struct PlanOwner {
    std::thread& t;
    gnm_plan*& p;
    ~PlanOwner() {
      if (t.joinable()) t.join();
      gnm_plan_destroy(p);
    }
  } owner{planner, p};
  if (v_first < V) issue_block(v_first, std::min(block, V - v_first), 0);
  planner.join();
  if (plan_error) std::rethrow_exception(plan_error);
  trace.mark("plan + first rows");

  plan_reset_impl(p, cs);
  std::vector<double> cb_sums;
  std::vector<uint32_t> cb_cnt;
  for (uint64_t b0 = v_first, bi = 0; b0 < V; b0 += block, ++bi) {
    const uint64_t nb = std::min(block, V - b0);
    const int slot = int(bi % nbuf);
    if (bi > 0) issue_block(b0, nb, slot);
    check_cuda(cudaStreamWaitEvent(cs, copied[slot], 0), "wait");
    accumulate_impl(p, dbuf[slot], pitch, b0, nb, cs);
    check_cuda(cudaEventRecord(consumed[slot], cs), "event");
    if (o.on_block) {
      finalize_impl(p, d_sums, d_cnt, resume == nullptr, cs);
      sync_impl(p, cs);
      cb_sums.resize(P * K);
      cb_cnt.resize(P * K);
      check_cuda(cudaMemcpy(cb_sums.data(), d_sums, P * K * 8, cudaMemcpyDeviceToHost), "D2H");
      check_cuda(cudaMemcpy(cb_cnt.data(), d_cnt, P * K * 4, cudaMemcpyDeviceToHost), "D2H");
      if (resume)
        for (uint64_t x = 0; x < P * K; ++x) {
          cb_sums[x] += resume->sums[x];
          cb_cnt[x] += resume->counts[x];
        }
      if (o.on_block(o.on_block_ctx, b0 + nb, cb_sums.data(), cb_cnt.data()) != 0)
        fail(GNM_ERR_PRODUCER, "block callback requested abort");
    }
  }
  if (trace.on) {   // (tracing serialises the last block's copy and compute)
    check_cuda(cudaStreamSynchronize(xs), "trace sync");
    check_cuda(cudaStreamSynchronize(rs), "trace sync");
    trace.mark("rows host->device");
    check_cuda(cudaStreamSynchronize(cs), "trace sync");
    trace.mark("accumulate");
  }
  finalize_impl(p, d_sums, d_cnt, resume == nullptr, cs);
  sync_impl(p, cs);
  copy_to_host(sums_out, d_sums, P * K * sizeof(double), cs);
  copy_to_host(missing_out, d_cnt, P * K * sizeof(uint32_t), cs);
  trace.mark("finalize + results");
  if (resume)
    for (uint64_t x = 0; x < P * K; ++x) {
      sums_out[x] += resume->sums[x];
      missing_out[x] += resume->counts[x];
    }
  if (trace.on) {
    res.release();
    gnm_plan_destroy(p);
    p = nullptr;
    trace.mark("release");
  }
}

// ---- HWE-PCA projection blocks (map/project.rs) --------------------------------
// The reference's GPU projection unpacks each variant block into a dense f32
// matrix, code 00 -> coeffs[0], 10 -> coeffs[1], 11 -> coeffs[2], missing -> 0
// (unpack_weighted_plink, map/project.rs:322-370), multiplies it by the
// block's loadings with an SGEMM accumulating into f32 [P][k]
// (compute_scores_block, :547-667) and adds that into f64 row-major scores
// (:669-733).  Here a block is a plain-engine plan whose cell records are the
// lookup values themselves: per (variant v, component c) baseline c0*L,
// code 01 -> -c0*L, 10 -> (c1 - c0)*L, 11 -> (c2 - c0)*L (FP64, rounded to
// FP32 records), so the 3-variant stage tables give exactly
// sum_v coeff(code) * L for any coefficients, accumulated in FP32 over 120
// variants and in FP64 beyond.
// Whether every variant's coefficients are linear in the dosage up to their
// own FP32 rounding, |(c2 - c0) - 2 (c1 - c0)| <= 4 ulp of the largest: true
// of the reference's HWE coefficients (g - 2p) * inv * weight, each rounded
// to FP32 on its own.
static bool projection_is_linear(const float* coeffs, uint64_t V) {
  for (uint64_t v = 0; v < V; ++v) {
    const double c0 = coeffs[3 * v], c1 = coeffs[3 * v + 1], c2 = coeffs[3 * v + 2];
    const double m = std::max({std::fabs(c0), std::fabs(c1), std::fabs(c2)});
    if (std::fabs((c2 - c0) - 2.0 * (c1 - c0)) > 4.0 * std::ldexp(m, -23)) return false;
  }
  return true;
}

// A block on the split-BF16 tensor engine, for 8 or more axes with linear
// coefficients: one pass over the rows for every axis.  The cells are the
// scoring engine's own: dosage weight (c1 - c0) * L, missing correction
// c0 * L and baseline sum c0 * L, so code 11 gets 2 (c1 - c0) * L, within
// the coefficients' FP32 rounding of (c2 - c0) * L.
static gnm_plan* plan_create_projection_tensor(int device, uint64_t n, uint64_t K, uint64_t V,
                                               const float* coeffs, const float* loadings_cm) {
  std::vector<float> w(V * K), c(V * K);
  std::vector<uint32_t> cols(V * K);
  std::vector<uint64_t> offs(V + 1);
  std::vector<double> base(K, 0.0);
  for (uint64_t v = 0; v < V; ++v) {
    offs[v] = v * K;
    const double c0 = coeffs[3 * v], c1 = coeffs[3 * v + 1];
    for (uint64_t k = 0; k < K; ++k) {
      const double l = loadings_cm[k * V + v];
      w[v * K + k] = float((c1 - c0) * l);
      c[v * K + k] = float(c0 * l);
      cols[v * K + k] = uint32_t(k);
      base[k] += c0 * l;
    }
  }
  offs[V] = V * K;
  gnm_prep_view view{};
  view.num_people = n;
  view.total_people_in_fam = n;
  view.bytes_per_variant = (n + 3) / 4;
  view.num_scores = K;
  view.num_variants = V;
  view.sparse_weights = w.data();
  view.sparse_missing_corrections = c.data();
  view.sparse_score_columns = cols.data();
  view.sparse_row_offsets = offs.data();
  view.baseline = base.data();
  return plan_create_impl(&view, GNM_ENGINE_TENSOR, device, true);
}

static gnm_plan* plan_create_projection(int device, uint64_t n, uint64_t K, uint64_t V,
                                        const float* coeffs, const float* loadings_cm) {
  PhaseTrace trace;
  DeviceGuard g(device);
  auto* p = new gnm_plan();
  try {
    p->device = device;
    p->P = n;
    p->fam = n;
    p->bpv = (n + 3) / 4;
    p->K = K;
    p->V = V;
    p->engine = GNM_ENGINE_PLAIN;
    p->h_baseline.assign(K, 0.0);
    p->rec_stride = V + kRecordPad;
    std::vector<float4> rec(K * p->rec_stride);
    // one axis per host thread: its records and its FP64 baseline
    auto fill = [&](uint64_t k0, uint64_t k1) {
      for (uint64_t k = k0; k < k1; ++k) {
        float4* r = rec.data() + k * p->rec_stride;
        const float* lk = loadings_cm + k * V;
        double b = 0.0;
        for (uint64_t v = 0; v < V; ++v) {
          const double l = lk[v];
          const double c0 = coeffs[3 * v], c1 = coeffs[3 * v + 1], c2 = coeffs[3 * v + 2];
          b += c0 * l;
          // member bits 0: the projection keeps no missing counts
          r[v] = make_float4(float(-c0 * l), float((c1 - c0) * l), float((c2 - c0) * l), 0.f);
        }
        std::fill(r + V, r + p->rec_stride, make_float4(0.f, 0.f, 0.f, 0.f));
        p->h_baseline[k] = b;
      }
    };
    const uint64_t nt = std::min<uint64_t>(K, std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
    if (nt <= 1 || K * V < (uint64_t(1) << 16)) {
      fill(0, K);
    } else {
      std::vector<std::thread> pool;
      const uint64_t per = (K + nt - 1) / nt;
      for (uint64_t i = 0; i < nt; ++i)
        pool.emplace_back(fill, std::min(K, i * per), std::min(K, (i + 1) * per));
      for (auto& th : pool) th.join();
    }
    p->d_baseline = dalloc<double>(p, K, "cudaMalloc(baseline)");
    check_cuda(cudaMemcpy(p->d_baseline, p->h_baseline.data(), K * sizeof(double),
                          cudaMemcpyHostToDevice),
               "upload baseline");
    p->d_zero_base = dalloc<double>(p, K, "cudaMalloc(zero baseline)");
    check_cuda(cudaMemset(p->d_zero_base, 0, K * sizeof(double)), "memset");
    p->d_err = dalloc<uint32_t>(p, 1, "cudaMalloc(error word)");
    check_cuda(cudaMemset(p->d_err, 0, 4), "memset");
    plain_geometry(p);
    upload_plain_records(p, rec, trace);
    check_cuda(cudaStreamSynchronize(0), "plan upload");
  } catch (...) {
    gnm_plan_destroy(p);
    throw;
  }
  return p;
}

static void project_block_impl(gnm_projector* pj, const uint8_t* packed, uint64_t filled,
                               const float* coeffs, const float* loadings_cm) {
  if (!pj) fail(GNM_ERR_INVALID, "projector is NULL");
  if (filled == 0) return;
  if (!packed || !coeffs || !loadings_cm) fail(GNM_ERR_INVALID, "block buffers are NULL");
  PhaseTrace trace;
  DeviceGuard g(pj->device);
  const uint64_t bpv = (pj->n + 3) / 4, pitch = (bpv + 127) / 128 * 128;
  struct Bufs {
    std::vector<void*> p;
    cudaStream_t s = nullptr;
    ~Bufs() {   // on an early exit, work on `s` may still use the buffers
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
      for (void* x : p) pool_free(x);
    }
  } b;
  b.p.push_back(pool_alloc(pj->device, filled * pitch, "projection rows"));
  auto* rows = static_cast<uint8_t*>(b.p.back());
  b.p.push_back(pool_alloc(pj->device, filled * bpv, "projection staging"));
  auto* staging = static_cast<uint8_t*>(b.p.back());
  b.p.push_back(pool_alloc(pj->device, pj->n * pj->K * 8, "projection sums"));
  auto* d_sums = static_cast<double*>(b.p.back());
  b.p.push_back(pool_alloc(pj->device, pj->n * pj->K * 4, "projection counts"));
  auto* d_counts = static_cast<uint32_t*>(b.p.back());
  check_cuda(cudaStreamCreateWithFlags(&b.s, cudaStreamNonBlocking), "cudaStreamCreate");
  // the plan (records, baseline, stage tables) is built on a helper thread
  // while the rows go up through the pinned ring on their own stream
  gnm_plan* built = nullptr;
  std::exception_ptr plan_error;
  const bool tensor = pj->K >= kTensorMinScores && projection_is_linear(coeffs, filled);
  std::thread planner([&] {
    try {
      built = tensor ? plan_create_projection_tensor(pj->device, pj->n, pj->K, filled, coeffs,
                                                     loadings_cm)
                     : plan_create_projection(pj->device, pj->n, pj->K, filled, coeffs,
                                              loadings_cm);
    } catch (...) {
      plan_error = std::current_exception();
    }
  });
  struct Join {   // on an early exit: wait for the planner, free what it built
    std::thread& t;
    gnm_plan*& built;
    ~Join() {
      if (t.joinable()) t.join();
      if (built) gnm_plan_destroy(built);
    }
  } join{planner, built};
  copy_to_device(staging, packed, filled * bpv, b.s);
  check_cuda(launch_repitch(staging, bpv, filled, rows, pitch, b.s), "repitch launch");
  trace.mark("project: rows");
  planner.join();
  if (plan_error) std::rethrow_exception(plan_error);
  std::unique_ptr<gnm_plan, void (*)(gnm_plan*)> plan(built, gnm_plan_destroy);
  built = nullptr;
  trace.mark("project: plan");
  plan_reset_impl(plan.get(), b.s);
  accumulate_impl(plan.get(), rows, pitch, 0, filled, b.s);
  finalize_impl(plan.get(), d_sums, d_counts, true, b.s);
  std::vector<double> s(pj->n * pj->K);
  check_cuda(cudaMemcpyAsync(s.data(), d_sums, s.size() * 8, cudaMemcpyDeviceToHost, b.s), "sums");
  sync_impl(plan.get(), b.s);
  trace.mark("project: accumulate");
  for (uint64_t i = 0; i < s.size(); ++i) pj->acc[i] += s[i];
  trace.mark("project: add");
}

// The .pgen counterpart of the end-to-end run: the file is uploaded once, the
// reconciled variants (required_bim_indices) are decoded on the device block
// by block into one row buffer, and each block is accumulated as it lands.
// With ALT counts, the .bim rows are a virtual .bim (the reference's split of
// multiallelic variants, shared/adapt_plink2.rs:1295-1330): row r holds ALT
// bim_alt[r] of .pgen variant bim_variant[r].
static void score_pgen_impl(const gnm_prep_view* prep, const uint8_t* pgen, uint64_t pgen_len,
                            const gnm_run_options* opts, double* sums_out,
                            uint32_t* missing_out, const uint32_t* alt_counts = nullptr,
                            const uint64_t* bim_variant = nullptr,
                            const uint32_t* bim_alt = nullptr, uint64_t bim_rows = 0) {
  if (!prep) fail(GNM_ERR_INVALID, "prep is NULL");
  if (!sums_out || !missing_out) fail(GNM_ERR_INVALID, "output buffers are NULL");
  const gnm_engine engine = opts ? opts->engine : GNM_ENGINE_AUTO;
  int device = opts ? opts->device : -1;
  device = resolve_device(device);
  validate_prep(prep);
  if (alt_counts && (!bim_variant || !bim_alt))
    fail(GNM_ERR_INVALID, "bim_variant and bim_alt are needed with alt_counts");
  std::unique_ptr<gnm_pgen, void (*)(gnm_pgen*)> pg(
      pgen_open_impl(pgen, pgen_len, device, alt_counts), gnm_pgen_close);
  const uint64_t n = pgen_samples(pg.get()), m = pgen_variants(pg.get());
  if (n != prep->total_people_in_fam || (n + 3) / 4 != prep->bytes_per_variant)
    fail(GNM_ERR_INVALID, "the .pgen has " + std::to_string(n) + " samples, the preparation " +
                              std::to_string(prep->total_people_in_fam));
  const uint64_t V = prep->num_variants;
  std::vector<uint64_t> req(V);
  std::vector<uint32_t> alts(alt_counts ? V : 0);
  for (uint64_t v = 0; v < V; ++v) {
    req[v] = prep->required_bim_indices ? prep->required_bim_indices[v] : v;
    if (alt_counts) {
      if (req[v] >= bim_rows)
        fail(GNM_ERR_INVALID, "required .bim row " + std::to_string(req[v]) + " is past the " +
                                  std::to_string(bim_rows) + " rows");
      alts[v] = bim_alt[req[v]];
      req[v] = bim_variant[req[v]];
    }
    if (req[v] >= m)
      fail(GNM_ERR_INVALID, "required variant " + std::to_string(req[v]) +
                                " is past the .pgen's " + std::to_string(m) + " variants");
  }
  std::unique_ptr<gnm_plan, void (*)(gnm_plan*)> plan(plan_create_impl(prep, engine, device, true),
                                                      gnm_plan_destroy);
  DeviceGuard g(device);
  struct Pool {
    std::vector<void*> p;
    ~Pool() {
      for (void* x : p) pool_free(x);
    }
    void* get(int dev, uint64_t bytes, const char* what) {
      p.push_back(pool_alloc(dev, bytes, what));
      return p.back();
    }
  } pool;
  struct Stream {   // destroyed before the pool: its work ends before buffers are freed
    cudaStream_t s = nullptr;
    ~Stream() {
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    }
  } st;
  check_cuda(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking), "cudaStreamCreate");
  const uint64_t pitch = (prep->bytes_per_variant + 127) / 128 * 128;
  // default block: every reconciled variant if its rows take at most 4 GiB
  uint64_t B = opts && opts->block_variants ? opts->block_variants
                                            : std::max<uint64_t>(1, (uint64_t(4) << 30) / pitch);
  B = std::max<uint64_t>(1, std::min<uint64_t>(B, std::max<uint64_t>(V, 1)));
  auto* rows = static_cast<uint8_t*>(pool.get(device, B * pitch, ".pgen row block"));
  const uint64_t PK = prep->num_people * prep->num_scores;
  auto* d_sums = static_cast<double*>(pool.get(device, std::max<uint64_t>(PK, 1) * 8, "sums"));
  auto* d_counts = static_cast<uint32_t*>(pool.get(device, std::max<uint64_t>(PK, 1) * 4, "counts"));
  plan_reset_impl(plan.get(), st.s);
  for (uint64_t b0 = 0; b0 < V; b0 += B) {
    const uint64_t nb = std::min(B, V - b0);
    pgen_decode_list_impl(pg.get(), req.data() + b0, nb, rows, pitch, st.s,
                          alt_counts ? alts.data() + b0 : nullptr);
    accumulate_impl(plan.get(), rows, pitch, b0, nb, st.s);
  }
  finalize_impl(plan.get(), d_sums, d_counts, true, st.s);
  check_cuda(cudaMemcpyAsync(sums_out, d_sums, PK * 8, cudaMemcpyDeviceToHost, st.s), "sums");
  check_cuda(cudaMemcpyAsync(missing_out, d_counts, PK * 4, cudaMemcpyDeviceToHost, st.s),
             "counts");
  pgen_check_impl(pg.get(), st.s);
  sync_impl(plan.get(), st.s);
}

}  // namespace gnm

using namespace gnm;

extern "C" {

int gnm_abi_version(void) { return GNM_ABI_VERSION; }

gnm_status gnm_score_run(const gnm_prep_view* prep, const gnm_bed_view* bed,
                         const gnm_resume* resume, double* sums_out, uint32_t* missing_out,
                         gnm_error* err) {
  return gnm_score_run_ex(prep, bed, resume, nullptr, sums_out, missing_out, err);
}

gnm_status gnm_score_pgen(const gnm_prep_view* prep, const uint8_t* pgen, uint64_t pgen_len,
                          const gnm_run_options* opts, double* sums_out, uint32_t* missing_out,
                          gnm_error* err) {
  return guarded(err, [&] { score_pgen_impl(prep, pgen, pgen_len, opts, sums_out, missing_out); });
}

gnm_status gnm_score_pgen_alleles(const gnm_prep_view* prep, const uint8_t* pgen,
                                  uint64_t pgen_len, const uint32_t* alt_counts,
                                  const uint64_t* bim_variant, const uint32_t* bim_alt,
                                  uint64_t bim_rows, const gnm_run_options* opts,
                                  double* sums_out, uint32_t* missing_out, gnm_error* err) {
  return guarded(err, [&] {
    if (!alt_counts) fail(GNM_ERR_INVALID, "alt_counts is NULL");
    score_pgen_impl(prep, pgen, pgen_len, opts, sums_out, missing_out, alt_counts, bim_variant,
                    bim_alt, bim_rows);
  });
}

gnm_status gnm_project_create(uint64_t n_samples, uint64_t components, int device,
                              gnm_projector** out, gnm_error* err) {
  return guarded(err, [&] {
    if (!out) fail(GNM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (n_samples == 0 || components == 0)
      fail(GNM_ERR_INVALID, "a projection needs samples and components");
    device = resolve_device(device);
    auto* pj = new gnm_projector;
    pj->device = device;
    pj->n = n_samples;
    pj->K = components;
    pj->acc.assign(n_samples * components, 0.0);
    *out = pj;
  });
}

void gnm_project_destroy(gnm_projector* pj) { delete pj; }

gnm_status gnm_project_block(gnm_projector* pj, const uint8_t* packed, uint64_t filled,
                             const float* coeffs, const float* loadings_col_major,
                             gnm_error* err) {
  return guarded(err, [&] { project_block_impl(pj, packed, filled, coeffs, loadings_col_major); });
}

gnm_status gnm_project_scores(const gnm_projector* pj, double* scores_row_major, gnm_error* err) {
  return guarded(err, [&] {
    if (!pj || !scores_row_major) fail(GNM_ERR_INVALID, "NULL argument");
    for (uint64_t i = 0; i < pj->acc.size(); ++i) scores_row_major[i] += pj->acc[i];
  });
}

gnm_status gnm_score_run_ex(const gnm_prep_view* prep, const gnm_bed_view* bed,
                            const gnm_resume* resume, const gnm_run_options* opts,
                            double* sums_out, uint32_t* missing_out, gnm_error* err) {
  return guarded(err, [&] { host_run_impl(prep, bed, resume, opts, sums_out, missing_out); });
}

gnm_status gnm_plan_create(const gnm_prep_view* prep, gnm_engine engine, int device,
                           gnm_plan** plan_out, gnm_error* err) {
  if (!plan_out) return GNM_ERR_INVALID;
  *plan_out = nullptr;
  return guarded(err, [&] { *plan_out = plan_create_impl(prep, engine, device); });
}

void gnm_plan_destroy(gnm_plan* p) {
  if (!p) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(p->device);
  cudaDeviceSynchronize();   // no kernel of any stream may still use the buffers
  if (p->tensor) tensor_plan_destroy(p);
  for (void* b : {static_cast<void*>(p->d_records), static_cast<void*>(p->d_tables),
                  static_cast<void*>(p->d_tab_scratch), static_cast<void*>(p->d_part_sum),
                  static_cast<void*>(p->d_part_cnt), static_cast<void*>(p->d_baseline),
                  static_cast<void*>(p->d_zero_base), static_cast<void*>(p->d_out_to_fam),
                  static_cast<void*>(p->d_err), static_cast<void*>(p->d_grad_fam),
                  static_cast<void*>(p->d_bw)})
    pool_free(b);
  cudaStreamSynchronize(0);
  if (prev >= 0) cudaSetDevice(prev);
  delete p;
}

gnm_engine gnm_plan_engine(const gnm_plan* p) { return p ? p->engine : GNM_ENGINE_AUTO; }
uint64_t gnm_plan_device_bytes(const gnm_plan* p) { return p ? p->device_bytes : 0; }
uint64_t gnm_plan_launch_count(const gnm_plan* p) { return p ? p->launches : 0; }

gnm_status gnm_plan_reset(gnm_plan* p, void* stream, gnm_error* err) {
  if (!p) return GNM_ERR_INVALID;
  return guarded(err, [&] { plan_reset_impl(p, static_cast<cudaStream_t>(stream)); });
}

gnm_status gnm_plan_accumulate_device(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch,
                                      uint64_t v0, uint64_t nv, void* stream, gnm_error* err) {
  if (!p) return GNM_ERR_INVALID;
  return guarded(err, [&] {
    accumulate_impl(p, d_rows, pitch, v0, nv, static_cast<cudaStream_t>(stream));
  });
}

gnm_status gnm_plan_finalize_device(gnm_plan* p, double* d_sums, uint32_t* d_counts, void* stream,
                                    gnm_error* err) {
  if (!p) return GNM_ERR_INVALID;
  return guarded(err, [&] {
    if (!d_sums || !d_counts) fail(GNM_ERR_INVALID, "output buffers are NULL");
    finalize_impl(p, d_sums, d_counts, true, static_cast<cudaStream_t>(stream));
  });
}

gnm_status gnm_plan_sync(gnm_plan* p, void* stream, gnm_error* err) {
  if (!p) return GNM_ERR_INVALID;
  return guarded(err, [&] { sync_impl(p, static_cast<cudaStream_t>(stream)); });
}

gnm_status gnm_score_device(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch, double* d_sums,
                            uint32_t* d_counts, void* stream, gnm_error* err) {
  if (!p) return GNM_ERR_INVALID;
  return guarded(err, [&] {
    if (!d_sums || !d_counts) fail(GNM_ERR_INVALID, "output buffers are NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    plan_reset_impl(p, s);
    accumulate_impl(p, d_rows, pitch, 0, p->V, s);
    finalize_impl(p, d_sums, d_counts, true, s);
  });
}

gnm_status gnm_plan_autotune(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch,
                             uint64_t variant_count, void* stream, gnm_error* err) {
  if (!p) return GNM_ERR_INVALID;
  return guarded(err, [&] {
    autotune_impl(p, d_rows, pitch, variant_count, static_cast<cudaStream_t>(stream));
  });
}

gnm_status gnm_plan_set_shape(gnm_plan* p, uint32_t shape, gnm_error* err) {
  if (!p) return GNM_ERR_INVALID;
  return guarded(err, [&] {
    if (p->engine != GNM_ENGINE_PLAIN) {
      if (shape > 15 || ((shape & 8u) && (shape & 6u) != 4u))
        fail(GNM_ERR_INVALID,
             "tensor engine shape is raster | (narrow << 1) | (8-bit limbs << 2) | "
             "(8-bit wide kernel on SM pairs << 3)");
      tensor_set_narrow(p, (shape & 2u) != 0);
      tensor_set_i8(p, (shape & 4u) != 0);
      tensor_set_pair(p, (shape & 8u) != 0);
      p->raster = shape & 1u;
      return;
    }
    const uint32_t kernel = shape >> 16;
    bool known = false;
    for (uint32_t kn : kPlainKernels) known |= kn == kernel;
    if (!known) fail(GNM_ERR_INVALID, "unknown plain kernel in shape " + std::to_string(shape));
    const uint32_t k0 = p->kernel, t0 = p->tiles, s0 = p->splits, l0 = p->last_splits,
                   n0 = p->slots;
    plain_shape_fixed(p, kernel, shape & 0xFFFFu);
    if (p->slots > p->splits_alloc) {
      const uint32_t need = p->slots;
      p->kernel = k0;
      p->tiles = t0;
      p->splits = s0;
      p->last_splits = l0;
      p->slots = n0;
      fail(GNM_ERR_INVALID, "shape needs " + std::to_string(need) + " partial slots; the plan has " +
                                std::to_string(p->splits_alloc));
    }
  });
}

uint32_t gnm_plan_tuned_shape(const gnm_plan* p) {
  if (!p) return 0;
  return p->engine == GNM_ENGINE_PLAIN ? (p->kernel << 16) | std::min<uint32_t>(p->splits, 0xFFFFu)
                                       : (p->raster | (tensor_is_narrow(p) ? 2u : 0u) |
                                          (tensor_is_i8(p) ? 4u : 0u) |
                                          (tensor_is_pair(p) ? 8u : 0u));
}

gnm_status gnm_decode_device(const uint8_t* d_rows, uint64_t pitch, uint64_t nv, uint64_t np,
                             int8_t* d_out, uint64_t out_pitch, void* stream, gnm_error* err) {
  return guarded(err, [&] {
    if (np > pitch * 4) fail(GNM_ERR_INVALID, "num_people exceeds 4*pitch");
    if (out_pitch < np) fail(GNM_ERR_INVALID, "out_pitch < num_people");
    check_cuda(launch_decode(d_rows, pitch, nv, np, d_out, out_pitch,
                             static_cast<cudaStream_t>(stream)),
               "decode launch");
  });
}

gnm_status gnm_release_cached_memory(int device, gnm_error* err) {
  return guarded(err, [&] {
    device = resolve_device(device);
    DeviceGuard g(device);
    check_cuda(cudaMemPoolTrimTo(run_pool(device), 0), "cudaMemPoolTrimTo");
    release_result_ring();
  });
}

gnm_status gnm_watchdog_selftest(int device, uint64_t wait_ns, uint64_t* waited_ns_out,
                                 gnm_error* err) {
  return guarded(err, [&] {
    device = resolve_device(device);
    DeviceGuard g(device);
    void* d = nullptr;
    check_cuda(cudaMalloc(&d, 16), "cudaMalloc(watchdog words)");
    struct Free {
      void* p;
      ~Free() { cudaFree(p); }
    } free_on_exit{d};
    uint64_t* waited = static_cast<uint64_t*>(d);
    uint32_t* word = reinterpret_cast<uint32_t*>(static_cast<char*>(d) + 8);
    check_cuda(cudaMemset(d, 0, 16), "memset");
    check_cuda(launch_watchdog_probe(wait_ns, word, waited, 0), "watchdog probe launch");
    check_cuda(cudaDeviceSynchronize(), "watchdog probe");
    uint64_t host[2] = {0, 0};
    check_cuda(cudaMemcpy(host, d, 16, cudaMemcpyDeviceToHost), "D2H");
    if (waited_ns_out) *waited_ns_out = host[0];
    if (uint32_t(host[1]) & kErrTmaTimeout)
      fail(GNM_ERR_TIMEOUT, "device watchdog: a bounded wait expired after " +
                                std::to_string(host[0]) + " ns (self-test)");
  });
}

gnm_status gnm_synth_fill_device(uint8_t* d_rows, uint64_t pitch, uint64_t v0, uint64_t nv,
                                 uint64_t i0, uint64_t np, const uint32_t* d_thr, uint64_t seed,
                                 void* stream, gnm_error* err) {
  return guarded(err, [&] {
    if (pitch % 16 != 0) fail(GNM_ERR_INVALID, "pitch must be a multiple of 16");
    if ((np + 3) / 4 > pitch) fail(GNM_ERR_INVALID, "pitch smaller than ceil(num_people/4)");
    check_cuda(launch_synth_fill(d_rows, pitch, v0, nv, i0, np, d_thr, seed,
                                 static_cast<cudaStream_t>(stream)),
               "synth launch");
  });
}

gnm_status gnm_backward_dw_device(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch,
                                  const float* d_grad_s, float* d_grad_w, float* d_grad_corr,
                                  void* stream, gnm_error* err) {
  if (!p) return GNM_ERR_INVALID;
  return guarded(err, [&] {
    DeviceGuard g(p->device);
    backward_dw(p, d_rows, pitch, d_grad_s, d_grad_w, d_grad_corr,
                static_cast<cudaStream_t>(stream));
  });
}

gnm_status gnm_plan_set_backward_limbs(gnm_plan* p, uint32_t bits, gnm_error* err) {
  if (!p) return GNM_ERR_INVALID;
  return guarded(err, [&] {
    if (bits != 8 && bits != 16) fail(GNM_ERR_INVALID, "backward limbs are 8 or 16 bits wide");
    p->bw_limb_bits = bits;
  });
}

}  // extern "C"
