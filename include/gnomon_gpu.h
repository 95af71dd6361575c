/*
 * gnomon_gpu.h — C ABI of the B200 (sm_100a) polygenic-score engine.
 *
 * This library stands in for gnomon's GPU scoring backend.  Its entry points
 * take exactly what gnomon's `score::pipeline` hands its engines: the prepared
 * CSR of (variant, score) cells, the packed PLINK .bed rows, and an optional
 * resume state.  They return gnomon's per-person result: row-major [P][K]
 * final sums (baseline included, not averaged) and [P][K] missing counts.
 *
 * Reference interfaces each declaration replaces are cited by file:line in
 * the SauersML/gnomon tree (crate `gnomon` v0.1.4).
 *
 * Conventions
 *   - Plain C types only; no exceptions or aborts cross this boundary.  Every
 *     CUDA error, invalid argument and device watchdog expiry becomes a
 *     gnm_status plus a message in the caller-owned gnm_error.
 *   - Outputs are caller-allocated.  Host entry points take host pointers;
 *     `*_device` entry points take device pointers and a cudaStream_t passed
 *     as `void*` (NULL = the legacy default stream).
 *   - PLINK code per person per variant (SNP-major, 4 people per byte, person
 *     i at bits 2*(i%4)): 00 -> dosage 0, 01 -> missing, 10 -> 1, 11 -> 2
 *     (allele-2 dosage).  Cited: score/batch.rs:489-503,
 *     score/cuda_backend.rs:106-117.
 *   - Per (variant v, score k) cell the prepared weights are
 *       dosage_weight  = +w (effect allele == BIM allele2) or -w (flipped),
 *       missing_correction = 2w if flipped else 0 (duplicates summed),
 *     and sum[p,k] = baseline[k] + sum_v dosage_weight*d(p,v)
 *                    - sum_{v missing for p} missing_correction.
 *     Cited: score/prepare.rs:197-208, 557-558, 630-650.
 */
#ifndef GNOMON_GPU_H
#define GNOMON_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GNM_ABI_VERSION 1

/* Status codes.  GNM_DECLINED mirrors `Ok(None)` of try_run_cuda
 * (score/cuda_backend.rs:604-657): the caller falls back to its CPU pipeline.
 * The error codes mirror PipelineError::{Io, Compute, Producer}
 * (shared/pipeline_error.rs:5-9). */
typedef enum gnm_status {
  GNM_OK = 0,
  GNM_DECLINED = 1,
  GNM_ERR_IO = 2,
  GNM_ERR_COMPUTE = 3,
  GNM_ERR_PRODUCER = 4,
  GNM_ERR_TIMEOUT = 5,  /* a bounded device wait expired; context still usable */
  GNM_ERR_INVALID = 6   /* argument / shape validation failed */
} gnm_status;

typedef struct gnm_error {
  char message[512];
} gnm_error;

/* Engine selection for gnm_score_run_ex. */
/* Device argument: pick the visible sm_100 device with the most free memory,
 * ties broken by SM count (the reference probes every visible device and
 * ranks them the same way, score/cuda_backend.rs:894-991). */
#define GNM_DEVICE_BEST (-2)

typedef enum gnm_engine {
  GNM_ENGINE_AUTO = 0,     /* plain below 8 score columns, split-BF16 tensor cores from 8 */
  GNM_ENGINE_PLAIN = 1,    /* FP32 CUDA-core LUT kernel, FP64 cross-block reduce */
  GNM_ENGINE_TENSOR = 2    /* split-BF16 (hi/mid/lo) tcgen05 GEMM, FP32 TMEM accum */
} gnm_engine;

/* Read-only view of gnomon's PreparationResult (score/types.rs:167-327) for
 * one scoring run.  All pointers are HOST pointers owned by the caller.
 *   sparse_row_offsets[v]..[v+1] delimit reconciled variant v's cells,
 *   columns strictly ascending within a row (prepare.rs:630-650). */
typedef struct gnm_prep_view {
  uint64_t num_people;            /* P = num_people_to_score                      */
  uint64_t total_people_in_fam;   /* people per .bed row (sets bytes_per_variant) */
  uint64_t bytes_per_variant;     /* ceil(total_people_in_fam / 4) (prepare.rs:811) */
  uint64_t num_scores;            /* K = score_names.len()                        */
  uint64_t num_variants;          /* V = num_reconciled_variants                  */
  const float* sparse_weights;              /* [nnz] dosage_weight                */
  const float* sparse_missing_corrections;  /* [nnz] missing_correction           */
  const uint32_t* sparse_score_columns;     /* [nnz] score column < K             */
  const uint64_t* sparse_row_offsets;       /* [V+1]                              */
  const uint64_t* required_bim_indices;     /* [V] .bed row of variant v; NULL = identity */
  const uint32_t* output_idx_to_fam_idx;    /* [P] fam index of output row; NULL = identity */
  const double* baseline;         /* [K] sum of missing_correction; NULL = computed here */
} gnm_prep_view;

/* Genotype byte source (shared/files.rs:187-292).  Either `data` points at
 * the .bed bytes AFTER the 3-byte magic (mmap or RAM; row r at r*bpv), or
 * `read_at` fills dst with `len` bytes starting at row-data offset `offset`
 * and returns 0 on success. */
typedef struct gnm_bed_view {
  const uint8_t* data;
  uint64_t data_len;
  int (*read_at)(void* user_ctx, uint64_t offset, uint8_t* dst, uint64_t len);
  void* user_ctx;
} gnm_bed_view;

/* Resume state of a checkpoint (score/checkpoint.rs:293-340,
 * score/pipeline.rs:1777-1800): the first `completed_variants` reconciled
 * variants are already folded into `sums`/`counts` ([P][K], baseline
 * included).  NULL = fresh run. */
typedef struct gnm_resume {
  uint64_t completed_variants;
  const double* sums;
  const uint32_t* counts;
} gnm_resume;

/* Optional progress / checkpoint callback, called on the calling thread after
 * each completed variant block with the running [P][K] state (host memory,
 * valid only during the call).  Return nonzero to abort with GNM_ERR_PRODUCER. */
typedef int (*gnm_block_callback)(void* user_ctx, uint64_t completed_variants,
                                  const double* sums, const uint32_t* counts);

typedef struct gnm_run_options {
  gnm_engine engine;
  int device;                     /* CUDA ordinal; -1 = current device;
                                     GNM_DEVICE_BEST = the visible sm_100 device
                                     with the most free memory (then SMs)        */
  uint64_t block_variants;        /* streaming block; 0 = default: the whole matrix
                                     if it fits (tensor engine: four blocks of at
                                     least 16,384 variants, each block's compute
                                     overlapping the next block's copy); the
                                     tensor engine rounds it up to a multiple of
                                     64 variants (its 8-bit kernels take blocks
                                     starting at multiples of 128; others run on
                                     BF16 limbs); its default blocks are
                                     multiples of 128                             */
  gnm_block_callback on_block;    /* may be NULL                                  */
  void* on_block_ctx;
} gnm_run_options;

/* Library / ABI identification.  Returns GNM_ABI_VERSION. */
int gnm_abi_version(void);

/* Drop-in for `try_run_cuda(context) -> Result<Option<(Vec<f64>, Vec<u32>)>>`
 * (score/cuda_backend.rs:604), called from pipeline::run
 * (score/pipeline.rs:480-482).  Host buffers in, host buffers out:
 *   sums_out    [P*K] row-major final sums (baseline included),
 *   missing_out [P*K] missing counts.
 * Returns GNM_DECLINED (leaving outputs untouched) when no usable CUDA device
 * exists, mirroring the reference's CPU fallback. */
gnm_status gnm_score_run(const gnm_prep_view* prep, const gnm_bed_view* bed,
                         const gnm_resume* resume, double* sums_out,
                         uint32_t* missing_out, gnm_error* err);

/* gnm_score_run with explicit engine / streaming options (NULL = defaults). */
gnm_status gnm_score_run_ex(const gnm_prep_view* prep, const gnm_bed_view* bed,
                            const gnm_resume* resume, const gnm_run_options* opts,
                            double* sums_out, uint32_t* missing_out, gnm_error* err);

/* ---- Device-resident API (genotypes already in HBM) ---------------------
 * A plan uploads the prepared weights once (the work of CudaRuntime::new,
 * score/cuda_backend.rs:994-1190, minus NVRTC/cuBLAS) and then scores packed
 * rows that already live in device memory. */
typedef struct gnm_plan gnm_plan;

gnm_status gnm_plan_create(const gnm_prep_view* prep, gnm_engine engine, int device,
                           gnm_plan** plan_out, gnm_error* err);
void gnm_plan_destroy(gnm_plan* plan);

/* Which engine the plan resolved to (GNM_ENGINE_PLAIN or GNM_ENGINE_TENSOR). */
gnm_engine gnm_plan_engine(const gnm_plan* plan);

/* Bytes of device scratch the plan holds (partials, tables). */
uint64_t gnm_plan_device_bytes(const gnm_plan* plan);

/* Zero the plan's accumulators (start of a run).  Asynchronous on `stream`. */
gnm_status gnm_plan_reset(gnm_plan* plan, void* stream, gnm_error* err);

/* Accumulate reconciled variants [variant_begin, variant_begin+variant_count)
 * whose packed rows sit at d_rows (row i of the block at d_rows + i*pitch;
 * pitch a multiple of 16; d_rows 16-byte aligned).  Asynchronous on `stream`. */
gnm_status gnm_plan_accumulate_device(gnm_plan* plan, const uint8_t* d_rows,
                                      uint64_t pitch, uint64_t variant_begin,
                                      uint64_t variant_count, void* stream,
                                      gnm_error* err);

/* Write final [P][K] sums (baseline added, output rows gathered through
 * output_idx_to_fam_idx) and counts to DEVICE buffers.  Asynchronous; the
 * status of the device watchdog is checked by gnm_plan_sync. */
gnm_status gnm_plan_finalize_device(gnm_plan* plan, double* d_sums_out,
                                    uint32_t* d_missing_out, void* stream,
                                    gnm_error* err);

/* Synchronize `stream` and report any device-side watchdog / error flag. */
gnm_status gnm_plan_sync(gnm_plan* plan, void* stream, gnm_error* err);

/* gnm_score_run / gnm_score_run_ex allocate their row blocks, staging and
 * output buffers from a per-device memory pool that keeps freed memory
 * reserved, so repeated runs on a device skip mapping and unmapping it, and
 * copy large results back through a cached 128 MB pinned host ring.  This
 * returns that reserve to the device (-1 = current device) and frees the
 * ring; it is safe to call at any time and frees nothing a running call
 * holds.  No reference counterpart (the reference's engine allocates and
 * frees per call). */
gnm_status gnm_release_cached_memory(int device, gnm_error* err);

/* Device watchdog self-test (no reference counterpart; the reference's GPU
 * engine has no bounded device waits).  Every wait in this library's kernels
 * gives up after 2 s, records the expiry in a device error word and returns,
 * which the host turns into GNM_ERR_TIMEOUT with the context still usable.
 * This runs that same bounded-wait code on an mbarrier that nothing ever
 * signals, with a limit of `wait_ns`, on device `device` (-1 = current), and
 * returns what a scoring call would: GNM_ERR_TIMEOUT once the wait expired.
 * *waited_ns_out (may be NULL) receives the measured wait. */
gnm_status gnm_watchdog_selftest(int device, uint64_t wait_ns, uint64_t* waited_ns_out,
                                 gnm_error* err);

/* One-shot device scoring: reset + accumulate(all V rows) + finalize. */
gnm_status gnm_score_device(gnm_plan* plan, const uint8_t* d_rows, uint64_t pitch,
                            double* d_sums_out, uint32_t* d_missing_out,
                            void* stream, gnm_error* err);

/* Number of kernel launches the last accumulate+finalize issued (for audit). */
uint64_t gnm_plan_launch_count(const gnm_plan* plan);

/* Autotuner (no reference counterpart; the reference sizes its tiles from free
 * memory only, score/cuda_backend.rs:803-975): times the plan's accumulate on
 * the first `variant_count` resident rows for each candidate launch shape —
 * plain engine (accumulate + finalize, which reads every split's partials):
 * the kernel (people tiles of 512 bytes with 4 warps, with or without a
 * producer warp; 1024 bytes with 8 warps, with or without one; 2048 bytes
 * with 16 warps and a producer warp) times the variant-split count (0.5x to
 * 8x the SMs' CTA slots, the same count for every people tile);
 * tensor engine: up to 64 scores the narrow kernel (people as the MMA's M)
 * on BF16 and on 8-bit limbs, against the wide kernel (scores as M) on BF16
 * limbs, on 8-bit integer limbs, and on 8-bit limbs over SM pairs (one MMA
 * across the two CTAs of a cluster), each wide form in both CTA raster
 * orders — keeps the fastest, and
 * leaves the plan reset.  Blocks until done.  With the environment variable
 * GNM_TRACE set, every candidate's time is printed on stderr. */
gnm_status gnm_plan_autotune(gnm_plan* plan, const uint8_t* d_rows, uint64_t pitch,
                             uint64_t variant_count, void* stream, gnm_error* err);

/* The tuned shape.  Plain engine: (kernel << 16) | splits per full people
 * tile, kernel = tile bytes (512, 1024, 2048) + 1 with a producer warp;
 * tensor engine: raster order | (2 if the narrow kernel runs the plan) |
 * (4 if it runs on 8-bit limbs; its blocks then start at multiples of 128
 * variants, others fall back to the BF16 limbs) | (8 if the wide kernel's
 * 8-bit MMAs span SM pairs; only with 4 and without 2). */
uint32_t gnm_plan_tuned_shape(const gnm_plan* plan);

/* Pin a shape (a value gnm_plan_tuned_shape returned, e.g. saved from an
 * earlier autotune of the same workload).  GNM_ERR_INVALID for an unknown
 * kernel, more splits than the plan's partial slots hold, or a tensor shape
 * with unknown bits or SM pairs on anything but the 8-bit wide kernel. */
gnm_status gnm_plan_set_shape(gnm_plan* plan, uint32_t shape, gnm_error* err);

/* ---- Packed-row utilities ------------------------------------------------ */

/* Decode packed rows to int8 dosage codes on the device: out[v*out_pitch + i]
 * = {0,1,2} or -1 for missing, for i < num_people.  Used for decode parity. */
gnm_status gnm_decode_device(const uint8_t* d_rows, uint64_t pitch,
                             uint64_t num_variants, uint64_t num_people,
                             int8_t* d_out, uint64_t out_pitch, void* stream,
                             gnm_error* err);

/* Fill a device matrix with the deterministic synthetic HWE genotype
 * generator: per-variant uint32 thresholds {t_missing, T0, T1},
 * code = u_m < t_m ? 01 : u_g < T0 ? 00 : u_g < T1 ? 10 : 11 with (u_m, u_g)
 * the two halves of mix64(key(seed, v, i)).  Column c of the matrix holds
 * cohort person i = person_begin + c, so a person shard can generate its own
 * column slice of a larger cohort.  Padding columns (c >= num_people) are 00. */
gnm_status gnm_synth_fill_device(uint8_t* d_rows, uint64_t pitch, uint64_t variant_begin,
                                 uint64_t num_variants, uint64_t person_begin,
                                 uint64_t num_people,
                                 const uint32_t* d_thresholds /* [num_variants][3] */,
                                 uint64_t seed, void* stream, gnm_error* err);

/* ---- Backward: dW = G^T dS by re-unpacking genotypes -------------------- */

/* d_grad_w[v*K + k] = sum_p dosage'(p,v) * d_grad_s[p*K + k] where dosage' is
 * the allele-2 dosage with missing -> 0 (the derivative of the plain score
 * w.r.t. dosage_weight), and d_grad_corr[v*K+k] = -sum_{p missing} dS[p,k]
 * (derivative w.r.t. missing_correction; may be NULL).  dS is [P][K] FP32
 * over output rows (gathered through output_idx_to_fam_idx). */
gnm_status gnm_backward_dw_device(gnm_plan* plan, const uint8_t* d_rows, uint64_t pitch,
                                  const float* d_grad_s, float* d_grad_w,
                                  float* d_grad_corr, void* stream, gnm_error* err);

/* Limb width of the backward's dS split: 8 (the default: signed 8-bit limbs,
 * tcgen05 kind::i8, 128 people per stage) or 16 (BF16 limbs, kind::f16, 64
 * people per stage).  Both leave each dS within 2^-31.9 (8) / 2^-33 (16) of
 * its score's largest |dS|.  GNM_ERR_INVALID for any other width. */
gnm_status gnm_plan_set_backward_limbs(gnm_plan* plan, uint32_t bits, gnm_error* err);

/* ---- PLINK 2 .pgen input ---------------------------------------------------
 * gnomon scores a .pgen through a virtual .bed (shared/adapt_plink2.rs:1093-
 * 1158, 2108-2666): each variant's hard calls are decoded and packed as the
 * .bed codes of the A1 = ALT dosage.  These entry points do that decode on the
 * GPU, straight into device rows the scoring plans read (gnm_plan_accumulate /
 * gnm_score_device), one row per .pgen variant in file order.
 *
 * Supported: storage modes 0x02 and 0x10 / 0x11, biallelic records
 * (main-track types 0-4, 6, 7), optionally followed by a phase track (skipped)
 * and a dosage track: a hard call that is missing takes the nearest whole
 * allele count of its dosage when that lies within 0.10, as the reference's
 * reader coerces dosages (shared/adapt_plink2.rs:14-18); phased-dosage
 * tracks are skipped.  Multiallelic records (vrtype bit 3) need the
 * variants' ALT counts (gnm_pgen_open_alleles): each decoded row then holds
 * the copies of one ALT, as the reference's virtual .bim splits a
 * multiallelic variant into one row per ALT (shared/adapt_plink2.rs:2704-
 * 2881).  Without ALT counts such records, external-index modes and more
 * than 2^31 samples are rejected with GNM_ERR_INVALID; truncated or
 * malformed files give GNM_ERR_IO.  The reference additionally applies
 * sex-chromosome ploidy from the .pvar / .psam; callers handle that. */

/* Variant and sample counts from a .pgen header (host bytes). */
gnm_status gnm_pgen_dims(const uint8_t* pgen, uint64_t pgen_len, uint64_t* num_variants,
                         uint64_t* num_samples, gnm_error* err);

/* Decode every variant of the .pgen (host bytes) into d_rows[v * pitch ..]
 * on `device` (-1 = current): ceil(samples / 4) bytes per row, padding fields
 * of the last byte set to 01 as the reference packs them; the other bytes of
 * each row keep their values.  d_rows 16-byte aligned, pitch a multiple of 16.
 * Synchronous on `stream` (NULL = default stream).  Same as gnm_pgen_open +
 * gnm_pgen_decode of every variant + gnm_pgen_check + gnm_pgen_close. */
gnm_status gnm_pgen_decode_device(const uint8_t* pgen, uint64_t pgen_len, int device,
                                  uint8_t* d_rows, uint64_t pitch, void* stream,
                                  gnm_error* err);

/* A .pgen resident on one device: the file's bytes and its record index are
 * copied to HBM once (the reference's reader keeps the same index,
 * shared/adapt_plink2.rs:1512-1716), then any variant range is decoded on
 * demand, e.g. block by block into a streaming buffer.  Use a handle from one
 * stream at a time. */
typedef struct gnm_pgen gnm_pgen;

/* Parse and validate the header, upload the file; GNM_DECLINED without a
 * device. */
gnm_status gnm_pgen_open(const uint8_t* pgen, uint64_t pgen_len, int device, gnm_pgen** out,
                         gnm_error* err);
void gnm_pgen_close(gnm_pgen* pg);

/* Bytes of device memory the handle holds (file, index, one scratch row). */
uint64_t gnm_pgen_device_bytes(const gnm_pgen* pg);

/* Decode variants [variant_begin, variant_begin + variant_count) into
 * d_rows[(v - variant_begin) * pitch ..], asynchronously on `stream`.  An
 * LD-compressed record whose anchor precedes the range is decoded from that
 * anchor, which the call decodes into the handle's scratch row.  Malformed
 * records set the handle's sticky error word; gnm_pgen_check reports it. */
gnm_status gnm_pgen_decode(gnm_pgen* pg, uint64_t variant_begin, uint64_t variant_count,
                           uint8_t* d_rows, uint64_t pitch, void* stream, gnm_error* err);

/* Decode the listed variants (`count` indices, any order, each below the
 * variant count) into d_rows[i * pitch ..] = variant variants[i],
 * asynchronously on `stream`: e.g. the reconciled variants of a preparation
 * (required_bim_indices), which the reference's virtual .bed serves.  LD
 * anchors that are not listed are decoded into the handle's scratch rows. */
gnm_status gnm_pgen_decode_list(gnm_pgen* pg, const uint64_t* variants, uint64_t count,
                                uint8_t* d_rows, uint64_t pitch, void* stream, gnm_error* err);

/* Wait for `stream`, then GNM_ERR_IO if any record decoded so far was
 * malformed (the message names the first such variant). */
gnm_status gnm_pgen_check(gnm_pgen* pg, void* stream, gnm_error* err);

/* gnm_pgen_open with each variant's ALT allele count (the .pvar's ALT column,
 * 1..65535; the reference's VariantPlan alts_per_in, shared/adapt_plink2.rs:
 * 740-768): multiallelic records are accepted and decode per ALT.  As in the
 * reference, a record without a patch gives every ALT row the plain
 * categories, a patched record of a variant with one ALT reads as
 * biallelic, and only ALT 1 rows take dosages.  GNM_ERR_INVALID above
 * 928,000 samples when the file holds patched multiallelic records. */
gnm_status gnm_pgen_open_alleles(const uint8_t* pgen, uint64_t pgen_len,
                                 const uint32_t* alt_counts, int device, gnm_pgen** out,
                                 gnm_error* err);

/* gnm_pgen_decode_list where row i holds the copies of ALT alt_ords[i]
 * (1-based, at most the variant's ALT count) of variant variants[i]: the
 * reference's (in_idx, alt_ord) mapping of a virtual .bim row
 * (shared/adapt_plink2.rs:1295-1330). */
gnm_status gnm_pgen_decode_alleles(gnm_pgen* pg, const uint64_t* variants,
                                   const uint32_t* alt_ords, uint64_t count, uint8_t* d_rows,
                                   uint64_t pitch, void* stream, gnm_error* err);

/* gnm_score_run_ex with a .pgen (host bytes) as the genotype source: the
 * reference's virtual-.bed route (shared/adapt_plink2.rs:1093-1158), with the
 * decode on the device.  The .pgen's variants are the .bim rows
 * required_bim_indices point at; its sample count must equal
 * total_people_in_fam.  The reconciled variants are decoded and scored in
 * blocks of opts->block_variants (0 = as many as 4 GiB of rows hold);
 * opts->on_block is not called.  Same outputs and statuses as
 * gnm_score_run. */
gnm_status gnm_score_pgen(const gnm_prep_view* prep, const uint8_t* pgen, uint64_t pgen_len,
                          const gnm_run_options* opts, double* sums_out, uint32_t* missing_out,
                          gnm_error* err);

/* gnm_score_pgen over a virtual .bim that splits multiallelic variants:
 * .bim row r (what required_bim_indices index, bim_rows of them) holds ALT
 * bim_alt[r] of .pgen variant bim_variant[r]; alt_counts as for
 * gnm_pgen_open_alleles. */
gnm_status gnm_score_pgen_alleles(const gnm_prep_view* prep, const uint8_t* pgen,
                                  uint64_t pgen_len, const uint32_t* alt_counts,
                                  const uint64_t* bim_variant, const uint32_t* bim_alt,
                                  uint64_t bim_rows, const gnm_run_options* opts,
                                  double* sums_out, uint32_t* missing_out, gnm_error* err);

/* ---- HWE-PCA projection blocks --------------------------------------------
 * The GPU part of gnomon's projection onto a fitted HWE-PCA model
 * (map/project.rs): per variant block, every sample's genotype codes are
 * mapped through the block's per-variant coefficients (code 00 ->
 * coeffs[3v], 10 -> coeffs[3v+1], 11 -> coeffs[3v+2], missing (01) -> 0;
 * unpack_weighted_plink, map/project.rs:322-370) and multiplied by the
 * block's loadings (compute_scores_block, :547-667); the blocks' sums are
 * added into row-major f64 scores (:669-733).  The missing-data scan and the
 * per-sample solves that follow stay with the caller, as in the reference.
 * Engine per block: with 8 or more axes and coefficients linear in the
 * dosage up to their FP32 rounding (the reference's HWE coefficients), the
 * split-BF16 tensor engine, one pass for all axes; otherwise exact 3-variant
 * FP32 lookup tables, one pass per axis.  Both sum in FP32 within a block of
 * variants and in FP64 across (the reference: an FP32 SGEMM over the whole
 * projection). */
typedef struct gnm_projector gnm_projector;

/* A projection of n_samples samples onto `components` axes; GNM_DECLINED
 * without a device. */
gnm_status gnm_project_create(uint64_t n_samples, uint64_t components, int device,
                              gnm_projector** out, gnm_error* err);
void gnm_project_destroy(gnm_projector* pj);

/* One block of `filled` variants: packed .bed rows (host, ceil(n_samples/4)
 * bytes each, back to back), coeffs [filled][3] and column-major loadings
 * [components][filled] (f32, as the reference stages them).  Synchronous. */
gnm_status gnm_project_block(gnm_projector* pj, const uint8_t* packed, uint64_t filled,
                             const float* coeffs, const float* loadings_col_major,
                             gnm_error* err);

/* Add the projection's sums over every block so far into
 * scores_row_major[n_samples][components] (+=, like the reference's
 * copy-back). */
gnm_status gnm_project_scores(const gnm_projector* pj, double* scores_row_major, gnm_error* err);

/* ---- Allocation-free scoring ---------------------------------------------
 * No counterpart in the reference: an extra entry point of this library.
 *
 * Some callers cannot allocate device memory while they score: an application
 * that has already handed the whole device to its own caching allocator (a
 * cudaMalloc would fail, or force that allocator to give back cached blocks),
 * or a host that calls the scorer from a callback in which a device
 * allocation would implicitly synchronise the device and stall its other
 * streams.  gnm_score_noalloc scores one score column with the plain kernel
 * and allocates nothing: its scratch (the 3-variant stage tables of one chunk
 * of up to 48,840 variants at a time, FP64 partial sums and counts, the
 * baseline and the watchdog word) lives in one statically sized
 * device array of GNM_NOALLOC_SCRATCH_BYTES that every GPU loading this
 * library holds until process exit.  The caller passes inputs and outputs:
 *   d_rows                 packed rows (row v at d_rows + v*pitch, pitch a
 *                          multiple of 16, 16-byte aligned), every person of
 *                          the row scored (identity output order);
 *   d_dosage_weight,       [num_variants] FP32 dosage_weight and
 *   d_missing_correction   missing_correction of the score's cell;
 *   d_member               [num_variants] 1 = the variant is in the score,
 *                          0 = it is not (contributes nothing, its missing
 *                          calls are not counted); NULL = all members;
 *   baseline               the score's baseline (sum of corrections);
 *   d_sums_out, d_missing_out [num_people].
 * Limits: num_variants <= GNM_NOALLOC_MAX_VARIANTS and num_people <=
 * GNM_NOALLOC_MAX_PEOPLE; larger inputs are rejected with GNM_ERR_INVALID
 * before any device work.  The first call on a device looks up the scratch
 * array's device address (once per device, that device current), so make
 * that first call before any stream capture.  Every call reuses the same
 * array and clears what must start at zero; calls that overlap on the GPU
 * (other streams, other host threads) race on it and corrupt each other's
 * partial sums, so serialise the calls per device.  The call returns after
 * the work on `stream` has finished. */
#define GNM_NOALLOC_MAX_VARIANTS 262144u
#define GNM_NOALLOC_MAX_PEOPLE 65536u
#define GNM_NOALLOC_SCRATCH_BYTES 16778496u
gnm_status gnm_score_noalloc(const uint8_t* d_rows, uint64_t pitch, uint64_t num_variants,
                             uint64_t num_people, const float* d_dosage_weight,
                             const float* d_missing_correction, const uint8_t* d_member,
                             double baseline, double* d_sums_out, uint32_t* d_missing_out,
                             void* stream, gnm_error* err);

#ifdef __cplusplus
}
#endif

#endif /* GNOMON_GPU_H */
