// gnm_tensor.h — split-BF16 tcgen05 engine and the backward kernel (host entry points).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

struct gnm_plan;
struct gnm_prep_view;

namespace gnm {

// AUTO picks the tensor engine from this many score columns on: one narrow
// tensor pass (a 16-score tile) costs about as much as seven single-score plain
// passes over the same rows (measured on B200: 20,000 x 200,000, 16 scores,
// 2.25 ms against 16 x 0.33 ms).
constexpr uint64_t kTensorMinScores = 8;

// Smallest row block the end-to-end call splits the tensor engine's rows into.
constexpr uint64_t kTensorMinBlock = 16384;

struct PhaseTrace;
// Builds the limb planes from the caller's CSR (read during the call only).
void tensor_plan_create(gnm_plan* p, const gnm_prep_view* prep, PhaseTrace* trace);
void tensor_plan_destroy(gnm_plan* p);
void tensor_reset(gnm_plan* p, cudaStream_t s);
// Up to 64 scores either tensor kernel can run a plan: the narrow one (people
// as the MMA's M, the default) or the wide one (scores as M).
bool tensor_can_narrow(const gnm_plan* p);
bool tensor_is_narrow(const gnm_plan* p);
void tensor_set_narrow(gnm_plan* p, bool narrow);
// The wide GEMM on 8-bit limbs (gnm_t8_accumulate) instead of BF16 limbs.
bool tensor_is_i8(const gnm_plan* p);
void tensor_set_i8(gnm_plan* p, bool i8);
// The 8-bit wide GEMM over SM pairs (gnm_t8_pair, cta_group::2).
bool tensor_is_pair(const gnm_plan* p);
void tensor_set_pair(gnm_plan* p, bool pair);
void tensor_accumulate(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch, uint64_t v0,
                       uint64_t nv, cudaStream_t s);
void tensor_finalize(gnm_plan* p, double* d_sums, uint32_t* d_counts, bool add_baseline,
                     cudaStream_t s);
void backward_dw(gnm_plan* p, const uint8_t* d_rows, uint64_t pitch, const float* d_grad_s,
                 float* d_grad_w, float* d_grad_corr, cudaStream_t s);

}  // namespace gnm
