// Learned scheduler of the tet clipper (lsm_sched.cu): parameter layout,
// device weight image and launchers.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace lsm {

// MLP 24 -> 64 -> 64 -> 4 (ReLU).  FP32 parameter vector, row-major
// [out][in] weight blocks, inputs padded to 32 and outputs of the last layer
// to 8 (the padding entries are zero and are never trained).
constexpr int kSchedIn = 24;
constexpr int kSchedInPad = 32;
constexpr int kSchedHidden = 64;
constexpr int kSchedClasses = 4;
constexpr int kSchedOffW1 = 0;                                     // [64][32]
constexpr int kSchedOffB1 = kSchedOffW1 + kSchedHidden * kSchedInPad;  // [64]
constexpr int kSchedOffW2 = kSchedOffB1 + kSchedHidden;             // [64][64]
constexpr int kSchedOffB2 = kSchedOffW2 + kSchedHidden * kSchedHidden;  // [64]
constexpr int kSchedOffW3 = kSchedOffB2 + kSchedHidden;             // [8][64]
constexpr int kSchedOffB3 = kSchedOffW3 + 8 * kSchedHidden;         // [8]
constexpr int kSchedParams = kSchedOffB3 + 8;                       // 6792
constexpr int kSchedBatch = 128;                                    // training minibatch (8 warps x 16)

// Device image used for inference: BF16 weights, FP32 biases (b3 of the
// padding classes is -FLT_MAX so they never win).
struct SchedWeights {
  __nv_bfloat16 w1[kSchedHidden * kSchedInPad];
  __nv_bfloat16 w2[kSchedHidden * kSchedHidden];
  __nv_bfloat16 w3[8 * kSchedHidden];
  float b1[kSchedHidden];
  float b2[kSchedHidden];
  float b3[8];
};

// Binning of the clipper's work list (see k_sched_bin).  Classes come from
// the MLP (weights) or, when cls_of_pair is set, from that per-candidate
// array; pred_of_pair (optional) receives each survivor's class.
struct SchedBin {
  const SchedWeights* weights = nullptr;
  const int8_t* cls_of_pair = nullptr;
  int8_t* pred_of_pair = nullptr;
  const double* screen_b = nullptr;  // B's vertices (kScreen3 rows)
  int4* out = nullptr;               // binned list, as many entries as the survivors
  int4* flat = nullptr;              // (optional) the survivor segments gathered into one list first
  int window = 1024;
};

constexpr int kSchedMaxWindow = 8192;

size_t sched_bin_smem_bytes(int window);
size_t sched_train_smem_bytes();
cudaError_t init_sched_attributes(int max_window);
cudaError_t launch_sched_pack(const float* params, SchedWeights* w, cudaStream_t s);
cudaError_t launch_sched_true_class(int64_t n, const int32_t* n_out, int8_t* cls, cudaStream_t s);
cudaError_t launch_sched_bin(const SchedBin& b, const int4* in, const unsigned long long* nlist, int4* out,
                             const double* coords_a, cudaStream_t s);
cudaError_t launch_sched_samples(const int4* list, const unsigned long long* nlist, int64_t cap, const double* coords_a,
                                 const double* screen_b, const int32_t* n_out, void* x, int8_t* y, cudaStream_t s);
cudaError_t launch_sched_predict(int64_t n, const void* x, const SchedWeights* w, float* logits, int8_t* cls,
                                 cudaStream_t s);
cudaError_t launch_sched_train(const void* x, const int8_t* y, int64_t n, float* params, float* adam, int steps,
                               float lr, float* loss_trace, int trace_every, float* grad_first, cudaStream_t s);

}  // namespace lsm
