// Measurement probe (not part of the supermesh API): the FP64 arithmetic
// ceiling that the clipping kernels run against.  The clipper is compiled
// without FMA contraction, so its ceiling is the issue rate of separate
// DADD/DMUL instructions; the probe measures that rate (and, for context,
// the DFMA rate) with long chains of independent operations.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) k_dadd_dmul(double seed, double* sink) {
  double x[kChains];
#pragma unroll
  for (int i = 0; i < kChains; ++i) x[i] = seed + i + threadIdx.x * 1e-9;
  const double m = 1.0000000001, a = 1e-12;
  for (int it = 0; it < kIters; ++it) {
#pragma unroll
    for (int i = 0; i < kChains; ++i) {
      x[i] = __dmul_rn(x[i], m);
      x[i] = __dadd_rn(x[i], a);
    }
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kChains; ++i) s += x[i];
  if (s == 12345.678) sink[0] = s;
}

__global__ void __launch_bounds__(256) k_dfma(double seed, double* sink) {
  double x[kChains];
#pragma unroll
  for (int i = 0; i < kChains; ++i) x[i] = seed + i + threadIdx.x * 1e-9;
  const double m = 1.0000000001, a = 1e-12;
  for (int it = 0; it < kIters; ++it) {
#pragma unroll
    for (int i = 0; i < kChains; ++i) x[i] = __fma_rn(x[i], m, a);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kChains; ++i) s += x[i];
  if (s == 12345.678) sink[0] = s;
}

}  // namespace

extern "C" {

// Returns FP64 operations per second: mode 0 = separate DADD+DMUL (1 op
// each), mode 1 = DFMA (2 ops each).  Timed with CUDA events, best of
// `reps` launches of blocks_per_sm * SMs blocks of 256 threads.
double lsm_probe_fp64_rate(int mode, int reps) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double* sink = nullptr;
  if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8;
  const double ops_per_thread = (double)kIters * kChains * 2.0;
  double best = 0.0;
  for (int r = 0; r < reps + 1; ++r) {
    cudaEventRecord(e0);
    if (mode == 0)
      k_dadd_dmul<<<blocks, 256>>>(1.0, sink);
    else
      k_dfma<<<blocks, 256>>>(1.0, sink);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r == 0 || ms <= 0.f) continue;  // first launch warms up
    const double rate = ops_per_thread * blocks * 256.0 / (ms * 1e-3);
    if (rate > best) best = rate;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  return cudaGetLastError() == cudaSuccess ? best : -1.0;
}

// Writes `bytes` of zeros to evict the L2 cache between timed steps.
int lsm_probe_flush_l2(void* buf, int64_t bytes, void* stream) {
  return (int)cudaMemsetAsync(buf, 0, (size_t)bytes, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
