// Allocation-free entry point: clipping of explicit tetrahedron pairs with
// all scratch memory in a fixed, file-scope device array.
//
// Some callers cannot let a library allocate device memory: applications
// whose GPU memory is owned by another pool allocator (a solver framework or
// a Python runtime that reserves the device up front, where a foreign
// cudaMalloc fails or disturbs the pool's accounting), and time-step loops
// that overlap work on several streams, where cudaFree's implicit device-wide
// synchronisation would serialise everything.  This entry point runs the same
// kernels as the context-based API (plane setup, exact early-out,
// persistent depth-first clipper, fixed-order reduction) but takes its
// scratch from g_scratch below, so it calls no cudaMalloc, cudaFree or other
// allocating routine.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/libsupermesh-gpu.h"
#include "lsm_geom.cuh"
#include "lsm_kernels.h"

namespace {

constexpr int64_t kMaxPairs = LSM_NOALLOC_MAX_PAIRS;
constexpr size_t kAlign = 256;

constexpr size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Scratch layout (byte offsets, 256-aligned).
constexpr size_t kOffSetup = 0;                                                      // [n][kSetup3] f64
constexpr size_t kOffTol = align_up(kOffSetup + sizeof(double) * lsm::kSetup3 * kMaxPairs);  // [n] f64
constexpr size_t kOffIota = align_up(kOffTol + sizeof(double) * kMaxPairs);              // [n] i32
constexpr size_t kOffList = align_up(kOffIota + sizeof(int32_t) * kMaxPairs);            // [n] survivor records
constexpr size_t kOffWork = align_up(kOffList + 4 * sizeof(int32_t) * kMaxPairs);        // misc counters
constexpr size_t kWorkBytes = 256;
constexpr size_t kOffPartials = align_up(kOffWork + kWorkBytes);                         // reduction partials
constexpr size_t kOffTotal = align_up(kOffPartials + sizeof(lsm::Partial) * lsm::kReduceBlocks);
constexpr size_t kScratchBytes = align_up(kOffTotal + sizeof(lsm::Partial));

static_assert(kScratchBytes == LSM_NOALLOC_SCRATCH_BYTES, "keep the header's scratch size in sync");
static_assert(lsm::kReduceBlocks == 1024, "the partials region holds one Partial per reduce block");

// Every GPU that loads the library holds this array until the process exits.
// All calls share it: it keeps the previous call's contents, and calls that
// overlap on the GPU (from different host threads or streams) race on it.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch per device, obtained once per device with that
// device current (the symbol's host-side name is not a device address).
std::mutex g_mu;
void* g_addr[64] = {};

int scratch_address(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return LSM_ERROR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) {
      (void)cudaGetLastError();
      return LSM_ERROR_CUDA;
    }
    if (lsm::init_device_attributes() != cudaSuccess) {
      (void)cudaGetLastError();
      return LSM_ERROR_CUDA;
    }
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return LSM_SUCCESS;
}

}  // namespace

extern "C" int libsupermesh_gpu_intersect_tets_noalloc(int64_t n, const double* tet_a, const double* tet_b,
                                                       double* measure, int32_t* n_out, double* total,
                                                       void* stream) {
  if (n < 0 || n > kMaxPairs) {
    fprintf(stderr,
            "libsupermesh_gpu_intersect_tets_noalloc: %lld pairs requested, the fixed scratch holds at most "
            "%lld\n",
            (long long)n, (long long)kMaxPairs);
    return LSM_ERROR_CAPACITY;
  }
  if (n > 0 && (!tet_a || !tet_b || !measure || !n_out)) return LSM_ERROR_INVALID_ARGUMENT;
  // the clipper reads each tetrahedron as six 16-byte loads: a pair array
  // that starts off a 16-byte boundary (a view at an odd double offset) is
  // refused here instead of faulting on the device
  if (n > 0 && (((uintptr_t)tet_a | (uintptr_t)tet_b) & 15u) != 0) {
    fprintf(stderr, "libsupermesh_gpu_intersect_tets_noalloc: tet_a and tet_b must be 16-byte aligned\n");
    return LSM_ERROR_INVALID_ARGUMENT;
  }
  void* base = nullptr;
  const int st = scratch_address(&base);
  if (st != LSM_SUCCESS) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char* b = static_cast<unsigned char*>(base);
  double* setup = reinterpret_cast<double*>(b + kOffSetup);
  double* tol = reinterpret_cast<double*>(b + kOffTol);
  int32_t* iota = reinterpret_cast<int32_t*>(b + kOffIota);
  int32_t* list = reinterpret_cast<int32_t*>(b + kOffList);
  unsigned long long* work = reinterpret_cast<unsigned long long*>(b + kOffWork);
  lsm::Partial* partials = reinterpret_cast<lsm::Partial*>(b + kOffPartials);
  lsm::Partial* tot = reinterpret_cast<lsm::Partial*>(b + kOffTotal);
  if (n > 0) {
    // B's planes and tolerance, A's tolerance and the identity pair indices
    if (lsm::launch_setup_pairs3(n, tet_a, tet_b, setup, tol, iota, nullptr, nullptr, s) != cudaSuccess)
      return LSM_ERROR_CUDA;
    // launch_clip clears the two work counters (survivors, progress) first
    if (lsm::launch_clip(3, n, iota, iota, tet_a, tol, setup, measure, n_out, list, nullptr, work, s) !=
        cudaSuccess)
      return LSM_ERROR_CUDA;
  }
  if (lsm::launch_reduce_pairs(n, measure, n_out, partials, s) != cudaSuccess ||
      lsm::launch_finalize(partials, lsm::reduce_pairs_blocks(), tot, s) != cudaSuccess)
    return LSM_ERROR_CUDA;
  if (total) {
    lsm::Partial h;
    if (cudaMemcpyAsync(&h, tot, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return LSM_ERROR_CUDA;
    *total = h.sum;
  }
  // every launch above was checked where it was issued; an error pending
  // from other work on this thread is left for its owner
  return LSM_SUCCESS;
}
