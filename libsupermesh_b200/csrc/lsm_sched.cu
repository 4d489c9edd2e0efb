// Learned scheduler of the tet clipper: a small MLP that predicts each
// surviving candidate pair's output-size class (0: no tets, 1: 1-3, 2: 4-7,
// 3: 8 or more) from the pair's normalised vertices, used only to reorder
// the clipper's work list into class-uniform runs.  Every pair is still
// clipped exactly; the order never changes a result (each pair's measure and
// count are stored at its own index).
//
// Network: 24 inputs (A's and B's four vertices, centred on the mean of the
// eight and divided by the longest of the twelve edges), two hidden layers of
// 64 ReLU units, 4 logits.  Weights BF16, accumulation FP32, on the tensor
// cores through mma.sync.m16n8k16 (one warp per 16-row tile); the output of
// one layer is turned into the next layer's A fragments in registers.
//
// Kernels
//   k_sched_bin       the prefilter's survivor records, window by window:
//                     classes (MLP, or given per pair), then a stable
//                     partition of the window by class, heaviest first
//   k_sched_samples   training samples (features, class) of the survivors of
//                     a plain narrow phase, labelled by the clipper's counts
//   k_sched_predict   logits and classes of given feature rows
//   k_sched_train     minibatch Adam on the cross-entropy loss, forward and
//                     backward on the tensor cores, one persistent block
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "lsm_geom.cuh"
#include "lsm_kernels.h"
#include "lsm_sched.h"

namespace lsm {

namespace {

constexpr int kSW1 = 40;  // bf16 row stride of W1 in shared memory (32 + pad)
constexpr int kSW2 = 72;  // W2, W3, activations (64 + pad)

// Weights staged in shared memory as BF16 (padded rows: the B-fragment loads
// of one mma hit 32 different banks) and biases as FP32.
struct SchedSmem {
  __nv_bfloat16 w1[kSchedHidden * kSW1];
  __nv_bfloat16 w2[kSchedHidden * kSW2];
  __nv_bfloat16 w3[8 * kSW2];
  float b1[kSchedHidden];
  float b2[kSchedHidden];
  float b3[8];
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// D += A (16x16, row-major bf16) * B (16x8, col-major bf16), FP32 accumulate.
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Stage the device weights (kSchedParams FP32 values in the layout of
// lsm_sched.h, or their BF16 image) into shared memory.
__device__ void stage_weights(const SchedWeights* __restrict__ w, SchedSmem& s) {
  for (int i = threadIdx.x; i < kSchedHidden * kSchedInPad; i += blockDim.x)
    s.w1[(i / kSchedInPad) * kSW1 + i % kSchedInPad] = w->w1[i];
  for (int i = threadIdx.x; i < kSchedHidden * kSchedHidden; i += blockDim.x)
    s.w2[(i / kSchedHidden) * kSW2 + i % kSchedHidden] = w->w2[i];
  for (int i = threadIdx.x; i < 8 * kSchedHidden; i += blockDim.x)
    s.w3[(i / kSchedHidden) * kSW2 + i % kSchedHidden] = w->w3[i];
  for (int i = threadIdx.x; i < kSchedHidden; i += blockDim.x) {
    s.b1[i] = w->b1[i];
    s.b2[i] = w->b2[i];
  }
  for (int i = threadIdx.x; i < 8; i += blockDim.x) s.b3[i] = w->b3[i];
}

// Forward pass of one 16-row tile whose inputs are rows r0 .. r0+15 of x
// (bf16, row stride kSW1).  h1 / h2 (optional, row stride kSW2) receive the
// post-ReLU activations as BF16 (training).  logit[0..3] of this lane: rows
// g (o[0], o[1]: classes 2t, 2t+1) and g+8 (o[2], o[3]).
__device__ __forceinline__ void mlp_tile(const SchedSmem& s, const __nv_bfloat16* x, float (&o)[4],
                                         __nv_bfloat16* h1 = nullptr, __nv_bfloat16* h2 = nullptr) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  uint32_t a[4][4];
#pragma unroll
  for (int kb = 0; kb < 2; ++kb) {
    a[kb][0] = ld32(x + g * kSW1 + kb * 16 + 2 * t);
    a[kb][1] = ld32(x + (g + 8) * kSW1 + kb * 16 + 2 * t);
    a[kb][2] = ld32(x + g * kSW1 + kb * 16 + 8 + 2 * t);
    a[kb][3] = ld32(x + (g + 8) * kSW1 + kb * 16 + 8 + 2 * t);
  }
  float h[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int c = nt * 8 + 2 * t;
    h[nt][0] = h[nt][2] = s.b1[c];
    h[nt][1] = h[nt][3] = s.b1[c + 1];
    const __nv_bfloat16* wr = s.w1 + (nt * 8 + g) * kSW1;
#pragma unroll
    for (int kb = 0; kb < 2; ++kb) mma16816(h[nt], a[kb], ld32(wr + kb * 16 + 2 * t), ld32(wr + kb * 16 + 8 + 2 * t));
  }
  // ReLU; the C fragments of n-tiles 2k and 2k+1 are the A fragment of k-block k
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int j = 0; j < 4; ++j) h[nt][j] = fmaxf(h[nt][j], 0.0f);
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    a[kb][0] = pack_bf16(h[2 * kb][0], h[2 * kb][1]);
    a[kb][1] = pack_bf16(h[2 * kb][2], h[2 * kb][3]);
    a[kb][2] = pack_bf16(h[2 * kb + 1][0], h[2 * kb + 1][1]);
    a[kb][3] = pack_bf16(h[2 * kb + 1][2], h[2 * kb + 1][3]);
  }
  if (h1) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      *reinterpret_cast<uint32_t*>(h1 + g * kSW2 + nt * 8 + 2 * t) = pack_bf16(h[nt][0], h[nt][1]);
      *reinterpret_cast<uint32_t*>(h1 + (g + 8) * kSW2 + nt * 8 + 2 * t) = pack_bf16(h[nt][2], h[nt][3]);
    }
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int c = nt * 8 + 2 * t;
    h[nt][0] = h[nt][2] = s.b2[c];
    h[nt][1] = h[nt][3] = s.b2[c + 1];
    const __nv_bfloat16* wr = s.w2 + (nt * 8 + g) * kSW2;
#pragma unroll
    for (int kb = 0; kb < 4; ++kb) mma16816(h[nt], a[kb], ld32(wr + kb * 16 + 2 * t), ld32(wr + kb * 16 + 8 + 2 * t));
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int j = 0; j < 4; ++j) h[nt][j] = fmaxf(h[nt][j], 0.0f);
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) {
    a[kb][0] = pack_bf16(h[2 * kb][0], h[2 * kb][1]);
    a[kb][1] = pack_bf16(h[2 * kb][2], h[2 * kb][3]);
    a[kb][2] = pack_bf16(h[2 * kb + 1][0], h[2 * kb + 1][1]);
    a[kb][3] = pack_bf16(h[2 * kb + 1][2], h[2 * kb + 1][3]);
  }
  if (h2) {
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      *reinterpret_cast<uint32_t*>(h2 + g * kSW2 + nt * 8 + 2 * t) = pack_bf16(h[nt][0], h[nt][1]);
      *reinterpret_cast<uint32_t*>(h2 + (g + 8) * kSW2 + nt * 8 + 2 * t) = pack_bf16(h[nt][2], h[nt][3]);
    }
  }
  o[0] = o[2] = s.b3[2 * t];
  o[1] = o[3] = s.b3[2 * t + 1];
  const __nv_bfloat16* wr = s.w3 + g * kSW2;
#pragma unroll
  for (int kb = 0; kb < 4; ++kb) mma16816(o, a[kb], ld32(wr + kb * 16 + 2 * t), ld32(wr + kb * 16 + 8 + 2 * t));
}

// Class of rows g and g+8 from a tile's logits (lanes t = 0, 1 of each quad
// hold classes 0-1 and 2-3; ties go to the lower class).  Valid in lanes
// with t == 0.
__device__ __forceinline__ void tile_argmax(const float (&o)[4], int& c_lo, int& c_hi) {
  const int t = threadIdx.x & 3;
  float v_lo = o[0] >= o[1] ? o[0] : o[1];
  int k_lo = o[0] >= o[1] ? 2 * t : 2 * t + 1;
  float v_hi = o[2] >= o[3] ? o[2] : o[3];
  int k_hi = o[2] >= o[3] ? 2 * t : 2 * t + 1;
  const float w_lo = __shfl_xor_sync(0xffffffffu, v_lo, 1), w_hi = __shfl_xor_sync(0xffffffffu, v_hi, 1);
  const int j_lo = __shfl_xor_sync(0xffffffffu, k_lo, 1), j_hi = __shfl_xor_sync(0xffffffffu, k_hi, 1);
  c_lo = w_lo > v_lo ? j_lo : k_lo;  // lane t = 0 holds classes 0-1, its partner 2-3
  c_hi = w_hi > v_hi ? j_hi : k_hi;
}

// Output-size class of a clipped pair from its number of output tets.
__device__ __forceinline__ int size_class(int n_out) { return n_out <= 0 ? 0 : (n_out <= 3 ? 1 : (n_out <= 7 ? 2 : 3)); }

// Features of one pair (FP64 arithmetic, BF16 result): A's vertices then B's,
// (x, y, z) each, minus the mean of the eight vertices, divided by the
// longest edge of the two tets.  Columns 24..31 are zero.
__device__ __forceinline__ void pair_features(const double* __restrict__ coords_a, const double* __restrict__ screen_b,
                                              int a, int b, __nv_bfloat16* row) {
  Tet ta, tb;
  {
    const double* p = coords_a + (int64_t)a * 12;
    const double* q = screen_b + (int64_t)b * kScreen3;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      ta.x[k] = __ldg(p + 3 * k);
      ta.y[k] = __ldg(p + 3 * k + 1);
      ta.z[k] = __ldg(p + 3 * k + 2);
      tb.x[k] = __ldg(q + 3 * k);
      tb.y[k] = __ldg(q + 3 * k + 1);
      tb.z[k] = __ldg(q + 3 * k + 2);
    }
  }
  double cx = 0.0, cy = 0.0, cz = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    cx += ta.x[k] + tb.x[k];
    cy += ta.y[k] + tb.y[k];
    cz += ta.z[k] + tb.z[k];
  }
  cx *= 0.125;
  cy *= 0.125;
  cz *= 0.125;
  double l2 = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = i + 1; j < 4; ++j) {
      const double ax = ta.x[i] - ta.x[j], ay = ta.y[i] - ta.y[j], az = ta.z[i] - ta.z[j];
      const double bx = tb.x[i] - tb.x[j], by = tb.y[i] - tb.y[j], bz = tb.z[i] - tb.z[j];
      l2 = fmax(l2, fmax(ax * ax + ay * ay + az * az, bx * bx + by * by + bz * bz));
    }
  const double inv = l2 > 0.0 ? 1.0 / sqrt(l2) : 0.0;
  float f[32];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    f[3 * k] = (float)((ta.x[k] - cx) * inv);
    f[3 * k + 1] = (float)((ta.y[k] - cy) * inv);
    f[3 * k + 2] = (float)((ta.z[k] - cz) * inv);
    f[12 + 3 * k] = (float)((tb.x[k] - cx) * inv);
    f[12 + 3 * k + 1] = (float)((tb.y[k] - cy) * inv);
    f[12 + 3 * k + 2] = (float)((tb.z[k] - cz) * inv);
  }
#pragma unroll
  for (int k = 24; k < 32; ++k) f[k] = 0.0f;
#pragma unroll
  for (int k = 0; k < 32; k += 2) *reinterpret_cast<uint32_t*>(row + k) = pack_bf16(f[k], f[k + 1]);
}

}  // namespace

// ---------------------------------------------------------------- binning
// One block per window of `window` survivor records (persistent over the
// windows).  Each warp classifies 32 records at a time: every lane builds
// one record's features in its warp's tile, then two 16-row MLP tiles run
// on the tensor cores (or the class comes from cls_of_pair).  The window is
// then written to `out` at the same offset, stably partitioned by class,
// heaviest class first, so the clipper's warps take class-uniform runs while
// the pairs stay within their window (spatially close: the survivor list
// follows the candidate order).
__global__ void __launch_bounds__(256) k_sched_bin(const int4* __restrict__ in, const unsigned long long* __restrict__ nlist,
                                                   int4* out, const double* __restrict__ coords_a,
                                                   const double* __restrict__ screen_b,
                                                   const SchedWeights* __restrict__ w,
                                                   const int8_t* __restrict__ cls_of_pair, int8_t* pred_of_pair,
                                                   int window) {
  extern __shared__ __align__(16) unsigned char sm[];
  SchedSmem& s = *reinterpret_cast<SchedSmem*>(sm);
  __nv_bfloat16* xt = reinterpret_cast<__nv_bfloat16*>(sm + sizeof(SchedSmem)) + (threadIdx.x >> 5) * 32 * kSW1;
  int4* rec = reinterpret_cast<int4*>(sm + sizeof(SchedSmem) + 8 * 32 * kSW1 * sizeof(__nv_bfloat16));
  unsigned char* cls = reinterpret_cast<unsigned char*>(rec + window);
  __shared__ int cnt[4], base[4], wsum[8][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const int64_t n = (int64_t)*nlist;
  if (!cls_of_pair) stage_weights(w, s);
  for (int64_t w0 = (int64_t)blockIdx.x * window; w0 < n; w0 += (int64_t)gridDim.x * window) {
    const int nw = (int)(n - w0 < window ? n - w0 : window);
    __syncthreads();  // previous window's records and classes are written out
    for (int i = threadIdx.x; i < nw; i += blockDim.x) rec[i] = in[w0 + i];
    if (threadIdx.x < 4) cnt[threadIdx.x] = 0;
    __syncthreads();
    for (int r0 = warp * 32; r0 < nw; r0 += 8 * 32) {
      const int r = r0 + lane;
      if (cls_of_pair) {
        if (r < nw) cls[r] = (unsigned char)cls_of_pair[rec[r].x];
        continue;
      }
      if (r < nw) {
        pair_features(coords_a, screen_b, rec[r].y, rec[r].z, xt + lane * kSW1);
      } else {
#pragma unroll
        for (int k = 0; k < 32; k += 2) *reinterpret_cast<uint32_t*>(xt + lane * kSW1 + k) = 0u;
      }
      __syncwarp();
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        float o[4];
        mlp_tile(s, xt + mt * 16 * kSW1, o);
        int c_lo, c_hi;
        tile_argmax(o, c_lo, c_hi);
        const int ra = r0 + mt * 16 + g, rb = ra + 8;
        if (t == 0) {
          if (ra < nw) cls[ra] = (unsigned char)c_lo;
          if (rb < nw) cls[rb] = (unsigned char)c_hi;
        }
      }
      __syncwarp();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nw; i += blockDim.x) {
      atomicAdd(&cnt[cls[i]], 1);
      if (pred_of_pair) pred_of_pair[rec[i].x] = (int8_t)cls[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // heaviest class first
      base[3] = 0;
      base[2] = cnt[3];
      base[1] = cnt[3] + cnt[2];
      base[0] = cnt[3] + cnt[2] + cnt[1];
    }
    // stable scatter, 256 records per round
    for (int c0 = 0; c0 < nw; c0 += 256) {
      __syncthreads();
      const int i = c0 + threadIdx.x;
      const int k = i < nw ? cls[i] : -1;
      unsigned m[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) m[q] = __ballot_sync(0xffffffffu, k == q);
      if (lane < 4) wsum[warp][lane] = __popc(m[lane]);
      __syncthreads();
      if (k >= 0) {
        int before = 0;
        for (int v = 0; v < warp; ++v) before += wsum[v][k];
        const int pos = base[k] + before + __popc(m[k] & ((1u << lane) - 1u));
        out[w0 + pos] = rec[i];
      }
      __syncthreads();
      if (threadIdx.x < 4) {
        int tot = 0;
        for (int v = 0; v < 8; ++v) tot += wsum[v][threadIdx.x];
        base[threadIdx.x] += tot;
      }
    }
  }
}

size_t sched_bin_smem_bytes(int window) {
  return sizeof(SchedSmem) + 8 * 32 * kSW1 * sizeof(__nv_bfloat16) + (size_t)window * (sizeof(int4) + 1);
}

// Classes per pair from the counts of an earlier narrow phase over the same
// candidates (the true classes: the scheduler's best case).
__global__ void k_sched_true_class(int64_t n, const int32_t* __restrict__ n_out, int8_t* cls) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    cls[i] = (int8_t)size_class(n_out[i]);
}

// ---------------------------------------------------------------- samples
// Training samples from the survivors of a plain narrow phase: features of
// survivor j in x[j], class of its output count in y[j] (j < min(n, cap)).
__global__ void k_sched_samples(const int4* __restrict__ list, const unsigned long long* __restrict__ nlist,
                                int64_t cap, const double* __restrict__ coords_a, const double* __restrict__ screen_b,
                                const int32_t* __restrict__ n_out, __nv_bfloat16* x, int8_t* y) {
  const int64_t n = (int64_t)*nlist < cap ? (int64_t)*nlist : cap;
  __nv_bfloat16 row[32];
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const int4 r = list[j];
    pair_features(coords_a, screen_b, r.y, r.z, row);
    uint4* dst = reinterpret_cast<uint4*>(x + j * kSchedInPad);
#pragma unroll
    for (int q = 0; q < 4; ++q) dst[q] = reinterpret_cast<const uint4*>(row)[q];
    y[j] = (int8_t)size_class(n_out[r.x]);
  }
}

// ---------------------------------------------------------------- predict
// Logits (optional, [n][4] FP32) and classes ([n]) of feature rows x[n][32].
__global__ void __launch_bounds__(256) k_sched_predict(int64_t n, const __nv_bfloat16* __restrict__ x,
                                                       const SchedWeights* __restrict__ w, float* logits,
                                                       int8_t* cls) {
  extern __shared__ __align__(16) unsigned char sm[];
  SchedSmem& s = *reinterpret_cast<SchedSmem*>(sm);
  __nv_bfloat16* xt = reinterpret_cast<__nv_bfloat16*>(sm + sizeof(SchedSmem)) + (threadIdx.x >> 5) * 16 * kSW1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  stage_weights(w, s);
  __syncthreads();
  for (int64_t r0 = ((int64_t)blockIdx.x * 8 + warp) * 16; r0 < n; r0 += (int64_t)gridDim.x * 8 * 16) {
    // lanes 0..15 copy one row each
    if (lane < 16) {
      const int64_t r = r0 + lane;
      uint4* d = reinterpret_cast<uint4*>(xt + lane * kSW1);
      if (r < n) {
        const uint4* src = reinterpret_cast<const uint4*>(x + r * kSchedInPad);
#pragma unroll
        for (int q = 0; q < 4; ++q) d[q] = src[q];
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) d[q] = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    __syncwarp();
    float o[4];
    mlp_tile(s, xt, o);
    int c_lo, c_hi;
    tile_argmax(o, c_lo, c_hi);
    const int64_t ra = r0 + g, rb = ra + 8;
    if (logits && t < 2) {
      if (ra < n) {
        logits[ra * 4 + 2 * t] = o[0];
        logits[ra * 4 + 2 * t + 1] = o[1];
      }
      if (rb < n) {
        logits[rb * 4 + 2 * t] = o[2];
        logits[rb * 4 + 2 * t + 1] = o[3];
      }
    }
    if (t == 0) {
      if (ra < n) cls[ra] = (int8_t)c_lo;
      if (rb < n) cls[rb] = (int8_t)c_hi;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- training
// One persistent block of 8 warps; a step takes a minibatch of 128 rows (16
// per warp: rows (step*128 + 16*warp + r) mod n, so callers shuffle the
// samples first), runs the forward pass, the softmax cross-entropy
// gradient, and the backward pass:
//   dW3 = dL^T H2, dH2 = (dL W3) * [H2 > 0], dW2 = dH2^T H1,
//   dH1 = (dH2 W2) * [H1 > 0],  dW1 = dH1^T X,  db = column sums,
// every product an mma.sync over 16-sample K blocks (BF16 operands, FP32
// accumulation, summed over the warps in shared memory), then an Adam step
// on the FP32 master weights (moments in `adam`, 2 * kSchedParams floats)
// with the learning rate decayed from lr to 0 along a half cosine.
// Padding entries (W1 columns 24..31, W3 rows 4..7, b3[4..7]) stay fixed.
namespace {
struct TrainWarp {
  __nv_bfloat16 x[16 * kSW1];
  __nv_bfloat16 h1[16 * kSW2];
  __nv_bfloat16 h2[16 * kSW2];
  __nv_bfloat16 d2[16 * kSW2];
  __nv_bfloat16 d1[16 * kSW2];
  __nv_bfloat16 dl[16 * 8];
  float dlf[16 * 4];
  int y[16];
};

__device__ __forceinline__ bool is_pad_param(int p) {
  if (p >= kSchedOffW1 && p < kSchedOffW1 + kSchedHidden * kSchedInPad) return (p - kSchedOffW1) % kSchedInPad >= kSchedIn;
  if (p >= kSchedOffW3 && p < kSchedOffW3 + 8 * kSchedHidden) return (p - kSchedOffW3) / kSchedHidden >= kSchedClasses;
  if (p >= kSchedOffB3 && p < kSchedOffB3 + 8) return p - kSchedOffB3 >= kSchedClasses;
  return false;
}

// BF16 image (and FP32 biases) of the master weights for the forward pass.
__device__ void refresh_smem(const float* __restrict__ P, SchedSmem& s) {
  for (int i = threadIdx.x; i < kSchedHidden * kSchedInPad; i += blockDim.x)
    s.w1[(i / kSchedInPad) * kSW1 + i % kSchedInPad] = __float2bfloat16_rn(P[kSchedOffW1 + i]);
  for (int i = threadIdx.x; i < kSchedHidden * kSchedHidden; i += blockDim.x)
    s.w2[(i / kSchedHidden) * kSW2 + i % kSchedHidden] = __float2bfloat16_rn(P[kSchedOffW2 + i]);
  for (int i = threadIdx.x; i < 8 * kSchedHidden; i += blockDim.x)
    s.w3[(i / kSchedHidden) * kSW2 + i % kSchedHidden] = __float2bfloat16_rn(P[kSchedOffW3 + i]);
  for (int i = threadIdx.x; i < kSchedHidden; i += blockDim.x) {
    s.b1[i] = P[kSchedOffB1 + i];
    s.b2[i] = P[kSchedOffB2 + i];
  }
  for (int i = threadIdx.x; i < 8; i += blockDim.x) s.b3[i] = P[kSchedOffB3 + i];
}
}  // namespace

__global__ void __launch_bounds__(256, 1) k_sched_train(const __nv_bfloat16* __restrict__ x, const int8_t* __restrict__ y,
                                                        int64_t n, float* params, float* adam, int steps, float lr,
                                                        float* loss_trace, int trace_every, float* grad_first) {
  extern __shared__ __align__(16) unsigned char sm[];
  float* P = reinterpret_cast<float*>(sm);
  float* G = P + kSchedParams;
  SchedSmem& s = *reinterpret_cast<SchedSmem*>(G + kSchedParams);
  TrainWarp& tw = reinterpret_cast<TrainWarp*>(reinterpret_cast<unsigned char*>(&s) + sizeof(SchedSmem))[threadIdx.x >> 5];
  __shared__ float loss_sum;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  const float inv_batch = 1.0f / (float)kSchedBatch;
  for (int i = threadIdx.x; i < kSchedParams; i += blockDim.x) {
    P[i] = params[i];
    G[i] = 0.0f;
    adam[i] = 0.0f;
    adam[kSchedParams + i] = 0.0f;
  }
  if (threadIdx.x == 0) loss_sum = 0.0f;
  __syncthreads();
  refresh_smem(P, s);
  __syncthreads();
  float b1t = 1.0f, b2t = 1.0f;
  for (int step = 0; step < steps; ++step) {
    // ---- minibatch rows of this warp
    if (lane < 16) {
      const int64_t r = ((int64_t)step * kSchedBatch + warp * 16 + lane) % n;
      const uint4* src = reinterpret_cast<const uint4*>(x + r * kSchedInPad);
      uint4* d = reinterpret_cast<uint4*>(tw.x + lane * kSW1);
#pragma unroll
      for (int q = 0; q < 4; ++q) d[q] = src[q];
      tw.y[lane] = y[r];
    }
    __syncwarp();
    // ---- forward
    float o[4];
    mlp_tile(s, tw.x, o, tw.h1, tw.h2);
    // ---- softmax cross-entropy: lanes t = 0, 1 of quad g hold rows g, g+8
    {
      float lo0 = o[0], lo1 = o[1], hi0 = o[2], hi1 = o[3];
      const float plo0 = __shfl_xor_sync(0xffffffffu, lo0, 1), plo1 = __shfl_xor_sync(0xffffffffu, lo1, 1);
      const float phi0 = __shfl_xor_sync(0xffffffffu, hi0, 1), phi1 = __shfl_xor_sync(0xffffffffu, hi1, 1);
      if (t < 2) {
        // the four logits of each row, in class order
        const float Llo[4] = {t == 0 ? lo0 : plo0, t == 0 ? lo1 : plo1, t == 0 ? plo0 : lo0, t == 0 ? plo1 : lo1};
        const float Lhi[4] = {t == 0 ? hi0 : phi0, t == 0 ? hi1 : phi1, t == 0 ? phi0 : hi0, t == 0 ? phi1 : hi1};
        float row_loss = 0.0f;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          const float* L = half ? Lhi : Llo;
          const int row = g + 8 * half;
          const int yl = tw.y[row];
          const float m = fmaxf(fmaxf(L[0], L[1]), fmaxf(L[2], L[3]));
          const float e0 = __expf(L[0] - m), e1 = __expf(L[1] - m), e2 = __expf(L[2] - m), e3 = __expf(L[3] - m);
          const float sum = e0 + e1 + e2 + e3;
          const float p[4] = {e0 / sum, e1 / sum, e2 / sum, e3 / sum};
          if (t == 0) row_loss += -__logf(fmaxf(p[yl], 1e-30f));
          // this lane writes classes 2t, 2t+1 of the row
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int k = 2 * t + q;
            const float d = (p[k] - (k == yl ? 1.0f : 0.0f)) * inv_batch;
            tw.dlf[row * 4 + k] = d;
            tw.dl[row * 8 + k] = __float2bfloat16_rn(d);
            tw.dl[row * 8 + 4 + k] = __float2bfloat16_rn(0.0f);
          }
        }
        if (t == 0) atomicAdd(&loss_sum, row_loss);
      }
    }
    __syncwarp();
    // ---- dW3 (rows 0..3) = dL^T H2 ; db3
    {
      uint32_t a[4];
      a[0] = pack2(tw.dl[(2 * t) * 8 + g], tw.dl[(2 * t + 1) * 8 + g]);
      a[1] = 0u;
      a[2] = pack2(tw.dl[(2 * t + 8) * 8 + g], tw.dl[(2 * t + 9) * 8 + g]);
      a[3] = 0u;
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const int col = nt * 8 + g;
        const uint32_t b0 = pack2(tw.h2[(2 * t) * kSW2 + col], tw.h2[(2 * t + 1) * kSW2 + col]);
        const uint32_t b1 = pack2(tw.h2[(2 * t + 8) * kSW2 + col], tw.h2[(2 * t + 9) * kSW2 + col]);
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        mma16816(c, a, b0, b1);
        if (g < kSchedClasses) {
          atomicAdd(&G[kSchedOffW3 + g * kSchedHidden + nt * 8 + 2 * t], c[0]);
          atomicAdd(&G[kSchedOffW3 + g * kSchedHidden + nt * 8 + 2 * t + 1], c[1]);
        }
      }
      if (lane < kSchedClasses) {
        float sb = 0.0f;
        for (int r = 0; r < 16; ++r) sb += tw.dlf[r * 4 + lane];
        atomicAdd(&G[kSchedOffB3 + lane], sb);
      }
    }
    // ---- dH2 = (dL W3) masked ; db2
    {
      uint32_t a[4];
      a[0] = ld32(tw.dl + g * 8 + 2 * t);
      a[1] = ld32(tw.dl + (g + 8) * 8 + 2 * t);
      a[2] = 0u;
      a[3] = 0u;
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const int col = nt * 8 + g;
        const uint32_t b0 = pack2(s.w3[(2 * t) * kSW2 + col], s.w3[(2 * t + 1) * kSW2 + col]);
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        mma16816(c, a, b0, 0u);
        const int cc = nt * 8 + 2 * t;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          if (__bfloat162float(tw.h2[g * kSW2 + cc + q]) <= 0.0f) c[q] = 0.0f;
          if (__bfloat162float(tw.h2[(g + 8) * kSW2 + cc + q]) <= 0.0f) c[2 + q] = 0.0f;
        }
        *reinterpret_cast<uint32_t*>(tw.d2 + g * kSW2 + cc) = pack_bf16(c[0], c[1]);
        *reinterpret_cast<uint32_t*>(tw.d2 + (g + 8) * kSW2 + cc) = pack_bf16(c[2], c[3]);
        float s0 = c[0] + c[2], s1 = c[1] + c[3];
#pragma unroll
        for (int off = 4; off < 32; off <<= 1) {
          s0 += __shfl_xor_sync(0xffffffffu, s0, off);
          s1 += __shfl_xor_sync(0xffffffffu, s1, off);
        }
        if (g == 0) {
          atomicAdd(&G[kSchedOffB2 + cc], s0);
          atomicAdd(&G[kSchedOffB2 + cc + 1], s1);
        }
      }
    }
    __syncwarp();
    // ---- dW2 = dH2^T H1 (M: 64 outputs, N: 64 inputs, K: 16 samples)
#pragma unroll 1
    for (int mt = 0; mt < 4; ++mt) {
      const int o0 = mt * 16 + g;
      uint32_t a[4];
      a[0] = pack2(tw.d2[(2 * t) * kSW2 + o0], tw.d2[(2 * t + 1) * kSW2 + o0]);
      a[1] = pack2(tw.d2[(2 * t) * kSW2 + o0 + 8], tw.d2[(2 * t + 1) * kSW2 + o0 + 8]);
      a[2] = pack2(tw.d2[(2 * t + 8) * kSW2 + o0], tw.d2[(2 * t + 9) * kSW2 + o0]);
      a[3] = pack2(tw.d2[(2 * t + 8) * kSW2 + o0 + 8], tw.d2[(2 * t + 9) * kSW2 + o0 + 8]);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const int col = nt * 8 + g;
        const uint32_t b0 = pack2(tw.h1[(2 * t) * kSW2 + col], tw.h1[(2 * t + 1) * kSW2 + col]);
        const uint32_t b1 = pack2(tw.h1[(2 * t + 8) * kSW2 + col], tw.h1[(2 * t + 9) * kSW2 + col]);
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        mma16816(c, a, b0, b1);
        const int ci = nt * 8 + 2 * t;
        atomicAdd(&G[kSchedOffW2 + o0 * kSchedHidden + ci], c[0]);
        atomicAdd(&G[kSchedOffW2 + o0 * kSchedHidden + ci + 1], c[1]);
        atomicAdd(&G[kSchedOffW2 + (o0 + 8) * kSchedHidden + ci], c[2]);
        atomicAdd(&G[kSchedOffW2 + (o0 + 8) * kSchedHidden + ci + 1], c[3]);
      }
    }
    // ---- dH1 = (dH2 W2) masked ; db1
    {
      uint32_t a[4][4];
#pragma unroll
      for (int kb = 0; kb < 4; ++kb) {
        a[kb][0] = ld32(tw.d2 + g * kSW2 + kb * 16 + 2 * t);
        a[kb][1] = ld32(tw.d2 + (g + 8) * kSW2 + kb * 16 + 2 * t);
        a[kb][2] = ld32(tw.d2 + g * kSW2 + kb * 16 + 8 + 2 * t);
        a[kb][3] = ld32(tw.d2 + (g + 8) * kSW2 + kb * 16 + 8 + 2 * t);
      }
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const int col = nt * 8 + g;
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kb = 0; kb < 4; ++kb) {
          const int k0 = kb * 16 + 2 * t;
          const uint32_t b0 = pack2(s.w2[k0 * kSW2 + col], s.w2[(k0 + 1) * kSW2 + col]);
          const uint32_t b1 = pack2(s.w2[(k0 + 8) * kSW2 + col], s.w2[(k0 + 9) * kSW2 + col]);
          mma16816(c, a[kb], b0, b1);
        }
        const int cc = nt * 8 + 2 * t;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          if (__bfloat162float(tw.h1[g * kSW2 + cc + q]) <= 0.0f) c[q] = 0.0f;
          if (__bfloat162float(tw.h1[(g + 8) * kSW2 + cc + q]) <= 0.0f) c[2 + q] = 0.0f;
        }
        *reinterpret_cast<uint32_t*>(tw.d1 + g * kSW2 + cc) = pack_bf16(c[0], c[1]);
        *reinterpret_cast<uint32_t*>(tw.d1 + (g + 8) * kSW2 + cc) = pack_bf16(c[2], c[3]);
        float s0 = c[0] + c[2], s1 = c[1] + c[3];
#pragma unroll
        for (int off = 4; off < 32; off <<= 1) {
          s0 += __shfl_xor_sync(0xffffffffu, s0, off);
          s1 += __shfl_xor_sync(0xffffffffu, s1, off);
        }
        if (g == 0) {
          atomicAdd(&G[kSchedOffB1 + cc], s0);
          atomicAdd(&G[kSchedOffB1 + cc + 1], s1);
        }
      }
    }
    __syncwarp();
    // ---- dW1 = dH1^T X (M: 64 outputs, N: 24 inputs, K: 16 samples)
#pragma unroll 1
    for (int mt = 0; mt < 4; ++mt) {
      const int o0 = mt * 16 + g;
      uint32_t a[4];
      a[0] = pack2(tw.d1[(2 * t) * kSW2 + o0], tw.d1[(2 * t + 1) * kSW2 + o0]);
      a[1] = pack2(tw.d1[(2 * t) * kSW2 + o0 + 8], tw.d1[(2 * t + 1) * kSW2 + o0 + 8]);
      a[2] = pack2(tw.d1[(2 * t + 8) * kSW2 + o0], tw.d1[(2 * t + 9) * kSW2 + o0]);
      a[3] = pack2(tw.d1[(2 * t + 8) * kSW2 + o0 + 8], tw.d1[(2 * t + 9) * kSW2 + o0 + 8]);
#pragma unroll
      for (int nt = 0; nt < 3; ++nt) {
        const int col = nt * 8 + g;
        const uint32_t b0 = pack2(tw.x[(2 * t) * kSW1 + col], tw.x[(2 * t + 1) * kSW1 + col]);
        const uint32_t b1 = pack2(tw.x[(2 * t + 8) * kSW1 + col], tw.x[(2 * t + 9) * kSW1 + col]);
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        mma16816(c, a, b0, b1);
        const int ci = nt * 8 + 2 * t;
        atomicAdd(&G[kSchedOffW1 + o0 * kSchedInPad + ci], c[0]);
        atomicAdd(&G[kSchedOffW1 + o0 * kSchedInPad + ci + 1], c[1]);
        atomicAdd(&G[kSchedOffW1 + (o0 + 8) * kSchedInPad + ci], c[2]);
        atomicAdd(&G[kSchedOffW1 + (o0 + 8) * kSchedInPad + ci + 1], c[3]);
      }
    }
    __syncthreads();
    // ---- Adam on the FP32 master weights
    if (grad_first && step == 0)
      for (int i = threadIdx.x; i < kSchedParams; i += blockDim.x) grad_first[i] = G[i];
    if (loss_trace && threadIdx.x == 0 && trace_every > 0 && step % trace_every == 0)
      loss_trace[step / trace_every] = loss_sum * inv_batch;
    b1t *= 0.9f;
    b2t *= 0.999f;
    const float c1 = 1.0f / (1.0f - b1t), c2 = 1.0f / (1.0f - b2t);
    const float lr_t = 0.5f * lr * (1.0f + cospif((float)step / (float)steps));
    for (int i = threadIdx.x; i < kSchedParams; i += blockDim.x) {
      const float gi = G[i];
      G[i] = 0.0f;
      if (is_pad_param(i)) continue;
      float m = adam[i], v = adam[kSchedParams + i];
      m = 0.9f * m + 0.1f * gi;
      v = 0.999f * v + 0.001f * gi * gi;
      adam[i] = m;
      adam[kSchedParams + i] = v;
      P[i] -= lr_t * (m * c1) / (sqrtf(v * c2) + 1e-8f);
    }
    __syncthreads();
    if (threadIdx.x == 0) loss_sum = 0.0f;
    refresh_smem(P, s);
    __syncthreads();
  }
  for (int i = threadIdx.x; i < kSchedParams; i += blockDim.x) params[i] = P[i];
}

size_t sched_train_smem_bytes() { return 2 * sizeof(float) * kSchedParams + sizeof(SchedSmem) + 8 * sizeof(TrainWarp); }

// ---------------------------------------------------------------- host side
__global__ void k_sched_pack(const float* __restrict__ p, SchedWeights* w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kSchedParams; i += gridDim.x * blockDim.x) {
    const float v = p[i];
    if (i < kSchedOffB1) {
      w->w1[i - kSchedOffW1] = __float2bfloat16_rn(v);
    } else if (i < kSchedOffW2) {
      w->b1[i - kSchedOffB1] = v;
    } else if (i < kSchedOffB2) {
      w->w2[i - kSchedOffW2] = __float2bfloat16_rn(v);
    } else if (i < kSchedOffW3) {
      w->b2[i - kSchedOffB2] = v;
    } else if (i < kSchedOffB3) {
      w->w3[i - kSchedOffW3] = __float2bfloat16_rn(v);
    } else {
      w->b3[i - kSchedOffB3] = (i - kSchedOffB3) < kSchedClasses ? v : -FLT_MAX;
    }
  }
}

cudaError_t launch_sched_pack(const float* params, SchedWeights* w, cudaStream_t s) {
  count_launch();
  k_sched_pack<<<(kSchedParams + 255) / 256, 256, 0, s>>>(params, w);
  return cudaGetLastError();
}

cudaError_t launch_sched_true_class(int64_t n, const int32_t* n_out, int8_t* cls, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launch();
  k_sched_true_class<<<grid_for(n, 256, 8), 256, 0, s>>>(n, n_out, cls);
  return cudaGetLastError();
}

cudaError_t launch_sched_bin(const SchedBin& b, const int4* in, const unsigned long long* nlist, int4* out,
                             const double* coords_a, cudaStream_t s) {
  count_launch();
  k_sched_bin<<<sm_count() * 4, 256, sched_bin_smem_bytes(b.window), s>>>(
      in, nlist, out, coords_a, b.screen_b, b.weights, b.cls_of_pair, b.pred_of_pair, b.window);
  return cudaGetLastError();
}

cudaError_t launch_sched_samples(const int4* list, const unsigned long long* nlist, int64_t cap, const double* coords_a,
                                 const double* screen_b, const int32_t* n_out, void* x, int8_t* y, cudaStream_t s) {
  if (cap <= 0) return cudaSuccess;
  count_launch();
  k_sched_samples<<<grid_for(cap, 256, 8), 256, 0, s>>>(list, nlist, cap, coords_a, screen_b, n_out,
                                                        static_cast<__nv_bfloat16*>(x), y);
  return cudaGetLastError();
}

cudaError_t launch_sched_predict(int64_t n, const void* x, const SchedWeights* w, float* logits, int8_t* cls,
                                 cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launch();
  const size_t smem = sizeof(SchedSmem) + 8 * 16 * kSW1 * sizeof(__nv_bfloat16);
  k_sched_predict<<<grid_for(n, 256, 4), 256, smem, s>>>(n, static_cast<const __nv_bfloat16*>(x), w, logits, cls);
  return cudaGetLastError();
}

cudaError_t launch_sched_train(const void* x, const int8_t* y, int64_t n, float* params, float* adam, int steps,
                               float lr, float* loss_trace, int trace_every, float* grad_first, cudaStream_t s) {
  if (n <= 0 || steps <= 0) return cudaSuccess;
  count_launch();
  k_sched_train<<<1, 256, sched_train_smem_bytes(), s>>>(static_cast<const __nv_bfloat16*>(x), y, n, params, adam,
                                                         steps, lr, loss_trace, trace_every, grad_first);
  return cudaGetLastError();
}

cudaError_t init_sched_attributes(int max_window) {
  cudaError_t e = cudaFuncSetAttribute(k_sched_bin, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sched_bin_smem_bytes(max_window));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_sched_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sched_train_smem_bytes());
}

}  // namespace lsm
