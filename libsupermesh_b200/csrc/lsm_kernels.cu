// Supermesh kernels for sm_100a.
//
//   K1  k_prep          element gather, FP64/FP32 boxes, measures, tolerances,
//                       B-element clip setup (lines / unit-normal planes)
//   K1b k_root_*        root box reduction;  k_morton  Morton keys
//   K2  radix sort      stable LSD, 8-bit digits, warp-match ranking;
//                       one digit-count kernel, then one kernel per pass
//                       with decoupled look-back (k_radix_onesweep)
//   K3  k_bvh_internal  Karras LBVH hierarchy + rope table;
//       k_bvh_refit     bottom-up FP32 box refit, escape links, leaf records
//   K4  k_query         stackless LBVH traversal per A element (FP32,
//                       outward-rounded boxes) + exact strict FP64 box test
//                       at the leaf records; the count pass caches rows,
//                       k_fill_from_cache copies
//   K5  k_clip_tris     one candidate pair per thread, polygon in shared
//                       memory, FP64 Sutherland-Hodgman
//   K6  k_prefilter_tets two exact early-outs and the no-op plane mask;
//                       k_clip_tets_ix depth-first clipping over point
//                       indices with a refill pipeline, templated on what it
//                       does with the kept tets (measures; explicit pairs'
//                       output tets; the supermesh's tets at their offsets;
//                       the P1 quadrature) and on the plane count (4: tets,
//                       6: hexahedra)
//   K7  compensated reductions (per-block (sum, err), then final; per mesh
//                       pair for the batched path)
//   K8  P1-P1 mixed mass blocks + u^T M v: 2D k_p1_mass; 3D the early-out
//                       pass and k_clip_tets_ix with the quadrature sink;
//                       k_p2_inner  P2 inner product
//   K9  1D sort finder  k_prep_1d, 64-bit stable sort, max segment tree,
//                       k_rows_1d, k_sweep_1d, k_emit_1d;  k_clip_intervals
//   K10 explicit pairs  k_pairs_tris / _tets and the mixed element pairs
//                       (intervals, tri-quad, quad-quad, tet-hex, hex-hex);
//                       large tet-tet / tet-hex batches: k_setup_pairs3 /
//                       k_setup_hex_pairs, then K6
//   K13 supermesh elements  K6's emit pass (3D), k_tris_emit (2D)
//
// Everything FP64 is compiled with -fmad=false so that each +,-,*,/ is a
// separately rounded IEEE operation, matching libsupermesh's gfortran build.
#include "lsm_geom.cuh"
#include "lsm_kernels.h"
#include "lsm_sched.h"

#include <cuda/atomic>

#include <cfloat>
#include <cstdio>
#include <cstdlib>

namespace lsm {

namespace {
unsigned long long g_launches = 0;
}  // namespace

unsigned long long launches() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

namespace {
int g_tri_bps = 8;
int g_query_block = 128;
int g_leaf_bucket = 1;
}  // namespace

int tri_blocks_per_sm() { return g_tri_bps; }
void set_tri_blocks_per_sm(int v) { g_tri_bps = v; }
int query_block() { return g_query_block; }
void set_query_block(int v) { g_query_block = v; }
int leaf_bucket() { return g_leaf_bucket; }
void set_leaf_bucket(int v) { g_leaf_bucket = v; }
int tree_bucket(int n, bool leaf_records) {
  // buckets need the leaf records and fit the node encoding (first leaf
  // below 2^27, at most 8 leaves)
  return leaf_records && g_leaf_bucket > 1 && n < (1 << 27) ? g_leaf_bucket : 1;
}

void count_launch(int n) { __atomic_fetch_add(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED); }

int sm_count() {
  static int cached = -1;
  if (cached < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cached = n;
  }
  return cached;
}

int grid_for(int64_t n, int block, int per_sm) {
  int64_t need = (n + block - 1) / block;
  int64_t cap = (int64_t)sm_count() * per_sm;
  if (need < 1) need = 1;
  return (int)(need < cap ? need : cap);
}

namespace {

// Compensated (sum, err) pair helpers: TwoSum-based merge.
__device__ __forceinline__ void cs_add(double& sum, double& err, double x) {
  // Kahan step (Precision.F90:89-95)
  const double cx = err + x;
  const double s = sum + cx;
  err = (sum - s) + cx;
  sum = s;
}

__device__ __forceinline__ void two_sum_merge(double& s, double& e, double s2, double e2) {
  const double t = s + s2;
  const double bp = t - s;
  const double err = (s - (t - bp)) + (s2 - bp);
  s = t;
  e = e + e2 + err;
}

template <int BLOCK>
__device__ void block_reduce_partial(double sum, double err, unsigned long long ni, unsigned long long no,
                                     Partial* out) {
  __shared__ double ss[BLOCK / 32], se[BLOCK / 32];
  __shared__ unsigned long long si[BLOCK / 32], so[BLOCK / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double s2 = __shfl_down_sync(0xffffffffu, sum, o);
    const double e2 = __shfl_down_sync(0xffffffffu, err, o);
    two_sum_merge(sum, err, s2, e2);
    ni += __shfl_down_sync(0xffffffffu, ni, o);
    no += __shfl_down_sync(0xffffffffu, no, o);
  }
  if (lane == 0) {
    ss[wid] = sum;
    se[wid] = err;
    si[wid] = ni;
    so[wid] = no;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    Partial p{ss[0], se[0], si[0], so[0]};
    for (int w = 1; w < BLOCK / 32; ++w) {
      two_sum_merge(p.sum, p.err, ss[w], se[w]);
      p.n_int += si[w];
      p.n_out += so[w];
    }
    *out = p;
  }
}

}  // namespace

// ======================================================================
// K1: element prep
// ======================================================================
// One element of the prep: gather, boxes, measure/tolerance, clip setup.
// LOC = DIM + 1 for simplices; other LOC (quads, hexes) only get boxes,
// which is all the candidate search needs.
template <int DIM, int LOC, typename IDX>
__device__ __forceinline__ void prep_element(int64_t e, const double* __restrict__ pos,
                                             const IDX* __restrict__ row, int64_t nnodes, double* coords,
                                             double* box64, float* box32, double* tolv, double* setup,
                                             int* bad, double* faces = nullptr, double* screen = nullptr) {
  constexpr bool SIMPLEX = LOC == DIM + 1;
  double v[LOC * DIM];
  bool ok = true;
#pragma unroll
  for (int k = 0; k < LOC; ++k) {
    int64_t node = (int64_t)row[k];
    if (node < 0 || node >= nnodes) {
      ok = false;
      node = 0;
    }
#pragma unroll
    for (int c = 0; c < DIM; ++c) v[k * DIM + c] = pos[node * DIM + c];
  }
  if (!ok) atomicExch(bad, 1);
  if (coords) {
    static_assert((LOC * DIM) % 2 == 0, "element rows of an even number of doubles");
#pragma unroll
    for (int j = 0; j < LOC * DIM; j += 2) st2(coords + e * LOC * DIM + j, v[j], v[j + 1]);
  }
  double lo[DIM], hi[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) lo[c] = hi[c] = v[c];
#pragma unroll
  for (int k = 1; k < LOC; ++k)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      lo[c] = fmin(lo[c], v[k * DIM + c]);
      hi[c] = fmax(hi[c], v[k * DIM + c]);
    }
  if (box64) {
    double* o = box64 + e * 2 * DIM;
    if (DIM == 3) {
      st2(o, lo[0], lo[1]);
      st2(o + 2, lo[DIM - 1], hi[0]);
      st2(o + 4, hi[1], hi[DIM - 1]);
    } else {
      st2(o, lo[0], lo[1]);
      st2(o + 2, hi[0], hi[1]);
    }
  }
  if (box32) {
    float4 l = make_float4(0.f, 0.f, 0.f, 0.f), h = make_float4(0.f, 0.f, 0.f, 0.f);
    l.x = __double2float_rd(lo[0]);
    l.y = __double2float_rd(lo[1]);
    h.x = __double2float_ru(hi[0]);
    h.y = __double2float_ru(hi[1]);
    if (DIM == 3) {
      l.z = __double2float_rd(lo[DIM - 1]);
      h.z = __double2float_ru(hi[DIM - 1]);
    }
    reinterpret_cast<float4*>(box32)[2 * e] = l;
    reinterpret_cast<float4*>(box32)[2 * e + 1] = h;
  }
  if (!SIMPLEX) return;
  double meas;
  Tet t;
  if (DIM == 2) {
    meas = tri_area(v[0], v[1], v[2], v[3], v[4], v[5]);
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      t.x[k] = v[k * DIM + 0];
      t.y[k] = v[k * DIM + 1];
      t.z[k] = v[k * DIM + DIM - 1];
    }
    meas = tet_volume_v4(t);
  }
  const double tol = 10.0 * spacing(meas);
  if (tolv) tolv[e] = tol;
  if (setup) {
    if (DIM == 2) {
      Lines L;
      tri_lines(v, L);
      double* o = setup + e * kSetup2;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        st2(o + 4 * i, L.nx[i], L.ny[i]);
        st2(o + 4 * i + 2, L.px[i], L.py[i]);
      }
      st2(o + 12, tol, 0.0);
    } else {
      Planes P;
      tet_planes(t, P);
      double* o = setup + e * kSetup3;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        st2(o + 4 * i, P.nx[i], P.ny[i]);
        st2(o + 4 * i + 2, P.nz[i], P.c[i]);
      }
      st2(o + 16, tol, 0.0);
      st2(o + 18, 0.0, 0.0);
      if (screen) tet_screen_b(t, P, screen + e * kScreen3);
    }
  }
  if constexpr (DIM == 3) {
    if (faces) tet_faces_screen(t, faces + e * kScreen3);
  }
}

template <int DIM, int LOC, typename IDX>
__global__ void k_prep(int64_t nel, const double* __restrict__ pos, const IDX* __restrict__ en,
                       double* coords, double* box64, float* box32, double* tolv, double* setup,
                       int* bad, int64_t nnodes, double* faces, double* screen) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel;
       e += (int64_t)gridDim.x * blockDim.x)
    prep_element<DIM, LOC, IDX>(e, pos, en + e * LOC, nnodes, coords, box64, box32, tolv, setup, bad, faces,
                                screen);
}

// Batched prep over the concatenation of many meshes.  Element e belongs to
// mesh p = the last p with elem_off[p] <= e; its nodes are read through the
// per-mesh pointer tables.  pair_of[e] receives p.
__device__ __forceinline__ int find_mesh(const int64_t* __restrict__ off, int nm, int64_t e) {
  int lo = 0, hi = nm;  // off[lo] <= e < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= e)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

template <int DIM, typename IDX>
__global__ void k_prep_batched(int64_t nel, int nm, const int64_t* __restrict__ elem_off,
                               const unsigned long long* __restrict__ pos_ptr,
                               const unsigned long long* __restrict__ en_ptr,
                               const int64_t* __restrict__ nnodes, double* coords, double* box64,
                               float* box32, double* tolv, double* setup, int32_t* pair_of, int* bad,
                               double* faces, double* screen) {
  constexpr int LOC = DIM + 1;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int p = find_mesh(elem_off, nm, e);
    const int64_t local = e - elem_off[p];
    const double* pos = reinterpret_cast<const double*>(pos_ptr[p]);
    const IDX* en = reinterpret_cast<const IDX*>(en_ptr[p]);
    prep_element<DIM, LOC, IDX>(e, pos, en + local * LOC, nnodes[p], coords, box64, box32, tolv, setup, bad,
                                faces, screen);
    pair_of[e] = p;
  }
}

template <int DIM, int LOC>
static void prep_dispatch_idx(int g, int B, cudaStream_t s, int64_t nel, const double* pos,
                              const void* enlist, int idx_bytes, double* coords, double* box64,
                              float* box32, double* tolv, double* setup, int* bad, int64_t nnodes,
                              double* faces, double* screen) {
  count_launch();
  if (idx_bytes == 4)
    k_prep<DIM, LOC, int32_t><<<g, B, 0, s>>>(nel, pos, (const int32_t*)enlist, coords, box64, box32, tolv, setup, bad,
                                              nnodes, faces, screen);
  else
    k_prep<DIM, LOC, int64_t><<<g, B, 0, s>>>(nel, pos, (const int64_t*)enlist, coords, box64, box32, tolv, setup, bad,
                                              nnodes, faces, screen);
}

cudaError_t launch_prep(int dim, int loc, int64_t nel, const double* pos, const void* enlist, int idx_bytes,
                        double* coords, double* box64, float* box32, double* tolv, double* setup,
                        int* bad_index, int64_t nnodes, cudaStream_t s, double* faces, double* screen) {
  if (nel <= 0) return cudaSuccess;
  const int B = 256;
  const int g = grid_for(nel, B, 8);
  if (dim == 2 && loc == 3)
    prep_dispatch_idx<2, 3>(g, B, s, nel, pos, enlist, idx_bytes, coords, box64, box32, tolv, setup, bad_index, nnodes,
                            nullptr, nullptr);
  else if (dim == 2 && loc == 4)
    prep_dispatch_idx<2, 4>(g, B, s, nel, pos, enlist, idx_bytes, coords, box64, box32, tolv, setup, bad_index, nnodes,
                            nullptr, nullptr);
  else if (dim == 3 && loc == 4)
    prep_dispatch_idx<3, 4>(g, B, s, nel, pos, enlist, idx_bytes, coords, box64, box32, tolv, setup, bad_index, nnodes,
                            faces, screen);
  else if (dim == 3 && loc == 8)
    prep_dispatch_idx<3, 8>(g, B, s, nel, pos, enlist, idx_bytes, coords, box64, box32, tolv, setup, bad_index, nnodes,
                            nullptr, nullptr);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_prep_batched(int dim, int64_t nel, int nm, const int64_t* elem_off,
                                const unsigned long long* pos_ptr, const unsigned long long* en_ptr,
                                const int64_t* nnodes, int idx_bytes, double* coords, double* box64,
                                float* box32, double* tolv, double* setup, int32_t* pair_of, int* bad,
                                cudaStream_t s, double* faces, double* screen) {
  if (nel <= 0) return cudaSuccess;
  const int B = 256;
  const int g = grid_for(nel, B, 8);
  count_launch();
  if (dim == 2 && idx_bytes == 4)
    k_prep_batched<2, int32_t><<<g, B, 0, s>>>(nel, nm, elem_off, pos_ptr, en_ptr, nnodes, coords, box64, box32,
                                                 tolv, setup, pair_of, bad, nullptr, nullptr);
  else if (dim == 2)
    k_prep_batched<2, int64_t><<<g, B, 0, s>>>(nel, nm, elem_off, pos_ptr, en_ptr, nnodes, coords, box64, box32,
                                                 tolv, setup, pair_of, bad, nullptr, nullptr);
  else if (idx_bytes == 4)
    k_prep_batched<3, int32_t><<<g, B, 0, s>>>(nel, nm, elem_off, pos_ptr, en_ptr, nnodes, coords, box64, box32,
                                                 tolv, setup, pair_of, bad, faces, screen);
  else
    k_prep_batched<3, int64_t><<<g, B, 0, s>>>(nel, nm, elem_off, pos_ptr, en_ptr, nnodes, coords, box64, box32,
                                                 tolv, setup, pair_of, bad, faces, screen);
  return cudaGetLastError();
}

// ======================================================================
// K1b: root box and Morton keys
// ======================================================================
template <int DIM>
__global__ void k_root_partial(int64_t nel, const double* __restrict__ box64, double* partial) {
  double lo[DIM], hi[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    lo[c] = DBL_MAX;
    hi[c] = -DBL_MAX;
  }
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel;
       e += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      lo[c] = fmin(lo[c], box64[e * 2 * DIM + c]);
      hi[c] = fmax(hi[c], box64[e * 2 * DIM + DIM + c]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      lo[c] = fmin(lo[c], __shfl_down_sync(0xffffffffu, lo[c], o));
      hi[c] = fmax(hi[c], __shfl_down_sync(0xffffffffu, hi[c], o));
    }
  __shared__ double sl[32][DIM], sh[32][DIM];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      sl[wid][c] = lo[c];
      sh[wid][c] = hi[c];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        lo[c] = fmin(lo[c], sl[w][c]);
        hi[c] = fmax(hi[c], sh[w][c]);
      }
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      partial[blockIdx.x * 2 * DIM + c] = lo[c];
      partial[blockIdx.x * 2 * DIM + DIM + c] = hi[c];
    }
  }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_root_final(int np, const double* partial, double* root) {
  double lo[DIM], hi[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    lo[c] = DBL_MAX;
    hi[c] = -DBL_MAX;
  }
  for (int b = threadIdx.x; b < np; b += blockDim.x)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      lo[c] = fmin(lo[c], partial[b * 2 * DIM + c]);
      hi[c] = fmax(hi[c], partial[b * 2 * DIM + DIM + c]);
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      lo[c] = fmin(lo[c], __shfl_down_sync(0xffffffffu, lo[c], o));
      hi[c] = fmax(hi[c], __shfl_down_sync(0xffffffffu, hi[c], o));
    }
  __shared__ double sl[8][DIM], sh[8][DIM];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      sl[wid][c] = lo[c];
      sh[wid][c] = hi[c];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; ++w)
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        lo[c] = fmin(lo[c], sl[w][c]);
        hi[c] = fmax(hi[c], sh[w][c]);
      }
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      root[c] = lo[c];
      root[DIM + c] = hi[c];
    }
  }
}

cudaError_t launch_root_box(int dim, int64_t nel, const double* box64, double* partial,
                            int partial_cap, double* rootbox, cudaStream_t s) {
  const int B = 256;
  int g = grid_for(nel, B, 2);
  if (g > partial_cap) g = partial_cap;
  count_launch(2);
  if (dim == 2) {
    k_root_partial<2><<<g, B, 0, s>>>(nel, box64, partial);
    k_root_final<2><<<1, 256, 0, s>>>(g, partial, rootbox);
  } else {
    k_root_partial<3><<<g, B, 0, s>>>(nel, box64, partial);
    k_root_final<3><<<1, 256, 0, s>>>(g, partial, rootbox);
  }
  return cudaGetLastError();
}

__device__ __forceinline__ uint32_t spread2(uint32_t x) {  // 16 bits -> even bits
  x &= 0xffffu;
  x = (x | (x << 8)) & 0x00ff00ffu;
  x = (x | (x << 4)) & 0x0f0f0f0fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}

__device__ __forceinline__ uint32_t spread3(uint32_t x) {  // 10 bits -> every 3rd bit
  x &= 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

template <int DIM>
__global__ void k_morton(int64_t nel, const double* __restrict__ box64, const double* __restrict__ root,
                         uint32_t* keys, int32_t* vals) {
  constexpr double kScale = DIM == 2 ? 65536.0 : 1024.0;
  constexpr uint32_t kMax = DIM == 2 ? 65535u : 1023u;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel;
       e += (int64_t)gridDim.x * blockDim.x) {
    uint32_t q[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      const double mid = 0.5 * (box64[e * 2 * DIM + c] + box64[e * 2 * DIM + DIM + c]);
      const double ext = root[DIM + c] - root[c];
      double u = ext > 0.0 ? (mid - root[c]) / ext : 0.0;
      u = fmin(fmax(u, 0.0), 1.0);
      const double f = u * kScale;
      q[c] = f >= (double)kMax ? kMax : (uint32_t)f;
    }
    uint32_t key;
    if (DIM == 2)
      key = (spread2(q[1]) << 1) | spread2(q[0]);
    else
      key = (spread3(q[DIM - 1]) << 2) | (spread3(q[1]) << 1) | spread3(q[0]);
    keys[e] = key;
    vals[e] = (int32_t)e;
  }
}

cudaError_t launch_morton(int dim, int64_t nel, const double* box64, const double* rootbox,
                          uint32_t* keys, int32_t* vals, cudaStream_t s) {
  if (nel <= 0) return cudaSuccess;
  const int B = 256;
  const int g = grid_for(nel, B, 8);
  count_launch();
  if (dim == 2)
    k_morton<2><<<g, B, 0, s>>>(nel, box64, rootbox, keys, vals);
  else
    k_morton<3><<<g, B, 0, s>>>(nel, box64, rootbox, keys, vals);
  return cudaGetLastError();
}

// ======================================================================
// K2: stable LSD radix sort (8-bit digits, one kernel per pass)
// ======================================================================
namespace {
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;                           // per thread
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per block
constexpr int kWarpTile = 32 * kSortItems;             // contiguous per warp
}  // namespace

// Single-pass digit binning per pass ("onesweep"): one kernel counts every
// digit of every pass over all keys; each pass is then one kernel in which
// block b (in ticket order) ranks its 2048 keys, publishes its digit counts,
// looks back over the blocks before it for their prefix (decoupled
// look-back: a block publishes its local count first and its inclusive
// prefix once known) and scatters.  Stable: ranks follow key order within a
// block and blocks follow key order.
//
// Scratch layout (uint32, radix_hist_entries(n)): counts[4][256] |
// tickets[4] | err | pad | status[4][nblocks][256].  A status word holds a
// 2-bit flag (0 not ready, 1 local count, 2 inclusive prefix) over a 30-bit
// count (n < 2^30).  Waits are bounded: a block that gives up sets err and
// treats the missing prefix as 0 (wrong order, never a hang); forward
// progress does not need the bound, since a block only waits for blocks
// that took earlier tickets and are running or done.  A partial prefix only
// lowers the scatter positions, so they stay inside [0, n); some keys then
// overwrite others, and k_sort_repair turns the output back into a
// permutation (identity values, equal keys) so that the kernels after the
// sort never read an element number that does not exist.  The caller sees
// err and reports the failure.
//
// Test hooks (process-wide, off by default): the bound of each wait
// (set_sort_spin_limit) and one block per pass that never publishes its
// counts (set_sort_stall_block, sorts given an err word only), which makes
// the waits of the blocks after it run out.
namespace {
constexpr int kSortPassesMax = 4;
constexpr int kSortHdr = kSortPassesMax * 256 + 8;
constexpr uint32_t kFlagLocal = 1u << 30, kFlagIncl = 2u << 30, kFlagMask = 3u << 30;
}  // namespace

namespace {
int g_sort_spin_limit = 1 << 22;
int g_sort_stall = -1;
}  // namespace

void set_sort_spin_limit(int v) { g_sort_spin_limit = v > 0 ? v : 1; }
int sort_spin_limit() { return g_sort_spin_limit; }
void set_sort_stall_block(int b) { g_sort_stall = b >= 1 ? b : -1; }
int sort_stall_block() { return g_sort_stall; }

int64_t radix_hist_entries(int64_t n) {
  const int64_t nb = (n + kSortTile - 1) / kSortTile;
  return kSortHdr + (int64_t)kSortPassesMax * 256 * (nb > 0 ? nb : 1);
}

__global__ void __launch_bounds__(kSortThreads) k_radix_counts(int64_t n, int passes,
                                                               const uint32_t* __restrict__ keys, uint32_t* counts) {
  __shared__ uint32_t h[kSortPassesMax][256];
  for (int i = threadIdx.x; i < kSortPassesMax * 256; i += blockDim.x) (&h[0][0])[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    for (int p = 0; p < passes; ++p) atomicAdd(&h[p][(k >> (8 * p)) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
    const uint32_t v = (&h[0][0])[i];
    if (v) atomicAdd(&counts[i], v);
  }
}

__global__ void __launch_bounds__(kSortThreads) k_radix_onesweep(int64_t n, int shift,
                                                                 const uint32_t* __restrict__ keys_in,
                                                                 const int32_t* __restrict__ vals_in,
                                                                 uint32_t* keys_out, int32_t* vals_out,
                                                                 const uint32_t* __restrict__ counts,
                                                                 uint32_t* status, uint32_t* ticket,
                                                                 uint32_t* err, int spin_limit, int stall) {
  __shared__ uint32_t wh[kSortWarps][256];
  __shared__ uint32_t base_s[256];
  __shared__ uint32_t wt[kSortWarps];
  __shared__ int bid_s;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  if (threadIdx.x == 0) bid_s = (int)atomicAdd(ticket, 1u);
  for (int i = lane; i < 256; i += 32) wh[wid][i] = 0;
  __syncthreads();
  const int b = bid_s;
  const int64_t base = (int64_t)b * kSortTile + (int64_t)wid * kWarpTile;
  uint32_t k[kSortItems];
  int dg[kSortItems];
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int64_t i = base + r * 32 + lane;
    k[r] = i < n ? keys_in[i] : 0u;
    dg[r] = i < n ? (int)((k[r] >> shift) & 255u) : 256;
    const unsigned peers = __match_any_sync(0xffffffffu, dg[r]);
    if (dg[r] < 256 && (peers & lt) == 0) wh[wid][dg[r]] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // thread d: this block's count of digit d, published, then the prefix of
  // the blocks before it; the warps' offsets within the block
  const int d = threadIdx.x;  // blockDim.x == 256
  uint32_t local = 0;
  for (int w = 0; w < kSortWarps; ++w) local += wh[w][d];
  cuda::atomic_ref<uint32_t, cuda::thread_scope_device> mine(status[(int64_t)b * 256 + d]);
  const bool publish = b != stall;
  if (publish) mine.store((b == 0 ? kFlagIncl : kFlagLocal) | local, cuda::memory_order_relaxed);
  uint32_t prefix = 0;
  for (int j = b - 1; j >= 0;) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> st(status[(int64_t)j * 256 + d]);
    uint32_t v = st.load(cuda::memory_order_relaxed);
    for (int spin = 0; (v & kFlagMask) == 0; ++spin) {
      if (spin > spin_limit) {
        atomicExch(err, 1u);
        v = kFlagIncl;
        break;
      }
      __nanosleep(64);
      v = st.load(cuda::memory_order_relaxed);
    }
    prefix += v & ~kFlagMask;
    if ((v & kFlagMask) == kFlagIncl) break;
    --j;
  }
  if (b > 0 && publish) mine.store(kFlagIncl | (prefix + local), cuda::memory_order_relaxed);
  // global start of digit d: exclusive scan of the pass's digit counts
  {
    const uint32_t c = counts[d];
    uint32_t inc = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) wt[wid] = inc;
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < wid; ++w) before += wt[w];
    base_s[d] = before + inc - c + prefix;
  }
  __syncthreads();
  {
    uint32_t run = base_s[d];
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = wh[w][d];
      wh[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortItems; ++r) {
    const int64_t i = base + r * 32 + lane;
    const unsigned peers = __match_any_sync(0xffffffffu, dg[r]);
    if (dg[r] < 256) {
      const uint32_t pos = wh[wid][dg[r]] + __popc(peers & lt);
      keys_out[pos] = k[r];
      vals_out[pos] = vals_in[i];
    }
    __syncwarp();
    if (dg[r] < 256 && (peers & lt) == 0) wh[wid][dg[r]] += __popc(peers);
    __syncwarp();
  }
}

// After a sort whose look-back gave up (*err != 0): identity values and
// equal keys, a permutation that every later kernel can read safely.
__global__ void k_sort_repair(int64_t n, const uint32_t* __restrict__ err, uint32_t* keys, int32_t* vals) {
  if (*err == 0u) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    keys[i] = 0u;
    vals[i] = (int32_t)i;
  }
}

cudaError_t radix_sort_pairs(int64_t n, int bits, uint32_t* keys, int32_t* vals, uint32_t* keys_tmp,
                             int32_t* vals_tmp, uint32_t* hist, cudaStream_t s, int* err) {
  if (n <= 1) return cudaSuccess;
  if (n >= (int64_t)1 << 30 || bits > 32) return cudaErrorInvalidValue;
  const int nb = (int)((n + kSortTile - 1) / kSortTile);
  const int passes = (bits + 7) / 8;
  uint32_t* counts = hist;
  uint32_t* tickets = hist + kSortPassesMax * 256;
  uint32_t* errw = err ? reinterpret_cast<uint32_t*>(err) : tickets + kSortPassesMax;
  uint32_t* status = hist + kSortHdr;
  cudaMemsetAsync(hist, 0, sizeof(uint32_t) * (kSortHdr - 4 + (int64_t)passes * 256 * nb + 4), s);
  uint32_t *ki = keys, *ko = keys_tmp;
  int32_t *vi = vals, *vo = vals_tmp;
  count_launch(1 + passes);
  k_radix_counts<<<grid_for(n, kSortThreads, 4), kSortThreads, 0, s>>>(n, passes, ki, counts);
  for (int p = 0; p < passes; ++p) {
    k_radix_onesweep<<<nb, kSortThreads, 0, s>>>(n, 8 * p, ki, vi, ko, vo, counts + 256 * p,
                                                 status + (int64_t)p * 256 * nb, tickets + p, errw,
                                                 g_sort_spin_limit, err ? g_sort_stall : -1);
    uint32_t* tk = ki;
    ki = ko;
    ko = tk;
    int32_t* tv = vi;
    vi = vo;
    vo = tv;
  }
  if (ki != keys) {
    cudaMemcpyAsync(keys, ki, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(vals, vi, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s);
  }
  if (err) {
    count_launch();
    k_sort_repair<<<grid_for(n, 256, 4), 256, 0, s>>>(n, errw, keys, vals);
  }
  return cudaGetLastError();
}

// ======================================================================
// K3: LBVH (Karras 2012) + ropes + refit
// ======================================================================
// Node ids: internal i in [0, n-2]; leaf k -> (n-1) + k.  Root = node 0.
__device__ __forceinline__ int bvh_delta(const uint32_t* __restrict__ codes, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const uint32_t a = codes[i], b = codes[j];
  if (a != b) return __clz(a ^ b);
  return 32 + __clz((uint32_t)i ^ (uint32_t)j);
}

// work layout (ints): parent[2n-1] | rope[n] | visit[n] | last[n] | left[n] | right[n] | first[n]
__global__ void k_bvh_internal(int n, const uint32_t* __restrict__ codes, int* parent, int* rope,
                               int* last, int* left, int* right, int* first_leaf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = (bvh_delta(codes, n, i, i + 1) - bvh_delta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = bvh_delta(codes, n, i, i - d);
  int lmax = 2;
  while (bvh_delta(codes, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (bvh_delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = bvh_delta(codes, n, i, j);
  int s = 0;
  int t = l;
  do {
    t = (t + 1) >> 1;
    if (bvh_delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  const int gamma = i + s * d + (d < 0 ? -1 : 0);
  const int first = i < j ? i : j;
  const int lst = i < j ? j : i;
  const int lc = (first == gamma) ? (n - 1) + gamma : gamma;
  const int rc = (lst == gamma + 1) ? (n - 1) + gamma + 1 : gamma + 1;
  left[i] = lc;
  right[i] = rc;
  parent[lc] = i;
  parent[rc] = i;
  rope[gamma + 1] = rc;
  last[i] = lst;
  if (first_leaf) first_leaf[i] = first;
}

__device__ __forceinline__ int bvh_escape(int n, int node, const int* __restrict__ rope, const int* __restrict__ last) {
  const int r = node >= n - 1 ? node - (n - 1) : last[node];
  return r == n - 1 ? -1 : rope[r + 1];
}

constexpr int kRefitBlock = 256;

template <bool BUCKET>
__global__ void __launch_bounds__(kRefitBlock) k_bvh_refit(int n, const int32_t* __restrict__ sorted_vals, const float4* __restrict__ box32,
                            const int* __restrict__ parent, const int* __restrict__ rope,
                            const int* __restrict__ last, const int* __restrict__ left,
                            const int* __restrict__ right, int* visit, float4* lo_left, float4* hi_esc,
                            int dim, const double* __restrict__ box64, double* leaf,
                            const int* __restrict__ first_leaf, int bucket) {
  // Nodes whose leaf range lies within this block's 256 leaves are merged
  // through shared memory (block-scope counters and boxes) when first_leaf
  // is given; the climb above them uses the device-scope counters.  Node i
  // is an end of its own range, so an in-block node i has i - L in [0, 256).
  __shared__ float4 s_lo[2 * kRefitBlock], s_hi[2 * kRefitBlock];  // leaves, then internal nodes
  __shared__ int s_vis[kRefitBlock];
  const int L = blockIdx.x * kRefitBlock;
  const int R = (L + kRefitBlock < n ? L + kRefitBlock : n) - 1;
  s_vis[threadIdx.x] = 0;
  __syncthreads();
  const int k = L + threadIdx.x;
  if (k >= n) return;
  const int elem = sorted_vals[k];
  int node = (n - 1) + k;
  float4 lo = box32[2 * elem], hi = box32[2 * elem + 1];
  lo.w = __int_as_float(elem);
  hi.w = __int_as_float(bvh_escape(n, node, rope, last));
  lo_left[2 * node] = lo;
  hi_esc[2 * node] = hi;
  s_lo[threadIdx.x] = lo;
  s_hi[threadIdx.x] = hi;
  if (leaf) {
    // leaf record in sorted order: FP64 box (lo at 0.., hi at 3..), element, escape
    double* o = leaf + (int64_t)k * 8;
    for (int c = 0; c < 3; ++c) {
      o[c] = c < dim ? box64[(int64_t)elem * 2 * dim + c] : 0.0;
      o[3 + c] = c < dim ? box64[(int64_t)elem * 2 * dim + dim + c] : 0.0;
    }
    reinterpret_cast<int2*>(o + 6)[0] = make_int2(elem, __float_as_int(hi.w));
    o[7] = 0.0;
  }
  if (n == 1) return;
  int p = parent[node];
  bool local = first_leaf != nullptr;
  for (int guard = 0; guard < 128 && p >= 0; ++guard) {
    if (local) {
      if (first_leaf[p] >= L && last[p] <= R) {
        // block scope: this thread's boxes out, the sibling's in
        __threadfence_block();
        if (atomicAdd_block(&s_vis[p - L], 1) == 0) return;  // sibling not done yet
        __threadfence_block();
        const int lc = left[p], rc = right[p];
        const int ia = lc >= n - 1 ? lc - (n - 1) - L : kRefitBlock + lc - L;
        const int ib = rc >= n - 1 ? rc - (n - 1) - L : kRefitBlock + rc - L;
        const float4 a0 = s_lo[ia], a1 = s_hi[ia], b0 = s_lo[ib], b1 = s_hi[ib];
        float4 l, h;
        l.x = fminf(a0.x, b0.x);
        l.y = fminf(a0.y, b0.y);
        l.z = fminf(a0.z, b0.z);
        l.w = __int_as_float(lc);
        if (BUCKET) {
          const int f = first_leaf[p], cnt = last[p] - f + 1;
          if (cnt <= bucket) l.w = __int_as_float((int)(0x80000000u | ((unsigned)(cnt - 1) << 27) | (unsigned)f));
        }
        h.x = fmaxf(a1.x, b1.x);
        h.y = fmaxf(a1.y, b1.y);
        h.z = fmaxf(a1.z, b1.z);
        h.w = __int_as_float(bvh_escape(n, p, rope, last));
        lo_left[2 * p] = l;
        hi_esc[2 * p] = h;
        s_lo[kRefitBlock + p - L] = l;
        s_hi[kRefitBlock + p - L] = h;
        if (p == 0) return;
        p = parent[p];
        continue;
      }
      local = false;  // above the block's subtrees: device scope from here on
    }
    // release: this thread's node boxes; acquire: the sibling's
    cuda::atomic_ref<int, cuda::thread_scope_device> vis(visit[p]);
    if (vis.fetch_add(1, cuda::memory_order_acq_rel) == 0) return;  // sibling not done yet
    const int lc = left[p], rc = right[p];
    const float4 a0 = __ldcg(&lo_left[2 * lc]), a1 = __ldcg(&hi_esc[2 * lc]);
    const float4 b0 = __ldcg(&lo_left[2 * rc]), b1 = __ldcg(&hi_esc[2 * rc]);
    float4 l, h;
    l.x = fminf(a0.x, b0.x);
    l.y = fminf(a0.y, b0.y);
    l.z = fminf(a0.z, b0.z);
    l.w = __int_as_float(lc);
    if (BUCKET) {
      // a subtree of at most `bucket` leaves becomes a bucket: the node
      // records its first sorted leaf and leaf count instead of its left
      // child, and the search scans those leaf records in order
      const int f = first_leaf[p], cnt = last[p] - f + 1;
      if (cnt <= bucket) l.w = __int_as_float((int)(0x80000000u | ((unsigned)(cnt - 1) << 27) | (unsigned)f));
    }
    h.x = fmaxf(a1.x, b1.x);
    h.y = fmaxf(a1.y, b1.y);
    h.z = fmaxf(a1.z, b1.z);
    h.w = __int_as_float(bvh_escape(n, p, rope, last));
    __stcg(&lo_left[2 * p], l);
    __stcg(&hi_esc[2 * p], h);
    if (p == 0) return;
    p = parent[p];
  }
}

cudaError_t launch_bvh_build(int dim, int n, const uint32_t* sorted_keys, const int32_t* sorted_vals,
                             const float* box32, BVH bvh, int* work, cudaStream_t s, const double* box64) {
  if (n <= 0) return cudaSuccess;
  int* parent = work;
  int* rope = parent + (2 * n - 1);
  int* visit = rope + n;
  int* last = visit + n;
  int* left = last + n;
  int* right = left + n;
  cudaMemsetAsync(visit, 0, sizeof(int) * n, s);
  cudaMemsetAsync(rope, 0xff, sizeof(int) * n, s);  // unset ropes read as "end"
  count_launch(n > 1 ? 2 : 1);
  // leaf buckets need the leaf records (box64) and fit the node encoding
  // (first leaf below 2^27, at most 8 leaves)
  int* first_leaf = right + n;
  const bool buckets = tree_bucket(n, box64 != nullptr) > 1;
  if (n > 1) {
    k_bvh_internal<<<(n - 1 + 255) / 256, 256, 0, s>>>(n, sorted_keys, parent, rope, last, left, right,
                                                       first_leaf);
  }
  cudaMemsetAsync(parent, 0xff, sizeof(int), s);  // parent[root] = -1
  if (buckets)
    k_bvh_refit<true><<<(n + kRefitBlock - 1) / kRefitBlock, kRefitBlock, 0, s>>>(
        n, sorted_vals, reinterpret_cast<const float4*>(box32), parent, rope, last, left, right, visit, bvh.lo_left,
        bvh.hi_esc, dim, box64, bvh.leaf, n > 1 ? first_leaf : nullptr, g_leaf_bucket);
  else
    k_bvh_refit<false><<<(n + kRefitBlock - 1) / kRefitBlock, kRefitBlock, 0, s>>>(
        n, sorted_vals, reinterpret_cast<const float4*>(box32), parent, rope, last, left, right, visit, bvh.lo_left,
        bvh.hi_esc, dim, box64, box64 ? bvh.leaf : nullptr, n > 1 ? first_leaf : nullptr, 1);
  return cudaGetLastError();
}

// ======================================================================
// K4: candidate search
// ======================================================================
// Row cache of the count pass: the first `cap` candidates of row a at
// cache[a * cap ..]; later ones spill into chunks of kSpillChunk entries
// taken from a pool (sp.next counts the chunks handed out), chained per row
// (sp.row_chunk[a] = first chunk, sp.chunk_next[c] = the next one) in
// traversal order.  A row that finds the pool exhausted, or runs without a
// pool, is `lost`: it is listed for a second traversal instead.  Only the
// batched search spills (its mesh pairs of unrelated resolutions give many
// long rows); the single-mesh search (k_query) keeps the tighter walk, with
// fewer registers, and lists its (rare) long rows.
__device__ __forceinline__ void cache_put(int32_t* cache, int cap, const Spill& sp, int64_t a, int cnt, int w,
                                          int& ch, bool& lost) {
  if (cnt < cap) {
    cache[a * cap + cnt] = w;
    return;
  }
  if (lost || !sp.pool) {
    lost = true;
    return;
  }
  const int q = cnt - cap, o = q & (kSpillChunk - 1);
  if (o == 0) {
    const int nc = atomicAdd(sp.next, 1);
    if (nc >= sp.chunks) {
      lost = true;
      return;
    }
    if (q == 0)
      sp.row_chunk[a] = nc;
    else
      sp.chunk_next[ch] = nc;
    ch = nc;
  }
  sp.pool[(int64_t)ch * kSpillChunk + o] = w;
}

// The count pass (FILL = false) also keeps the first `cap` candidates of
// every row in cache[a * cap ..] (when cache is given) and lists rows with
// more than cap candidates in over_rows; the fill then copies cached rows
// (k_fill_from_cache) and traverses again only for the listed rows
// (FILL = true with `rows`).
// With leaf records (`leaf`, in sorted order: FP64 box, element, escape) a
// leaf visit is one load that gives the exact box test and the next node;
// without them it reads the leaf's FP32 node and then the element's FP64
// box, two dependent loads.  Both give the same candidates in the same order.
template <int DIM, bool FILL, bool BUCKET>
__global__ void __launch_bounds__(256) k_query(int64_t nel_a, const double* __restrict__ box64_a,
                                               const float4* __restrict__ lo_left,
                                               const float4* __restrict__ hi_esc, int n,
                                               const double* __restrict__ box64_b, int* counts,
                                               const int64_t* __restrict__ offsets, int32_t* pair_a,
                                               int32_t* pair_b, int32_t* cache, int cap,
                                               const int32_t* __restrict__ rows, int* over_rows,
                                               const double* __restrict__ leaf, int64_t pair_cap) {
  const int64_t nrows = rows ? (int64_t)*over_rows : nel_a;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = rows ? rows[r] : r;
    double lo[DIM], hi[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      lo[c] = box64_a[a * 2 * DIM + c];
      hi[c] = box64_a[a * 2 * DIM + DIM + c];
    }
    float ql[3], qh[3];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      ql[c] = __double2float_rd(lo[c]);
      qh[c] = __double2float_ru(hi[c]);
    }
    int cnt = 0;
    int64_t out = FILL ? offsets[a] : 0;
    int node = 0;
    // Each step moves forward in depth-first order; 2n-1 nodes bound it.
    const int nodes = 2 * n - 1;
    for (int guard = 0; node >= 0 && guard < 2 * n + 1; ++guard) {
      if (node >= nodes) break;  // never taken for a well-formed hierarchy
      if (leaf && node >= n - 1) {
        const double2* q = reinterpret_cast<const double2*>(leaf + (int64_t)(node - (n - 1)) * 8);
        const double2 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2), q3 = __ldg(q + 3);
        const double blo[3] = {q0.x, q0.y, q1.x}, bhi[3] = {q1.y, q2.x, q2.y};
        const int2 meta = make_int2(__double2loint(q3.x), __double2hiint(q3.x));
        bool ex = true;
#pragma unroll
        for (int c = 0; c < DIM; ++c) ex = ex && (hi[c] > blo[c]) && (lo[c] < bhi[c]);
        if (ex) {
          if (FILL) {
            if (out + cnt < pair_cap) {
              pair_a[out + cnt] = (int32_t)a;
              pair_b[out + cnt] = meta.x;
            }
          } else if (cache) {
            if (cnt < cap) cache[a * cap + cnt] = meta.x;
          }
          ++cnt;
        }
        node = meta.y;
        continue;
      }
      const float4 L = __ldg(&lo_left[2 * node]);
      const float4 H = __ldg(&hi_esc[2 * node]);
      bool ov = H.x > ql[0] && L.x < qh[0] && H.y > ql[1] && L.y < qh[1];
      if (DIM == 3) ov = ov && H.z > ql[2] && L.z < qh[2];
      if (ov) {
        const int w = __float_as_int(L.w);
        if (BUCKET && node < n - 1 && w < 0) {
          // leaf bucket: its sorted leaves in order, exact FP64 test each
          // (independent loads), then on past the subtree
          const int f = w & 0x07ffffff, nl = ((w >> 27) & 7) + 1;
          for (int k = 0; k < nl; ++k) {
            const double2* q = reinterpret_cast<const double2*>(leaf + (int64_t)(f + k) * 8);
            const double2 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2), q3 = __ldg(q + 3);
            const double blo[3] = {q0.x, q0.y, q1.x}, bhi[3] = {q1.y, q2.x, q2.y};
            bool ex = true;
#pragma unroll
            for (int c = 0; c < DIM; ++c) ex = ex && (hi[c] > blo[c]) && (lo[c] < bhi[c]);
            if (ex) {
              const int e = __double2loint(q3.x);
              if (FILL) {
                if (out + cnt < pair_cap) {
                  pair_a[out + cnt] = (int32_t)a;
                  pair_b[out + cnt] = e;
                }
              } else if (cache) {
                if (cnt < cap) cache[a * cap + cnt] = e;
              }
              ++cnt;
            }
          }
          node = __float_as_int(H.w);
          continue;
        }
        if (node < n - 1) {
          node = w;
          continue;
        }
        const double* bb = box64_b + (int64_t)w * 2 * DIM;
        bool ex = true;
#pragma unroll
        for (int c = 0; c < DIM; ++c) ex = ex && (hi[c] > bb[c]) && (lo[c] < bb[DIM + c]);
        if (ex) {
          if (FILL) {
            if (out + cnt < pair_cap) {
              pair_a[out + cnt] = (int32_t)a;
              pair_b[out + cnt] = w;
            }
          } else if (cache) {
            if (cnt < cap) cache[a * cap + cnt] = w;
          }
          ++cnt;
        }
      }
      node = __float_as_int(H.w);
    }
    if (!FILL) {
      counts[a] = cnt;
      if (cache && cnt > cap) over_rows[1 + atomicAdd(over_rows, 1)] = (int32_t)a;
    }
  }
}

// Fill of the rows whose candidates the count pass cached: each warp copies
// its 32 rows one after the other, lanes striding over the row (coalesced
// reads of the cache and writes of the pair arrays).
__global__ void __launch_bounds__(256) k_fill_from_cache(int64_t nel_a, const int* __restrict__ counts,
                                                         const int64_t* __restrict__ offsets,
                                                         const int32_t* __restrict__ cache, int cap,
                                                         int32_t* pair_a, int32_t* pair_b, Spill sp,
                                                         int64_t pair_cap) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < nel_a;
       base += warps * 32) {
    const int64_t a = base + lane;
    int cnt = 0;
    int64_t off = 0;
    if (a < nel_a) {
      cnt = counts[a];
      off = offsets[a];
    }
    for (int r = 0; r < 32; ++r) {
      const int c = __shfl_sync(0xffffffffu, cnt, r);
      const int64_t o = __shfl_sync(0xffffffffu, off, r);
      const int64_t row = base + r;
      // entries of this row that fit the pair arrays (all of them unless a
      // capacity-mode call outgrew its arrays)
      const int64_t room = pair_cap - o;
      const int lim = room >= c ? c : (room > 0 ? (int)room : 0);
      if (c > cap) {
        // the cached head, then the row's chain of spill chunks; rows that
        // lost theirs (-2) are filled by the traversal over the listed rows
        const int first = sp.row_chunk ? sp.row_chunk[row] : -2;
        if (first < 0) continue;
        const int head = lim < cap ? lim : cap;
        for (int k = lane; k < head; k += 32) {
          pair_a[o + k] = (int32_t)row;
          pair_b[o + k] = cache[row * cap + k];
        }
        int ch = first;
        for (int k0 = cap; k0 < c; k0 += kSpillChunk) {
          for (int k = lane; k < kSpillChunk && k0 + k < lim; k += 32) {
            pair_a[o + k0 + k] = (int32_t)row;
            pair_b[o + k0 + k] = sp.pool[(int64_t)ch * kSpillChunk + k];
          }
          if (k0 + kSpillChunk < c) ch = sp.chunk_next[ch];
        }
        continue;
      }
      for (int k = lane; k < lim; k += 32) {
        pair_a[o + k] = (int32_t)row;
        pair_b[o + k] = cache[row * cap + k];
      }
    }
  }
}

cudaError_t launch_query(int dim, bool fill, int64_t nel_a, const double* box64_a, BVH bvh,
                         const double* box64_b, int* counts, const int64_t* offsets, int32_t* pair_a,
                         int32_t* pair_b, cudaStream_t s, int32_t* cache, int cap, int* over_rows, Spill sp,
                         int64_t pair_cap) {
  if (nel_a <= 0 || bvh.n <= 0) return cudaSuccess;
  const int B = query_block();
  const int g = grid_for(nel_a, B, 2048 / B);
  if (fill && cache) {
    count_launch(2);
    k_fill_from_cache<<<grid_for(nel_a, 256, 8), 256, 0, s>>>(nel_a, counts, offsets, cache, cap, pair_a, pair_b,
                                                              sp, pair_cap);
  } else {
    count_launch();
  }
  const int32_t* rows = (fill && cache) ? over_rows + 1 : nullptr;
  int32_t* cc = fill ? nullptr : cache;
#define LSM_QUERY_ARGS                                                                                    \
  nel_a, box64_a, bvh.lo_left, bvh.hi_esc, bvh.n, box64_b, counts, offsets, pair_a, pair_b, cc, cap, rows, \
      over_rows, bvh.leaf, pair_cap
  // the bucket scan is compiled in only where the hierarchy has buckets:
  // without them its branch alone slows the walk (2D count pass +27%)
  const bool bk = bvh.bucket > 1;
  if (dim == 2) {
    if (fill)
      bk ? k_query<2, true, true><<<g, B, 0, s>>>(LSM_QUERY_ARGS) : k_query<2, true, false><<<g, B, 0, s>>>(LSM_QUERY_ARGS);
    else
      bk ? k_query<2, false, true><<<g, B, 0, s>>>(LSM_QUERY_ARGS) : k_query<2, false, false><<<g, B, 0, s>>>(LSM_QUERY_ARGS);
  } else {
    if (fill)
      bk ? k_query<3, true, true><<<g, B, 0, s>>>(LSM_QUERY_ARGS) : k_query<3, true, false><<<g, B, 0, s>>>(LSM_QUERY_ARGS);
    else
      bk ? k_query<3, false, true><<<g, B, 0, s>>>(LSM_QUERY_ARGS) : k_query<3, false, false><<<g, B, 0, s>>>(LSM_QUERY_ARGS);
  }
#undef LSM_QUERY_ARGS
  return cudaGetLastError();
}

// ======================================================================
// Scan of int32 counts -> int64 offsets
// ======================================================================
namespace {
constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;
}  // namespace

int64_t scan_tmp_entries(int64_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

template <int BLOCK>
__device__ int64_t block_excl_scan(int64_t v, int64_t* total) {
  __shared__ int64_t wt[BLOCK / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int64_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) wt[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int64_t w = lane < BLOCK / 32 ? wt[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < BLOCK / 32) wt[lane] = w;
  }
  __syncthreads();
  const int64_t r = inc - v + (wid > 0 ? wt[wid - 1] : 0);
  if (total) *total = wt[BLOCK / 32 - 1];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(int64_t n, const int* __restrict__ counts, int64_t* tmp) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) s += counts[base + i];
  int64_t tot;
  block_excl_scan<kScanThreads>(s, &tot);
  if (threadIdx.x == 0) tmp[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_scan_top(int nb, int64_t* tmp) {
  // exclusive scan of tmp[0..nb) in place; tmp[nb] = total
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += 1024) {
    const int i = base + threadIdx.x;
    const int64_t v = i < nb ? tmp[i] : 0;
    int64_t tot;
    const int64_t ex = block_excl_scan<1024>(v, &tot);
    if (i < nb) tmp[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) tmp[nb] = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_down(int64_t n, const int* __restrict__ counts,
                                                            const int64_t* __restrict__ tmp, int64_t* out,
                                                            int nb) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int v[kScanItems];
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = base + i < n ? counts[base + i] : 0;
    s += v[i];
  }
  int64_t run = block_excl_scan<kScanThreads>(s, nullptr) + tmp[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = run;
    run += v[i];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tmp[nb];
}

cudaError_t launch_scan(int64_t n, const int* counts, int64_t* offsets, int64_t* tmp, cudaStream_t s) {
  if (n <= 0) {
    cudaMemsetAsync(offsets, 0, sizeof(int64_t), s);
    return cudaGetLastError();
  }
  const int nb = (int)((n + kScanTile - 1) / kScanTile);
  count_launch(3);
  k_scan_reduce<<<nb, kScanThreads, 0, s>>>(n, counts, tmp);
  k_scan_top<<<1, 1024, 0, s>>>(nb, tmp);
  k_scan_down<<<nb, kScanThreads, 0, s>>>(n, counts, tmp, offsets, nb);
  return cudaGetLastError();
}

// ======================================================================
// K5: triangle clipping
// ======================================================================
namespace {
constexpr int kTriBlock = 128;
constexpr int kTriCap = 8;  // fast-path polygon slots (geometric max is 6)
constexpr int kTriWideCap = 24;
constexpr int kTetStack = 6;      // max pending tets: 2 per level for planes 0-2
}  // namespace

// Polygon in shared memory: slot i, coord c at base[(2*i + c) * BLOCK].
template <int BLOCK>
struct SmemPoly {
  double* base;
  __device__ __forceinline__ double x(int i) const { return base[(2 * i) * BLOCK]; }
  __device__ __forceinline__ double y(int i) const { return base[(2 * i + 1) * BLOCK]; }
  __device__ __forceinline__ void set(int i, double px, double py) {
    base[(2 * i) * BLOCK] = px;
    base[(2 * i + 1) * BLOCK] = py;
  }
};

template <int CAP>
struct LocalPoly {
  double px[CAP], py[CAP];
  __device__ __forceinline__ double x(int i) const { return px[i]; }
  __device__ __forceinline__ double y(int i) const { return py[i]; }
  __device__ __forceinline__ void set(int i, double a, double b) {
    px[i] = a;
    py[i] = b;
  }
};

struct NoEmit {
  __device__ __forceinline__ void operator()(int, double, double, double, double, double, double) const {}
};

// A setup row of kSetup2 doubles (16-byte aligned) in seven 16-byte loads.
__device__ __forceinline__ void load_lines(const double* __restrict__ o, Lines& L, double& tol) {
  const double2* q = reinterpret_cast<const double2*>(o);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double2 n = __ldg(q + 2 * i), pt = __ldg(q + 2 * i + 1);
    L.nx[i] = n.x;
    L.ny[i] = n.y;
    L.px[i] = pt.x;
    L.py[i] = pt.y;
  }
  tol = __ldg(q + 6).x;
}

__global__ void __launch_bounds__(kTriBlock) k_clip_tris(int64_t npairs, const int32_t* __restrict__ pa,
                                                         const int32_t* __restrict__ pb,
                                                         const double* __restrict__ coords_a,
                                                         const double* __restrict__ tol_a,
                                                         const double* __restrict__ setup_b,
                                                         double* pair_measure, int32_t* pair_nout,
                                                         int32_t* ovf_list, int* ovf_count,
                                                         const int32_t* __restrict__ order,
                                                         const int64_t* __restrict__ n_dev) {
  // n_dev (optional): the pair count on the device, npairs its upper bound
  if (n_dev && *n_dev < npairs) npairs = *n_dev;
  __shared__ double poly[2 * 2 * kTriCap * kTriBlock];
  SmemPoly<kTriBlock> p{poly + threadIdx.x}, q{poly + 2 * kTriCap * kTriBlock + threadIdx.x};
  // each iteration loads the next one's pair indices (which stream from
  // DRAM) before it clips its own pair
  const int64_t stride = (int64_t)gridDim.x * kTriBlock;
  int64_t ni = (int64_t)blockIdx.x * kTriBlock + threadIdx.x;
  int na = 0, nb = 0;
  if (ni < npairs) {
    if (order) ni = order[ni];
    na = pa[ni];
    nb = pb[ni];
  }
  for (int64_t j = (int64_t)blockIdx.x * kTriBlock + threadIdx.x; j < npairs; j += stride) {
    const int64_t i = ni;
    const int a = na, b = nb;
    if (j + stride < npairs) {
      ni = order ? (int64_t)order[j + stride] : j + stride;
      na = pa[ni];
      nb = pb[ni];
    }
    const double2* va = reinterpret_cast<const double2*>(coords_a + (int64_t)a * 6);
    const double2 v0 = __ldg(va), v1 = __ldg(va + 1), v2 = __ldg(va + 2);
    Lines L;
    double tolb;
    load_lines(setup_b + (int64_t)b * kSetup2, L, tolb);
    const double tol = fmin(tol_a[a], tolb);
    double m;
    const int n = clip_tri(v0.x, v0.y, v1.x, v1.y, v2.x, v2.y, L, tol, p, q, kTriCap, m, NoEmit{});
    if (n < 0) {
      const int k = atomicAdd(ovf_count, 1);
      ovf_list[k] = (int32_t)i;
      continue;
    }
    pair_measure[i] = m;
    pair_nout[i] = n;
  }
}

__global__ void __launch_bounds__(32) k_clip_tris_wide(const int32_t* __restrict__ list, const int* __restrict__ count,
                                                       int64_t cap, const int32_t* __restrict__ pa,
                                                       const int32_t* __restrict__ pb,
                                                       const double* __restrict__ coords_a,
                                                       const double* __restrict__ tol_a,
                                                       const double* __restrict__ setup_b,
                                                       double* pair_measure, int32_t* pair_nout) {
  int64_t nl = *count;
  if (nl > cap) nl = cap;
  for (int64_t j = threadIdx.x; j < nl; j += 32) {
    const int64_t i = list[j];
    const int a = pa[i], b = pb[i];
    const double* va = coords_a + (int64_t)a * 6;
    Lines L;
    double tolb;
    load_lines(setup_b + (int64_t)b * kSetup2, L, tolb);
    const double tol = fmin(tol_a[a], tolb);
    LocalPoly<kTriWideCap> p, q;
    double m;
    int n = clip_tri(va[0], va[1], va[2], va[3], va[4], va[5], L, tol, p, q, kTriWideCap, m, NoEmit{});
    if (n < 0) {  // cannot happen: 3 -> 6 -> 12 -> 24 vertices at most
      n = 0;
      m = 0.0;
    }
    pair_measure[i] = m;
    pair_nout[i] = n;
  }
}

// ======================================================================
// K6: tetrahedron clipping, depth-first
// ======================================================================
struct TetStackLocal {
  Tet slot[kTetStack];
  __device__ __forceinline__ void store(int s, const Tet& t) { slot[s] = t; }
  __device__ __forceinline__ void load(int s, Tet& t) const { t = slot[s]; }
};

// Sink for clip_tet_plane inside the depth-first walk: at the last plane it
// evaluates final tets (vol_v4 >= tol, then the vertex-1 volume) in order;
// before that it parks children 1..k-1 on the stack so that child 1 is on
// top (pre-order = the reference's breadth-first output order).
template <class Stack, class Leaf>
struct DfsSink {
  Stack& stk;
  Leaf& leaf;
  int sp;
  bool last;
  double tol;
  int k;
  int kept;
  __device__ __forceinline__ void begin(int kk) { k = kk; }
  __device__ __forceinline__ void child(int j, const Tet& c) {
    if (last) {
      if (tet_volume_v4(c) >= tol) {
        leaf(c);
        ++kept;
      }
    } else if (j > 0) {
      stk.store(sp + (k - 1) - j, c);
    }
  }
};

__device__ __forceinline__ void load_plane(const double* __restrict__ planes, int L, double& nx, double& ny,
                                           double& nz, double& c) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(planes + 4 * L));
  const double2 b = __ldg(reinterpret_cast<const double2*>(planes + 4 * L + 2));
  nx = a.x;
  ny = a.y;
  nz = b.x;
  c = b.y;
}

// Plane source for the depth-first walk: planes computed in registers.
struct RegPlanes {
  const Planes& P;
  __device__ __forceinline__ void get(int L, double& nx, double& ny, double& nz, double& c) const {
    nx = sel4(L, P.nx[0], P.nx[1], P.nx[2], P.nx[3]);
    ny = sel4(L, P.ny[0], P.ny[1], P.ny[2], P.ny[3]);
    nz = sel4(L, P.nz[0], P.nz[1], P.nz[2], P.nz[3]);
    c = sel4(L, P.c[0], P.c[1], P.c[2], P.c[3]);
  }
};

// Depth-first clip of tet `t` by NP planes; calls leaf(tet) for each final
// tet with vol_v4 >= tol, in the reference's output order.  Returns the
// number of kept tets.  The stack needs 2*(NP-1) slots.
template <int NP = 4, class Src, class Stack, class Leaf>
__device__ __forceinline__ int clip_tet_dfs(Tet t, const Src& planes, double tol, Stack& stk, Leaf leaf) {
  int sp = 0;
  unsigned long long levels = 0;  // 3 bits per stack slot
  int L = 0;
  int kept = 0;
  for (int guard = 0; guard < 1200; ++guard) {  // at most (3^NP - 1)/2 tets are clipped
    double nx, ny, nz, c;
    planes.get(L, nx, ny, nz, c);
    DfsSink<Stack, Leaf> sink{stk, leaf, sp, L == NP - 1, tol, 0, 0};
    const int k = clip_tet_plane(t, nx, ny, nz, c, sink);
    kept += sink.kept;
    if (L < NP - 1 && k > 0) {
      if (k > 1) levels |= (unsigned long long)(L + 1) << (3 * sp);
      if (k > 2) levels |= (unsigned long long)(L + 1) << (3 * (sp + 1));
      sp += k - 1;
      ++L;
      continue;
    }
    if (sp == 0) break;
    --sp;
    stk.load(sp, t);
    L = (int)((levels >> (3 * sp)) & 7ull);
    levels &= ~(7ull << (3 * sp));
  }
  return kept;
}

// Planes in a per-thread array (explicit pairs: hex faces).
template <int NP>
struct ArrPlanes {
  double nx[NP], ny[NP], nz[NP], c[NP];
  __device__ __forceinline__ void get(int L, double& a, double& b, double& d, double& e) const {
    a = nx[L];
    b = ny[L];
    d = nz[L];
    e = c[L];
  }
};

template <int N>
struct TetStackN {
  Tet slot[N];
  __device__ __forceinline__ void store(int s, const Tet& t) { slot[s] = t; }
  __device__ __forceinline__ void load(int s, Tet& t) const { t = slot[s]; }
};

__device__ __forceinline__ void load_tet(const double* __restrict__ v, Tet& t) {
  const double2* q = reinterpret_cast<const double2*>(v);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double2 a = __ldg(q + 3 * k), b = __ldg(q + 3 * k + 1), c = __ldg(q + 3 * k + 2);
    // vertices 2k and 2k+1: (a.x a.y b.x) (b.y c.x c.y)
    t.x[2 * k] = a.x;
    t.y[2 * k] = a.y;
    t.z[2 * k] = b.x;
    t.x[2 * k + 1] = b.y;
    t.y[2 * k + 1] = c.x;
    t.z[2 * k + 1] = c.y;
  }
}

// Exact early-out for the tet clipper.  If every vertex of A lies at
// distance >= eps + margin on the outer side of one of B's face planes, then
// so does every tet the reference's clipping derives from A: derived
// vertices are convex combinations of A's vertices, and the rounding of at
// most three nested interpolations plus the distance evaluation moves them by
// far less than margin = 64*eps*(1 + 2M) (M bounds the coordinates and plane
// offsets involved).  Such a tet is classified entirely positive at that
// plane and discarded, so the reference returns no tets: the pair's result is
// written here (0 tets, measure 0) and only the remaining pairs are listed
// for the clipper.
// With faces_a / screen_b (optional) a pair that passes this test gets the
// second one: B beyond a face plane of A by the margin derived next to
// tet_screen_b, which again proves that the reference returns no tets.
// `order` (optional) lists the pairs in the order the clipper should take
// them (a schedule); survivors are appended in that order, warp by warp.
// A plane of B with every vertex of A at distance <= -(eps + margin) keeps
// every tet derived from A whole (all its vertices classify negative), so it
// changes nothing in the reference's result; such planes form the pair's
// no-op mask.  With all four planes no-op the reference returns A itself,
// which is settled here (volume test and measure as in the clipper).
// Survivors are written as {pair, a, b, no-op mask} so that the clipper
// gets the element numbers and the planes to skip in one load.
// kSettle false (the P1 mass pass, explicit pairs with output tets): pairs
// with all four planes no-op are listed too, for the clipper to emit A
// itself; rejected pairs get measure 0 and count 0 where pair_measure is
// given (the P1 pass passes none and zero-fills its blocks).
#ifndef LSM_PREFILTER_BPS
#define LSM_PREFILTER_BPS 2
#endif
// NP planes per B element in setup rows of clip_row(NP) doubles (4: tets,
// 6: hexahedra; the second early-out is for tets only).  The margin covers
// the up to NP-1 nested interpolations of a derived vertex (each within
// ~7 eps M of an exact convex combination) with room to spare.
__host__ __device__ constexpr int clip_row(int np) { return 4 * np + 4; }

// Pairs per block of the early-out pass (256 threads): one contiguous range
// each, a multiple of the block size.
constexpr int kSegChunk = 64;
__host__ __device__ inline int64_t seg_per(int64_t npairs, int grid) {
  return ((npairs + grid - 1) / grid + 255) / 256 * 256;
}

template <bool kSettle, int NP = 4, bool kSeg = false>
__global__ void __launch_bounds__(256, LSM_PREFILTER_BPS) k_prefilter_tets(int64_t npairs, const int32_t* __restrict__ order,
                                                        const int32_t* __restrict__ pa,
                                                        const int32_t* __restrict__ pb,
                                                        const double* __restrict__ coords_a,
                                                        const double* __restrict__ tol_a,
                                                        const double* __restrict__ setup_b,
                                                        double* pair_measure, int32_t* pair_nout,
                                                        int32_t* survivors, unsigned long long* nsurv,
                                                        const double* __restrict__ faces_a,
                                                        const double* __restrict__ screen_b,
                                                        const int64_t* __restrict__ n_dev, int* seg_count = nullptr) {
  // n_dev (optional): the pair count on the device, npairs its upper bound
  if (n_dev && *n_dev < npairs) npairs = *n_dev;
  __shared__ unsigned s_cnt;
  if (kSeg) {
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  // each block takes one contiguous range of pairs (consecutive iterations
  // then share A rows and most B elements in L1)
  const int64_t per = seg_per(npairs, gridDim.x);  // a multiple of the block size (256)
  const int64_t beg = (int64_t)blockIdx.x * per;
  const int64_t end = beg + per < npairs ? beg + per : npairs;
  // the pair indices stream from DRAM: each iteration loads the next one's
  // (ni, na, nb) while it tests its own pair
  int64_t ni = beg + threadIdx.x;
  int na = 0, nb = 0;
  if (ni < end) {
    if (order) ni = order[ni];
    na = pa[ni];
    nb = pb[ni];
  }
  for (int64_t base = beg; base < end; base += blockDim.x) {
    const int64_t j = base + threadIdx.x;
    bool live = false;
    const int64_t i = ni;
    const int a = na, b = nb;
    int noop = 0;
    {
      const int64_t jn = j + blockDim.x;
      if (jn < end) {
        ni = order ? (int64_t)order[jn] : jn;
        na = pa[ni];
        nb = pb[ni];
      }
    }
    if (j < end) {
      Tet t;
      load_tet(coords_a + (int64_t)a * 12, t);
      const double* pl = setup_b + (int64_t)b * clip_row(NP);
      double M = 0.0;
#pragma unroll
      for (int k = 0; k < 4; ++k) M = fmax(M, fmax(fabs(t.x[k]), fmax(fabs(t.y[k]), fabs(t.z[k]))));
      bool reject = false;
#pragma unroll
      for (int L = 0; L < NP; ++L) {
        double nx, ny, nz, c;
        load_plane(pl, L, nx, ny, nz, c);
        const double thr = kEps + 64.0 * kEps * (1.0 + 2.0 * fmax(M, fabs(c)));
        double dmin = DBL_MAX, dmax = -DBL_MAX;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double d = ((nx * t.x[k] + ny * t.y[k]) + nz * t.z[k]) - c;
          dmin = fmin(dmin, d);
          dmax = fmax(dmax, d);
        }
        reject = reject || dmin >= thr;
        noop |= dmax <= -thr ? 1 << L : 0;
      }
      if (NP == 4 && !reject && faces_a) {
        const double2* sb = reinterpret_cast<const double2*>(screen_b + (int64_t)b * kScreen3);
        const double2 gt = __ldg(sb + 6), mz = __ldg(sb + 7);
        if (gt.x < DBL_MAX) {  // B's planes bound a proper tet
          Tet u;
          load_tet(screen_b + (int64_t)b * kScreen3, u);
          const double Mp = fmax(M, mz.x);
          const double e = kEps + 128.0 * kEps * (1.0 + 2.0 * Mp);
          const double slack = 1.01 * gt.x * (gt.y + e) + 16.0 * kEps * (1.0 + Mp);
          const double2* fa = reinterpret_cast<const double2*>(faces_a + (int64_t)a * kScreen3);
#pragma unroll
          for (int P = 0; P < 4; ++P) {
            const double2 n01 = __ldg(fa + 2 * P), n2h = __ldg(fa + 2 * P + 1);
            double m = DBL_MAX;
#pragma unroll
            for (int k = 0; k < 4; ++k) m = fmin(m, (n01.x * u.x[k] + n01.y * u.y[k]) + n2h.x * u.z[k]);
            reject = reject || m >= n2h.y + slack;
          }
        }
      }
      if (!kSettle) {
        live = !reject;
        if (reject && pair_measure) {
          pair_measure[i] = 0.0;
          pair_nout[i] = 0;
        }
      } else if (reject) {
        pair_measure[i] = 0.0;
        pair_nout[i] = 0;
      } else if (noop == (1 << NP) - 1) {
        // A inside all planes: the reference keeps A as its one tet
        double v1;
        const bool keep = final_tet_keep(t, fmin(tol_a[a], pl[4 * NP]), v1);
        pair_measure[i] = keep ? v1 : 0.0;
        pair_nout[i] = keep ? 1 : 0;
      } else {
        live = true;
      }
    }
    const unsigned mask = __ballot_sync(0xffffffffu, live);
    if (mask) {
      const int leader = __ffs(mask) - 1;
      unsigned long long off = 0;
      if (lane == leader)
        off = kSeg ? (unsigned long long)beg + atomicAdd(&s_cnt, (unsigned)__popc(mask))
                   : atomicAdd(nsurv, (unsigned long long)__popc(mask));
      off = __shfl_sync(0xffffffffu, off, leader);
      if (live) {
        const int64_t o = (int64_t)off + __popc(mask & lt);
        reinterpret_cast<int4*>(survivors)[o] = make_int4((int)i, a, b, noop);
      }
    }
  }
  if (kSeg) {
    __syncthreads();
    if (threadIdx.x == 0) seg_count[blockIdx.x] = (int)s_cnt;
  }
}

// Segmented survivor lists.  With kSeg the early-out pass takes no global
// atomic per warp: block k appends its survivors at k * per (per = the pairs
// a block takes, so a segment never outgrows its range) through a counter
// in shared memory and writes the segment's length to seg_count[k].  The
// clipper then claims whole chunks of at most kIxChunk records that lie in
// one segment from a table, in segment order: {first, end, position in the
// compacted list, 0}.  The table kernel runs one block per segment (the
// early-out pass's grid) and writes the survivor count (work[0]) and the
// chunk count (work[2]).
int64_t seg_table_entries(int64_t npairs) { return npairs / kSegChunk + (int64_t)sm_count() * 8 + 1; }
int seg_blocks(int64_t npairs) { return grid_for(npairs, 256, 8); }

__global__ void __launch_bounds__(256) k_seg_chunks(int64_t npairs, const int64_t* __restrict__ n_dev,
                                                    const int* __restrict__ seg_count, int4* table,
                                                    unsigned long long* work) {
  if (n_dev && *n_dev < npairs) npairs = *n_dev;
  const int64_t per = seg_per(npairs, gridDim.x);
  __shared__ long long part[2][8];
  long long sn = 0, sc = 0;
  for (int k = threadIdx.x; k < (int)blockIdx.x; k += blockDim.x) {
    const int c = seg_count[k];
    sn += c;
    sc += (c + kSegChunk - 1) / kSegChunk;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sn += __shfl_xor_sync(0xffffffffu, sn, o);
    sc += __shfl_xor_sync(0xffffffffu, sc, o);
  }
  if ((threadIdx.x & 31) == 0) {
    part[0][threadIdx.x >> 5] = sn;
    part[1][threadIdx.x >> 5] = sc;
  }
  __syncthreads();
  long long pn = 0, pc = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    pn += part[0][w];
    pc += part[1][w];
  }
  const int cnt = seg_count[blockIdx.x];
  const int nch = (cnt + kSegChunk - 1) / kSegChunk;
  const int64_t first = (int64_t)blockIdx.x * per;
  for (int j = threadIdx.x; j < nch; j += blockDim.x) {
    const int lo = j * kSegChunk, hi = lo + kSegChunk < cnt ? lo + kSegChunk : cnt;
    table[pc + j] = make_int4((int)(first + lo), (int)(first + hi), (int)(pn + lo), 0);
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
    work[0] = (unsigned long long)(pn + cnt);
    work[2] = (unsigned long long)(pc + nch);
  }
}

// The segmented list gathered into one compacted list (in table order): for
// consumers that index survivors directly.  One warp per chunk.
__global__ void __launch_bounds__(256) k_seg_compact(int64_t max_chunks, const unsigned long long* __restrict__ nchunks,
                                                     const int4* __restrict__ table, const int4* __restrict__ seg,
                                                     int4* out) {
  const int64_t nc = (int64_t)*nchunks < max_chunks ? (int64_t)*nchunks : max_chunks;
  const int lane = threadIdx.x & 31;
  for (int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nc;
       c += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int4 t = table[c];
    for (int k = lane; k < t.y - t.x; k += 32) out[(int64_t)t.z + k] = seg[(int64_t)t.x + k];
  }
}

cudaError_t launch_seg_compact(int64_t npairs, const unsigned long long* nchunks, const int4* table,
                               const int4* seg, int4* out, cudaStream_t s) {
  const int64_t maxc = seg_table_entries(npairs);
  count_launch();
  k_seg_compact<<<grid_for(maxc * 32, 256, 8), 256, 0, s>>>(maxc, nchunks, table, seg, out);
  return cudaGetLastError();
}

// The early-out pass over n pairs into `survivors`: one list counted in
// work[0], or, with seg, per-block segments and their chunk table (work[0]
// survivors, work[2] chunks).  The clipper then takes seg_nlist(seg, work)
// and seg_table(seg).
namespace {
inline bool seg_on(const SegList* seg) { return seg && seg->count && seg->table; }
inline const unsigned long long* seg_nlist(const SegList* seg, const unsigned long long* work) {
  return seg_on(seg) ? work + 2 : work;
}
inline const int4* seg_table(const SegList* seg) { return seg_on(seg) ? seg->table : nullptr; }
template <bool kSettle, int NP>
void run_prefilter(int64_t n, const int32_t* order, const int32_t* pa, const int32_t* pb, const double* coords_a,
                   const double* tol_a, const double* setup, double* measure, int32_t* nout, int32_t* survivors,
                   unsigned long long* work, const double* faces_a, const double* screen_b, const int64_t* n_dev,
                   const SegList* seg, cudaStream_t s) {
  const int gp = grid_for(n, 256, 8);
  if (seg_on(seg)) {
    count_launch(2);
    k_prefilter_tets<kSettle, NP, true><<<gp, 256, 0, s>>>(n, order, pa, pb, coords_a, tol_a, setup, measure, nout,
                                                           survivors, work, faces_a, screen_b, n_dev, seg->count);
    k_seg_chunks<<<gp, 256, 0, s>>>(n, n_dev, seg->count, seg->table, work);
  } else {
    count_launch();
    k_prefilter_tets<kSettle, NP><<<gp, 256, 0, s>>>(n, order, pa, pb, coords_a, tol_a, setup, measure, nout,
                                                     survivors, work, faces_a, screen_b, n_dev);
  }
}
}  // namespace

// ----------------------------------------------------------------------
// K6: depth-first tet clipper over point indices
// ----------------------------------------------------------------------
// One pair per lane, depth-first, lanes refilled from the survivor list; a
// tet is four 5-bit indices into the lane's point pool in shared memory
// instead of twelve doubles in registers.  Pool slots 0-3 hold A's vertices; the split at
// plane L writes its (at most four) new points to slots 4+4L .. 7+4L.  In
// depth-first order that is safe: a tet at plane L references only points of
// planes < L, and when a sibling is taken from the stack every point written
// by the previous sibling's subtree belongs to planes >= its own.  Child
// assembly becomes integer work on index tuples, a pending tet is one word,
// and vertices are fetched by index with shared-memory loads instead of
// chains of selects.
constexpr int kIxPoints = 20;  // 4 + 4 per plane
#ifndef LSM_IX_BLOCK
#define LSM_IX_BLOCK 480
#endif
#ifndef LSM_IX_BPS
#define LSM_IX_BPS 1
#endif
// 480 B of shared memory per lane (the point pool; pending tets are kept in
// registers): one block of 480 threads (15 warps) fills the 228 KB of an SM.
constexpr int kIxBlock = LSM_IX_BLOCK;
constexpr int kIxBlocksPerSm = LSM_IX_BPS;

__device__ __forceinline__ unsigned ix_pack(unsigned a, unsigned b, unsigned c, unsigned d) {
  return a | b << 5 | c << 10 | d << 15;
}

__device__ __forceinline__ unsigned ix_vert(unsigned tet, int v) { return (tet >> (5 * v)) & 31u; }

__device__ __forceinline__ unsigned ix_set(unsigned tet, int v, unsigned j) {
  return (tet & ~(31u << (5 * v))) | j << (5 * v);
}

// A lane's point pool: point j, coordinate c at pool[(3j + c) * BLOCK]
// (consecutive lanes hit consecutive banks).
template <int BLOCK>
struct IxPool {
  double* pool;
  __device__ __forceinline__ V3 get(unsigned j) const {
    const double* q = pool + 3 * j * BLOCK;
    return V3{q[0], q[BLOCK], q[2 * BLOCK]};
  }
  __device__ __forceinline__ void put(unsigned j, const V3& v) const {
    double* q = pool + 3 * j * BLOCK;
    q[0] = v.x;
    q[BLOCK] = v.y;
    q[2 * BLOCK] = v.z;
  }
};

template <class Pool>
__device__ __forceinline__ void ix_gather(const Pool& pool, unsigned tet, Tet& t) {
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const V3 q = pool.get(ix_vert(tet, v));
    t.x[v] = q.x;
    t.y[v] = q.y;
    t.z[v] = q.z;
  }
}

// Split of tet `cur` (coordinates t, classification k) at the plane whose new
// points go to pool slots base .. base+3 (Tetrahedron_Intersection.F90:290-434,
// same cases, interpolations and child order as split_tet).  Returns the
// number of children; c0..c2 receive their index tuples.
template <class Pool>
__device__ __forceinline__ int ix_split(unsigned cur, const TetClass& k, const Pool& pool, unsigned base,
                                        unsigned& c0, unsigned& c1, unsigned& c2) {
  const int nn = k.nn, np = k.np;
  const int n0 = k.negl & 3, n1 = (k.negl >> 2) & 3, n2 = (k.negl >> 4) & 3;
  const int p0 = k.posl & 3, p1 = (k.posl >> 2) & 3, p2 = (k.posl >> 4) & 3;
  int ni;
  unsigned pairs;
  if (nn == 1) {
    ni = np;
    pairs = (unsigned)(p0 | n0 << 2) | (unsigned)(p1 | n0 << 2) << 4 | (unsigned)(p2 | n0 << 2) << 8;
  } else if (np == 2) {
    ni = 4;
    pairs = (unsigned)(p0 | n0 << 2) | (unsigned)(p1 | n0 << 2) << 4 | (unsigned)(p0 | n1 << 2) << 8 |
            (unsigned)(p1 | n1 << 2) << 12;
  } else {
    ni = nn;
    pairs = (unsigned)(p0 | n0 << 2) | (unsigned)(p0 | n1 << 2) << 4 | (unsigned)(p0 | n2 << 2) << 8;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (i < ni) {
      const int P = (pairs >> (4 * i)) & 3, N = (pairs >> (4 * i + 2)) & 3;
      const V3 T = interp(pool.get(ix_vert(cur, P)), pool.get(ix_vert(cur, N)),
                          sel4(P, k.d[0], k.d[1], k.d[2], k.d[3]), sel4(N, k.d[0], k.d[1], k.d[2], k.d[3]));
      pool.put(base + i, T);
    }
  }
  if (nn == 1) {  // +++-, ++-0, +-00: the r-th positive vertex becomes new point r
    unsigned c = cur;
#pragma unroll
    for (int r = 0; r < 3; ++r)
      if (r < np) c = ix_set(c, (k.posl >> (2 * r)) & 3, base + r);
    c0 = c;
    return 1;
  }
  if (np == 2) {  // ++--
    c0 = ix_set(ix_set(cur, p0, base + 2), p1, base + 1);
    c1 = ix_pack(ix_vert(cur, n1), base + 3, base + 2, base + 1);
    c2 = ix_pack(ix_vert(cur, n0), base + 0, base + 1, base + 2);
    return 3;
  }
  c0 = ix_set(cur, p0, base);
  if (nn == 3) {  // +---
    c1 = ix_pack(base + 0, ix_vert(cur, n1), ix_vert(cur, n2), base + 1);
    c2 = ix_pack(ix_vert(cur, n2), base + 1, base + 2, base + 0);
    return 3;
  }
  // +--0
  c1 = ix_pack(base + 1, ix_vert(cur, k.zerl & 3), ix_vert(cur, n1), base + 0);
  return 2;
}

// Pairs reach the lanes through a software pipeline so that the dependent
// loads of a new pair (survivor record {pair, a, b} -> A coordinates and
// tolerances) never stall the warp: every lane prefetches its next pair one
// stage per loop iteration while it clips the current one.  Records are
// taken from a warp-private cursor over chunks of kIxChunk list entries (one
// atomic per chunk).
constexpr int kIxChunk = 64;

// What the clipper does with a pair's kept output tets (each passed with
// its vertex-1 volume, in the reference's output order).  kInside: the list
// may hold pairs whose every plane is a no-op (A inside B: its one output
// tet is A itself), which the supermesh's early-out pass settles itself.
struct IxMeasureSink {
  static constexpr bool kInside = false;
  static constexpr int kLaneDoubles = 0;  // shared memory per lane behind the point pool
  double* pair_measure;
  int32_t* pair_nout;
  double m;
  int kept;
  __device__ __forceinline__ void bind(double*) {}
  __device__ __forceinline__ void begin(const int4&) {
    m = 0.0;
    kept = 0;
  }
  __device__ __forceinline__ void tet(const Tet&, double v1) {
    m = m + v1;
    ++kept;
  }
  __device__ __forceinline__ void end(int64_t p) {
    pair_measure[p] = m;
    pair_nout[p] = kept;
  }
  template <int BLOCK>
  __device__ __forceinline__ void finish() {}
};

// Measure and count per pair and, for explicit pairs, the output tets:
// elems (optional) [n][kCap][4][3] in the reference's order (tets beyond
// kCap are counted, not stored: 81 for tet-tet, 729 for tet-hex).  The list
// includes pairs with every plane a no-op.
template <int kCap>
struct IxElemSinkT {
  static constexpr bool kInside = true;
  static constexpr int kLaneDoubles = 0;
  double* pair_measure;
  int32_t* pair_nout;
  double* elems;
  double m;
  int kept;
  int pid;
  __device__ __forceinline__ void bind(double*) {}
  __device__ __forceinline__ void begin(const int4& r) {
    m = 0.0;
    kept = 0;
    pid = r.x;
  }
  __device__ __forceinline__ void tet(const Tet& o, double v1) {
    if (elems && kept < kCap) {
      double2* e = reinterpret_cast<double2*>(elems + ((int64_t)pid * kCap + kept) * 12);
      e[0] = make_double2(o.x[0], o.y[0]);
      e[1] = make_double2(o.z[0], o.x[1]);
      e[2] = make_double2(o.y[1], o.z[1]);
      e[3] = make_double2(o.x[2], o.y[2]);
      e[4] = make_double2(o.z[2], o.x[3]);
      e[5] = make_double2(o.y[3], o.z[3]);
    }
    m = m + v1;
    ++kept;
  }
  __device__ __forceinline__ void end(int64_t p) {
    pair_measure[p] = m;
    pair_nout[p] = kept;
  }
  template <int NT>
  __device__ __forceinline__ void finish() {}
};

using IxElemSink = IxElemSinkT<81>;

// As IxElemSinkT, but a pair's sum, count and output tets continue from
// what an earlier launch left in pair_measure / pair_nout / elems: the
// hexahedron-hexahedron pairs clip A's five tets in five launches, and the
// reference sums and lists all their output tets in one running order.
template <int kCap>
struct IxCarrySinkT {
  static constexpr bool kInside = true;
  static constexpr int kLaneDoubles = 0;
  double* pair_measure;
  int32_t* pair_nout;
  double* elems;
  double m;
  int kept;
  int pid;
  __device__ __forceinline__ void bind(double*) {}
  __device__ __forceinline__ void begin(const int4& r) {
    pid = r.x;
    m = pair_measure[pid];
    kept = pair_nout[pid];
  }
  __device__ __forceinline__ void tet(const Tet& o, double v1) {
    if (elems && kept < kCap) {
      double2* e = reinterpret_cast<double2*>(elems + ((int64_t)pid * kCap + kept) * 12);
      e[0] = make_double2(o.x[0], o.y[0]);
      e[1] = make_double2(o.z[0], o.x[1]);
      e[2] = make_double2(o.y[1], o.z[1]);
      e[3] = make_double2(o.x[2], o.y[2]);
      e[4] = make_double2(o.z[2], o.x[3]);
      e[5] = make_double2(o.y[3], o.z[3]);
    }
    m = m + v1;
    ++kept;
  }
  __device__ __forceinline__ void end(int64_t p) {
    pair_measure[p] = m;
    pair_nout[p] = kept;
  }
  template <int NT>
  __device__ __forceinline__ void finish() {}
};
constexpr int kHexHexCap = 5 * 729;  // output tets per hexahedron pair

// The supermesh's tets, written where the scan of the per-pair counts puts
// them: tet j of pair p at elems[pair_off[p] + j], with its parents.
struct IxEmitSink {
  static constexpr bool kInside = true;
  static constexpr int kLaneDoubles = 0;
  const int64_t* pair_off;
  double* elems;
  int64_t* parent_a;
  int64_t* parent_b;
  int64_t at;
  int a, b;
  __device__ __forceinline__ void bind(double*) {}
  __device__ __forceinline__ void begin(const int4& r) {
    at = pair_off[r.x];
    a = r.y;
    b = r.z;
  }
  __device__ __forceinline__ void tet(const Tet& o, double) {
    double2* e = reinterpret_cast<double2*>(elems + at * 12);
    e[0] = make_double2(o.x[0], o.y[0]);
    e[1] = make_double2(o.z[0], o.x[1]);
    e[2] = make_double2(o.y[1], o.z[1]);
    e[3] = make_double2(o.x[2], o.y[2]);
    e[4] = make_double2(o.z[2], o.x[3]);
    e[5] = make_double2(o.y[3], o.z[3]);
    if (parent_a) parent_a[at] = a;
    if (parent_b) parent_b[at] = b;
    ++at;
  }
  __device__ __forceinline__ void end(int64_t) {}
  template <int NT>
  __device__ __forceinline__ void finish() {}
};

// Points in a lane's pool for NP planes: A's 4 vertices + 4 per plane.
__host__ __device__ constexpr int ix_points(int np) { return 4 + 4 * np; }

template <class Sink, int BLOCK, int BPS, int NP = 4>
__global__ void __launch_bounds__(BLOCK, BPS) k_clip_tets_ix(
    const int4* __restrict__ list, const unsigned long long* __restrict__ nlist, const double* __restrict__ coords_a,
    const double* __restrict__ tol_a, const double* __restrict__ setup_b, Sink sk, unsigned long long* work,
    const int4* __restrict__ chunks = nullptr) {
  // chunks (optional): the list is segmented; nlist then counts the table's
  // chunks and work counts the chunks taken
  static_assert(ix_points(NP) <= 32, "pool indices are 5 bits");
  extern __shared__ double ix_mem[];
  IxPool<BLOCK> pool{ix_mem + threadIdx.x};
  sk.bind(ix_mem + 3 * ix_points(NP) * BLOCK + threadIdx.x);
  // pending tets (at most 2 per plane but the last): a shift register of
  // 20-bit index tuples over kW words (stk[kW-1]:...:stk[0], newest in the
  // low bits) and their planes, kLB bits each (stk_lv)
  constexpr int kW = NP <= 4 ? 2 : 4;
  constexpr int kLB = NP <= 4 ? 2 : 3;
  static_assert(2 * (NP - 1) * 20 <= 64 * kW && 2 * (NP - 1) * kLB <= 32, "pending-tet stack too small");
  unsigned long long stk[kW];
#pragma unroll
  for (int w = 0; w < kW; ++w) stk[w] = 0;
  unsigned stk_lv = 0;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t npairs = (int64_t)*nlist;
  // warp cursor over the list (warp-uniform)
  int64_t cbeg = 0, cend = 0;
  bool exhausted = false;
  // prefetch pipeline of the next pair: stage 0 idle, 1 record loading,
  // 2 element data loading (ready for the next refill)
  int nstage = 0;
  int4 nrec = make_int4(0, 0, 0, 0);
  Tet nt;
  double ntol = 0.0;
  // current pair
  int64_t p = -1;
  const double* planes = setup_b;
  unsigned cur = 0;
  double tol = 0.0;
  int L = 0, sp = 0;
  // planes this pair clips at (bit L; the prefilter's no-op planes are
  // skipped) and the last of them
  constexpr unsigned kAll = (1u << NP) - 1u;
  unsigned act = kAll;
  int lastL = NP - 1;
  for (;;) {
    // ---- prefetch pipeline
    if (nstage == 1) {
      load_tet(coords_a + (int64_t)nrec.y * 12, nt);
      ntol = fmin(tol_a[nrec.y], setup_b[(int64_t)nrec.z * clip_row(NP) + 4 * NP]);
      nstage = 2;
    }
    if (p < 0 && nstage == 2) {
      p = nrec.x;
#pragma unroll
      for (int v = 0; v < 4; ++v) pool.put(v, V3{nt.x[v], nt.y[v], nt.z[v]});
      planes = setup_b + (int64_t)nrec.z * clip_row(NP);
      tol = ntol;
      cur = ix_pack(0, 1, 2, 3);
      sk.begin(nrec);
      act = ~(unsigned)nrec.w & kAll;  // never 0 unless Sink::kInside
      L = __ffs(act) - 1;
      lastL = 31 - __clz(act);
      sp = 0;
      nstage = 0;
#pragma unroll
      for (int w = 0; w < kW; ++w) stk[w] = 0;
      stk_lv = 0;
      if (Sink::kInside && act == 0u) {
        // A inside all four planes: the reference keeps A as its one tet
        Tet o;
        ix_gather(pool, cur, o);
        double v1;
        if (final_tet_keep(o, tol, v1)) sk.tet(o, v1);
        sk.end(p);
        p = -1;
      }
    }
    {
      const bool want = nstage == 0 && !exhausted;
      unsigned wm = __ballot_sync(full, want);
      while (wm) {
        if (cbeg >= cend) {
          unsigned long long base = 0;
          if (lane == 0) base = atomicAdd(work, chunks ? 1ull : (unsigned long long)kIxChunk);
          base = __shfl_sync(full, base, 0);
          if ((int64_t)base >= npairs) {
            exhausted = true;
            break;
          }
          if (chunks) {
            const int4 ch = chunks[base];
            cbeg = ch.x;
            cend = ch.y;
          } else {
            cbeg = (int64_t)base;
            cend = cbeg + kIxChunk < npairs ? cbeg + kIxChunk : npairs;
          }
        }
        const int navail = (int)(cend - cbeg);
        const int rank = __popc(wm & lt);
        const bool take = want && ((wm >> lane) & 1u) && rank < navail;
        if (take) {
          nrec = list[cbeg + rank];
          nstage = 1;
        }
        const unsigned tm = __ballot_sync(full, take);
        cbeg += __popc(tm);
        wm &= ~tm;
      }
    }
    if (__all_sync(full, p < 0 && nstage == 0 && exhausted)) break;
    if (p < 0) continue;
    Tet t;
    ix_gather(pool, cur, t);
    double nx, ny, nz, c;
    load_plane(planes, L, nx, ny, nz, c);
    TetClass cls;
    classify_tet(t, nx, ny, nz, c, cls);
    int k = 0;
    unsigned c0 = cur, c1 = 0, c2 = 0;
    if (cls.nn > 0) k = cls.np == 0 ? 1 : ix_split(cur, cls, pool, 4 + 4 * L, c0, c1, c2);
    if (L == lastL) {
      // final tets, in the reference's order
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        if (j < k) {
          Tet o;
          ix_gather(pool, j == 0 ? c0 : (j == 1 ? c1 : c2), o);
          double v1;
          if (final_tet_keep(o, tol, v1)) sk.tet(o, v1);
        }
      }
      k = 0;
    }
    if (k > 0) {
      const unsigned lv = (unsigned)(__ffs(act & (~0u << (L + 1))) - 1);  // next plane clipped at
      if (k == 3) {
#pragma unroll
        for (int w = kW - 1; w > 0; --w) stk[w] = (stk[w] << 20) | (stk[w - 1] >> 44);
        stk[0] = (stk[0] << 20) | c2;
        stk_lv = (stk_lv << kLB) | lv;
        ++sp;
      }
      if (k >= 2) {
#pragma unroll
        for (int w = kW - 1; w > 0; --w) stk[w] = (stk[w] << 20) | (stk[w - 1] >> 44);
        stk[0] = (stk[0] << 20) | c1;
        stk_lv = (stk_lv << kLB) | lv;
        ++sp;
      }
      cur = c0;
      L = (int)lv;
      continue;
    }
    if (sp > 0) {
      cur = (unsigned)(stk[0] & 0xfffffull);
      L = (int)(stk_lv & ((1u << kLB) - 1u));
#pragma unroll
      for (int w = 0; w < kW - 1; ++w) stk[w] = (stk[w] >> 20) | (stk[w + 1] << 44);
      stk[kW - 1] >>= 20;
      stk_lv >>= kLB;
      --sp;
      continue;
    }
    sk.end(p);
    p = -1;
  }
  sk.template finish<BLOCK>();
}

size_t ix_smem_bytes() { return (size_t)kIxBlock * 3 * kIxPoints * sizeof(double); }

// Per-pair setup of explicit tetrahedron pairs (the prep kernel's work for
// one-element meshes): B's planes and tolerance (setup row), A's tolerance,
// identity pair indices and, optionally, the rows of the second early-out
// (A's face planes, B's screen row).
__global__ void k_setup_pairs3(int64_t n, const double* __restrict__ tet_a, const double* __restrict__ tet_b,
                               double* setup, double* tol_a, int32_t* iota, double* faces_a, double* screen_b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    // both pair arrays are 16-byte aligned (checked by the entry points)
    Tet a, b;
    load_tet(tet_a + 12 * i, a);
    load_tet(tet_b + 12 * i, b);
    Planes P;
    tet_planes(b, P);
    double* o = setup + i * kSetup3;
#pragma unroll
    for (int L = 0; L < 4; ++L) {
      st2(o + 4 * L, P.nx[L], P.ny[L]);
      st2(o + 4 * L + 2, P.nz[L], P.c[L]);
    }
    st2(o + 16, 10.0 * spacing(tet_volume_v4(b)), 0.0);
    st2(o + 18, 0.0, 0.0);
    tol_a[i] = 10.0 * spacing(tet_volume_v4(a));
    iota[i] = (int32_t)i;
    if (screen_b) tet_screen_b(b, P, screen_b + i * kScreen3);
    if (faces_a) tet_faces_screen(a, faces_a + i * kScreen3);
  }
}

cudaError_t launch_setup_pairs3(int64_t n, const double* tet_a, const double* tet_b, double* setup, double* tol_a,
                                int32_t* iota, double* faces_a, double* screen_b, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launch();
  k_setup_pairs3<<<grid_for(n, 256, 8), 256, 0, s>>>(n, tet_a, tet_b, setup, tol_a, iota, faces_a, screen_b);
  return cudaGetLastError();
}

// Explicit tet-hexahedron pairs through the same pipeline with six planes
// (Supermesh.F90:262-280 planes, tolerance from the tet alone): per-pair
// setup rows of clip_row(6) doubles (planes, +inf in the tolerance slot so
// that fmin keeps A's), the first early-out and the no-op planes, then the
// index clipper with a pool of 28 points.  320 threads per SM: 672 B of pool
// per lane.
constexpr int kIxHexBlock = 320;

size_t ix_hex_smem_bytes() { return (size_t)kIxHexBlock * 3 * ix_points(6) * sizeof(double); }

// kVec: hex_b is 16-byte aligned, each hexahedron is read in 12 16-byte loads
template <bool kVec>
__global__ void k_setup_hex_pairs(int64_t n, const double* __restrict__ tet_a, const double* __restrict__ hex_b,
                                  double* setup, double* tol_a, int32_t* iota) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double nx[6], ny[6], nz[6], c[6];
    if (kVec) {
      double h[24];
      const double2* q = reinterpret_cast<const double2*>(hex_b + 24 * i);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        const double2 v = __ldg(q + k);
        h[2 * k] = v.x;
        h[2 * k + 1] = v.y;
      }
      hex_planes(h, nx, ny, nz, c);
    } else {
      hex_planes(hex_b + 24 * i, nx, ny, nz, c);
    }
    double* o = setup + i * clip_row(6);
#pragma unroll
    for (int L = 0; L < 6; ++L) {
      st2(o + 4 * L, nx[L], ny[L]);
      st2(o + 4 * L + 2, nz[L], c[L]);
    }
    st2(o + 24, pos_inf(), 0.0);
    st2(o + 26, 0.0, 0.0);
    Tet a;
    load_tet(tet_a + 12 * i, a);
    tol_a[i] = 10.0 * spacing(tet_volume_v4(a));
    iota[i] = (int32_t)i;
  }
}

cudaError_t launch_tet_hex_pairs(int64_t n, const double* tet_a, const double* hex_b, double* measure, int32_t* nout,
                                 double* elems, double* setup, double* tol_a, int32_t* iota, int32_t* survivors,
                                 unsigned long long* work, cudaStream_t s, const SegList* seg) {
  cudaMemsetAsync(work, 0, 2 * sizeof(unsigned long long), s);
  if (n <= 0) return cudaGetLastError();
  count_launch(2);
  if ((reinterpret_cast<uintptr_t>(hex_b) & 15u) == 0)
    k_setup_hex_pairs<true><<<grid_for(n, 256, 8), 256, 0, s>>>(n, tet_a, hex_b, setup, tol_a, iota);
  else
    k_setup_hex_pairs<false><<<grid_for(n, 256, 8), 256, 0, s>>>(n, tet_a, hex_b, setup, tol_a, iota);
  const int4* list = reinterpret_cast<const int4*>(survivors);
  const int g = sm_count();
  if (elems) {
    run_prefilter<false, 6>(n, nullptr, iota, iota, tet_a, tol_a, setup, measure, nout, survivors, work, nullptr,
                            nullptr, nullptr, seg, s);
    k_clip_tets_ix<IxElemSinkT<729>, kIxHexBlock, 1, 6><<<g, kIxHexBlock, ix_hex_smem_bytes(), s>>>(
        list, seg_nlist(seg, work), tet_a, tol_a, setup, IxElemSinkT<729>{measure, nout, elems}, work + 1,
        seg_table(seg));
  } else {
    run_prefilter<true, 6>(n, nullptr, iota, iota, tet_a, tol_a, setup, measure, nout, survivors, work, nullptr,
                           nullptr, nullptr, seg, s);
    k_clip_tets_ix<IxMeasureSink, kIxHexBlock, 1, 6><<<g, kIxHexBlock, ix_hex_smem_bytes(), s>>>(
        list, seg_nlist(seg, work), tet_a, tol_a, setup, IxMeasureSink{measure, nout, 0.0, 0}, work + 1,
        seg_table(seg));
  }
  return cudaGetLastError();
}

// A hexahedron (Gmsh node order) as five tets, in the order and with the
// vertex order of the reference's slicing (Supermesh.F90:303-334).
__device__ constexpr int kHexTets[5][4] = {{2, 5, 6, 7}, {0, 2, 3, 7}, {0, 4, 5, 7}, {0, 1, 2, 5}, {0, 2, 5, 7}};

// Hexahedron-hexahedron pairs: B's six face planes (setup rows of
// clip_row(6) doubles with +inf in the tolerance slot), and A's five tets
// in the reference's slicing order (Supermesh.F90:303-334), tet k
// of pair i at sub[(k * n + i) * 12] with its tolerance at tol[k * n + i].
__global__ void k_setup_hex_hex(int64_t n, const double* __restrict__ hex_a, const double* __restrict__ hex_b,
                                double* setup, double* sub, double* tol, int32_t* iota) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double nx[6], ny[6], nz[6], c[6];
    hex_planes(hex_b + 24 * i, nx, ny, nz, c);
    double* o = setup + i * clip_row(6);
#pragma unroll
    for (int L = 0; L < 6; ++L) {
      st2(o + 4 * L, nx[L], ny[L]);
      st2(o + 4 * L + 2, nz[L], c[L]);
    }
    st2(o + 24, pos_inf(), 0.0);
    st2(o + 26, 0.0, 0.0);
    const double* h = hex_a + 24 * i;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      Tet t;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        t.x[v] = h[3 * kHexTets[k][v]];
        t.y[v] = h[3 * kHexTets[k][v] + 1];
        t.z[v] = h[3 * kHexTets[k][v] + 2];
      }
      double* q = sub + ((int64_t)k * n + i) * 12;
      st2(q + 0, t.x[0], t.y[0]);
      st2(q + 2, t.z[0], t.x[1]);
      st2(q + 4, t.y[1], t.z[1]);
      st2(q + 6, t.x[2], t.y[2]);
      st2(q + 8, t.z[2], t.x[3]);
      st2(q + 10, t.y[3], t.z[3]);
      tol[(int64_t)k * n + i] = 10.0 * spacing(tet_volume_v4(t));
    }
    iota[i] = (int32_t)i;
  }
}

cudaError_t launch_hex_hex_pairs(int64_t n, const double* hex_a, const double* hex_b, double* measure, int32_t* nout,
                                 double* elems, double* setup, double* sub, double* tol, int32_t* iota,
                                 int32_t* survivors, unsigned long long* work, cudaStream_t s, const SegList* seg) {
  if (n <= 0) return cudaSuccess;
  count_launch();
  k_setup_hex_hex<<<grid_for(n, 256, 8), 256, 0, s>>>(n, hex_a, hex_b, setup, sub, tol, iota);
  cudaMemsetAsync(measure, 0, sizeof(double) * n, s);
  cudaMemsetAsync(nout, 0, sizeof(int32_t) * n, s);
  const int4* list = reinterpret_cast<const int4*>(survivors);
  for (int k = 0; k < 5; ++k) {
    // tet k of every pair: rejected pairs keep their carried results, the
    // others (A's tet inside all six planes included) add to them
    const double* tk = sub + (int64_t)k * n * 12;
    const double* lk = tol + (int64_t)k * n;
    cudaMemsetAsync(work, 0, 2 * sizeof(unsigned long long), s);
    run_prefilter<false, 6>(n, nullptr, iota, iota, tk, lk, setup, nullptr, nullptr, survivors, work, nullptr,
                            nullptr, nullptr, seg, s);
    count_launch();
    k_clip_tets_ix<IxCarrySinkT<kHexHexCap>, kIxHexBlock, 1, 6><<<sm_count(), kIxHexBlock, ix_hex_smem_bytes(), s>>>(
        list, seg_nlist(seg, work), tk, lk, setup, IxCarrySinkT<kHexHexCap>{measure, nout, elems}, work + 1,
        seg_table(seg));
  }
  return cudaGetLastError();
}

cudaError_t launch_clip_elems(int64_t n, const int32_t* pair_a, const int32_t* pair_b, const double* tet_a,
                              const double* tol_a, const double* setup, double* measure, int32_t* nout,
                              double* elems, int32_t* survivors, unsigned long long* work, const double* faces_a,
                              const double* screen_b, cudaStream_t s, const SegList* seg) {
  cudaMemsetAsync(work, 0, 2 * sizeof(unsigned long long), s);
  if (n <= 0) return cudaGetLastError();
  run_prefilter<false, 4>(n, nullptr, pair_a, pair_b, tet_a, tol_a, setup, measure, nout, survivors, work, faces_a,
                          screen_b, nullptr, seg, s);
  count_launch();
  k_clip_tets_ix<IxElemSink, kIxBlock, kIxBlocksPerSm><<<sm_count() * kIxBlocksPerSm, kIxBlock, ix_smem_bytes(), s>>>(
      reinterpret_cast<const int4*>(survivors), seg_nlist(seg, work), tet_a, tol_a, setup,
      IxElemSink{measure, nout, elems}, work + 1, seg_table(seg));
  return cudaGetLastError();
}




// Deterministic per-block partials of the pair measures: block b reduces the
// contiguous range [b*chunk, (b+1)*chunk) in a fixed thread order.
__global__ void __launch_bounds__(256) k_reduce_pairs(int64_t npairs, const double* __restrict__ pm,
                                                      const int32_t* __restrict__ pn, Partial* partials,
                                                      const int64_t* __restrict__ n_dev) {
  if (n_dev && *n_dev < npairs) npairs = *n_dev;
  const int64_t chunk = (npairs + gridDim.x - 1) / gridDim.x;
  const int64_t beg = (int64_t)blockIdx.x * chunk;
  const int64_t end = beg + chunk < npairs ? beg + chunk : npairs;
  double sum = 0.0, err = 0.0;
  unsigned long long ni = 0, no = 0;
  for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
    cs_add(sum, err, pm[i]);
    const int k = pn ? pn[i] : 0;
    ni += k > 0;
    no += k;
  }
  block_reduce_partial<256>(sum, err, ni, no, &partials[blockIdx.x]);
}

int clip_grid_blocks(int dim) { return sm_count() * (dim == 2 ? tri_blocks_per_sm() : kIxBlocksPerSm); }

cudaError_t launch_clip(int dim, int64_t npairs, const int32_t* pair_a, const int32_t* pair_b,
                        const double* coords_a, const double* tol_a, const double* setup_b,
                        double* pair_measure, int32_t* pair_nout, int32_t* overflow_list,
                        int* overflow_count, unsigned long long* work, cudaStream_t s,
                        const int32_t* order, cudaEvent_t ev_begin, cudaEvent_t ev_end, const double* faces_a,
                        const double* screen_b, const SchedBin* bin, const int64_t* n_dev, const SegList* seg) {
  const int g = clip_grid_blocks(dim);
  count_launch();
  if (dim == 2) {
    if (ev_begin) cudaEventRecord(ev_begin, s);
    k_clip_tris<<<g, kTriBlock, 0, s>>>(npairs, pair_a, pair_b, coords_a, tol_a, setup_b, pair_measure,
                                        pair_nout, overflow_list, overflow_count, order, n_dev);
  } else {
    // work[0]: survivor count, work[1]: clipper pair counter
    // the timed span covers the early-out pass and the clipper: together
    // they settle every candidate
    if (ev_begin) cudaEventRecord(ev_begin, s);
    cudaMemsetAsync(work, 0, 2 * sizeof(unsigned long long), s);
    // the binned orders read one list: with bin->flat the segments are
    // gathered into it first
    const SegList sg = (bin && !bin->flat) ? SegList{} : (seg ? *seg : SegList{});
    run_prefilter<true, 4>(npairs, order, pair_a, pair_b, coords_a, tol_a, setup_b, pair_measure, pair_nout,
                           overflow_list, work, faces_a, screen_b, n_dev, &sg, s);
    const int4* list = reinterpret_cast<const int4*>(overflow_list);
    if (bin) {
      if (seg_on(&sg)) {
        cudaError_t e = launch_seg_compact(npairs, work + 2, sg.table, list, bin->flat, s);
        if (e != cudaSuccess) return e;
        list = bin->flat;
      }
      // the survivors reordered into class-uniform runs within windows
      cudaError_t e = launch_sched_bin(*bin, list, work, bin->out, coords_a, s);
      if (e != cudaSuccess) return e;
      list = bin->out;
    }
    k_clip_tets_ix<IxMeasureSink, kIxBlock, kIxBlocksPerSm><<<sm_count() * kIxBlocksPerSm, kIxBlock, ix_smem_bytes(), s>>>(
        list, bin ? work : seg_nlist(&sg, work), coords_a, tol_a, setup_b,
        IxMeasureSink{pair_measure, pair_nout, 0.0, 0}, work + 1, bin ? nullptr : seg_table(&sg));
  }
  if (ev_end) cudaEventRecord(ev_end, s);
  return cudaGetLastError();
}

int reduce_pairs_blocks() { return kReduceBlocks; }

cudaError_t launch_reduce_pairs(int64_t npairs, const double* pair_measure, const int32_t* pair_nout,
                                Partial* partials, cudaStream_t s, const int64_t* n_dev) {
  count_launch();
  k_reduce_pairs<<<kReduceBlocks, 256, 0, s>>>(npairs, pair_measure, pair_nout, partials, n_dev);
  return cudaGetLastError();
}

// 2D supermesh triangles: one candidate pair per thread, clipped again with
// the narrow phase's arithmetic; pairs without output triangles are skipped
// (their offsets are equal).
__global__ void __launch_bounds__(128) k_tris_emit(int64_t npairs, const int32_t* __restrict__ pa,
                                                   const int32_t* __restrict__ pb, const double* __restrict__ coords_a,
                                                   const double* __restrict__ tol_a, const double* __restrict__ setup_b,
                                                   const int64_t* __restrict__ pair_off, double* elems,
                                                   int64_t* parent_a, int64_t* parent_b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npairs;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t at = pair_off[i];
    if (pair_off[i + 1] == at) continue;
    const int a = pa[i], b = pb[i];
    const double* ca = coords_a + (int64_t)a * 6;
    Lines L;
    double tolb;
    load_lines(setup_b + (int64_t)b * kSetup2, L, tolb);
    const double tol = fmin(tol_a[a], tolb);
    LocalPoly<kTriWideCap> p, q;
    double m;
    clip_tri(ca[0], ca[1], ca[2], ca[3], ca[4], ca[5], L, tol, p, q, kTriWideCap, m,
             [&](int k, double x0, double y0, double x1, double y1, double x2, double y2) {
               double2* e = reinterpret_cast<double2*>(elems + (at + k) * 6);
               e[0] = make_double2(x0, y0);
               e[1] = make_double2(x1, y1);
               e[2] = make_double2(x2, y2);
               if (parent_a) parent_a[at + k] = a;
               if (parent_b) parent_b[at + k] = b;
             });
  }
}

cudaError_t launch_emit_elements(int dim, int64_t npairs, const int32_t* pair_a, const int32_t* pair_b,
                                 const double* coords_a, const double* tol_a, const double* setup_b,
                                 const int32_t* survivors, unsigned long long* work, const int64_t* pair_off,
                                 double* elems, int64_t* parent_a, int64_t* parent_b, cudaStream_t s,
                                 const SegList* seg) {
  if (npairs <= 0) return cudaSuccess;
  count_launch();
  if (dim == 2) {
    k_tris_emit<<<grid_for(npairs, 128, 8), 128, 0, s>>>(npairs, pair_a, pair_b, coords_a, tol_a, setup_b, pair_off,
                                                         elems, parent_a, parent_b);
    return cudaGetLastError();
  }
  // the survivors of the counting pass again (work[0] holds their number);
  // only the clipper's pair counter starts over
  cudaMemsetAsync(work + 1, 0, sizeof(unsigned long long), s);
  k_clip_tets_ix<IxEmitSink, kIxBlock, kIxBlocksPerSm><<<sm_count() * kIxBlocksPerSm, kIxBlock, ix_smem_bytes(), s>>>(
      reinterpret_cast<const int4*>(survivors), seg_nlist(seg, work), coords_a, tol_a, setup_b,
      IxEmitSink{pair_off, elems, parent_a, parent_b}, work + 1, seg_table(seg));
  return cudaGetLastError();
}

cudaError_t init_p1_attributes();

cudaError_t init_device_attributes() {
  cudaError_t e = cudaFuncSetAttribute(k_clip_tets_ix<IxMeasureSink, kIxBlock, kIxBlocksPerSm>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ix_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_clip_tets_ix<IxElemSink, kIxBlock, kIxBlocksPerSm>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ix_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_clip_tets_ix<IxEmitSink, kIxBlock, kIxBlocksPerSm>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ix_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_clip_tets_ix<IxMeasureSink, kIxHexBlock, 1, 6>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ix_hex_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_clip_tets_ix<IxCarrySinkT<kHexHexCap>, kIxHexBlock, 1, 6>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ix_hex_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_clip_tets_ix<IxElemSinkT<729>, kIxHexBlock, 1, 6>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ix_hex_smem_bytes());
  if (e == cudaSuccess) e = init_p1_attributes();
  if (e != cudaSuccess) return e;
  return init_sched_attributes(kSchedMaxWindow);
}



cudaError_t launch_clip_tris_wide(const int32_t* overflow_list, const int* overflow_count, int64_t cap,
                                  const int32_t* pair_a, const int32_t* pair_b,
                                  const double* coords_a, const double* tol_a,
                                  const double* setup_b, double* pair_measure, int32_t* pair_nout,
                                  cudaStream_t s) {
  count_launch();
  k_clip_tris_wide<<<1, 32, 0, s>>>(overflow_list, overflow_count, cap, pair_a, pair_b, coords_a, tol_a,
                                    setup_b, pair_measure, pair_nout);
  return cudaGetLastError();
}

// ======================================================================
// K7: finalize totals and per-row sums
// ======================================================================
// Merges the per-block partials in a fixed tree order (deterministic).
__global__ void __launch_bounds__(1024) k_finalize(const Partial* __restrict__ partials, int np, Partial* out) {
  double sum = 0.0, err = 0.0;
  unsigned long long ni = 0, no = 0;
  for (int b = threadIdx.x; b < np; b += blockDim.x) {
    two_sum_merge(sum, err, partials[b].sum, partials[b].err);
    ni += partials[b].n_int;
    no += partials[b].n_out;
  }
  __shared__ Partial r;
  block_reduce_partial<1024>(sum, err, ni, no, &r);
  __syncthreads();
  if (threadIdx.x == 0) {
    Partial p = r;
    p.sum = p.sum + p.err;
    *out = p;
  }
}

cudaError_t launch_finalize(const Partial* partials, int npartials, Partial* out, cudaStream_t s) {
  count_launch();
  k_finalize<<<1, 1024, 0, s>>>(partials, npartials, out);
  return cudaGetLastError();
}

__global__ void k_row_sums(int64_t nel_a, const int64_t* __restrict__ off, const double* __restrict__ pm,
                           double* em) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < nel_a;
       a += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int64_t p = off[a]; p < off[a + 1]; ++p) s = s + pm[p];
    em[a] = s;
  }
}

cudaError_t launch_row_sums(int64_t nel_a, const int64_t* offsets, const double* pair_measure,
                            double* elem_measure, cudaStream_t s) {
  if (nel_a <= 0) return cudaSuccess;
  count_launch();
  k_row_sums<<<grid_for(nel_a, 256, 8), 256, 0, s>>>(nel_a, offsets, pair_measure, elem_measure);
  return cudaGetLastError();
}

__global__ void k_i32_to_i64(int64_t n, const int32_t* __restrict__ in, int64_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[i];
}

cudaError_t launch_i32_to_i64(int64_t n, const int32_t* in, int64_t* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launch();
  k_i32_to_i64<<<grid_for(n, 256, 8), 256, 0, s>>>(n, in, out);
  return cudaGetLastError();
}

// ======================================================================
// Batched search: one LBVH over many meshes, one subtree per mesh
// ======================================================================
// After sorting the B elements of all meshes by (mesh, Morton) the combined
// 64-bit keys (mesh << 32 | Morton) give a Karras hierarchy in which every
// mesh's elements form one subtree (they share the mesh-id prefix, no other
// key does).  A query of mesh p starts at p's subtree root and stops at the
// root's escape node.
__global__ void k_pair_keys(int64_t n, const int32_t* __restrict__ vals, const int32_t* __restrict__ pair_of,
                            uint32_t* keys) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    keys[i] = (uint32_t)pair_of[vals[i]];
}

// After a sort whose look-back wait gave up (*err != 0, values repaired to
// the identity) the Morton part is left out: equal codes within a mesh give
// a well-formed hierarchy (ties break by position), so the kernels after it
// stay in bounds while the host reports the failure.
__global__ void k_combined_codes(int64_t n, const int32_t* __restrict__ vals, const int32_t* __restrict__ pair_of,
                                 const uint32_t* __restrict__ mort, unsigned long long* codes,
                                 const uint32_t* __restrict__ err) {
  const bool failed = err && *err != 0u;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = vals[i];
    codes[i] = ((unsigned long long)(uint32_t)pair_of[v] << 32) | (failed ? 0ull : (unsigned long long)mort[v]);
  }
}

__device__ __forceinline__ int bvh_delta64(const unsigned long long* __restrict__ codes, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const unsigned long long a = codes[i], b = codes[j];
  if (a != b) return __clzll((long long)(a ^ b));
  return 64 + __clz((uint32_t)i ^ (uint32_t)j);
}

__global__ void k_bvh_internal64(int n, const unsigned long long* __restrict__ codes, int* parent, int* rope,
                                 int* last, int* left, int* right, const int64_t* __restrict__ mesh_off,
                                 int* roots) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = (bvh_delta64(codes, n, i, i + 1) - bvh_delta64(codes, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = bvh_delta64(codes, n, i, i - d);
  int lmax = 2;
  while (bvh_delta64(codes, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (bvh_delta64(codes, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = bvh_delta64(codes, n, i, j);
  int s = 0;
  int t = l;
  do {
    t = (t + 1) >> 1;
    if (bvh_delta64(codes, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  const int gamma = i + s * d + (d < 0 ? -1 : 0);
  const int first = i < j ? i : j;
  const int lst = i < j ? j : i;
  const int lc = (first == gamma) ? (n - 1) + gamma : gamma;
  const int rc = (lst == gamma + 1) ? (n - 1) + gamma + 1 : gamma + 1;
  left[i] = lc;
  right[i] = rc;
  parent[lc] = i;
  parent[rc] = i;
  rope[gamma + 1] = rc;
  last[i] = lst;
  const int mesh = (int)(codes[first] >> 32);
  if (mesh_off[mesh] == first && mesh_off[mesh + 1] - 1 == lst) roots[mesh] = i;
}

// Roots of single-element meshes, and the stop node (the root's escape) of
// every mesh.  Meshes without elements get root -1.
__global__ void k_mesh_roots(int nm, int n, const int64_t* __restrict__ mesh_off, const int* __restrict__ rope,
                             const int* __restrict__ last, int* roots, int* stops) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nm) return;
  const int64_t cnt = mesh_off[p + 1] - mesh_off[p];
  int r = -1;
  if (cnt == 1)
    r = (n - 1) + (int)mesh_off[p];
  else if (cnt > 1)
    r = roots[p];
  roots[p] = r;
  stops[p] = r >= 0 ? bvh_escape(n, r, rope, last) : -1;
}

cudaError_t launch_batched_tree(int n, int nm, const int32_t* sorted_vals, const int32_t* pair_of_b,
                                const uint32_t* mort, unsigned long long* codes, const float* box32,
                                const int64_t* mesh_off_b, BVH bvh, int* work, int* roots, int* stops,
                                cudaStream_t s, int dim, const double* box64, const int* sort_err) {
  if (n <= 0) return cudaSuccess;
  int* parent = work;
  int* rope = parent + (2 * n - 1);
  int* visit = rope + n;
  int* last = visit + n;
  int* left = last + n;
  int* right = left + n;
  count_launch(4);
  k_combined_codes<<<grid_for(n, 256, 8), 256, 0, s>>>(n, sorted_vals, pair_of_b, mort, codes,
                                                       reinterpret_cast<const uint32_t*>(sort_err));
  cudaMemsetAsync(visit, 0, sizeof(int) * n, s);
  cudaMemsetAsync(rope, 0xff, sizeof(int) * n, s);
  cudaMemsetAsync(roots, 0xff, sizeof(int) * nm, s);
  if (n > 1) k_bvh_internal64<<<(n - 1 + 255) / 256, 256, 0, s>>>(n, codes, parent, rope, last, left, right, mesh_off_b, roots);
  cudaMemsetAsync(parent, 0xff, sizeof(int), s);
  k_mesh_roots<<<(nm + 255) / 256, 256, 0, s>>>(nm, n, mesh_off_b, rope, last, roots, stops);
  k_bvh_refit<false><<<(n + kRefitBlock - 1) / kRefitBlock, kRefitBlock, 0, s>>>(n, sorted_vals, reinterpret_cast<const float4*>(box32), parent,
                                                     rope, last, left, right, visit, bvh.lo_left, bvh.hi_esc, dim,
                                                     box64, box64 ? bvh.leaf : nullptr, nullptr, 1);
  return cudaGetLastError();
}

cudaError_t launch_pair_keys(int64_t n, const int32_t* vals, const int32_t* pair_of, uint32_t* keys,
                             cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launch();
  k_pair_keys<<<grid_for(n, 256, 8), 256, 0, s>>>(n, vals, pair_of, keys);
  return cudaGetLastError();
}

template <int DIM, bool FILL>
__global__ void __launch_bounds__(256) k_query_batched(int64_t nel_a, const double* __restrict__ box64_a,
                                                       const int32_t* __restrict__ pair_of_a,
                                                       const int* __restrict__ roots, const int* __restrict__ stops,
                                                       const float4* __restrict__ lo_left,
                                                       const float4* __restrict__ hi_esc, int n,
                                                       const double* __restrict__ box64_b, int* counts,
                                                       const int64_t* __restrict__ offsets, int32_t* pair_a,
                                                       int32_t* pair_b, int32_t* cache, int cap,
                                                       const int32_t* __restrict__ rows, int* over_rows,
                                                       const double* __restrict__ leaf, Spill sp,
                                                       int64_t pair_cap) {
  // cache / rows / over_rows / leaf: as k_query
  const int64_t nrows = rows ? (int64_t)*over_rows : nel_a;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = rows ? rows[r] : r;
    double lo[DIM], hi[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      lo[c] = box64_a[a * 2 * DIM + c];
      hi[c] = box64_a[a * 2 * DIM + DIM + c];
    }
    float ql[3], qh[3];
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      ql[c] = __double2float_rd(lo[c]);
      qh[c] = __double2float_ru(hi[c]);
    }
    const int mesh = pair_of_a[a];
    int node = roots[mesh];
    const int stop = stops[mesh];
    int cnt = 0;
    int64_t out = FILL ? offsets[a] : 0;
    int chunk = -1;     // current spill chunk of this row
    bool lost = false;  // the row goes to the second traversal
    const int nodes = 2 * n - 1;
    for (int guard = 0; node >= 0 && node != stop && guard < 2 * n + 1; ++guard) {
      if (node >= nodes) break;  // never taken for a well-formed hierarchy
      if (leaf && node >= n - 1) {
        const double2* q = reinterpret_cast<const double2*>(leaf + (int64_t)(node - (n - 1)) * 8);
        const double2 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2), q3 = __ldg(q + 3);
        const double blo[3] = {q0.x, q0.y, q1.x}, bhi[3] = {q1.y, q2.x, q2.y};
        const int2 meta = make_int2(__double2loint(q3.x), __double2hiint(q3.x));
        bool ex = true;
#pragma unroll
        for (int c = 0; c < DIM; ++c) ex = ex && (hi[c] > blo[c]) && (lo[c] < bhi[c]);
        if (ex) {
          if (FILL) {
            if (out + cnt < pair_cap) {
              pair_a[out + cnt] = (int32_t)a;
              pair_b[out + cnt] = meta.x;
            }
          } else if (cache) {
            cache_put(cache, cap, sp, a, cnt, meta.x, chunk, lost);
          }
          ++cnt;
        }
        node = meta.y;
        continue;
      }
      const float4 L = __ldg(&lo_left[2 * node]);
      const float4 H = __ldg(&hi_esc[2 * node]);
      bool ov = H.x > ql[0] && L.x < qh[0] && H.y > ql[1] && L.y < qh[1];
      if (DIM == 3) ov = ov && H.z > ql[2] && L.z < qh[2];
      if (ov) {
        const int w = __float_as_int(L.w);
        if (node < n - 1) {
          node = w;
          continue;
        }
        const double* bb = box64_b + (int64_t)w * 2 * DIM;
        bool ex = true;
#pragma unroll
        for (int c = 0; c < DIM; ++c) ex = ex && (hi[c] > bb[c]) && (lo[c] < bb[DIM + c]);
        if (ex) {
          if (FILL) {
            if (out + cnt < pair_cap) {
              pair_a[out + cnt] = (int32_t)a;
              pair_b[out + cnt] = w;
            }
          } else if (cache) {
            cache_put(cache, cap, sp, a, cnt, w, chunk, lost);
          }
          ++cnt;
        }
      }
      node = __float_as_int(H.w);
    }
    if (!FILL) {
      counts[a] = cnt;
      if (cache && lost) {
        if (sp.row_chunk) sp.row_chunk[a] = -2;
        over_rows[1 + atomicAdd(over_rows, 1)] = (int32_t)a;
      }
    }
  }
}


cudaError_t launch_query_batched(int dim, bool fill, int64_t nel_a, const double* box64_a,
                                 const int32_t* pair_of_a, const int* roots, const int* stops, BVH bvh,
                                 const double* box64_b, int* counts, const int64_t* offsets, int32_t* pair_a,
                                 int32_t* pair_b, cudaStream_t s, int32_t* cache, int cap, int* over_rows,
                                 Spill sp, int64_t pair_cap) {
  if (nel_a <= 0 || bvh.n <= 0) return cudaSuccess;
  const int B = query_block();
  const int g = grid_for(nel_a, B, 2048 / B);
  if (fill && cache) {
    count_launch(2);
    k_fill_from_cache<<<grid_for(nel_a, 256, 8), 256, 0, s>>>(nel_a, counts, offsets, cache, cap, pair_a, pair_b,
                                                              sp, pair_cap);
  } else {
    count_launch();
  }
  const int32_t* rows = (fill && cache) ? over_rows + 1 : nullptr;
  int32_t* cc = fill ? nullptr : cache;
#define LSM_QUERY_ARGS                                                                                         \
  nel_a, box64_a, pair_of_a, roots, stops, bvh.lo_left, bvh.hi_esc, bvh.n, box64_b, counts, offsets, pair_a, \
      pair_b, cc, cap, rows, over_rows, bvh.leaf, sp, pair_cap
  if (dim == 2) {
    if (fill)
      k_query_batched<2, true><<<g, B, 0, s>>>(LSM_QUERY_ARGS);
    else
      k_query_batched<2, false><<<g, B, 0, s>>>(LSM_QUERY_ARGS);
  } else {
    if (fill)
      k_query_batched<3, true><<<g, B, 0, s>>>(LSM_QUERY_ARGS);
    else
      k_query_batched<3, false><<<g, B, 0, s>>>(LSM_QUERY_ARGS);
  }
#undef LSM_QUERY_ARGS
  return cudaGetLastError();
}

// Per-mesh-pair totals of the batched path (mesh pair p owns the CSR rows
// elem_off_a[p] .. elem_off_a[p+1]-1).  Mesh pairs differ in size by
// 100x, so each pair's candidate range is split into kMeshSplit contiguous
// pieces reduced by separate blocks (grid nm x kMeshSplit), and the pieces
// are merged in piece order by k_mesh_combine: deterministic, and no block
// walks a whole large mesh alone.
constexpr int kMeshSplit = 32;

__global__ void __launch_bounds__(256) k_mesh_totals(int nm, const int64_t* __restrict__ elem_off_a,
                                                     const int64_t* __restrict__ offsets,
                                                     const double* __restrict__ pm, const int32_t* __restrict__ pn,
                                                     Partial* pieces, int64_t cap) {
  const int p = blockIdx.x, g = blockIdx.y;
  if (p >= nm) return;
  // cap: entries the pair arrays hold (a count beyond it is reported by the
  // host, which then runs the batch again with larger arrays)
  const int64_t beg = min(offsets[elem_off_a[p]], cap), end = min(offsets[elem_off_a[p + 1]], cap);
  const int64_t len = end - beg;
  const int64_t b0 = beg + len * g / kMeshSplit, b1 = beg + len * (g + 1) / kMeshSplit;
  double sum = 0.0, err = 0.0;
  unsigned long long ni = 0, no = 0;
  for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
    cs_add(sum, err, pm[i]);
    const int k = pn[i];
    ni += k > 0;
    no += k;
  }
  block_reduce_partial<256>(sum, err, ni, no, &pieces[(int64_t)p * kMeshSplit + g]);
}

__global__ void k_mesh_combine(int nm, const int64_t* __restrict__ elem_off_a, const int64_t* __restrict__ offsets,
                               const Partial* __restrict__ pieces, Partial* out, int64_t* ncand) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nm) return;
  Partial q = pieces[(int64_t)p * kMeshSplit];
  for (int g = 1; g < kMeshSplit; ++g) {
    const Partial r = pieces[(int64_t)p * kMeshSplit + g];
    two_sum_merge(q.sum, q.err, r.sum, r.err);
    q.n_int += r.n_int;
    q.n_out += r.n_out;
  }
  q.sum = q.sum + q.err;
  out[p] = q;
  ncand[p] = offsets[elem_off_a[p + 1]] - offsets[elem_off_a[p]];
}

int64_t mesh_totals_pieces(int nm) { return (int64_t)nm * kMeshSplit; }

// Per-pair CSR of a batch group in the get_output layout of the C API
// (C_bindings.F90:377-391): mesh pair k owns rows eoa[k] .. eoa[k+1]-1 and
// writes out[rowbase[k] + r] = offsets[eoa[k] + r] - offsets[eoa[k]] for
// r = 0 .. nel_a(k) (the last entry is the pair's candidate count).
__global__ void k_batch_indptr(int64_t na, int nm, const int32_t* __restrict__ pair_of_a,
                               const int64_t* __restrict__ eoa, const int64_t* __restrict__ offsets,
                               const int64_t* __restrict__ rowbase, int64_t* out) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < na + nm; e += (int64_t)gridDim.x * blockDim.x) {
    if (e < na) {
      const int k = pair_of_a[e];
      out[rowbase[k] + (e - eoa[k])] = offsets[e] - offsets[eoa[k]];
    } else {
      const int k = (int)(e - na);
      out[rowbase[k] + (eoa[k + 1] - eoa[k])] = offsets[eoa[k + 1]] - offsets[eoa[k]];
    }
  }
}

// Candidate B elements as numbers local to their mesh pair, int64.
__global__ void k_batch_indices(int64_t n, const int32_t* __restrict__ pair_b, const int32_t* __restrict__ pair_of_b,
                                const int64_t* __restrict__ eob, int64_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = pair_b[i];
    out[i] = (int64_t)b - eob[pair_of_b[b]];
  }
}

cudaError_t launch_batch_csr(int64_t na, int nm, const int32_t* pair_of_a, const int64_t* eoa, const int64_t* offsets,
                             const int64_t* rowbase, int64_t* ind_ptr, int64_t ncand, const int32_t* pair_b,
                             const int32_t* pair_of_b, const int64_t* eob, int64_t* indices, cudaStream_t s) {
  if (ind_ptr && na + nm > 0) {
    count_launch();
    k_batch_indptr<<<grid_for(na + nm, 256, 8), 256, 0, s>>>(na, nm, pair_of_a, eoa, offsets, rowbase, ind_ptr);
  }
  if (indices && ncand > 0) {
    count_launch();
    k_batch_indices<<<grid_for(ncand, 256, 8), 256, 0, s>>>(ncand, pair_b, pair_of_b, eob, indices);
  }
  return cudaGetLastError();
}

cudaError_t launch_mesh_totals(int nm, const int64_t* elem_off_a, const int64_t* offsets, const double* pm,
                               const int32_t* pn, Partial* pieces, Partial* out, int64_t* ncand, cudaStream_t s,
                               int64_t cap) {
  if (nm <= 0) return cudaSuccess;
  count_launch(2);
  k_mesh_totals<<<dim3(nm, kMeshSplit), 256, 0, s>>>(nm, elem_off_a, offsets, pm, pn, pieces, cap);
  k_mesh_combine<<<(nm + 127) / 128, 128, 0, s>>>(nm, elem_off_a, offsets, pieces, out, ncand);
  return cudaGetLastError();
}

// ======================================================================
// Explicit element pairs (the single-pair C API and its batched form)
// ======================================================================
struct TriEmit {
  double* out;  // [22][3][2] for this pair, or nullptr
  __device__ __forceinline__ void operator()(int k, double x0, double y0, double x1, double y1, double x2,
                                             double y2) const {
    if (!out || k >= 22) return;
    double* o = out + 6 * k;
    o[0] = x0;
    o[1] = y0;
    o[2] = x1;
    o[3] = y1;
    o[4] = x2;
    o[5] = y2;
  }
};

__global__ void k_pairs_tris(int64_t n, const double* __restrict__ A, const double* __restrict__ B,
                             double* measure, int32_t* nout, double* out_elems) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* va = A + 6 * i;
    const double* vb = B + 6 * i;
    Lines L;
    tri_lines(vb, L);
    const double tol = 10.0 * fmin(spacing(tri_area(va[0], va[1], va[2], va[3], va[4], va[5])),
                                   spacing(tri_area(vb[0], vb[1], vb[2], vb[3], vb[4], vb[5])));
    LocalPoly<kTriWideCap> p, q;
    double m;
    int k = clip_tri(va[0], va[1], va[2], va[3], va[4], va[5], L, tol, p, q, kTriWideCap, m,
                     TriEmit{out_elems ? out_elems + 22 * 6 * i : nullptr});
    if (k < 0) {
      k = 0;
      m = 0.0;
    }
    if (measure) measure[i] = m;
    if (nout) nout[i] = k;
  }
}

__global__ void k_pairs_tets(int64_t n, const double* __restrict__ A, const double* __restrict__ B,
                             double* measure, int32_t* nout, double* out_elems) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Tet ta, tb;
    load_tet(A + 12 * i, ta);
    load_tet(B + 12 * i, tb);
    Planes P;
    tet_planes(tb, P);
    const double tol = 10.0 * fmin(spacing(tet_volume_v4(ta)), spacing(tet_volume_v4(tb)));
    TetStackLocal stk;
    double m = 0.0;
    int idx = 0;
    double* o = out_elems ? out_elems + (int64_t)81 * 12 * i : nullptr;
    const int k = clip_tet_dfs(ta, RegPlanes{P}, tol, stk, [&](const Tet& t) {
      m = m + tet_volume_v1(t);
      if (o && idx < 81) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          o[12 * idx + 3 * v + 0] = t.x[v];
          o[12 * idx + 3 * v + 1] = t.y[v];
          o[12 * idx + 3 * v + 2] = t.z[v];
        }
      }
      ++idx;
    });
    if (measure) measure[i] = m;
    if (nout) nout[i] = k;
  }
}

// Triangle vs quadrilateral (Supermesh.F90:211-228): clip by the quad's 4
// edge lines, tolerance from the triangle's area only.
struct TriQuadEmit {
  double* out;  // [46][3][2] for this pair, or nullptr
  __device__ __forceinline__ void operator()(int k, double x0, double y0, double x1, double y1, double x2,
                                             double y2) const {
    if (!out || k >= 46) return;
    double* o = out + 6 * k;
    o[0] = x0;
    o[1] = y0;
    o[2] = x1;
    o[3] = y1;
    o[4] = x2;
    o[5] = y2;
  }
};

__global__ void k_pairs_tri_quad(int64_t n, const double* __restrict__ A, const double* __restrict__ B,
                                 double* measure, int32_t* nout, double* out_elems) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* va = A + 6 * i;
    double nx[4], ny[4], px[4], py[4];
    poly_lines<4>(B + 8 * i, nx, ny, px, py);
    const double tol = 10.0 * spacing(tri_area(va[0], va[1], va[2], va[3], va[4], va[5]));
    LocalPoly<48> p, q;
    p.set(0, va[0], va[1]);
    p.set(1, va[2], va[3]);
    p.set(2, va[4], va[5]);
    int m = 3;
    bool empty = false;
    for (int l = 0; l < 4 && !empty; ++l) {
      m = (l & 1) ? clip_stage(q, p, m, 48, nx[l], ny[l], px[l], py[l])
                  : clip_stage(p, q, m, 48, nx[l], ny[l], px[l], py[l]);
      empty = m < 3;
    }
    double meas = 0.0;
    int kept = 0;
    if (!empty) {  // after 4 stages the polygon is back in p
      TriQuadEmit emit{out_elems ? out_elems + 46 * 6 * i : nullptr};
      const double x0 = p.x(0), y0 = p.y(0);
      for (int j = 1; j < m - 1; ++j) {
        const double xi = p.x(j), yi = p.y(j), xj = p.x(j + 1), yj = p.y(j + 1);
        const double ar = tri_area(x0, y0, xi, yi, xj, yj);
        if (!(ar < tol)) {
          meas = meas + ar;
          emit(kept, x0, y0, xi, yi, xj, yj);
          ++kept;
        }
      }
    }
    if (measure) measure[i] = meas;
    if (nout) nout[i] = kept;
  }
}

// Tetrahedron vs hexahedron (Supermesh.F90:248-295): clip by the hex's 6
// face planes, tolerance from the tet's volume only.
__global__ void __launch_bounds__(64) k_pairs_tet_hex(int64_t n, const double* __restrict__ A,
                                                      const double* __restrict__ B, double* measure,
                                                      int32_t* nout, double* out_elems) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Tet ta;
    load_tet(A + 12 * i, ta);
    ArrPlanes<6> P;
    hex_planes(B + 24 * i, P.nx, P.ny, P.nz, P.c);
    const double tol = 10.0 * spacing(tet_volume_v4(ta));
    TetStackN<10> stk;
    double m = 0.0;
    int idx = 0;
    double* o = out_elems ? out_elems + (int64_t)729 * 12 * i : nullptr;
    const int k = clip_tet_dfs<6>(ta, P, tol, stk, [&](const Tet& t) {
      m = m + tet_volume_v1(t);
      if (o && idx < 729) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          o[12 * idx + 3 * v + 0] = t.x[v];
          o[12 * idx + 3 * v + 1] = t.y[v];
          o[12 * idx + 3 * v + 2] = t.z[v];
        }
      }
      ++idx;
    });
    if (measure) measure[i] = m;
    if (nout) nout[i] = k;
  }
}

// Quadrilateral vs quadrilateral (Supermesh.F90:230-246): clip quad A by
// quad B's 4 edge lines; no element area is given, so the fan keeps
// triangles with area >= 10*tiny (Triangle_Intersection.F90:255-264).
__global__ void k_pairs_quad_quad(int64_t n, const double* __restrict__ A, const double* __restrict__ B,
                                  double* measure, int32_t* nout, double* out_elems) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* va = A + 8 * i;
    double nx[4], ny[4], px[4], py[4];
    poly_lines<4>(B + 8 * i, nx, ny, px, py);
    LocalPoly<16> p, q;
#pragma unroll
    for (int v = 0; v < 4; ++v) p.set(v, va[2 * v], va[2 * v + 1]);
    int m = 4;
    bool empty = false;
    for (int l = 0; l < 4 && !empty; ++l) {
      m = (l & 1) ? clip_stage(q, p, m, 16, nx[l], ny[l], px[l], py[l])
                  : clip_stage(p, q, m, 16, nx[l], ny[l], px[l], py[l]);
      empty = m < 3;
    }
    double meas = 0.0;
    int kept = 0;
    if (!empty) {
      const double tol = 10.0 * DBL_MIN;
      double* o = out_elems ? out_elems + 62 * 6 * i : nullptr;
      const double x0 = p.x(0), y0 = p.y(0);
      for (int j = 1; j < m - 1; ++j) {
        const double xi = p.x(j), yi = p.y(j), xj = p.x(j + 1), yj = p.y(j + 1);
        const double ar = tri_area(x0, y0, xi, yi, xj, yj);
        if (!(ar < tol)) {
          meas = meas + ar;
          if (o && kept < 62) {
            double* t = o + 6 * kept;
            t[0] = x0;
            t[1] = y0;
            t[2] = xi;
            t[3] = yi;
            t[4] = xj;
            t[5] = yj;
          }
          ++kept;
        }
      }
    }
    if (measure) measure[i] = meas;
    if (nout) nout[i] = kept;
  }
}

// Hexahedron vs hexahedron (Supermesh.F90:303-334): hex A sliced into five
// tets (Gmsh corners 3,6,7,8 / 1,3,4,8 / 1,5,6,8 / 1,2,3,6 / 1,3,6,8), each
// clipped by hex B as in intersect_tet_hex; outputs concatenated.
__global__ void __launch_bounds__(64) k_pairs_hex_hex(int64_t n, const double* __restrict__ A,
                                                      const double* __restrict__ B, double* measure,
                                                      int32_t* nout, double* out_elems) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* h = A + 24 * i;
    ArrPlanes<6> P;
    hex_planes(B + 24 * i, P.nx, P.ny, P.nz, P.c);
    double m = 0.0;
    int total = 0;
    double* o = out_elems ? out_elems + (int64_t)5 * 729 * 12 * i : nullptr;
    for (int s = 0; s < 5; ++s) {
      Tet ta;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        ta.x[v] = h[3 * kHexTets[s][v]];
        ta.y[v] = h[3 * kHexTets[s][v] + 1];
        ta.z[v] = h[3 * kHexTets[s][v] + 2];
      }
      const double tol = 10.0 * spacing(tet_volume_v4(ta));
      TetStackN<10> stk;
      const int k = clip_tet_dfs<6>(ta, P, tol, stk, [&](const Tet& t) {
        m = m + tet_volume_v1(t);
        if (o && total < 5 * 729) {
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            o[12 * total + 3 * v + 0] = t.x[v];
            o[12 * total + 3 * v + 1] = t.y[v];
            o[12 * total + 3 * v + 2] = t.z[v];
          }
        }
        ++total;
      });
      (void)k;
    }
    if (measure) measure[i] = m;
    if (nout) nout[i] = total;
  }
}

__global__ void k_pairs_intervals(int64_t n, const double* __restrict__ A, const double* __restrict__ B,
                                  double* measure, int32_t* nout, double* out_elems) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double c0 = 0.0, c1 = 0.0;
    const int k = intersect_intervals(A[2 * i], A[2 * i + 1], B[2 * i], B[2 * i + 1], c0, c1);
    if (out_elems && k) {
      out_elems[2 * i] = c0;
      out_elems[2 * i + 1] = c1;
    }
    if (measure) measure[i] = k ? interval_size(c0, c1) : 0.0;
    if (nout) nout[i] = k;
  }
}

cudaError_t launch_pairs_mixed(int kind, int64_t n, const double* a, const double* b, double* measure,
                               int32_t* nout, double* out_elems, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launch();
  if (kind == 0)
    k_pairs_intervals<<<grid_for(n, 256, 8), 256, 0, s>>>(n, a, b, measure, nout, out_elems);
  else if (kind == 1)
    k_pairs_tri_quad<<<grid_for(n, 128, 8), 128, 0, s>>>(n, a, b, measure, nout, out_elems);
  else if (kind == 2)
    k_pairs_tet_hex<<<grid_for(n, 64, 8), 64, 0, s>>>(n, a, b, measure, nout, out_elems);
  else if (kind == 3)
    k_pairs_quad_quad<<<grid_for(n, 128, 8), 128, 0, s>>>(n, a, b, measure, nout, out_elems);
  else
    k_pairs_hex_hex<<<grid_for(n, 64, 8), 64, 0, s>>>(n, a, b, measure, nout, out_elems);
  return cudaGetLastError();
}

// ======================================================================
// 1D sort finder (Intersection_Finder.F90:811-921): elements sorted by left
// end, then one sweep pointer over the sorted B elements.  Restated as
//   E_i  = first sorted B element whose left end >= right end of sorted A_i
//   L_i  = last sorted B element before E_i whose right end > left end of A_i
//   row_i records {j in [js_i, E_i) : right_B(j) > left_A(i)}
//   js_{i+1} = y_i - [js_i <= L_i],  y_i = max(js_i, E_i) advanced past B
//              points equal to a point A_i
// E_i and L_i (binary search, max segment tree) and the rows are computed in
// parallel; only the integer recurrence for js runs on one warp.
// ======================================================================
__device__ __forceinline__ uint64_t ordered_key(double x) {
  if (x == 0.0) x = 0.0;  // -0 and +0 compare equal: give them one key
  const uint64_t u = (uint64_t)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

__global__ void k_prep_1d(int64_t nel, const double* __restrict__ pos, int stride, const void* __restrict__ en,
                          int idx_bytes, int64_t nnodes, double* coords, uint32_t* key_lo, uint32_t* key_hi,
                          int32_t* vals, int* bad) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t n0, n1;
    if (idx_bytes == 8) {
      n0 = static_cast<const int64_t*>(en)[2 * e];
      n1 = static_cast<const int64_t*>(en)[2 * e + 1];
    } else {
      n0 = static_cast<const int32_t*>(en)[2 * e];
      n1 = static_cast<const int32_t*>(en)[2 * e + 1];
    }
    if (n0 < 0 || n0 >= nnodes || n1 < 0 || n1 >= nnodes) {
      atomicExch(bad, 1);
      n0 = n1 = 0;
    }
    const double x0 = pos[n0 * stride], x1 = pos[n1 * stride];
    coords[2 * e] = x0;
    coords[2 * e + 1] = x1;
    const uint64_t k = ordered_key(x1 < x0 ? x1 : x0);
    key_lo[e] = (uint32_t)k;
    key_hi[e] = (uint32_t)(k >> 32);
    vals[e] = (int32_t)e;
  }
}

__global__ void k_permute_u32(int64_t n, const int32_t* __restrict__ perm, const uint32_t* __restrict__ in,
                              uint32_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[perm[i]];
}

__global__ void k_sorted_ends_1d(int64_t n, const int32_t* __restrict__ perm, const double* __restrict__ coords,
                                 double* lo, double* hi) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t e = perm[i];
    const double x0 = coords[2 * e], x1 = coords[2 * e + 1];
    lo[i] = x1 < x0 ? x1 : x0;
    hi[i] = x1 > x0 ? x1 : x0;
  }
}

__global__ void k_tree_leaves(int64_t n, int64_t P, const double* __restrict__ v, double* tree) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += (int64_t)gridDim.x * blockDim.x)
    tree[P + i] = i < n ? v[i] : -INFINITY;
}

__global__ void k_tree_level(int64_t w, double* tree) {
  for (int64_t k = w + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < 2 * w; k += (int64_t)gridDim.x * blockDim.x)
    tree[k] = fmax(tree[2 * k], tree[2 * k + 1]);
}

// Last leaf index < E whose value is > t, or -1 (tree over P leaves).
__device__ __forceinline__ int rightmost_greater(const double* __restrict__ tree, int64_t P, int64_t E, double t) {
  if (E <= 0) return -1;
  int64_t node = P + E - 1;
  for (int guard = 0; guard < 256; ++guard) {
    if (tree[node] > t) {
      while (node < P) node = tree[2 * node + 1] > t ? 2 * node + 1 : 2 * node;
      return (int)(node - P);
    }
    // move to the subtree just left of `node`
    while ((node & (node - 1)) != 0 && (node & 1) == 0) node >>= 1;
    if ((node & (node - 1)) == 0) return -1;  // leftmost at its level
    node -= 1;
  }
  return -1;
}

__global__ void k_rows_1d(int64_t na, const double* __restrict__ lo_a, const double* __restrict__ hi_a, int64_t nb,
                          const double* __restrict__ lo_b, const double* __restrict__ tree, int64_t P, int32_t* E,
                          int32_t* L) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (int64_t)gridDim.x * blockDim.x) {
    const double h = hi_a[i];
    int64_t lo = 0, hi = nb;  // first j with lo_b[j] >= h
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (lo_b[mid] < h)
        lo = mid + 1;
      else
        hi = mid;
    }
    E[i] = (int32_t)lo;
    L[i] = nb > 0 ? rightmost_greater(tree, P, lo, lo_a[i]) : -1;
  }
}

__global__ void __launch_bounds__(32) k_sweep_1d(int64_t na, int64_t nb, const int32_t* __restrict__ E,
                                                 const int32_t* __restrict__ L, const double* __restrict__ lo_a,
                                                 const double* __restrict__ hi_a, const double* __restrict__ hi_b,
                                                 int32_t* JS) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x;
  int64_t js = 0;
  for (int64_t base = 0; base < na; base += 32) {
    const int64_t i = base + lane;
    int e = 0, l = -1;
    double lo = 0.0, hi = 1.0;
    if (i < na) {
      e = E[i];
      l = L[i];
      lo = lo_a[i];
      hi = hi_a[i];
    }
    const unsigned point = __ballot_sync(full, i < na && !(lo < hi));
    const int cnt = (int)(na - base < 32 ? na - base : 32);
    int64_t mine = 0;
    for (int k = 0; k < cnt; ++k) {
      const int ek = __shfl_sync(full, e, k);
      const int lk = __shfl_sync(full, l, k);
      if (lane == k) mine = js;
      int64_t y = js > ek ? js : ek;
      if ((point >> k) & 1u) {
        const double t = __shfl_sync(full, lo, k);
        while (y < nb && hi_b[y] <= t) ++y;
      }
      js = js <= lk ? y - 1 : y;
    }
    if (i < na) JS[i] = (int32_t)mine;
  }
}

template <bool FILL>
__global__ void k_emit_1d(int64_t na, const int32_t* __restrict__ JS, const int32_t* __restrict__ E,
                          const double* __restrict__ lo_a, const double* __restrict__ hi_b,
                          const int32_t* __restrict__ perm_a, const int32_t* __restrict__ perm_b, int* counts,
                          const int64_t* __restrict__ offsets, int32_t* pair_a, int32_t* pair_b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < na; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = perm_a[i];
    const double t = lo_a[i];
    const int32_t end = E[i];
    int64_t out = FILL ? offsets[a] : 0;
    int cnt = 0;
    for (int32_t j = JS[i]; j < end; ++j) {
      if (hi_b[j] > t) {
        if (FILL) {
          pair_a[out + cnt] = a;
          pair_b[out + cnt] = perm_b[j];
        }
        ++cnt;
      }
    }
    if (!FILL) counts[a] = cnt;
  }
}

cudaError_t launch_prep_1d(int64_t nel, const double* pos, int stride, const void* en, int idx_bytes,
                           int64_t nnodes, double* coords, uint32_t* key_lo, uint32_t* key_hi, int32_t* vals,
                           int* bad, cudaStream_t s) {
  if (nel <= 0) return cudaSuccess;
  count_launch();
  k_prep_1d<<<grid_for(nel, 256, 8), 256, 0, s>>>(nel, pos, stride, en, idx_bytes, nnodes, coords, key_lo, key_hi,
                                                  vals, bad);
  return cudaGetLastError();
}

cudaError_t sort_by_key64(int64_t n, uint32_t* key_lo, const uint32_t* key_hi, int32_t* vals, uint32_t* keys_tmp,
                          int32_t* vals_tmp, uint32_t* hist, cudaStream_t s) {
  if (n <= 1) return cudaSuccess;
  cudaError_t e = radix_sort_pairs(n, 32, key_lo, vals, keys_tmp, vals_tmp, hist, s);
  if (e != cudaSuccess) return e;
  count_launch();
  k_permute_u32<<<grid_for(n, 256, 8), 256, 0, s>>>(n, vals, key_hi, key_lo);
  return radix_sort_pairs(n, 32, key_lo, vals, keys_tmp, vals_tmp, hist, s);
}

cudaError_t launch_sorted_ends_1d(int64_t n, const int32_t* perm, const double* coords, double* lo, double* hi,
                                  cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launch();
  k_sorted_ends_1d<<<grid_for(n, 256, 8), 256, 0, s>>>(n, perm, coords, lo, hi);
  return cudaGetLastError();
}

int64_t tree_leaves_1d(int64_t n) {
  int64_t P = 1;
  while (P < n) P <<= 1;
  return P;
}

cudaError_t launch_max_tree(int64_t n, const double* v, double* tree, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int64_t P = tree_leaves_1d(n);
  count_launch();
  k_tree_leaves<<<grid_for(P, 256, 8), 256, 0, s>>>(n, P, v, tree);
  for (int64_t w = P / 2; w >= 1; w /= 2) {
    count_launch();
    k_tree_level<<<grid_for(w, 256, 8), 256, 0, s>>>(w, tree);
  }
  return cudaGetLastError();
}

cudaError_t launch_rows_1d(int64_t na, const double* lo_a, const double* hi_a, int64_t nb, const double* lo_b,
                           const double* tree, int32_t* E, int32_t* L, cudaStream_t s) {
  if (na <= 0) return cudaSuccess;
  count_launch();
  k_rows_1d<<<grid_for(na, 256, 8), 256, 0, s>>>(na, lo_a, hi_a, nb, lo_b, tree, tree_leaves_1d(nb), E, L);
  return cudaGetLastError();
}

cudaError_t launch_sweep_1d(int64_t na, int64_t nb, const int32_t* E, const int32_t* L, const double* lo_a,
                            const double* hi_a, const double* hi_b, int32_t* JS, cudaStream_t s) {
  if (na <= 0) return cudaSuccess;
  count_launch();
  k_sweep_1d<<<1, 32, 0, s>>>(na, nb, E, L, lo_a, hi_a, hi_b, JS);
  return cudaGetLastError();
}

cudaError_t launch_emit_1d(bool fill, int64_t na, const int32_t* JS, const int32_t* E, const double* lo_a,
                           const double* hi_b, const int32_t* perm_a, const int32_t* perm_b, int* counts,
                           const int64_t* offsets, int32_t* pair_a, int32_t* pair_b, cudaStream_t s) {
  if (na <= 0) return cudaSuccess;
  count_launch();
  if (fill)
    k_emit_1d<true><<<grid_for(na, 256, 8), 256, 0, s>>>(na, JS, E, lo_a, hi_b, perm_a, perm_b, counts, offsets,
                                                         pair_a, pair_b);
  else
    k_emit_1d<false><<<grid_for(na, 256, 8), 256, 0, s>>>(na, JS, E, lo_a, hi_b, perm_a, perm_b, counts, offsets,
                                                          pair_a, pair_b);
  return cudaGetLastError();
}

// Narrow phase of 1D candidates: intersect_intervals per pair.
__global__ void k_clip_intervals(int64_t n, const int32_t* __restrict__ pa, const int32_t* __restrict__ pb,
                                 const double* __restrict__ ca, const double* __restrict__ cb, double* measure,
                                 int32_t* nout) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = pa[i], b = pb[i];
    double c0 = 0.0, c1 = 0.0;
    const int k = intersect_intervals(ca[2 * a], ca[2 * a + 1], cb[2 * b], cb[2 * b + 1], c0, c1);
    measure[i] = k ? interval_size(c0, c1) : 0.0;
    nout[i] = k;
  }
}

cudaError_t launch_clip_intervals(int64_t n, const int32_t* pa, const int32_t* pb, const double* ca,
                                  const double* cb, double* measure, int32_t* nout, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launch();
  k_clip_intervals<<<grid_for(n, 256, 8), 256, 0, s>>>(n, pa, pb, ca, cb, measure, nout);
  return cudaGetLastError();
}

cudaError_t launch_pairs_explicit(int dim, int64_t n, const double* a, const double* b,
                                  double* measure, int32_t* nout, double* out_elems,
                                  cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int B = 128;
  const int g = grid_for(n, B, 8);
  count_launch();
  if (dim == 2)
    k_pairs_tris<<<g, B, 0, s>>>(n, a, b, measure, nout, out_elems);
  else
    k_pairs_tets<<<g, B, 0, s>>>(n, a, b, measure, nout, out_elems);
  return cudaGetLastError();
}

__global__ void k_measure_explicit(int dim, int64_t n, const double* __restrict__ e, double* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (dim == 1) {
      out[i] = interval_size(e[2 * i], e[2 * i + 1]);
    } else if (dim == 2) {
      const double* v = e + 6 * i;
      out[i] = tri_area(v[0], v[1], v[2], v[3], v[4], v[5]);
    } else {
      Tet t;
      load_tet(e + 12 * i, t);
      out[i] = tet_volume_v1(t);
    }
  }
}

cudaError_t launch_measure_explicit(int dim, int64_t n, const double* elems, double* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launch();
  k_measure_explicit<<<grid_for(n, 256, 8), 256, 0, s>>>(dim, n, elems, out);
  return cudaGetLastError();
}

// ======================================================================
// K8: P1-P1 mixed mass matrix
// ======================================================================
// P1 basis on a triangle (test_parallel_p1_inner_product_2d.F90:206-229):
// the inverse Jacobian (divided by the determinant entry by entry) depends
// only on the element and is formed once per pair; each point then takes
// the same products and sums as the reference.
struct P1Fac2 {
  double ox, oy, j11, j12, j21, j22;
};

__device__ __forceinline__ P1Fac2 p1_factor_2d(const double* cc) {
  const double e1x = cc[2] - cc[0], e1y = cc[3] - cc[1];
  const double e2x = cc[4] - cc[0], e2y = cc[5] - cc[1];
  double j11 = e2y, j12 = -e2x, j21 = -e1y, j22 = e1x;
  const double det = j11 * j22 - j12 * j21;
  return P1Fac2{cc[0], cc[1], j11 / det, j12 / det, j21 / det, j22 / det};
}

__device__ __forceinline__ void p1_apply_2d(const P1Fac2& F, double x, double y, double f[3]) {
  const double dx = x - F.ox, dy = y - F.oy;
  f[1] = F.j11 * dx + F.j12 * dy;
  f[2] = F.j21 * dx + F.j22 * dy;
  f[0] = 1.0 - f[1] - f[2];
}

template <typename IDX>
__device__ __forceinline__ int64_t node_of(const void* en, int64_t e, int loc, int k) {
  return (int64_t)((const IDX*)en)[e * loc + k];
}

// P1 basis on a tetrahedron (test_parallel_p1_inner_product_3d.F90:215-250):
// the local coordinates of point x solve [v1-v0 | v2-v0 | v3-v0] l = x - v0
// by Gaussian elimination with partial pivoting on the augmented 3x4 matrix
// (pivot search, row swap, pivot row divided by the pivot, rows below
// reduced; then back substitution from the last row), f = (1 - l1 - l2 - l3,
// l1, l2, l3).  The pivot choices, pivots and multipliers depend only on the
// element's edge matrix, so p1_factor_3d runs that elimination on the three
// matrix columns once per element and stores, at stride S: the origin v0
// (3), the pivots (3), the forward multipliers of rows (1,0) (2,0) (2,1) and
// the back-substitution multipliers of rows (1,2) (0,2) (0,1); it returns the
// row swaps (row exchanged with row 0 in bits 0-1, with row 1 in bits 2-3).
// p1_apply_3d applies to the point's right-hand side exactly the operations
// the elimination applies to the augmented column, in the same order.
constexpr int kP1Fac3 = 12;

template <int S>
__device__ __forceinline__ int p1_factor_3d(const double* cc, double* F) {
  double m[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
#pragma unroll
    for (int c = 0; c < 3; ++c) m[r][c] = cc[3 * (c + 1) + r] - cc[r];
    F[r * S] = cc[r];
  }
  int sw = 0, nl = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    int j = i;
    double best = fabs(m[i][i]);
#pragma unroll
    for (int k = i + 1; k < 3; ++k)
      if (fabs(m[k][i]) > best) {
        best = fabs(m[k][i]);
        j = k;
      }
#pragma unroll
    for (int k = i + 1; k < 3; ++k) {
      if (j == k) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double t = m[i][c];
          m[i][c] = m[k][c];
          m[k][c] = t;
        }
      }
    }
    sw |= j << (2 * i);
    const double piv = m[i][i];
    F[(3 + i) * S] = piv;
#pragma unroll
    for (int c = 0; c < 3; ++c) m[i][c] = m[i][c] / piv;
#pragma unroll
    for (int k = i + 1; k < 3; ++k) {
      const double fk = m[k][i];
      F[(6 + nl++) * S] = fk;
#pragma unroll
      for (int c = 0; c < 3; ++c) m[k][c] = m[k][c] - fk * m[i][c];
    }
  }
  int nu = 0;
#pragma unroll
  for (int i = 2; i >= 0; --i)
#pragma unroll
    for (int k = i - 1; k >= 0; --k) {
      const double fk = m[k][i];
      F[(9 + nu++) * S] = fk;
#pragma unroll
      for (int c = 0; c < 3; ++c) m[k][c] = m[k][c] - fk * m[i][c];
    }
  return sw;
}

template <int S>
__device__ __forceinline__ void p1_apply_3d(const double* F, int sw, double x, double y, double z, double f[4]) {
  double r0 = x - F[0], r1 = y - F[S], r2 = z - F[2 * S];
  const int j0 = sw & 3, j1 = (sw >> 2) & 3;
  {
    const double t0 = r0;
    r0 = j0 == 1 ? r1 : (j0 == 2 ? r2 : r0);
    r1 = j0 == 1 ? t0 : r1;
    r2 = j0 == 2 ? t0 : r2;
  }
  r0 = r0 / F[3 * S];
  r1 = r1 - F[6 * S] * r0;
  r2 = r2 - F[7 * S] * r0;
  {
    const double t1 = r1;
    r1 = j1 == 2 ? r2 : r1;
    r2 = j1 == 2 ? t1 : r2;
  }
  r1 = r1 / F[4 * S];
  r2 = r2 - F[8 * S] * r1;
  r2 = r2 / F[5 * S];
  r1 = r1 - F[9 * S] * r2;
  r0 = r0 - F[10 * S] * r2;
  r0 = r0 - F[11 * S] * r1;
  f[1] = r0;
  f[2] = r1;
  f[3] = r2;
  f[0] = 1.0 - f[1] - f[2] - f[3];
}

// P1-P1 mixed mass block of a pair (test_parallel_p1_inner_product_3d.F90:
// four-point rule, P1 bases of A and B by elimination at each point), per
// kept output tet in the reference's order; at the end of the pair the block
// is stored and u^T M v written per pair (lanes take pairs in a dynamic order;
// the caller sums them in pair order).  The per-element part of
// both eliminations is done once per pair (p1_factor_3d) into the lane's
// slice of shared memory behind the point pool (kLaneDoubles per lane).
template <typename IDX, int BLOCK>
struct IxP1Sink {
  static constexpr bool kInside = true;
  static constexpr int kLaneDoubles = 2 * kP1Fac3;
  const double* coords_a;
  const double* coords_b;
  const void* en_a;
  const void* en_b;
  const double* u_a;
  const double* v_b;
  double* blocks;
  double* pair_uv;  // u^T M v per pair (when u_a and v_b are given), summed in pair order afterwards
  double blk[16];
  double* fac;  // this lane's factors: A's at fac, B's at fac + kP1Fac3 * BLOCK
  int a, b, swa, swb;
  __device__ __forceinline__ void bind(double* lane_mem) { fac = lane_mem; }
  __device__ __forceinline__ void begin(const int4& r) {
    a = r.y;
    b = r.z;
    swa = p1_factor_3d<BLOCK>(coords_a + (int64_t)a * 12, fac);
    swb = p1_factor_3d<BLOCK>(coords_b + (int64_t)b * 12, fac + kP1Fac3 * BLOCK);
#pragma unroll
    for (int j = 0; j < 16; ++j) blk[j] = 0.0;
  }
  __device__ __forceinline__ void tet(const Tet& o, double v1) {
    const double qa = 5.8541019662496852e-1, qb = 1.3819660112501050e-1;
    const double w = 0.25 * v1;
#pragma unroll
    for (int qq = 0; qq < 4; ++qq) {
      double x = 0.0, y = 0.0, z = 0.0;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const double wv = v == qq ? qa : qb;
        x = x + wv * o.x[v];
        y = y + wv * o.y[v];
        z = z + wv * o.z[v];
      }
      double fa[4], fb[4];
      p1_apply_3d<BLOCK>(fac, swa, x, y, z, fa);
      p1_apply_3d<BLOCK>(fac + kP1Fac3 * BLOCK, swb, x, y, z, fb);
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) blk[r * 4 + c] += w * fa[r] * fb[c];
    }
  }
  __device__ __forceinline__ void end(int64_t p) {
    if (blocks) {
#pragma unroll
      for (int j = 0; j < 16; ++j) blocks[p * 16 + j] = blk[j];
    }
    if (u_a && v_b) {
      double sv = 0.0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const double ur = u_a[node_of<IDX>(en_a, a, 4, r)];
#pragma unroll
        for (int c = 0; c < 4; ++c) sv += ur * blk[r * 4 + c] * v_b[node_of<IDX>(en_b, b, 4, c)];
      }
      pair_uv[p] = sv;
    }
  }
  template <int NT>
  __device__ __forceinline__ void finish() {}
};


// 2D: one pair per thread, clipped with the triangle clipper; per supermesh
// triangle the degree-2 rule (three points), P1 bases of A and B, 3x3 block.
template <typename IDX>
__global__ void __launch_bounds__(128) k_p1_mass(int64_t npairs, const int32_t* __restrict__ pa,
                                                 const int32_t* __restrict__ pb,
                                                 const double* __restrict__ coords_a,
                                                 const double* __restrict__ tol_a,
                                                 const double* __restrict__ coords_b,
                                                 const double* __restrict__ setup_b, const void* en_a,
                                                 const void* en_b, const double* __restrict__ u_a,
                                                 const double* __restrict__ v_b, double* blocks,
                                                 Partial* partials) {
  double sum = 0.0, err = 0.0;
  unsigned long long ni = 0;
  // each iteration loads the next one's pair indices (which stream from
  // DRAM) before it works on its own pair
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int na = 0, nb = 0;
  {
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i0 < npairs) {
      na = pa[i0];
      nb = pb[i0];
    }
  }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npairs; i += stride) {
    const int a = na, b = nb;
    if (i + stride < npairs) {
      na = pa[i + stride];
      nb = pb[i + stride];
    }
    const double* ca = coords_a + (int64_t)a * 6;
    double blk[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) blk[j] = 0.0;
    Lines L;
    double tolb;
    load_lines(setup_b + (int64_t)b * kSetup2, L, tolb);
    const double tol = fmin(tol_a[a], tolb);
    const P1Fac2 fa_ = p1_factor_2d(ca), fb_ = p1_factor_2d(coords_b + (int64_t)b * 6);
    LocalPoly<kTriWideCap> p, q;
    double m;
    const double qp0 = 4.0 / 6.0, qp1 = 1.0 / 6.0;
    clip_tri(ca[0], ca[1], ca[2], ca[3], ca[4], ca[5], L, tol, p, q, kTriWideCap, m,
             [&](int, double x0, double y0, double x1, double y1, double x2, double y2) {
               const double meas = tri_area(x0, y0, x1, y1, x2, y2);
               const double w = (1.0 / 3.0) * meas;
#pragma unroll
               for (int qq = 0; qq < 3; ++qq) {
                 const double w0 = qq == 0 ? qp0 : qp1;
                 const double w1 = qq == 1 ? qp0 : qp1;
                 const double w2 = qq == 2 ? qp0 : qp1;
                 const double x = (w0 * x0 + w1 * x1) + w2 * x2;
                 const double y = (w0 * y0 + w1 * y1) + w2 * y2;
                 double fa[3], fb[3];
                 p1_apply_2d(fa_, x, y, fa);
                 p1_apply_2d(fb_, x, y, fb);
#pragma unroll
                 for (int r = 0; r < 3; ++r)
#pragma unroll
                   for (int c = 0; c < 3; ++c) blk[r * 3 + c] += w * fa[r] * fb[c];
               }
             });
    if (blocks) {
#pragma unroll
      for (int j = 0; j < 9; ++j) blocks[i * 9 + j] = blk[j];
    }
    if (u_a && v_b) {
      double sv = 0.0;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const double ur = u_a[node_of<IDX>(en_a, a, 3, r)];
#pragma unroll
        for (int c = 0; c < 3; ++c) sv += ur * blk[r * 3 + c] * v_b[node_of<IDX>(en_b, b, 3, c)];
      }
      cs_add(sum, err, sv);
    }
    ++ni;
  }
  block_reduce_partial<128>(sum, err, ni, 0ull, &partials[blockIdx.x]);
}

// ----------------------------------------------------------------------
// P2 inner product (test_parallel_p2_inner_product_2d.F90:398-522)
// ----------------------------------------------------------------------
// P2 basis of triangle cc ([3][2]) at point (x, y), basis_functions_p2
// (:399-433): local coordinates through the inverse Jacobian, then the six
// quadratic Lagrange functions (vertices 1-3, edge midpoints 1-2, 2-3, 1-3).
__device__ __forceinline__ void p2_basis_2d(const double* cc, double x, double y, double f[6]) {
  const double e10 = cc[2] - cc[0], e11 = cc[3] - cc[1];
  const double e20 = cc[4] - cc[0], e21 = cc[5] - cc[1];
  double j11 = e21, j12 = -e20, j21 = -e11, j22 = e10;
  const double det = j11 * j22 - j12 * j21;
  j11 = j11 / det;
  j12 = j12 / det;
  j21 = j21 / det;
  j22 = j22 / det;
  const double d1 = x - cc[0], d2 = y - cc[1];
  const double lx = j11 * d1 + j12 * d2, ly = j21 * d1 + j22 * d2;
  f[0] = ((1.0 - lx) - ly) * ((1.0 - 2.0 * lx) - 2.0 * ly);
  f[1] = lx * (2.0 * lx - 1.0);
  f[2] = ly * (2.0 * ly - 1.0);
  f[3] = (4.0 * lx) * ((1.0 - lx) - ly);
  f[4] = (4.0 * lx) * ly;
  f[5] = (4.0 * ly) * ((1.0 - lx) - ly);
}

__device__ __forceinline__ double p2_interp_2d(const double* cc, const double v[6], double x, double y) {
  double f[6];
  p2_basis_2d(cc, x, y, f);
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 6; ++k) s = s + f[k] * v[k];
  return s;
}

// Per candidate pair: clip, then for every supermesh triangle c the P2
// fields of A and B at c's vertices and edge midpoints and the contribution
// 2 |c| f_b . (M f_a), summed over c in output order.
template <class IDX>
__global__ void __launch_bounds__(128) k_p2_inner(int64_t npairs, const int32_t* __restrict__ pa,
                                                  const int32_t* __restrict__ pb,
                                                  const double* __restrict__ coords_a,
                                                  const double* __restrict__ tol_a,
                                                  const double* __restrict__ coords_b,
                                                  const double* __restrict__ setup_b, const void* en_p2_a,
                                                  const double* __restrict__ field_a, const void* en_p2_b,
                                                  const double* __restrict__ field_b, double* pair_value,
                                                  double* pair_area, int32_t* pair_n) {
  constexpr double M[6][6] = {
      {6.0 / 360.0, -1.0 / 360.0, -1.0 / 360.0, 0.0 / 360.0, -4.0 / 360.0, 0.0 / 360.0},
      {-1.0 / 360.0, 6.0 / 360.0, -1.0 / 360.0, 0.0 / 360.0, 0.0 / 360.0, -4.0 / 360.0},
      {-1.0 / 360.0, -1.0 / 360.0, 6.0 / 360.0, -4.0 / 360.0, 0.0 / 360.0, 0.0 / 360.0},
      {0.0 / 360.0, 0.0 / 360.0, -4.0 / 360.0, 32.0 / 360.0, 16.0 / 360.0, 16.0 / 360.0},
      {-4.0 / 360.0, 0.0 / 360.0, 0.0 / 360.0, 16.0 / 360.0, 32.0 / 360.0, 16.0 / 360.0},
      {0.0 / 360.0, -4.0 / 360.0, 0.0 / 360.0, 16.0 / 360.0, 16.0 / 360.0, 32.0 / 360.0}};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npairs;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int a = pa[i], b = pb[i];
    const double* ca = coords_a + (int64_t)a * 6;
    const double* cb = coords_b + (int64_t)b * 6;
    double va[6], vb[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      va[k] = field_a[node_of<IDX>(en_p2_a, a, 6, k)];
      vb[k] = field_b[node_of<IDX>(en_p2_b, b, 6, k)];
    }
    Lines L;
    double tolb;
    load_lines(setup_b + (int64_t)b * kSetup2, L, tolb);
    const double tol = fmin(tol_a[a], tolb);
    LocalPoly<kTriWideCap> p, q;
    double m;
    double sp = 0.0, sa = 0.0;
    int nt = 0;
    clip_tri(ca[0], ca[1], ca[2], ca[3], ca[4], ca[5], L, tol, p, q, kTriWideCap, m,
             [&](int, double x0, double y0, double x1, double y1, double x2, double y2) {
               const double ar = tri_area(x0, y0, x1, y1, x2, y2);
               sa = sa + ar;
               ++nt;
               const double px[6] = {x0, x1, x2, 0.5 * (x0 + x1), 0.5 * (x1 + x2), 0.5 * (x0 + x2)};
               const double py[6] = {y0, y1, y2, 0.5 * (y0 + y1), 0.5 * (y1 + y2), 0.5 * (y0 + y2)};
               double fa[6], fb[6];
#pragma unroll
               for (int l = 0; l < 6; ++l) {
                 fb[l] = p2_interp_2d(cb, vb, px[l], py[l]);
                 fa[l] = p2_interp_2d(ca, va, px[l], py[l]);
               }
               double dot = 0.0;
#pragma unroll
               for (int r = 0; r < 6; ++r) {
                 double mi = 0.0;
#pragma unroll
                 for (int k = 0; k < 6; ++k) mi = mi + M[r][k] * fa[k];
                 dot = dot + fb[r] * mi;
               }
               sp = sp + (2.0 * ar) * dot;
             });
    pair_value[i] = sp;
    pair_area[i] = sa;
    pair_n[i] = nt;
  }
}

__global__ void k_check_index(int64_t n, const void* en, int idx_bytes, int64_t limit, int* bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = idx_bytes == 8 ? static_cast<const int64_t*>(en)[i] : static_cast<const int32_t*>(en)[i];
    if (v < 0 || v >= limit) atomicExch(bad, 1);
  }
}

cudaError_t launch_check_index(int64_t n, const void* en, int idx_bytes, int64_t limit, int* bad, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  count_launch();
  k_check_index<<<grid_for(n, 256, 8), 256, 0, s>>>(n, en, idx_bytes, limit, bad);
  return cudaGetLastError();
}

cudaError_t launch_p2_inner(int64_t npairs, const int32_t* pair_a, const int32_t* pair_b, const double* coords_a,
                            const double* tol_a, const double* coords_b, const double* setup_b,
                            const void* en_p2_a, const double* field_a, const void* en_p2_b,
                            const double* field_b, int idx_bytes, double* pair_value, double* pair_area,
                            int32_t* pair_n, cudaStream_t s) {
  if (npairs <= 0) return cudaSuccess;
  count_launch();
  const int g = sm_count() * 4;
  if (idx_bytes == 4)
    k_p2_inner<int32_t><<<g, 128, 0, s>>>(npairs, pair_a, pair_b, coords_a, tol_a, coords_b, setup_b, en_p2_a,
                                          field_a, en_p2_b, field_b, pair_value, pair_area, pair_n);
  else
    k_p2_inner<int64_t><<<g, 128, 0, s>>>(npairs, pair_a, pair_b, coords_a, tol_a, coords_b, setup_b, en_p2_a,
                                          field_a, en_p2_b, field_b, pair_value, pair_area, pair_n);
  return cudaGetLastError();
}

// 3D: the index clipper with the P1 sink, one block per SM.  The sink's
// 4x4 block accumulator and the quadrature raise the register need to about
// 250: 8 warps (2 per SM sub-partition) can hold them without spilling,
// while 9-12 warps are capped at 168 registers by the sub-partitions'
// register files and spill (pool: 256 x 480 B of shared memory).
#ifndef LSM_IX_P1_BLOCK
#define LSM_IX_P1_BLOCK 256
#endif
constexpr int kIxP1Block = LSM_IX_P1_BLOCK;

size_t p1_smem_bytes() {
  return (size_t)kIxP1Block * (3 * kIxPoints + IxP1Sink<int32_t, kIxP1Block>::kLaneDoubles) * sizeof(double);
}

// partials written by launch_p1_mass: one per 2D block, or the fixed-order
// reduction's blocks in 3D
int p1_grid_blocks(int dim) { return dim == 2 ? sm_count() * 4 : kReduceBlocks; }

cudaError_t launch_p1_mass(int dim, int64_t npairs, const int32_t* pair_a, const int32_t* pair_b,
                           const double* coords_a, const double* tol_a, const double* coords_b,
                           const double* setup_b, const void* enlist_a, const void* enlist_b,
                           int idx_bytes, const double* u_a, const double* v_b, double* blocks,
                           Partial* partials, cudaStream_t s, int32_t* survivors, unsigned long long* work,
                           const double* faces_a, const double* screen_b, double* pair_uv, const SegList* seg) {
  const int g = dim == 2 ? p1_grid_blocks(2) : sm_count();
  if (dim == 2) {
    count_launch();
    if (idx_bytes == 4)
      k_p1_mass<int32_t><<<g, 128, 0, s>>>(npairs, pair_a, pair_b, coords_a, tol_a, coords_b, setup_b, enlist_a, enlist_b, u_a, v_b, blocks, partials);
    else
      k_p1_mass<int64_t><<<g, 128, 0, s>>>(npairs, pair_a, pair_b, coords_a, tol_a, coords_b, setup_b, enlist_a, enlist_b, u_a, v_b, blocks, partials);
    return cudaGetLastError();
  }
  // the early-out pass lists the pairs with output tets (blocks and u^T M v
  // of the others stay zero), then the index clipper integrates their tets;
  // u^T M v per pair is summed in pair order (a fixed-order reduction into
  // reduce_pairs_blocks() partials), so the integral does not depend on the
  // order in which the lanes took the pairs
  const bool uv = u_a && v_b;
  cudaMemsetAsync(work, 0, 2 * sizeof(unsigned long long), s);
  if (blocks && npairs > 0) cudaMemsetAsync(blocks, 0, sizeof(double) * 16 * npairs, s);
  if (uv && npairs > 0) cudaMemsetAsync(pair_uv, 0, sizeof(double) * npairs, s);
  if (npairs > 0)
    run_prefilter<false, 4>(npairs, nullptr, pair_a, pair_b, coords_a, tol_a, setup_b, nullptr, nullptr, survivors,
                            work, faces_a, screen_b, nullptr, seg, s);
  const bool sg = seg_on(seg) && npairs > 0;
  const int4* list = reinterpret_cast<const int4*>(survivors);
  count_launch();
  if (idx_bytes == 4) {
    using Sk = IxP1Sink<int32_t, kIxP1Block>;
    Sk sk{coords_a, coords_b, enlist_a, enlist_b, u_a, v_b, blocks, pair_uv};
    k_clip_tets_ix<Sk, kIxP1Block, 1><<<g, kIxP1Block, p1_smem_bytes(), s>>>(
        list, sg ? work + 2 : work, coords_a, tol_a, setup_b, sk, work + 1, sg ? seg->table : nullptr);
  } else {
    using Sk = IxP1Sink<int64_t, kIxP1Block>;
    Sk sk{coords_a, coords_b, enlist_a, enlist_b, u_a, v_b, blocks, pair_uv};
    k_clip_tets_ix<Sk, kIxP1Block, 1><<<g, kIxP1Block, p1_smem_bytes(), s>>>(
        list, sg ? work + 2 : work, coords_a, tol_a, setup_b, sk, work + 1, sg ? seg->table : nullptr);
  }
  if (uv) {
    count_launch();
    k_reduce_pairs<<<kReduceBlocks, 256, 0, s>>>(npairs, pair_uv, nullptr, partials, nullptr);
  } else {
    cudaMemsetAsync(partials, 0, sizeof(Partial) * kReduceBlocks, s);
  }
  return cudaGetLastError();
}

cudaError_t init_p1_attributes() {
  const int smem = (int)p1_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(k_clip_tets_ix<IxP1Sink<int32_t, kIxP1Block>, kIxP1Block, 1>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_clip_tets_ix<IxP1Sink<int64_t, kIxP1Block>, kIxP1Block, 1>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  return e;
}

}  // namespace lsm
