// C-ABI of the B200 supermesh library: the drop-in entries of
// include/libsupermesh-c.h and the GPU extension of include/libsupermesh-gpu.h.
//
// Pipeline per mesh pair (all on one stream):
//   prep A, prep B            gather coords, boxes, tolerances, B clip setup
//   root box, Morton, sort    LBVH leaves in Morton order
//   LBVH build + refit
//   query (count) -> scan -> [host reads n_candidates] -> query (fill)
//   clip (+ overflow re-run) -> finalize (compensated totals, counts)
// The only host synchronisation inside the pipeline is the read of the
// candidate count, needed to size the pair arrays.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/libsupermesh-c.h"
#include "../../include/libsupermesh-gpu.h"
#include "lsm_kernels.h"
#include "lsm_sched.h"

namespace {

// Option time_kernels: record events around the clip kernel of every narrow
// phase (libsupermesh_gpu_clip_kernel_ms reads them).
bool g_time_kernels = false;
// second exact early-out of the tet clipper (B beyond a face of A)
bool g_tet_screen = true;
// spill chunks of the batched search's row cache: -1 automatic, 0 none (long
// rows traversed again), n > 0 at most n
int64_t g_spill_chunks = -1;
// Test hook of the allocation-failure path: -1 off; n >= 0: the next n
// device allocations of the contexts succeed and the one after fails as if
// cudaMalloc had run out of memory (the hook then switches itself off).
int64_t g_fail_alloc_after = -1;
// Schedule of the 3D clipper's work list: 0 plain (the early-out pass's
// order), 1 learned (survivors binned by the MLP's predicted output-size
// class within windows of g_sched_window), 2 true classes (binned by the
// output counts of the previous narrow phase over the same candidates: the
// best any predictor can do; a measurement, not a production mode).
int g_tet_schedule = 0;
int g_sched_window = 1024;
// Device-resident batched calls replay a CUDA graph of the whole batch when
// the same meshes come again (1), or always run eagerly (0, default).
int g_batch_graph = 0;

// ------------------------------------------------------------------ buffers
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

struct Ctx {
  int device = 0;
  int64_t device_mem = 0;  // total device memory
  cudaStream_t stream = nullptr;
  std::string last_error;
  int64_t bytes = 0;

  // mesh A (query side)
  DevBuf a_pos, a_en, a_coords, a_box64, a_tol, a_faces, surv;
  // mesh B (tree side)
  DevBuf b_pos, b_en, b_coords, b_box64, b_box32, b_setup, b_screen;
  // tree
  DevBuf keys, vals, keys_tmp, vals_tmp, hist, root_partial, rootbox, bvh_lo, bvh_work, bvh_leaf;
  // candidates
  DevBuf counts, offsets, scan_tmp, pair_a, pair_b, i64_tmp, q_cache, q_over, q_pool, q_next, q_first;
  // narrow phase
  DevBuf pair_measure, pair_nout, partials, ovf_list, misc, elem_measure, totals;
  DevBuf p1_list;  // survivors of the P1 pass's early-out (kept apart from the narrow phase's)
  // 3D narrow phase: per-block survivor segment lengths, the clipper's chunk
  // table, and the compacted list for the consumers that index survivors
  DevBuf seg_cnt, seg_tab, surv_list;
  DevBuf p1_seg_cnt, p1_seg_tab, x_seg_cnt, x_seg_tab;  // the same for the P1 pass and explicit pairs
  // explicit pairs / p1 / batched
  DevBuf x_a, x_b, x_measure, x_nout, x_elems, u_a, v_b, blocks;
  DevBuf x_setup, x_tol, x_iota, x_faces, x_screen, x_list;  // explicit tet pairs through the early-out pass
  DevBuf x_sub;  // hexahedron pairs: A's five tets
  DevBuf elem_off, x_pa, x_pb;  // supermesh elements: per-pair offsets, parents
  DevBuf bt_tabs, bt_pair_a, bt_pair_b, bt_mort, bt_codes, bt_roots, bt_stops, bt_tot, bt_ncand, bt_indptr;
  // host meshes of a batch staged on the device, one set per dimension (the
  // 3D set is copied on the side stream while the 2D group computes)
  DevBuf bt_stage_pa[2], bt_stage_ea[2], bt_stage_pb[2], bt_stage_eb[2];
  // learned scheduler: BF16 weight image, binned survivor list, classes
  DevBuf sched_w, sched_list, sched_cls, sched_adam;
  bool have_sched = false;
  // 1D sort finder
  DevBuf d1_keyhi, d1_perm_a, d1_perm_b, d1_lo_a, d1_hi_a, d1_lo_b, d1_hi_b, d1_tree, d1_e, d1_l, d1_js;
  void* host_stage = nullptr;  // pinned, grow-only
  size_t host_stage_cap = 0;
  // pinned host scalars
  void* host_scalars = nullptr;
  // pinned staging of the single-pair entries (inputs and the whole output
  // buffer travel through it, one host wait per call)
  void* pair_io = nullptr;
  void* pair_io_dev = nullptr;  // the same pinned buffer as seen by kernels (mapped), or null
  // events around the clip kernel of the last narrow phase (option time_kernels)
  cudaEvent_t clip_ev[2] = {nullptr, nullptr};
  // side stream for mesh A's upload and prep (overlaps B's tree build) and
  // the events that order it with the caller's stream
  cudaStream_t side = nullptr;
  cudaEvent_t side_ev[2] = {nullptr, nullptr};
  // large host meshes: element lists copied in chunks on their own stream,
  // each chunk's prep waiting for its copy (events: B's chunks, A's chunks,
  // and the copy stream's waits for earlier work)
  cudaStream_t copy = nullptr;
  cudaEvent_t chunk_ev[10] = {};
  bool clip_timed = false;
  bool surv_valid = false;  // surv holds the clipper's pair count of the last 3D narrow phase
  bool surv_seg = false;    // ... and ovf_list holds its survivors as segments (seg_tab)
  int64_t surv_npairs = 0;  // the pair count that narrow phase was sized for
  // bumped whenever a device buffer is (re)allocated: a captured graph holds
  // buffer addresses and is only replayed while this is unchanged
  uint64_t gen = 0;
  // graph of a device-resident batched call (option batch_graph)
  struct BatchGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> sig;
    uint64_t gen = 0;
    unsigned long long launches = 0;
    void* host = nullptr;  // pinned: both groups' tables and result areas
    size_t host_cap = 0;
    std::vector<int> idx[2];
    int64_t cap[2] = {0, 0};
    size_t res_off[2] = {0, 0};
    int last_dim = 0, last_loc = 0;
    int64_t last_na = 0, last_nb = 0;
    bool last_seg = false;
    int64_t last_surv_npairs = 0;
  } bg;

  // state of the last candidate search
  int dim = 0;
  int loc_a = 0, loc_b = 0;
  int64_t nel_a = 0, nel_b = 0;
  int64_t ncand = -1;
  bool have_pairs = false;
  bool simplex_prep = false;  // A coords/tol and B clip setup are current
};

struct Fail {
  int status;
};

void set_error(Ctx* c, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  c->last_error = buf;
}

#define CU(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      set_error(c, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                __LINE__);                                                           \
      throw Fail{e_ == cudaErrorMemoryAllocation ? LSM_ERROR_OUT_OF_MEMORY           \
                                                 : LSM_ERROR_CUDA};                  \
    }                                                                                \
  } while (0)

#define REQUIRE(cond, ...)         \
  do {                             \
    if (!(cond)) {                 \
      set_error(c, __VA_ARGS__);   \
      throw Fail{LSM_ERROR_INVALID_ARGUMENT}; \
    }                              \
  } while (0)

// When an exception leaves its scope, waits for both streams, so that a
// failed call returns with no copy or kernel of its own still reading the
// caller's meshes.
struct SyncOnThrow {
  cudaStream_t s0, s1, s2 = nullptr;
  int depth = std::uncaught_exceptions();
  ~SyncOnThrow() {
    if (std::uncaught_exceptions() > depth) {
      cudaStreamSynchronize(s0);
      cudaStreamSynchronize(s1);
      if (s2) cudaStreamSynchronize(s2);
    }
  }
};

template <class T>
T* ensure(Ctx* c, DevBuf& b, int64_t count) {
  size_t need = sizeof(T) * (size_t)(count > 0 ? count : 1);
  need = (need + 255) & ~(size_t)255;
  if (b.cap < need) {
    if (b.p) {
      cudaFree(b.p);
      c->bytes -= (int64_t)b.cap;
      b.p = nullptr;
      b.cap = 0;
    }
    size_t want = need + need / 4;  // growth headroom
    if (g_fail_alloc_after >= 0 && g_fail_alloc_after-- == 0) {
      set_error(c, "cudaMalloc of %zu bytes failed: out of memory (forced by option fail_alloc_after)", want);
      throw Fail{LSM_ERROR_OUT_OF_MEMORY};
    }
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      want = need;
      e = cudaMalloc(&b.p, want);
    }
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      set_error(c, "cudaMalloc of %zu bytes failed: %s", want, cudaGetErrorString(e));
      throw Fail{LSM_ERROR_OUT_OF_MEMORY};
    }
    b.cap = want;
    c->bytes += (int64_t)want;
    ++c->gen;
  }
  return static_cast<T*>(b.p);
}

void free_buf(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int init_ctx(int device, Ctx* c) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    (void)cudaGetLastError();
    return LSM_ERROR_CUDA;
  }
  if (device < 0 || device >= n) return LSM_ERROR_INVALID_ARGUMENT;
  DeviceGuard g(device);
  c->device = device;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) c->device_mem = (int64_t)total_b;
  (void)cudaGetLastError();
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocHost(&c->host_scalars, 4096) != cudaSuccess || lsm::init_device_attributes() != cudaSuccess ||
      cudaEventCreate(&c->clip_ev[0]) != cudaSuccess || cudaEventCreate(&c->clip_ev[1]) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->side_ev[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->side_ev[1], cudaEventDisableTiming) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking) != cudaSuccess) {
    (void)cudaGetLastError();
    return LSM_ERROR_CUDA;
  }
  for (cudaEvent_t& e : c->chunk_ev)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      (void)cudaGetLastError();
      return LSM_ERROR_CUDA;
  }
  return LSM_SUCCESS;
}

void fini_ctx(Ctx* c) {
  DeviceGuard g(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  DevBuf* all[] = {&c->a_pos, &c->a_en, &c->a_coords, &c->a_box64, &c->a_tol, &c->b_pos, &c->b_en,
                   &c->b_coords, &c->b_box64, &c->b_box32, &c->b_setup, &c->keys, &c->vals,
                   &c->keys_tmp, &c->vals_tmp, &c->hist, &c->root_partial, &c->rootbox, &c->bvh_lo,
                   &c->bvh_work, &c->bvh_leaf, &c->counts, &c->offsets, &c->scan_tmp, &c->pair_a,
                   &c->pair_b, &c->i64_tmp, &c->pair_measure, &c->pair_nout, &c->partials,
                   &c->ovf_list, &c->p1_list, &c->misc, &c->elem_measure, &c->totals, &c->x_a, &c->x_b, &c->x_measure,
                   &c->x_nout, &c->x_elems, &c->x_setup, &c->x_tol, &c->x_iota, &c->x_faces, &c->x_screen,
                   &c->x_list, &c->elem_off, &c->x_pa, &c->x_pb, &c->u_a, &c->v_b, &c->blocks, &c->bt_tabs, &c->bt_pair_a,
                   &c->bt_pair_b, &c->bt_mort, &c->bt_codes, &c->bt_roots, &c->bt_stops, &c->bt_tot,
                   &c->bt_ncand, &c->bt_stage_pa[0], &c->bt_stage_ea[0], &c->bt_stage_pb[0],
                   &c->bt_stage_eb[0], &c->bt_stage_pa[1], &c->bt_stage_ea[1], &c->bt_stage_pb[1],
                   &c->bt_stage_eb[1],
                   &c->d1_keyhi, &c->d1_perm_a, &c->d1_perm_b, &c->d1_lo_a, &c->d1_hi_a, &c->d1_lo_b,
                   &c->d1_hi_b, &c->d1_tree, &c->d1_e, &c->d1_l, &c->d1_js, &c->q_cache, &c->q_over, &c->q_pool, &c->q_next, &c->q_first,
                   &c->a_faces, &c->b_screen, &c->surv, &c->sched_w, &c->sched_list, &c->sched_cls,
                   &c->sched_adam, &c->bt_indptr, &c->seg_cnt, &c->seg_tab, &c->surv_list,
                   &c->p1_seg_cnt, &c->p1_seg_tab, &c->x_seg_cnt, &c->x_seg_tab, &c->x_sub};
  for (DevBuf* b : all) free_buf(*b);
  for (cudaEvent_t& e : c->clip_ev)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  for (cudaEvent_t& e : c->side_ev)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  for (cudaEvent_t& e : c->chunk_ev)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  if (c->copy) {
    cudaStreamSynchronize(c->copy);
    cudaStreamDestroy(c->copy);
    c->copy = nullptr;
  }
  if (c->side) {
    cudaStreamSynchronize(c->side);
    cudaStreamDestroy(c->side);
    c->side = nullptr;
  }
  if (c->bg.exec) cudaGraphExecDestroy(c->bg.exec);
  c->bg.exec = nullptr;
  if (c->bg.host) cudaFreeHost(c->bg.host);
  c->bg.host = nullptr;
  if (c->host_scalars) cudaFreeHost(c->host_scalars);
  if (c->pair_io) cudaFreeHost(c->pair_io);
  c->pair_io = nullptr;
  if (c->host_stage) cudaFreeHost(c->host_stage);
  if (c->stream) cudaStreamDestroy(c->stream);
  c->host_stage = nullptr;
  c->host_stage_cap = 0;
  c->host_scalars = nullptr;
  c->stream = nullptr;
}

cudaStream_t pick(Ctx* c, void* s) { return s ? static_cast<cudaStream_t>(s) : c->stream; }

// ------------------------------------------------------------- mesh upload
struct MeshDev {
  int dim, loc, idx_bytes;
  int64_t nnodes, nel;
  const double* pos;
  const void* en;
};

// intervals = true: 2-node elements whose nodes' first coordinates are read
// (the sort finder's input), any dimension.
void check_mesh(Ctx* c, const lsm_gpu_mesh* m, const char* name, bool simplex, bool intervals = false) {
  REQUIRE(m != nullptr, "mesh %s is NULL", name);
  if (intervals)
    REQUIRE(m->dim >= 1 && m->loc == 2, "mesh %s: the sort finder takes 2-node elements (loc %d)", name, m->loc);
  else
    REQUIRE(m->dim >= 1 && m->dim <= 3, "Invalid dimension %d for mesh %s", m->dim, name);
  if (intervals) {
  } else if (simplex)
    REQUIRE(m->loc == m->dim + 1, "mesh %s: loc %d is not a simplex of dimension %d", name, m->loc, m->dim);
  else
    REQUIRE(m->loc == m->dim + 1 || m->loc == (1 << m->dim), "mesh %s: unsupported loc %d", name, m->loc);
  REQUIRE(m->index_bytes == 4 || m->index_bytes == 8, "mesh %s: index_bytes must be 4 or 8", name);
  REQUIRE(m->nnodes >= 0 && m->nelements >= 0, "mesh %s: negative size", name);
  REQUIRE(m->nelements < (int64_t)0x7fffffff, "mesh %s: more than 2^31-1 elements", name);
  REQUIRE(m->nelements == 0 || (m->positions && m->enlist), "mesh %s: NULL arrays", name);
  REQUIRE(m->nelements == 0 || m->nnodes > 0, "mesh %s: No nodes", name);
}

MeshDev upload(Ctx* c, const lsm_gpu_mesh* m, int on_device, DevBuf& pos, DevBuf& en, cudaStream_t s) {
  MeshDev d{m->dim, m->loc, m->index_bytes, m->nnodes, m->nelements, m->positions, m->enlist};
  if (!on_device && m->nelements > 0) {
    double* p = ensure<double>(c, pos, m->nnodes * m->dim);
    CU(cudaMemcpyAsync(p, m->positions, sizeof(double) * m->nnodes * m->dim, cudaMemcpyHostToDevice, s));
    char* e = ensure<char>(c, en, m->nelements * m->loc * m->index_bytes);
    CU(cudaMemcpyAsync(e, m->enlist, (size_t)m->nelements * m->loc * m->index_bytes, cudaMemcpyHostToDevice, s));
    d.pos = p;
    d.en = e;
  }
  return d;
}

int* bad_flag(Ctx* c) { return ensure<int>(c, c->misc, 64); }

// The narrow phase's work lists carry candidate indices as 32-bit ints
// (survivor records, overflow lists): more candidates than that are refused
// (the search alone, with its 64-bit offsets, has no such limit).
void require_pair_index(Ctx* c, int64_t n) {
  if (n > INT32_MAX) {
    set_error(c, "%lld candidate pairs: the narrow phase takes at most 2^31-1 per call (split the meshes)",
              (long long)n);
    throw Fail{LSM_ERROR_CAPACITY};
  }
}

// Explicit tet pair batches of at least this many pairs run through the
// early-out pass and the index clipper (work counters: misc ints 24-29).
constexpr int64_t kPairsPipelineMin = 2048;
unsigned long long* pairs_work(Ctx* c) { return reinterpret_cast<unsigned long long*>(bad_flag(c) + 24); }

// Survivor segments of a 3D early-out pass over n pairs (lengths and chunk
// table) in the given buffers.
lsm::SegList seg_list(Ctx* c, DevBuf& cnt, DevBuf& tab, int64_t n) {
  return lsm::SegList{ensure<int>(c, cnt, lsm::seg_blocks(n)), ensure<int4>(c, tab, lsm::seg_table_entries(n))};
}

// P1 mass pass (3D): its survivor list, segments and three counters (misc
// ints 16-21)
int32_t* p1_survivors(Ctx* c, int dim, int64_t nnz) {
  return dim == 3 ? ensure<int32_t>(c, c->p1_list, 4 * std::max<int64_t>(nnz, 1)) : nullptr;
}
unsigned long long* p1_work(Ctx* c) { return reinterpret_cast<unsigned long long*>(bad_flag(c) + 16); }
lsm::SegList p1_seg(Ctx* c, int dim, int64_t nnz) {
  return dim == 3 ? seg_list(c, c->p1_seg_cnt, c->p1_seg_tab, nnz) : lsm::SegList{};
}

// Device memory the candidate-row cache of the search may hold: min(4 GiB,
// 1/32 of the device).  Only rows' actual candidates are written (4 B each);
// the cap only bounds the row length that avoids a second traversal.
int64_t cache_budget(Ctx* c) { return std::min<int64_t>(4ll << 30, c->device_mem / 32); }

// Spill pool for rows longer than the cache: what the budget leaves after
// the dense part, at most 4 chunks (256 candidates) per row on average.  Its
// chunk counter is bad_flag(c)[4], zeroed with the flags.  row_chunk needs no
// clearing: the count pass writes it for every row longer than the cache,
// and only those rows read it.
lsm::Spill make_spill(Ctx* c, int64_t nel, int cap) {
  lsm::Spill sp;
  const int64_t chunk_bytes = sizeof(int32_t) * lsm::kSpillChunk + sizeof(int);
  int64_t chunks = (cache_budget(c) - (int64_t)sizeof(int32_t) * nel * cap) / chunk_bytes;
  chunks = std::min<int64_t>(std::min<int64_t>(chunks, 4 * nel), INT32_MAX);
  if (g_spill_chunks >= 0) chunks = std::min<int64_t>(chunks, g_spill_chunks);
  if (nel <= 0 || chunks < 1) return sp;
  sp.pool = ensure<int32_t>(c, c->q_pool, chunks * lsm::kSpillChunk);
  sp.chunk_next = ensure<int>(c, c->q_next, chunks);
  sp.row_chunk = ensure<int>(c, c->q_first, nel);
  sp.next = bad_flag(c) + 4;
  sp.chunks = (int)chunks;
  return sp;
}

// prep of the query mesh A: coords (simplices only), box64, tol; tets also
// get their face planes for the clipper's separation screen
// Prep of elements [e0, e0 + n) of A or B (every per-element output at its
// element's offset); the buffers are sized for the whole mesh first.
void prep_a_range(Ctx* c, const MeshDev& a, bool simplex, int64_t e0, int64_t n, cudaStream_t s) {
  double* coords = simplex ? ensure<double>(c, c->a_coords, a.nel * a.loc * a.dim) : nullptr;
  double* box = ensure<double>(c, c->a_box64, a.nel * 2 * a.dim);
  double* tol = simplex ? ensure<double>(c, c->a_tol, a.nel) : nullptr;
  double* faces = simplex && a.dim == 3 ? ensure<double>(c, c->a_faces, a.nel * lsm::kScreen3) : nullptr;
  if (n <= 0) return;
  const char* en = static_cast<const char*>(a.en) + e0 * a.loc * a.idx_bytes;
  CU(lsm::launch_prep(a.dim, a.loc, n, a.pos, en, a.idx_bytes, coords ? coords + e0 * a.loc * a.dim : nullptr,
                      box + e0 * 2 * a.dim, nullptr, tol ? tol + e0 : nullptr, nullptr, bad_flag(c), a.nnodes, s,
                      faces ? faces + e0 * lsm::kScreen3 : nullptr));
}

void prep_b_range(Ctx* c, const MeshDev& b, bool simplex, bool want_coords, int64_t e0, int64_t n, cudaStream_t s) {
  double* coords = want_coords ? ensure<double>(c, c->b_coords, b.nel * b.loc * b.dim) : nullptr;
  double* box = ensure<double>(c, c->b_box64, b.nel * 2 * b.dim);
  float* box32 = ensure<float>(c, c->b_box32, b.nel * 8);
  const int srow = b.dim == 2 ? lsm::kSetup2 : lsm::kSetup3;
  double* setup = simplex ? ensure<double>(c, c->b_setup, b.nel * srow) : nullptr;
  double* screen = simplex && b.dim == 3 ? ensure<double>(c, c->b_screen, b.nel * lsm::kScreen3) : nullptr;
  if (n <= 0) return;
  const char* en = static_cast<const char*>(b.en) + e0 * b.loc * b.idx_bytes;
  CU(lsm::launch_prep(b.dim, b.loc, n, b.pos, en, b.idx_bytes, coords ? coords + e0 * b.loc * b.dim : nullptr,
                      box + e0 * 2 * b.dim, box32 + e0 * 8, nullptr, setup ? setup + e0 * srow : nullptr,
                      bad_flag(c), b.nnodes, s, nullptr, screen ? screen + e0 * lsm::kScreen3 : nullptr));
}

// Large host meshes: the element list is copied in kPrepChunks pieces on the
// context's copy stream (after the node positions), and the prep of each
// piece, on the mesh's own stream, waits only for that piece's copy, so the
// copies and the prep overlap.  ev[k] marks piece k's copy.
constexpr int64_t kPrepChunkMin = 1 << 18;
constexpr int kPrepChunks = 4;

MeshDev upload_chunks(Ctx* c, const lsm_gpu_mesh* m, DevBuf& pos, DevBuf& en, int chunks, cudaEvent_t* ev) {
  MeshDev d{m->dim, m->loc, m->index_bytes, m->nnodes, m->nelements, m->positions, m->enlist};
  double* p = ensure<double>(c, pos, m->nnodes * m->dim);
  char* e = ensure<char>(c, en, m->nelements * m->loc * m->index_bytes);
  d.pos = p;
  d.en = e;
  if (m->nelements > 0)
    CU(cudaMemcpyAsync(p, m->positions, sizeof(double) * m->nnodes * m->dim, cudaMemcpyHostToDevice, c->copy));
  const size_t row = (size_t)m->loc * m->index_bytes;
  for (int k = 0; k < chunks; ++k) {
    const int64_t e0 = m->nelements * k / chunks, e1 = m->nelements * (k + 1) / chunks;
    if (e1 > e0)
      CU(cudaMemcpyAsync(e + e0 * row, static_cast<const char*>(m->enlist) + e0 * row, (size_t)(e1 - e0) * row,
                         cudaMemcpyHostToDevice, c->copy));
    CU(cudaEventRecord(ev[k], c->copy));
  }
  return d;
}

template <class Prep>
void prep_chunks(Ctx* c, const MeshDev& d, int chunks, const cudaEvent_t* ev, cudaStream_t s, Prep prep) {
  for (int k = 0; k < chunks; ++k) {
    const int64_t e0 = d.nel * k / chunks, e1 = d.nel * (k + 1) / chunks;
    CU(cudaStreamWaitEvent(s, ev[k], 0));
    prep(e0, e1 - e0);
  }
}

lsm::BVH build_tree(Ctx* c, const MeshDev& b, cudaStream_t s) {
  const int64_t n = b.nel;
  lsm::BVH bvh;
  bvh.n = (int)n;
  if (n == 0) return bvh;
  const int dim = b.dim;
  uint32_t* keys = ensure<uint32_t>(c, c->keys, n);
  int32_t* vals = ensure<int32_t>(c, c->vals, n);
  uint32_t* kt = ensure<uint32_t>(c, c->keys_tmp, n);
  int32_t* vt = ensure<int32_t>(c, c->vals_tmp, n);
  uint32_t* hist = ensure<uint32_t>(c, c->hist, lsm::radix_hist_entries(n));
  const int pcap = 4096;
  double* part = ensure<double>(c, c->root_partial, (int64_t)pcap * 2 * dim);
  double* root = ensure<double>(c, c->rootbox, 2 * dim);
  CU(lsm::launch_root_box(dim, n, static_cast<double*>(c->b_box64.p), part, pcap, root, s));
  CU(lsm::launch_morton(dim, n, static_cast<double*>(c->b_box64.p), root, keys, vals, s));
  CU(lsm::radix_sort_pairs(n, dim == 2 ? 32 : 30, keys, vals, kt, vt, hist, s, bad_flag(c) + 3));
  bvh.lo_left = ensure<float4>(c, c->bvh_lo, 2 * (2 * n - 1));
  bvh.hi_esc = bvh.lo_left + 1;
  bvh.leaf = ensure<double>(c, c->bvh_leaf, 8 * n);
  int* work = ensure<int>(c, c->bvh_work, 8 * n);
  bvh.bucket = lsm::tree_bucket((int)n, true);
  CU(lsm::launch_bvh_build(dim, (int)n, keys, vals, static_cast<float*>(c->b_box32.p), bvh, work, s,
                           static_cast<double*>(c->b_box64.p)));
  return bvh;
}

// Gather, sort by left end (stable) and take sorted left/right ends of one
// interval mesh; coords[2*nel] keeps the element's two node coordinates.
void sort_intervals(Ctx* c, const MeshDev& m, DevBuf& coords_buf, DevBuf& perm_buf, DevBuf& lo_buf, DevBuf& hi_buf,
                    cudaStream_t s) {
  const int64_t n = m.nel;
  double* coords = ensure<double>(c, coords_buf, 2 * n);
  uint32_t* klo = ensure<uint32_t>(c, c->keys, n);
  uint32_t* khi = ensure<uint32_t>(c, c->d1_keyhi, n);
  int32_t* perm = ensure<int32_t>(c, perm_buf, n);
  uint32_t* kt = ensure<uint32_t>(c, c->keys_tmp, n);
  int32_t* vt = ensure<int32_t>(c, c->vals_tmp, n);
  uint32_t* hist = ensure<uint32_t>(c, c->hist, lsm::radix_hist_entries(n));
  CU(lsm::launch_prep_1d(n, m.pos, m.dim, m.en, m.idx_bytes, m.nnodes, coords, klo, khi, perm, bad_flag(c), s));
  CU(lsm::sort_by_key64(n, klo, khi, perm, kt, vt, hist, s));
  CU(lsm::launch_sorted_ends_1d(n, perm, coords, ensure<double>(c, lo_buf, n), ensure<double>(c, hi_buf, n), s));
}

// 1D sort finder (Intersection_Finder.F90:811-921) on the GPU; the first
// coordinate of each node is used, positions have stride dim.
void find_candidates_1d(Ctx* c, const MeshDev& a, const MeshDev& b, cudaStream_t s) {
  const int64_t na = a.nel, nb = b.nel;
  CU(cudaMemsetAsync(bad_flag(c), 0, sizeof(int) * 64, s));
  sort_intervals(c, a, c->a_coords, c->d1_perm_a, c->d1_lo_a, c->d1_hi_a, s);
  sort_intervals(c, b, c->b_coords, c->d1_perm_b, c->d1_lo_b, c->d1_hi_b, s);
  const double* lo_a = static_cast<double*>(c->d1_lo_a.p);
  const double* hi_a = static_cast<double*>(c->d1_hi_a.p);
  const double* lo_b = static_cast<double*>(c->d1_lo_b.p);
  const double* hi_b = static_cast<double*>(c->d1_hi_b.p);
  double* tree = nb > 0 ? ensure<double>(c, c->d1_tree, 2 * lsm::tree_leaves_1d(nb)) : nullptr;
  CU(lsm::launch_max_tree(nb, hi_b, tree, s));
  int32_t* E = ensure<int32_t>(c, c->d1_e, na);
  int32_t* L = ensure<int32_t>(c, c->d1_l, na);
  int32_t* JS = ensure<int32_t>(c, c->d1_js, na);
  CU(lsm::launch_rows_1d(na, lo_a, hi_a, nb, lo_b, tree, E, L, s));
  CU(lsm::launch_sweep_1d(na, nb, E, L, lo_a, hi_a, hi_b, JS, s));
  int64_t* offsets = ensure<int64_t>(c, c->offsets, na + 1);
  int* counts = ensure<int>(c, c->counts, na);
  int64_t* stmp = ensure<int64_t>(c, c->scan_tmp, lsm::scan_tmp_entries(na) + 1);
  const int32_t* perm_a = static_cast<int32_t*>(c->d1_perm_a.p);
  const int32_t* perm_b = static_cast<int32_t*>(c->d1_perm_b.p);
  CU(lsm::launch_emit_1d(false, na, JS, E, lo_a, hi_b, perm_a, perm_b, counts, nullptr, nullptr, nullptr, s));
  CU(lsm::launch_scan(na, counts, offsets, stmp, s));
  int64_t* h = static_cast<int64_t*>(c->host_scalars) + 8;
  CU(cudaMemcpyAsync(h, offsets + na, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  int* hb = static_cast<int*>(c->host_scalars);
  CU(cudaMemcpyAsync(hb, c->misc.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  REQUIRE(hb[0] == 0, "Invalid node index in an element list");
  const int64_t nnz = *h;
  int32_t* pa = ensure<int32_t>(c, c->pair_a, nnz);
  int32_t* pb = ensure<int32_t>(c, c->pair_b, nnz);
  if (nnz > 0) CU(lsm::launch_emit_1d(true, na, JS, E, lo_a, hi_b, perm_a, perm_b, nullptr, offsets, pa, pb, s));
  c->dim = 1;
  c->loc_a = 2;
  c->loc_b = 2;
  c->nel_a = na;
  c->nel_b = nb;
  c->ncand = nnz;
  c->simplex_prep = true;  // coords of both meshes are current
}

// Broad phase: candidates as CSR (offsets) + pair arrays.  1D meshes (and
// intervals = true, the sort finder's entry) take the sort-and-sweep
// search, 2D/3D the LBVH search.
void find_candidates(Ctx* c, const lsm_gpu_mesh* ma, const lsm_gpu_mesh* mb, int on_device, bool simplex,
                     bool want_b_coords, cudaStream_t s, bool intervals = false) {
  intervals = intervals || (ma && ma->dim == 1);
  c->surv_valid = false;
  check_mesh(c, ma, "A", simplex, intervals);
  check_mesh(c, mb, "B", simplex, intervals);
  c->have_pairs = false;
  c->ncand = -1;
  c->simplex_prep = false;
  if (intervals) {
    MeshDev a = upload(c, ma, on_device, c->a_pos, c->a_en, s);
    MeshDev b = upload(c, mb, on_device, c->b_pos, c->b_en, s);
    find_candidates_1d(c, a, b, s);
    return;
  }
  REQUIRE(ma->dim == mb->dim, "Invalid dimension: A is %dD, B is %dD", ma->dim, mb->dim);
  c->have_pairs = false;
  c->ncand = -1;
  c->simplex_prep = false;
  simplex = simplex || (ma->loc == ma->dim + 1 && mb->loc == mb->dim + 1);
  // A's upload and prep run on the side stream, overlapping B's prep and
  // tree build on s; s waits for them before the search.  A's copies start
  // once B's are done, so B's (on the critical path) get the whole link;
  // large host meshes come in chunks whose prep overlaps the next copy.
  SyncOnThrow sync_on_throw{s, c->side};
  CU(cudaMemsetAsync(bad_flag(c), 0, sizeof(int) * 64, s));
  MeshDev a, b;
  if (!on_device && std::max(ma->nelements, mb->nelements) >= kPrepChunkMin) {
    // chunked copies on the copy stream (B's first: B is on the critical
    // path), once earlier work that may still read these buffers is done
    sync_on_throw.s2 = c->copy;
    cudaEvent_t* ev = c->chunk_ev;
    CU(cudaEventRecord(ev[8], s));
    CU(cudaEventRecord(ev[9], c->side));
    CU(cudaStreamWaitEvent(c->copy, ev[8], 0));
    CU(cudaStreamWaitEvent(c->copy, ev[9], 0));
    const int kb = mb->nelements >= kPrepChunkMin ? kPrepChunks : 1;
    const int ka = ma->nelements >= kPrepChunkMin ? kPrepChunks : 1;
    b = upload_chunks(c, mb, c->b_pos, c->b_en, kb, ev);
    a = upload_chunks(c, ma, c->a_pos, c->a_en, ka, ev + 4);
    prep_chunks(c, b, kb, ev, s,
                [&](int64_t e0, int64_t n) { prep_b_range(c, b, simplex, want_b_coords, e0, n, s); });
    prep_chunks(c, a, ka, ev + 4, c->side,
                [&](int64_t e0, int64_t n) { prep_a_range(c, a, simplex, e0, n, c->side); });
  } else {
    b = upload(c, mb, on_device, c->b_pos, c->b_en, s);
    CU(cudaEventRecord(c->side_ev[0], s));
    CU(cudaStreamWaitEvent(c->side, c->side_ev[0], 0));
    a = upload(c, ma, on_device, c->a_pos, c->a_en, c->side);
    prep_a_range(c, a, simplex, 0, a.nel, c->side);
    prep_b_range(c, b, simplex, want_b_coords, 0, b.nel, s);
  }
  CU(cudaEventRecord(c->side_ev[1], c->side));
  const int64_t nel_a = a.nel;
  int64_t* offsets = ensure<int64_t>(c, c->offsets, nel_a + 1);
  int* counts = ensure<int>(c, c->counts, nel_a);
  int64_t* stmp = ensure<int64_t>(c, c->scan_tmp, lsm::scan_tmp_entries(nel_a) + 1);
  lsm::BVH bvh{};
  // candidate cache of the count pass: at most 256 per row
  const int cap = nel_a > 0 ? (int)std::min<int64_t>(256, cache_budget(c) / (4 * nel_a)) : 0;
  int32_t* cache = cap >= 8 ? ensure<int32_t>(c, c->q_cache, nel_a * cap) : nullptr;
  int* over = cache ? ensure<int>(c, c->q_over, nel_a + 1) : nullptr;
  // (the single-mesh search keeps the tighter walk of a cache without spill
  // chunks: its long rows are traversed again)
  const lsm::Spill spill{};
  if (b.nel > 0 && nel_a > 0) {
    bvh = build_tree(c, b, s);
    if (over) CU(cudaMemsetAsync(over, 0, sizeof(int), s));
    CU(cudaStreamWaitEvent(s, c->side_ev[1], 0));
    CU(lsm::launch_query(a.dim, false, nel_a, static_cast<double*>(c->a_box64.p), bvh,
                         static_cast<double*>(c->b_box64.p), counts, nullptr, nullptr, nullptr, s, cache, cap,
                         over, spill));
  } else {
    CU(cudaStreamWaitEvent(s, c->side_ev[1], 0));
    if (nel_a > 0) CU(cudaMemsetAsync(counts, 0, sizeof(int) * nel_a, s));
  }
  CU(lsm::launch_scan(nel_a, counts, offsets, stmp, s));
  int64_t* h = static_cast<int64_t*>(c->host_scalars) + 8;
  CU(cudaMemcpyAsync(h, offsets + nel_a, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  int* hb = static_cast<int*>(c->host_scalars);
  CU(cudaMemcpyAsync(hb, c->misc.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  REQUIRE(hb[0] == 0, "Invalid node index in an element list");
  if (hb[3] != 0) {
    set_error(c, "tree build: the sort's look-back wait gave up");
    throw Fail{LSM_ERROR_TIMEOUT};
  }
  const int64_t nnz = *h;
  int32_t* pa = ensure<int32_t>(c, c->pair_a, nnz);
  int32_t* pb = ensure<int32_t>(c, c->pair_b, nnz);
  if (nnz > 0)
    CU(lsm::launch_query(a.dim, true, nel_a, static_cast<double*>(c->a_box64.p), bvh,
                         static_cast<double*>(c->b_box64.p), counts, offsets, pa, pb, s, cache, cap, over,
                         spill));
  c->dim = a.dim;
  c->loc_a = a.loc;
  c->loc_b = b.loc;
  c->nel_a = a.nel;
  c->nel_b = b.nel;
  c->ncand = nnz;
  c->simplex_prep = simplex;
}

// Narrow phase over the current candidates.  Leaves the merged totals in
// c->totals (one lsm::Partial).
// n_dev (optional): the candidate count on the device; c->ncand is then only
// its upper bound, the capacity of the pair arrays.
// list_inside (3D): the survivor list also holds the pairs whose every plane
// is a no-op, for a second pass over the list (the supermesh's elements);
// no schedule then.
void narrow(Ctx* c, cudaStream_t s, const int32_t* order = nullptr, const int64_t* n_dev = nullptr,
            bool list_inside = false) {
  const int64_t nnz = c->ncand;
  require_pair_index(c, nnz);
  double* pm = ensure<double>(c, c->pair_measure, nnz);
  int32_t* pn = ensure<int32_t>(c, c->pair_nout, nnz);
  const int nred = lsm::reduce_pairs_blocks();
  lsm::Partial* part = ensure<lsm::Partial>(c, c->partials, nred);
  lsm::Partial* tot = ensure<lsm::Partial>(c, c->totals, 1);
  // 2D: overflow list of the fast-path clipper; 3D: list of pairs that
  // survive the exact early-out.
  // (the default 3D clipper takes {pair, a, b, 0} records: 4 ints per pair)
  int32_t* ovf = ensure<int32_t>(c, c->ovf_list, c->dim == 3 ? 4 * nnz : nnz);
  int* ovf_count = bad_flag(c) + 2;
  if (c->dim == 2) CU(cudaMemsetAsync(ovf_count, 0, sizeof(int), s));
  unsigned long long* work = reinterpret_cast<unsigned long long*>(bad_flag(c) + 8);
  if (c->dim == 1) {
    CU(lsm::launch_clip_intervals(nnz, static_cast<int32_t*>(c->pair_a.p), static_cast<int32_t*>(c->pair_b.p),
                                  static_cast<double*>(c->a_coords.p), static_cast<double*>(c->b_coords.p), pm, pn,
                                  s));
    CU(lsm::launch_reduce_pairs(nnz, pm, pn, part, s));
    CU(lsm::launch_finalize(part, nred, tot, s));
    c->have_pairs = true;
    return;
  }
  const bool screen = c->dim == 3 && g_tet_screen;
  lsm::SchedBin bin;
  const bool binned = c->dim == 3 && g_tet_schedule != 0 && !list_inside;
  if (binned) {
    if (g_tet_schedule == 1 && !c->have_sched) {
      set_error(c, "tet_schedule 1 needs scheduler weights (libsupermesh_gpu_sched_set_weights)");
      throw Fail{LSM_ERROR_STATE};
    }
    if (g_tet_schedule == 2) {
      if (!c->have_pairs) {
        set_error(c, "tet_schedule 2 needs a narrow phase over the same candidates first");
        throw Fail{LSM_ERROR_STATE};
      }
      int8_t* cls = ensure<int8_t>(c, c->sched_cls, nnz);
      CU(lsm::launch_sched_true_class(nnz, pn, cls, s));
      bin.cls_of_pair = cls;
    } else {
      bin.weights = static_cast<const lsm::SchedWeights*>(c->sched_w.p);
    }
    bin.screen_b = static_cast<double*>(c->b_screen.p);
    bin.out = ensure<int4>(c, c->sched_list, nnz);
    bin.flat = ensure<int4>(c, c->surv_list, std::max<int64_t>(nnz, 1));
    bin.window = g_sched_window;
  }
  if (c->dim == 3 && list_inside) {
    const lsm::SegList sg = seg_list(c, c->seg_cnt, c->seg_tab, nnz);
    CU(lsm::launch_clip_elems(nnz, static_cast<int32_t*>(c->pair_a.p), static_cast<int32_t*>(c->pair_b.p),
                              static_cast<double*>(c->a_coords.p), static_cast<double*>(c->a_tol.p),
                              static_cast<double*>(c->b_setup.p), pm, pn, nullptr, ovf, work,
                              screen ? static_cast<double*>(c->a_faces.p) : nullptr,
                              screen ? static_cast<double*>(c->b_screen.p) : nullptr, s, &sg));
    c->clip_timed = false;
    c->surv_seg = false;
  } else {
    // 3D: survivors as per-block segments, taken by chunks (the binned
    // orders gather them into one list first)
    const bool seg = c->dim == 3;
    const lsm::SegList sg = seg ? seg_list(c, c->seg_cnt, c->seg_tab, nnz) : lsm::SegList{};
    CU(lsm::launch_clip(c->dim, nnz, static_cast<int32_t*>(c->pair_a.p), static_cast<int32_t*>(c->pair_b.p),
                        static_cast<double*>(c->a_coords.p), static_cast<double*>(c->a_tol.p),
                        static_cast<double*>(c->b_setup.p), pm, pn, ovf, ovf_count, work, s, order,
                        g_time_kernels ? c->clip_ev[0] : nullptr, g_time_kernels ? c->clip_ev[1] : nullptr,
                        screen ? static_cast<double*>(c->a_faces.p) : nullptr,
                        screen ? static_cast<double*>(c->b_screen.p) : nullptr, binned ? &bin : nullptr, n_dev,
                        &sg));
    c->clip_timed = g_time_kernels;
    c->surv_seg = seg;
    c->surv_npairs = nnz;
  }
  if (c->dim == 3) {
    CU(cudaMemcpyAsync(ensure<unsigned long long>(c, c->surv, 1), work, sizeof(unsigned long long),
                       cudaMemcpyDeviceToDevice, s));
    c->surv_valid = true;
  }
  if (c->dim == 2)
    CU(lsm::launch_clip_tris_wide(ovf, ovf_count, nnz, static_cast<int32_t*>(c->pair_a.p),
                                  static_cast<int32_t*>(c->pair_b.p), static_cast<double*>(c->a_coords.p),
                                  static_cast<double*>(c->a_tol.p), static_cast<double*>(c->b_setup.p), pm,
                                  pn, s));
  CU(lsm::launch_reduce_pairs(nnz, pm, pn, part, s, n_dev));
  CU(lsm::launch_finalize(part, nred, tot, s));
  c->have_pairs = true;
}

void read_stats(Ctx* c, lsm_gpu_stats* st, cudaStream_t s) {
  lsm::Partial* h = reinterpret_cast<lsm::Partial*>(static_cast<char*>(c->host_scalars) + 256);
  CU(cudaMemcpyAsync(h, c->totals.p, sizeof(lsm::Partial), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (st) {
    st->n_candidates = c->ncand;
    st->total_measure = h->sum;
    st->total_measure_err = h->err;
    st->n_intersecting = (int64_t)h->n_int;
    st->n_out_simplices = (int64_t)h->n_out;
  }
}

template <class F>
int guarded(Ctx* c, F&& f) {
  if (!c) return LSM_ERROR_INVALID_ARGUMENT;
  try {
    DeviceGuard g(c->device);
    f();
    return LSM_SUCCESS;
  } catch (const Fail& e) {
    return e.status;
  } catch (const std::bad_alloc&) {
    set_error(c, "host allocation failed");
    return LSM_ERROR_OUT_OF_MEMORY;
  }
}

// ------------------------------------------------------------ batched path
void* host_stage(Ctx* c, size_t bytes) {
  if (c->host_stage_cap < bytes) {
    if (c->host_stage) cudaFreeHost(c->host_stage);
    c->host_stage = nullptr;
    c->host_stage_cap = 0;
    const size_t want = bytes + bytes / 2 + 4096;
    if (cudaMallocHost(&c->host_stage, want) != cudaSuccess) {
      (void)cudaGetLastError();
      set_error(c, "pinned host allocation of %zu bytes failed", want);
      throw Fail{LSM_ERROR_OUT_OF_MEMORY};
    }
    c->host_stage_cap = want;
  }
  return c->host_stage;
}

// Copies the host meshes of one batch group into the context's staging
// buffers for that dimension (one copy per array and mesh, issued on st).
// ptr receives their device addresses as four tables of idx.size() entries:
// A's positions, A's element lists, B's positions, B's element lists.
void stage_batch_group(Ctx* c, int dim, const std::vector<int>& idx, const lsm_gpu_mesh* ma,
                       const lsm_gpu_mesh* mb, cudaStream_t st, std::vector<uint64_t>& ptr) {
  const int nm = (int)idx.size();
  const int ib = ma[idx[0]].index_bytes;
  const int loc = dim + 1;
  const int g = dim - 2;
  int64_t na = 0, nb = 0, va = 0, vb = 0;
  for (int i : idx) {
    na += ma[i].nelements;
    nb += mb[i].nelements;
    va += ma[i].nnodes;
    vb += mb[i].nnodes;
  }
  REQUIRE(na < (int64_t)0x7fffffff && nb < (int64_t)0x7fffffff, "batch has more than 2^31-1 elements");
  double* spa = ensure<double>(c, c->bt_stage_pa[g], va * dim);
  double* spb = ensure<double>(c, c->bt_stage_pb[g], vb * dim);
  char* sea = ensure<char>(c, c->bt_stage_ea[g], na * loc * ib);
  char* seb = ensure<char>(c, c->bt_stage_eb[g], nb * loc * ib);
  ptr.assign(4 * (size_t)nm, 0);
  int64_t oa = 0, ob = 0, ea = 0, eb = 0;
  for (int i = 0; i < nm; ++i) {
    const lsm_gpu_mesh& A = ma[idx[i]];
    const lsm_gpu_mesh& B = mb[idx[i]];
    ptr[i] = (uint64_t)(spa + oa * dim);
    ptr[nm + i] = (uint64_t)(sea + ea * loc * ib);
    ptr[2 * nm + i] = (uint64_t)(spb + ob * dim);
    ptr[3 * nm + i] = (uint64_t)(seb + eb * loc * ib);
    if (A.nnodes) CU(cudaMemcpyAsync(spa + oa * dim, A.positions, sizeof(double) * A.nnodes * dim, cudaMemcpyHostToDevice, st));
    if (B.nnodes) CU(cudaMemcpyAsync(spb + ob * dim, B.positions, sizeof(double) * B.nnodes * dim, cudaMemcpyHostToDevice, st));
    if (A.nelements) CU(cudaMemcpyAsync(sea + ea * loc * ib, A.enlist, (size_t)A.nelements * loc * ib, cudaMemcpyHostToDevice, st));
    if (B.nelements) CU(cudaMemcpyAsync(seb + eb * loc * ib, B.enlist, (size_t)B.nelements * loc * ib, cudaMemcpyHostToDevice, st));
    oa += A.nnodes;
    ob += B.nnodes;
    ea += A.nelements;
    eb += B.nelements;
  }
}

// Per-pair outputs of a batched call (libsupermesh_gpu_supermesh_batched_ex):
// the caller's arrays, each pair's first CSR row in them (caller order), and
// the next free slot of the per-candidate arrays (groups are written one
// after the other).  ind_ptr of host calls goes through a device image of
// the whole array, copied out once at the end.
struct BatchOut {
  const lsm_gpu_batch_out* o = nullptr;
  std::vector<int64_t> rowbase;  // caller order
  int64_t total_rows = 0;
  int64_t next = 0;
  int64_t p1_next = 0;  // next free double of the P1 blocks
  bool overflow = false;
  int64_t* dev_indptr = nullptr;  // where the kernels write ind_ptr
};

// All mesh pairs of one dimension through each phase in one launch:
// batched prep (pointer tables), one sort by (mesh, Morton), one LBVH with a
// subtree per mesh, one traversal, the usual clipper over all candidates,
// and a per-mesh-pair reduction.  One host synchronisation (candidate count).
// staged: the device addresses from stage_batch_group (host meshes), or
// null when the meshes are on the device.
// Pinned area a launched group's results are copied to: totals[nm],
// counts[nm], the candidate count, the error words.
struct GroupRes {
  lsm::Partial* tot;
  int64_t* nc;
  int64_t* count;
  int* flags;
};
size_t group_res_bytes(int nm) { return (sizeof(lsm::Partial) + sizeof(int64_t)) * (size_t)nm + 64; }
GroupRes group_res(char* base, int nm) {
  GroupRes r;
  r.tot = reinterpret_cast<lsm::Partial*>(base);
  r.nc = reinterpret_cast<int64_t*>(base + sizeof(lsm::Partial) * nm);
  r.count = r.nc + nm;
  r.flags = reinterpret_cast<int*>(r.count + 1);
  return r;
}

// The host half of a group: errors, overflow, per-pair results.  Returns
// false if the candidates did not fit a capacity-mode launch (pair_cap).
bool finish_batch_group(Ctx* c, const std::vector<int>& idx, int loc, const GroupRes& r, int64_t pair_cap,
                        double* totals, int64_t* ncand, int64_t* nint, BatchOut* bo, int64_t group_base,
                        int64_t p1_base) {
  const int nm = (int)idx.size();
  REQUIRE(r.flags[0] == 0, "Invalid node index in an element list");
  if (r.flags[3] != 0) {
    set_error(c, "tree build: the sort's look-back wait gave up");
    throw Fail{LSM_ERROR_TIMEOUT};
  }
  if (pair_cap > 0 && *r.count > pair_cap) return false;
  c->ncand = *r.count;
  int64_t run = group_base;
  for (int i = 0; i < nm; ++i) {
    if (totals) totals[idx[i]] = r.tot[i].sum;
    if (ncand) ncand[idx[i]] = r.nc[i];
    if (nint) nint[idx[i]] = (int64_t)r.tot[i].n_int;
    if (bo && bo->o && bo->o->cand_offset) bo->o->cand_offset[idx[i]] = group_base >= 0 ? run : -1;
    if (bo && bo->o && bo->o->p1_offset)
      bo->o->p1_offset[idx[i]] = p1_base >= 0 ? p1_base + (run - group_base) * loc * loc : -1;
    if (group_base >= 0) run += r.nc[i];
  }
  return true;
}

// pair_cap > 0 (capacity mode): the pair arrays hold pair_cap candidates and
// no count is read back mid-call: the fill and the narrow phase read the
// count on the device and write nothing beyond the arrays; host_tab (pinned,
// group-owned) holds the tables and res_area receives the results, which
// finish_batch_group reads after the caller waits for the stream.  Nothing in
// that mode synchronises or allocates once the buffers have their sizes, so
// it can run under stream capture.  Returns false in capacity mode with the
// results pending; true when the group is finished (sync mode).
bool run_batch_group(Ctx* c, int dim, const std::vector<int>& idx, const lsm_gpu_mesh* ma,
                     const lsm_gpu_mesh* mb, const uint64_t* staged, double* totals, int64_t* ncand,
                     int64_t* nint, cudaStream_t s, BatchOut* bo = nullptr, int on_device = 0,
                     int64_t pair_cap = 0, void* host_tab = nullptr, char* res_area = nullptr) {
  REQUIRE(pair_cap == 0 || (!(bo && bo->o) && host_tab && res_area), "capacity mode without per-pair outputs");
  const int nm = (int)idx.size();
  const int ib = ma[idx[0]].index_bytes;
  const int loc = dim + 1;
  c->surv_valid = false;
  // host tables: elem_off_a[nm+1] elem_off_b[nm+1] nnodes_a[nm] nnodes_b[nm]
  //              pos_a[nm] en_a[nm] pos_b[nm] en_b[nm] rowbase[nm]
  const size_t tab_words = 2 * (nm + 1) + 7 * (size_t)nm;
  std::vector<int64_t> tab(tab_words);
  int64_t* eoa = tab.data();
  int64_t* eob = eoa + (nm + 1);
  int64_t* nna = eob + (nm + 1);
  int64_t* nnb = nna + nm;
  uint64_t* pta = reinterpret_cast<uint64_t*>(nnb + nm);
  uint64_t* eta = pta + nm;
  uint64_t* ptb = eta + nm;
  uint64_t* etb = ptb + nm;
  int64_t* rbase = reinterpret_cast<int64_t*>(etb + nm);
  for (int i = 0; i < nm; ++i) rbase[i] = bo && bo->o ? bo->rowbase[idx[i]] : 0;
  int64_t na = 0, nb = 0;
  for (int i = 0; i < nm; ++i) {
    const lsm_gpu_mesh& A = ma[idx[i]];
    const lsm_gpu_mesh& B = mb[idx[i]];
    eoa[i] = na;
    eob[i] = nb;
    nna[i] = A.nnodes;
    nnb[i] = B.nnodes;
    na += A.nelements;
    nb += B.nelements;
  }
  eoa[nm] = na;
  eob[nm] = nb;
  REQUIRE(na < (int64_t)0x7fffffff && nb < (int64_t)0x7fffffff, "batch has more than 2^31-1 elements");
  if (!staged) {
    for (int i = 0; i < nm; ++i) {
      pta[i] = (uint64_t)ma[idx[i]].positions;
      eta[i] = (uint64_t)ma[idx[i]].enlist;
      ptb[i] = (uint64_t)mb[idx[i]].positions;
      etb[i] = (uint64_t)mb[idx[i]].enlist;
    }
  } else {
    // pta, eta, ptb, etb are consecutive tables of nm entries, as in staged
    memcpy(pta, staged, sizeof(uint64_t) * 4 * (size_t)nm);
  }
  int64_t* dtab = ensure<int64_t>(c, c->bt_tabs, (int64_t)tab_words);
  void* htab = host_tab;
  if (!htab) {
    htab = host_stage(c, sizeof(int64_t) * tab_words);
    CU(cudaStreamSynchronize(s));  // the pinned stage may still feed a previous copy
  }
  memcpy(htab, tab.data(), sizeof(int64_t) * tab_words);
  CU(cudaMemcpyAsync(dtab, htab, sizeof(int64_t) * tab_words, cudaMemcpyHostToDevice, s));
  const int64_t* d_eoa = dtab;
  const int64_t* d_eob = d_eoa + (nm + 1);
  const int64_t* d_nna = d_eob + (nm + 1);
  const int64_t* d_nnb = d_nna + nm;
  const unsigned long long* d_pta = reinterpret_cast<const unsigned long long*>(d_nnb + nm);
  const unsigned long long* d_eta = d_pta + nm;
  const unsigned long long* d_ptb = d_eta + nm;
  const unsigned long long* d_etb = d_ptb + nm;
  const int64_t* d_rbase = reinterpret_cast<const int64_t*>(d_etb + nm);

  int* bad = bad_flag(c);
  CU(cudaMemsetAsync(bad, 0, sizeof(int) * 64, s));
  double* a_coords = ensure<double>(c, c->a_coords, na * loc * dim);
  double* a_box = ensure<double>(c, c->a_box64, na * 2 * dim);
  double* a_tol = ensure<double>(c, c->a_tol, na);
  int32_t* pair_of_a = ensure<int32_t>(c, c->bt_pair_a, na);
  double* b_box = ensure<double>(c, c->b_box64, nb * 2 * dim);
  float* b_box32 = ensure<float>(c, c->b_box32, nb * 8);
  double* b_setup = ensure<double>(c, c->b_setup, nb * (dim == 2 ? lsm::kSetup2 : lsm::kSetup3));
  int32_t* pair_of_b = ensure<int32_t>(c, c->bt_pair_b, nb);
  const bool want_p1 = bo && bo->o && bo->o->p1_blocks;
  double* b_coords = want_p1 ? ensure<double>(c, c->b_coords, nb * loc * dim) : nullptr;
  double* a_faces = dim == 3 ? ensure<double>(c, c->a_faces, na * lsm::kScreen3) : nullptr;
  double* b_screen = dim == 3 ? ensure<double>(c, c->b_screen, nb * lsm::kScreen3) : nullptr;
  CU(lsm::launch_prep_batched(dim, na, nm, d_eoa, d_pta, d_eta, d_nna, ib, a_coords, a_box, nullptr, a_tol,
                              nullptr, pair_of_a, bad, s, a_faces));
  CU(lsm::launch_prep_batched(dim, nb, nm, d_eob, d_ptb, d_etb, d_nnb, ib, b_coords, b_box, b_box32, nullptr,
                              b_setup, pair_of_b, bad, s, nullptr, b_screen));
  // tree over all B meshes
  lsm::BVH bvh;
  bvh.n = (int)nb;
  int* roots = ensure<int>(c, c->bt_roots, nm);
  int* stops = ensure<int>(c, c->bt_stops, nm);
  if (nb > 0) {
    uint32_t* keys = ensure<uint32_t>(c, c->keys, nb);
    int32_t* vals = ensure<int32_t>(c, c->vals, nb);
    uint32_t* kt = ensure<uint32_t>(c, c->keys_tmp, nb);
    int32_t* vt = ensure<int32_t>(c, c->vals_tmp, nb);
    uint32_t* hist = ensure<uint32_t>(c, c->hist, lsm::radix_hist_entries(nb));
    uint32_t* mort = ensure<uint32_t>(c, c->bt_mort, nb);
    const int pcap = 4096;
    double* part = ensure<double>(c, c->root_partial, (int64_t)pcap * 2 * dim);
    double* root = ensure<double>(c, c->rootbox, 2 * dim);
    CU(lsm::launch_root_box(dim, nb, b_box, part, pcap, root, s));
    CU(lsm::launch_morton(dim, nb, b_box, root, keys, vals, s));
    CU(cudaMemcpyAsync(mort, keys, sizeof(uint32_t) * nb, cudaMemcpyDeviceToDevice, s));
    CU(lsm::radix_sort_pairs(nb, dim == 2 ? 32 : 30, keys, vals, kt, vt, hist, s, bad + 3));
    int mbits = 1;
    while ((1 << mbits) < nm) ++mbits;
    CU(lsm::launch_pair_keys(nb, vals, pair_of_b, keys, s));
    CU(lsm::radix_sort_pairs(nb, mbits, keys, vals, kt, vt, hist, s, bad + 3));
    bvh.lo_left = ensure<float4>(c, c->bvh_lo, 2 * (2 * nb - 1));
    bvh.hi_esc = bvh.lo_left + 1;
    bvh.leaf = ensure<double>(c, c->bvh_leaf, 8 * nb);
    int* work = ensure<int>(c, c->bvh_work, 8 * nb);
    unsigned long long* codes = ensure<unsigned long long>(c, c->bt_codes, nb);
    CU(lsm::launch_batched_tree((int)nb, nm, vals, pair_of_b, mort, codes, b_box32, d_eob, bvh, work, roots,
                                stops, s, dim, b_box, bad + 3));
  } else {
    CU(cudaMemsetAsync(roots, 0xff, sizeof(int) * nm, s));
    CU(cudaMemsetAsync(stops, 0xff, sizeof(int) * nm, s));
  }
  int64_t* offsets = ensure<int64_t>(c, c->offsets, na + 1);
  int* counts = ensure<int>(c, c->counts, na);
  int64_t* stmp = ensure<int64_t>(c, c->scan_tmp, lsm::scan_tmp_entries(na) + 1);
  // candidate cache of the count pass, as in find_candidates
  const int cap = na > 0 ? (int)std::min<int64_t>(256, cache_budget(c) / (4 * na)) : 0;
  int32_t* cache = cap >= 8 ? ensure<int32_t>(c, c->q_cache, na * cap) : nullptr;
  int* over = cache ? ensure<int>(c, c->q_over, na + 1) : nullptr;
  const lsm::Spill spill = cache ? make_spill(c, na, cap) : lsm::Spill{};
  if (na > 0 && nb > 0) {
    if (over) CU(cudaMemsetAsync(over, 0, sizeof(int), s));
    CU(lsm::launch_query_batched(dim, false, na, a_box, pair_of_a, roots, stops, bvh, b_box, counts, nullptr,
                                 nullptr, nullptr, s, cache, cap, over, spill));
  }
  else if (na > 0)
    CU(cudaMemsetAsync(counts, 0, sizeof(int) * na, s));
  CU(lsm::launch_scan(na, counts, offsets, stmp, s));
  int64_t nnz = pair_cap;
  if (pair_cap == 0) {
    int64_t* h = static_cast<int64_t*>(c->host_scalars) + 8;
    int* hb = static_cast<int*>(c->host_scalars);
    CU(cudaMemcpyAsync(h, offsets + na, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(hb, bad, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    REQUIRE(hb[0] == 0, "Invalid node index in an element list");
    if (hb[3] != 0) {
      set_error(c, "tree build: the sort's look-back wait gave up");
      throw Fail{LSM_ERROR_TIMEOUT};
    }
    nnz = *h;
  }
  int32_t* pa = ensure<int32_t>(c, c->pair_a, nnz);
  int32_t* pb = ensure<int32_t>(c, c->pair_b, nnz);
  if (nnz > 0)
    CU(lsm::launch_query_batched(dim, true, na, a_box, pair_of_a, roots, stops, bvh, b_box, counts, offsets,
                                 pa, pb, s, cache, cap, over, spill, pair_cap > 0 ? pair_cap : INT64_MAX));
  c->dim = dim;
  c->loc_a = c->loc_b = loc;
  c->nel_a = na;
  c->nel_b = nb;
  c->ncand = nnz;
  c->simplex_prep = true;
  narrow(c, s, nullptr, pair_cap > 0 ? offsets + na : nullptr);
  lsm::Partial* tot = ensure<lsm::Partial>(c, c->bt_tot, nm);
  int64_t* nc = ensure<int64_t>(c, c->bt_ncand, nm);
  lsm::Partial* pieces = ensure<lsm::Partial>(c, c->partials, lsm::mesh_totals_pieces(nm));
  CU(lsm::launch_mesh_totals(nm, d_eoa, offsets, static_cast<double*>(c->pair_measure.p),
                             static_cast<int32_t*>(c->pair_nout.p), pieces, tot, nc, s,
                             pair_cap > 0 ? pair_cap : INT64_MAX));
  if (pair_cap > 0) {
    const GroupRes r = group_res(res_area, nm);
    CU(cudaMemcpyAsync(r.tot, tot, sizeof(lsm::Partial) * nm, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(r.nc, nc, sizeof(int64_t) * nm, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(r.count, offsets + na, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(r.flags, bad, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
    return false;
  }
  // per-pair outputs: CSR rows at the caller's row bases; the group's
  // per-candidate arrays (pair-major, as the caller's) as one block at the
  // next free slot, if they fit
  int64_t group_base = -1, p1_base = -1;
  if (bo && bo->o) {
    const lsm_gpu_batch_out* o = bo->o;
    const bool fits = bo->next + nnz <= o->cand_capacity;
    if (!fits) bo->overflow = true;
    const bool want_ind = fits && o->indices && nnz > 0;
    int64_t* ind_dst = nullptr;
    if (want_ind) ind_dst = on_device ? o->indices + bo->next : ensure<int64_t>(c, c->i64_tmp, nnz);
    CU(lsm::launch_batch_csr(na, nm, pair_of_a, d_eoa, offsets, d_rbase, o->ind_ptr ? bo->dev_indptr : nullptr,
                             want_ind ? nnz : 0, pb, pair_of_b, d_eob, ind_dst, s));
    if (fits) {
      const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
      if (want_ind && !on_device)
        CU(cudaMemcpyAsync(o->indices + bo->next, ind_dst, sizeof(int64_t) * nnz, k, s));
      if (o->pair_measure && nnz > 0)
        CU(cudaMemcpyAsync(o->pair_measure + bo->next, c->pair_measure.p, sizeof(double) * nnz, k, s));
      if (o->pair_n_out && nnz > 0)
        CU(cudaMemcpyAsync(o->pair_n_out + bo->next, c->pair_nout.p, sizeof(int32_t) * nnz, k, s));
      group_base = bo->next;
      bo->next += nnz;
    }
    // P1-P1 mass blocks of every candidate (a second clipping pass with the
    // quadrature; blocks dense, loc x loc per candidate, CSR order)
    const int64_t p1_need = nnz * loc * loc;
    if (want_p1 && fits && bo->p1_next + p1_need <= o->p1_capacity) {
      p1_base = bo->p1_next;
      if (nnz > 0) {
        double* dst = on_device ? o->p1_blocks + bo->p1_next : ensure<double>(c, c->blocks, p1_need);
        lsm::Partial* pp = ensure<lsm::Partial>(c, c->partials, std::max<int64_t>(lsm::p1_grid_blocks(dim),
                                                                                  lsm::mesh_totals_pieces(nm)));
        const lsm::SegList p1sg = p1_seg(c, dim, nnz);
        CU(lsm::launch_p1_mass(dim, nnz, pa, pb, a_coords, a_tol, b_coords, b_setup, nullptr, nullptr, ib, nullptr,
                               nullptr, dst, pp, s, p1_survivors(c, dim, nnz), p1_work(c),
                               g_tet_screen ? a_faces : nullptr, g_tet_screen ? b_screen : nullptr, nullptr,
                               &p1sg));
        if (!on_device)
          CU(cudaMemcpyAsync(o->p1_blocks + bo->p1_next, dst, sizeof(double) * p1_need, cudaMemcpyDeviceToHost, s));
      }
      bo->p1_next += p1_need;
    } else if (want_p1) {
      bo->overflow = true;
    }
  }
  const GroupRes r = group_res(static_cast<char*>(host_stage(c, group_res_bytes(nm))), nm);
  CU(cudaMemcpyAsync(r.tot, tot, sizeof(lsm::Partial) * nm, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(r.nc, nc, sizeof(int64_t) * nm, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(r.count, offsets + na, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(r.flags, bad, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  finish_batch_group(c, idx, loc, r, 0, totals, ncand, nint, bo, group_base, p1_base);
  return true;
}

// ------------------------------------------------------------- legacy API
std::mutex g_mutex;
Ctx* g_ctx = nullptr;
bool g_tree_state = false;

[[noreturn]] void legacy_abort(const char* what) {
  fprintf(stderr, "libsupermesh (B200) error: %s\n", what);
  fflush(stderr);
  exit(1);
}

Ctx* legacy_ctx() {
  if (!g_ctx) {
    int dev = 0;
    const char* env = getenv("LIBSUPERMESH_CUDA_DEVICE");
    if (env && *env) dev = atoi(env);
    g_ctx = new Ctx();
    const int st = init_ctx(dev, g_ctx);
    if (st != LSM_SUCCESS) legacy_abort("no usable CUDA device for libsupermesh");
  }
  return g_ctx;
}

void legacy_check(Ctx* c, int st) {
  if (st != LSM_SUCCESS) legacy_abort(c->last_error.empty() ? "CUDA failure" : c->last_error.c_str());
}

// Pinned staging area of the single-pair entries: inputs at 0, the count
// and the output simplices after them.
constexpr size_t kPairIoBytes = 16384;
char* pair_io(Ctx* c) {
  if (!c->pair_io) {
    if (cudaMallocHost(&c->pair_io, kPairIoBytes) != cudaSuccess) {
      (void)cudaGetLastError();
      c->pair_io = nullptr;
      set_error(c, "pinned host allocation of %zu bytes failed", kPairIoBytes);
      throw Fail{LSM_ERROR_OUT_OF_MEMORY};
    }
    // page-locked memory is mapped for the device under unified addressing:
    // the per-pair kernels then read their inputs and write their outputs
    // there directly (no copy calls); without a mapping the copies stay
    if (cudaHostGetDevicePointer(&c->pair_io_dev, c->pair_io, 0) != cudaSuccess) {
      (void)cudaGetLastError();
      c->pair_io_dev = nullptr;
    }
  }
  return static_cast<char*>(c->pair_io);
}

// One pair through the batched kernels: inputs staged in a pinned buffer
// that the kernel reads and writes directly (mapped), or, without a mapping,
// sent in one copy with the count and the output buffer back in one copy;
// one host wait.
void single_pair(int dim, const double* a, const double* b, double* out_elems, int* n_out) {
  std::lock_guard<std::mutex> lk(g_mutex);
  Ctx* c = legacy_ctx();
  const int per = dim == 2 ? 6 : 12;
  const int cap = dim == 2 ? 22 : 81;
  legacy_check(c, guarded(c, [&] {
    cudaStream_t s = c->stream;
    char* io = pair_io(c);
    double* hin = reinterpret_cast<double*>(io);
    memcpy(hin, a, sizeof(double) * per);
    memcpy(hin + per, b, sizeof(double) * per);
    char* hout = io + 1024;
    if (c->pair_io_dev) {
      // the kernel reads the pair from the pinned buffer and writes the count
      // and the simplices back into it: one launch, one wait
      char* dio = static_cast<char*>(c->pair_io_dev);
      const double* din = reinterpret_cast<const double*>(dio);
      CU(lsm::launch_pairs_explicit(dim, 1, din, din + per, nullptr, reinterpret_cast<int32_t*>(dio + 1024),
                                    reinterpret_cast<double*>(dio + 1024 + 16), s));
    } else {
      double* din = ensure<double>(c, c->x_a, 2 * per);
      const size_t out_bytes = 16 + sizeof(double) * (size_t)cap * per;
      char* dout = ensure<char>(c, c->x_elems, (int64_t)out_bytes);
      CU(cudaMemcpyAsync(din, hin, sizeof(double) * 2 * per, cudaMemcpyHostToDevice, s));
      CU(lsm::launch_pairs_explicit(dim, 1, din, din + per, nullptr, reinterpret_cast<int32_t*>(dout),
                                    reinterpret_cast<double*>(dout + 16), s));
      CU(cudaMemcpyAsync(hout, dout, out_bytes, cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
    const int k = *reinterpret_cast<int32_t*>(hout);
    *n_out = k;
    if (k > 0) memcpy(out_elems, hout + 16, sizeof(double) * per * k);
  }));
}

// Element shapes of the mixed pair kinds: doubles per A and B element, output
// capacity and doubles per output element.
struct MixedShape {
  int per_a, per_b, cap, per_out;
};

MixedShape mixed_shape(int kind) {
  if (kind == LSM_PAIR_INTERVALS) return {2, 2, 1, 2};
  if (kind == LSM_PAIR_TRI_QUAD) return {6, 8, 46, 6};
  if (kind == LSM_PAIR_QUAD_QUAD) return {8, 8, 62, 6};
  if (kind == LSM_PAIR_HEX_HEX) return {24, 24, 5 * 729, 12};
  return {12, 24, 729, 12};
}

void single_mixed(int kind, const double* a, const double* b, double* out_elems, int* n_out) {
  std::lock_guard<std::mutex> lk(g_mutex);
  Ctx* c = legacy_ctx();
  const MixedShape m = mixed_shape(kind);
  legacy_check(c, guarded(c, [&] {
    cudaStream_t s = c->stream;
    char* io = pair_io(c);
    double* hin = reinterpret_cast<double*>(io);
    memcpy(hin, a, sizeof(double) * m.per_a);
    memcpy(hin + m.per_a, b, sizeof(double) * m.per_b);
    double* din = ensure<double>(c, c->x_a, m.per_a + m.per_b);
    const size_t elem_bytes = sizeof(double) * (size_t)m.cap * m.per_out;
    char* dout = ensure<char>(c, c->x_elems, (int64_t)(16 + elem_bytes));
    CU(cudaMemcpyAsync(din, hin, sizeof(double) * (m.per_a + m.per_b), cudaMemcpyHostToDevice, s));
    CU(lsm::launch_pairs_mixed(kind, 1, din, din + m.per_a, nullptr, reinterpret_cast<int32_t*>(dout),
                               reinterpret_cast<double*>(dout + 16), s));
    // small output buffers come back whole with the count; large ones
    // (tet-hex, hex-hex) only up to the count, after a first wait
    char* hout = io + 1024;
    const bool whole = 16 + elem_bytes <= kPairIoBytes - 1024;
    CU(cudaMemcpyAsync(hout, dout, whole ? 16 + elem_bytes : 16, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const int k = *reinterpret_cast<int32_t*>(hout);
    *n_out = k;
    if (k > 0) {
      const size_t bytes = sizeof(double) * m.per_out * (size_t)k;
      if (whole) {
        memcpy(out_elems, hout + 16, bytes);
      } else {
        CU(cudaMemcpyAsync(out_elems, dout + 16, bytes, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
      }
    }
  }));
}
double single_measure(int dim, const double* e) {
  std::lock_guard<std::mutex> lk(g_mutex);
  Ctx* c = legacy_ctx();
  const int per = dim == 1 ? 2 : dim == 2 ? 6 : 12;
  double r = 0.0;
  legacy_check(c, guarded(c, [&] {
    cudaStream_t s = c->stream;
    double* de = ensure<double>(c, c->x_a, per);
    double* dm = ensure<double>(c, c->x_measure, 1);
    double* hin = reinterpret_cast<double*>(pair_io(c));
    memcpy(hin, e, sizeof(double) * per);
    CU(cudaMemcpyAsync(de, hin, sizeof(double) * per, cudaMemcpyHostToDevice, s));
    CU(lsm::launch_measure_explicit(dim, 1, de, dm, s));
    double* h = static_cast<double*>(c->host_scalars);
    CU(cudaMemcpyAsync(h, dm, sizeof(double), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    r = h[0];
  }));
  return r;
}

}  // namespace

struct lsm_gpu_context {
  Ctx c;
};

static Ctx* C(lsm_gpu_context* p) { return p ? &p->c : nullptr; }

// ---------------------------------------------------- batched CUDA graph
// Signature of a device-resident batch: the meshes' shapes and addresses and
// the options that shape the launches.  A graph replays only for the same
// signature (the caller may change the coordinates in place).
std::vector<uint64_t> batch_signature(int npairs, const lsm_gpu_mesh* a, const lsm_gpu_mesh* b) {
  std::vector<uint64_t> v;
  v.reserve(10 + 14 * (size_t)npairs);
  v.push_back((uint64_t)npairs);
  v.push_back((uint64_t)lsm::query_block());
  v.push_back((uint64_t)lsm::tri_blocks_per_sm());
  v.push_back((uint64_t)g_tet_screen);
  v.push_back((uint64_t)g_tet_schedule);
  v.push_back((uint64_t)g_sched_window);
  v.push_back((uint64_t)g_spill_chunks);
  v.push_back((uint64_t)lsm::sort_spin_limit());
  v.push_back((uint64_t)(int64_t)lsm::sort_stall_block());
  for (int i = 0; i < npairs; ++i)
    for (const lsm_gpu_mesh* m : {&a[i], &b[i]}) {
      v.push_back((uint64_t)m->dim);
      v.push_back((uint64_t)m->loc);
      v.push_back((uint64_t)m->nnodes);
      v.push_back((uint64_t)m->nelements);
      v.push_back((uint64_t)m->positions);
      v.push_back((uint64_t)m->enlist);
      v.push_back((uint64_t)m->index_bytes);
    }
  return v;
}

void drop_batch_graph(Ctx* c) {
  if (c->bg.exec) cudaGraphExecDestroy(c->bg.exec);
  c->bg.exec = nullptr;
  c->bg.sig.clear();
}

// One launch of the batch's graph and one host wait.  False if there is no
// graph for this signature, a device buffer was reallocated since its
// capture, or the candidates outgrew its arrays (the caller then runs the
// batch eagerly and captures again).
bool replay_batch_graph(Ctx* c, const std::vector<uint64_t>& sig, cudaStream_t s, double* totals, int64_t* ncand,
                        int64_t* nint) {
  Ctx::BatchGraph& g = c->bg;
  if (!g.exec || g.sig != sig || g.gen != c->gen) return false;
  CU(cudaGraphLaunch(g.exec, s));
  lsm::count_launch((int)g.launches);
  CU(cudaStreamSynchronize(s));
  char* host = static_cast<char*>(g.host);
  for (int k = 0; k < 2; ++k) {
    if (g.idx[k].empty()) continue;
    const int nm = (int)g.idx[k].size();
    if (!finish_batch_group(c, g.idx[k], k + 3, group_res(host + g.res_off[k], nm), g.cap[k], totals, ncand, nint,
                            nullptr, -1, -1)) {
      drop_batch_graph(c);
      return false;
    }
  }
  c->dim = g.last_dim;
  c->loc_a = c->loc_b = g.last_loc;
  c->nel_a = g.last_na;
  c->nel_b = g.last_nb;
  c->simplex_prep = true;
  c->have_pairs = true;
  c->surv_valid = g.last_dim == 3;
  c->surv_seg = g.last_seg;
  c->surv_npairs = g.last_surv_npairs;
  return true;
}

// Graph of a batch that has just run eagerly: pair arrays sized from that
// run's counts (+1/8), a dry run in capacity mode (it sizes every buffer, so
// the captured run allocates nothing) and the capture of the same launches.
// Leaves no graph if anything in the capture would allocate.
void capture_batch_graph(Ctx* c, std::vector<uint64_t> sig, const std::vector<int>& g2, const std::vector<int>& g3,
                         const int64_t cnt[2], const lsm_gpu_mesh* a, const lsm_gpu_mesh* b, cudaStream_t s,
                         double* totals, int64_t* ncand, int64_t* nint) {
  drop_batch_graph(c);
  Ctx::BatchGraph& g = c->bg;
  const std::vector<int>* grp[2] = {&g2, &g3};
  size_t tab_off[2] = {0, 0}, bytes = 0;
  for (int k = 0; k < 2; ++k) {
    const size_t nm = grp[k]->size();
    tab_off[k] = bytes;
    bytes += (sizeof(int64_t) * (2 * (nm + 1) + 7 * nm) + 255) & ~(size_t)255;
    g.res_off[k] = bytes;
    bytes += (group_res_bytes((int)nm) + 255) & ~(size_t)255;
    g.idx[k] = *grp[k];
    g.cap[k] = cnt[k] + cnt[k] / 8 + 1024;
  }
  if (g.host_cap < bytes) {
    if (g.host) cudaFreeHost(g.host);
    g.host = nullptr;
    g.host_cap = 0;
    if (cudaMallocHost(&g.host, bytes) != cudaSuccess) {
      (void)cudaGetLastError();
      set_error(c, "pinned host allocation of %zu bytes failed", bytes);
      throw Fail{LSM_ERROR_OUT_OF_MEMORY};
    }
    g.host_cap = bytes;
  }
  char* host = static_cast<char*>(g.host);
  auto run = [&]() {
    for (int k = 0; k < 2; ++k)
      if (!grp[k]->empty())
        run_batch_group(c, k + 2, *grp[k], a, b, nullptr, nullptr, nullptr, nullptr, s, nullptr, 1, g.cap[k],
                        host + tab_off[k], host + g.res_off[k]);
  };
  run();
  CU(cudaStreamSynchronize(s));
  for (int k = 0; k < 2; ++k)
    if (!grp[k]->empty() && !finish_batch_group(c, *grp[k], k + 3, group_res(host + g.res_off[k], (int)grp[k]->size()),
                                                g.cap[k], totals, ncand, nint, nullptr, -1, -1))
      return;
  const uint64_t gen0 = c->gen;
  const unsigned long long l0 = lsm::launches();
  CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  cudaGraph_t graph = nullptr;
  try {
    run();
  } catch (...) {
    cudaStreamEndCapture(s, &graph);
    if (graph) cudaGraphDestroy(graph);
    (void)cudaGetLastError();
    throw;
  }
  CU(cudaStreamEndCapture(s, &graph));
  if (c->gen != gen0) {
    cudaGraphDestroy(graph);
    return;
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return;
  }
  g.exec = exec;
  g.sig = std::move(sig);
  g.gen = c->gen;
  g.launches = lsm::launches() - l0;
  g.last_dim = c->dim;
  g.last_loc = c->loc_a;
  g.last_na = c->nel_a;
  g.last_nb = c->nel_b;
  g.last_seg = c->surv_seg;
  g.last_surv_npairs = c->surv_npairs;
}

// Both batched entries.
static int batched(Ctx* c, int npairs, const lsm_gpu_mesh* a, const lsm_gpu_mesh* b, int on_device, double* totals,
            int64_t* n_candidates, int64_t* n_intersecting, const lsm_gpu_batch_out* out, void* stream) {
  return guarded(c, [&] {
    REQUIRE(npairs >= 0 && (npairs == 0 || (a && b)), "invalid batch");
    cudaStream_t s = pick(c, stream);
    std::vector<int> g2, g3;
    for (int i = 0; i < npairs; ++i) {
      check_mesh(c, &a[i], "A", true);
      check_mesh(c, &b[i], "B", true);
      REQUIRE(a[i].dim >= 2, "batched supermesh: pair %d is 1D (use libsupermesh_gpu_supermesh)", i);
      REQUIRE(a[i].dim == b[i].dim, "Invalid dimension: pair %d mixes %dD and %dD", i, a[i].dim, b[i].dim);
      REQUIRE(a[i].index_bytes == a[0].index_bytes && b[i].index_bytes == a[0].index_bytes,
              "all meshes of a batch must use the same index width");
      (a[i].dim == 2 ? g2 : g3).push_back(i);
    }
    BatchOut bo;
    if (out) {
      REQUIRE(out->cand_capacity >= 0, "negative candidate capacity");
      bo.o = out;
      bo.rowbase.resize(npairs);
      for (int i = 0; i < npairs; ++i) {
        bo.rowbase[i] = bo.total_rows;
        bo.total_rows += a[i].nelements + 1;
      }
      if (out->ind_ptr)
        bo.dev_indptr = on_device ? out->ind_ptr : ensure<int64_t>(c, c->bt_indptr, bo.total_rows);
    }
    // device-resident batches without per-pair outputs can replay a graph
    const bool graph_mode = g_batch_graph && on_device && !out && !g_time_kernels;
    std::vector<uint64_t> sig;
    if (graph_mode) {
      sig = batch_signature(npairs, a, b);
      if (replay_batch_graph(c, sig, s, totals, n_candidates, n_intersecting)) return;
    }
    c->have_pairs = false;
    c->ncand = -1;
    // Host meshes: the 2D group's copies go on the caller's stream; the 3D
    // group's go on the side stream, where they overlap the 2D group's work
    // (the side stream first waits for earlier work on s, which may still
    // read the 3D staging buffers).
    std::vector<uint64_t> st2, st3;
    const bool side3 = !on_device && !g2.empty() && !g3.empty();
    SyncOnThrow sync_on_throw{s, c->side};
    if (!on_device && !g2.empty()) stage_batch_group(c, 2, g2, a, b, s, st2);
    if (!on_device && !g3.empty()) {
      if (side3) {
        CU(cudaEventRecord(c->side_ev[0], s));
        CU(cudaStreamWaitEvent(c->side, c->side_ev[0], 0));
      }
      stage_batch_group(c, 3, g3, a, b, side3 ? c->side : s, st3);
      if (side3) CU(cudaEventRecord(c->side_ev[1], c->side));
    }
    BatchOut* bp = out ? &bo : nullptr;
    int64_t cnt[2] = {0, 0};
    if (!g2.empty()) {
      run_batch_group(c, 2, g2, a, b, on_device ? nullptr : st2.data(), totals, n_candidates, n_intersecting, s, bp,
                      on_device);
      cnt[0] = c->ncand;
    }
    if (!g3.empty()) {
      if (side3) CU(cudaStreamWaitEvent(s, c->side_ev[1], 0));
      run_batch_group(c, 3, g3, a, b, on_device ? nullptr : st3.data(), totals, n_candidates, n_intersecting, s, bp,
                      on_device);
      cnt[1] = c->ncand;
    }
    if (graph_mode && npairs > 0)
      capture_batch_graph(c, std::move(sig), g2, g3, cnt, a, b, s, totals, n_candidates, n_intersecting);
    if (out && out->ind_ptr && !on_device && bo.total_rows > 0) {
      CU(cudaMemcpyAsync(out->ind_ptr, bo.dev_indptr, sizeof(int64_t) * bo.total_rows, cudaMemcpyDeviceToHost, s));
      CU(cudaStreamSynchronize(s));
    }
    if (out) {
      if (out->total_candidates) *out->total_candidates = bo.next;
      if (bo.overflow) {
        int64_t need = 0, need_p1 = 0;
        if (n_candidates)
          for (int i = 0; i < npairs; ++i) {
            need += n_candidates[i];
            need_p1 += n_candidates[i] * (a[i].dim + 1) * (a[i].dim + 1);
          }
        set_error(c,
                  "batched supermesh: %lld candidates (%lld block doubles) do not fit the per-candidate arrays "
                  "(capacity %lld, %lld)",
                  (long long)need, (long long)need_p1, (long long)out->cand_capacity, (long long)out->p1_capacity);
        throw Fail{LSM_ERROR_CAPACITY};
      }
    }
  });
}

extern "C" {

// ---------------------------------------------------------------- legacy
void libsupermesh_tree_intersection_finder_set_input(long* nnodes_a, int* dim_a, long* nelements_a, int* loc_a,
                                                     long* nnodes_b, int* dim_b, long* nelements_b, int* loc_b,
                                                     double* positions_a, long* enlist_a, double* positions_b,
                                                     long* enlist_b) {
  std::lock_guard<std::mutex> lk(g_mutex);
  if (g_tree_state) legacy_abort("tree intersection finder: set_input called again before get_output");
  if (*dim_a != 2 && *dim_a != 3) legacy_abort("Invalid dimension");
  if (*dim_b != *dim_a) legacy_abort("Invalid dimension");
  Ctx* c = legacy_ctx();
  lsm_gpu_mesh a{*dim_a, *loc_a, (int64_t)*nnodes_a, (int64_t)*nelements_a, positions_a, enlist_a, (int)sizeof(long)};
  lsm_gpu_mesh b{*dim_b, *loc_b, (int64_t)*nnodes_b, (int64_t)*nelements_b, positions_b, enlist_b, (int)sizeof(long)};
  legacy_check(c, guarded(c, [&] { find_candidates(c, &a, &b, 0, false, false, c->stream); }));
  g_tree_state = true;
}

void libsupermesh_tree_intersection_finder_query_output(long* nindices) {
  std::lock_guard<std::mutex> lk(g_mutex);
  if (!g_tree_state) legacy_abort("intersection finder: query_output without set_input");
  *nindices = (long)g_ctx->ncand;
}

void libsupermesh_tree_intersection_finder_get_output(long* nelements, long* nindices, long* indices, long* ind_ptr) {
  std::lock_guard<std::mutex> lk(g_mutex);
  if (!g_tree_state) legacy_abort("intersection finder: get_output without set_input");
  Ctx* c = g_ctx;
  if (*nelements != (long)c->nel_a || *nindices != (long)c->ncand)
    legacy_abort("intersection finder: get_output sizes do not match set_input");
  legacy_check(c, guarded(c, [&] {
    cudaStream_t s = c->stream;
    const int64_t nnz = c->ncand;
    if (nnz > 0) {
      int64_t* tmp = ensure<int64_t>(c, c->i64_tmp, nnz);
      CU(lsm::launch_i32_to_i64(nnz, static_cast<int32_t*>(c->pair_b.p), tmp, s));
      CU(cudaMemcpyAsync(indices, tmp, sizeof(int64_t) * nnz, cudaMemcpyDeviceToHost, s));
    }
    CU(cudaMemcpyAsync(ind_ptr, c->offsets.p, sizeof(int64_t) * (c->nel_a + 1), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
  }));
  g_tree_state = false;
}

void libsupermesh_intersect_tris_real(double* tri_a, double* tri_b, double* tris_c, int* n_tris_c) {
  single_pair(2, tri_a, tri_b, tris_c, n_tris_c);
}

void libsupermesh_intersect_tets_real(double* tet_a, double* tet_b, double* tets_c, int* n_tets_c) {
  single_pair(3, tet_a, tet_b, tets_c, n_tets_c);
}

void libsupermesh_triangle_area(double* tri, double* area) { *area = single_measure(2, tri); }

void libsupermesh_tetrahedron_volume(double* tet, double* volume) { *volume = single_measure(3, tet); }

void libsupermesh_sort_intersection_finder_set_input(long* nnodes_a, int* dim_a, long* nelements_a, int* loc_a,
                                                     long* nnodes_b, int* dim_b, long* nelements_b, int* loc_b,
                                                     double* positions_a, long* enlist_a, double* positions_b,
                                                     long* enlist_b) {
  std::lock_guard<std::mutex> lk(g_mutex);
  if (g_tree_state) legacy_abort("sort intersection finder: set_input called again before get_output");
  if (*dim_a < 1 || *dim_b < 1) legacy_abort("Invalid dimension");
  if (*loc_a != 2 || *loc_b != 2) legacy_abort("sort intersection finder: elements must have 2 nodes");
  Ctx* c = legacy_ctx();
  lsm_gpu_mesh a{*dim_a, 2, (int64_t)*nnodes_a, (int64_t)*nelements_a, positions_a, enlist_a, (int)sizeof(long)};
  lsm_gpu_mesh b{*dim_b, 2, (int64_t)*nnodes_b, (int64_t)*nelements_b, positions_b, enlist_b, (int)sizeof(long)};
  legacy_check(c, guarded(c, [&] { find_candidates(c, &a, &b, 0, false, false, c->stream, true); }));
  g_tree_state = true;
}

// The reference's tree and sort finders keep their output in the same module
// arrays (C_bindings.F90:30-32), so either query/get_output pair reads the
// result of the last set_input.
void libsupermesh_sort_intersection_finder_query_output(long* nindices) {
  libsupermesh_tree_intersection_finder_query_output(nindices);
}

void libsupermesh_sort_intersection_finder_get_output(long* nelements, long* nindices, long* indices, long* ind_ptr) {
  libsupermesh_tree_intersection_finder_get_output(nelements, nindices, indices, ind_ptr);
}

void libsupermesh_interval_size(double* interval, double* size) { *size = single_measure(1, interval); }

void libsupermesh_intersect_intervals(double* interval_a, double* interval_b, double* intervals_c,
                                      int* n_intervals_c) {
  single_mixed(LSM_PAIR_INTERVALS, interval_a, interval_b, intervals_c, n_intervals_c);
}

void libsupermesh_intersect_tet_hex(double* tet_a, double* hex_b, double* tets_c, int* n_tets_c) {
  single_mixed(LSM_PAIR_TET_HEX, tet_a, hex_b, tets_c, n_tets_c);
}

void libsupermesh_intersect_tri_quad(double* tri_a, double* quad_b, double* tris_c, int* n_tris_c) {
  single_mixed(LSM_PAIR_TRI_QUAD, tri_a, quad_b, tris_c, n_tris_c);
}

// ------------------------------------------------------------- GPU API
int libsupermesh_gpu_context_create(int device, lsm_gpu_context** ctx) {
  if (!ctx) return LSM_ERROR_INVALID_ARGUMENT;
  *ctx = nullptr;
  lsm_gpu_context* p = new lsm_gpu_context();
  const int st = init_ctx(device, &p->c);
  if (st != LSM_SUCCESS) {
    fini_ctx(&p->c);
    delete p;
    return st;
  }
  *ctx = p;
  return LSM_SUCCESS;
}

int libsupermesh_gpu_context_destroy(lsm_gpu_context* ctx) {
  if (!ctx) return LSM_ERROR_INVALID_ARGUMENT;
  fini_ctx(&ctx->c);
  delete ctx;
  return LSM_SUCCESS;
}

const char* libsupermesh_gpu_status_string(int status) {
  switch (status) {
    case LSM_SUCCESS: return "success";
    case LSM_ERROR_INVALID_ARGUMENT: return "invalid argument";
    case LSM_ERROR_OUT_OF_MEMORY: return "out of device memory";
    case LSM_ERROR_CAPACITY: return "output capacity exceeded";
    case LSM_ERROR_TIMEOUT: return "timed out";
    case LSM_ERROR_CUDA: return "CUDA error";
    case LSM_ERROR_STATE: return "invalid call sequence";
    default: return "unknown status";
  }
}

const char* libsupermesh_gpu_last_error(const lsm_gpu_context* ctx) {
  return ctx ? ctx->c.last_error.c_str() : "NULL context";
}

int64_t libsupermesh_gpu_context_bytes(const lsm_gpu_context* ctx) {
  return ctx ? ctx->c.bytes : 0;
}

int64_t libsupermesh_gpu_kernel_launches(void) { return (int64_t)lsm::launches(); }

int libsupermesh_gpu_set_option(const char* name, int64_t value) {
  if (!name) return LSM_ERROR_INVALID_ARGUMENT;
  const std::string n(name);
  if (n == "tri_blocks_per_sm" && (value == 4 || value == 8 || value == 16)) {
    lsm::set_tri_blocks_per_sm((int)value);
  } else if (n == "query_block" && (value == 64 || value == 128 || value == 256)) {
    lsm::set_query_block((int)value);
  } else if (n == "time_kernels" && (value == 0 || value == 1)) {
    g_time_kernels = value == 1;
  } else if (n == "tet_screen" && (value == 0 || value == 1)) {
    g_tet_screen = value == 1;
  } else if (n == "spill_chunks" && value >= -1 && value <= INT32_MAX) {
    g_spill_chunks = value;
  } else if (n == "tet_schedule" && value >= 0 && value <= 2) {
    g_tet_schedule = (int)value;
  } else if (n == "sched_window" && value >= 256 && value <= lsm::kSchedMaxWindow && value % 256 == 0) {
    g_sched_window = (int)value;
  } else if (n == "leaf_bucket" && (value == 1 || value == 2 || value == 4 || value == 8)) {
    lsm::set_leaf_bucket((int)value);
  } else if (n == "batch_graph" && (value == 0 || value == 1)) {
    g_batch_graph = (int)value;
  } else if (n == "fail_alloc_after" && value >= -1 && value <= INT32_MAX) {
    g_fail_alloc_after = value;
  } else if (n == "sort_spin_limit" && value >= 1 && value <= (1 << 22)) {
    lsm::set_sort_spin_limit((int)value);
  } else if (n == "sort_stall_block" && (value == -1 || (value >= 1 && value <= INT32_MAX))) {
    lsm::set_sort_stall_block((int)value);
  } else {
    return LSM_ERROR_INVALID_ARGUMENT;
  }
  return LSM_SUCCESS;
}

int libsupermesh_gpu_get_option(const char* name, int64_t* value) {
  if (!name || !value) return LSM_ERROR_INVALID_ARGUMENT;
  const std::string n(name);
  if (n == "tri_blocks_per_sm")
    *value = lsm::tri_blocks_per_sm();
  else if (n == "query_block")
    *value = lsm::query_block();
  else if (n == "time_kernels")
    *value = g_time_kernels ? 1 : 0;
  else if (n == "tet_screen")
    *value = g_tet_screen ? 1 : 0;
  else if (n == "spill_chunks")
    *value = g_spill_chunks;
  else if (n == "fail_alloc_after")
    *value = g_fail_alloc_after;
  else if (n == "tet_schedule")
    *value = g_tet_schedule;
  else if (n == "sched_window")
    *value = g_sched_window;
  else if (n == "batch_graph")
    *value = g_batch_graph;
  else if (n == "leaf_bucket")
    *value = lsm::leaf_bucket();
  else if (n == "sort_spin_limit")
    *value = lsm::sort_spin_limit();
  else if (n == "sort_stall_block")
    *value = lsm::sort_stall_block();
  else
    return LSM_ERROR_INVALID_ARGUMENT;
  return LSM_SUCCESS;
}

int libsupermesh_gpu_clip_kernel_ms(lsm_gpu_context* ctx, double* ms) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    REQUIRE(ms != nullptr, "NULL output");
    if (!c->clip_timed) {
      set_error(c, "the last narrow phase ran without the time_kernels option");
      throw Fail{LSM_ERROR_STATE};
    }
    CU(cudaEventSynchronize(c->clip_ev[1]));
    float f = 0.0f;
    CU(cudaEventElapsedTime(&f, c->clip_ev[0], c->clip_ev[1]));
    *ms = (double)f;
  });
}

int libsupermesh_gpu_clip_survivors(lsm_gpu_context* ctx, int64_t* n) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    REQUIRE(n != nullptr, "NULL output");
    if (!c->surv_valid) {
      set_error(c, "no 3D narrow phase since the last candidate search");
      throw Fail{LSM_ERROR_STATE};
    }
    CU(cudaDeviceSynchronize());
    unsigned long long v = 0;
    CU(cudaMemcpy(&v, c->surv.p, sizeof(v), cudaMemcpyDeviceToHost));
    *n = (int64_t)v;
  });
}

int libsupermesh_gpu_find_candidates(lsm_gpu_context* ctx, const lsm_gpu_mesh* a, const lsm_gpu_mesh* b,
                                     int on_device, int64_t* n_candidates, void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    find_candidates(c, a, b, on_device, false, false, pick(c, stream));
    if (n_candidates) *n_candidates = c->ncand;
  });
}

int libsupermesh_gpu_get_candidates(lsm_gpu_context* ctx, int64_t* ind_ptr, int64_t* indices, int on_device,
                                    void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    if (c->ncand < 0) {
      set_error(c, "no candidate search has run on this context");
      throw Fail{LSM_ERROR_STATE};
    }
    cudaStream_t s = pick(c, stream);
    const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (indices && c->ncand > 0) {
      if (on_device) {
        CU(lsm::launch_i32_to_i64(c->ncand, static_cast<int32_t*>(c->pair_b.p), indices, s));
      } else {
        int64_t* tmp = ensure<int64_t>(c, c->i64_tmp, c->ncand);
        CU(lsm::launch_i32_to_i64(c->ncand, static_cast<int32_t*>(c->pair_b.p), tmp, s));
        CU(cudaMemcpyAsync(indices, tmp, sizeof(int64_t) * c->ncand, k, s));
      }
    }
    if (ind_ptr) CU(cudaMemcpyAsync(ind_ptr, c->offsets.p, sizeof(int64_t) * (c->nel_a + 1), k, s));
    CU(cudaStreamSynchronize(s));
  });
}

int libsupermesh_gpu_supermesh(lsm_gpu_context* ctx, const lsm_gpu_mesh* a, const lsm_gpu_mesh* b, int on_device,
                               double* elem_measure_a, lsm_gpu_stats* stats, void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    cudaStream_t s = pick(c, stream);
    find_candidates(c, a, b, on_device, true, false, s);
    narrow(c, s);
    if (elem_measure_a && c->nel_a > 0) {
      double* em = on_device ? elem_measure_a : ensure<double>(c, c->elem_measure, c->nel_a);
      CU(lsm::launch_row_sums(c->nel_a, static_cast<int64_t*>(c->offsets.p), static_cast<double*>(c->pair_measure.p),
                              em, s));
      if (!on_device)
        CU(cudaMemcpyAsync(elem_measure_a, em, sizeof(double) * c->nel_a, cudaMemcpyDeviceToHost, s));
    }
    read_stats(c, stats, s);
  });
}

int libsupermesh_gpu_supermesh_out(lsm_gpu_context* ctx, const lsm_gpu_mesh* a, const lsm_gpu_mesh* b,
                                   int on_device, lsm_gpu_pair_out* out, lsm_gpu_stats* stats, void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    REQUIRE(out != nullptr, "NULL output descriptor");
    cudaStream_t s = pick(c, stream);
    SyncOnThrow sync_on_throw{s, c->side};
    find_candidates(c, a, b, on_device, true, false, s);
    const int64_t n = c->ncand, na = c->nel_a;
    out->n_candidates = n;
    const bool fits = n <= out->cand_capacity;
    const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    // the CSR is final once the search is done: its conversion and copy run
    // on the side stream while the narrow phase runs on s
    const bool csr = out->ind_ptr || (fits && out->indices && n > 0);
    if (csr) {
      CU(cudaEventRecord(c->side_ev[0], s));
      CU(cudaStreamWaitEvent(c->side, c->side_ev[0], 0));
      if (out->ind_ptr)
        CU(cudaMemcpyAsync(out->ind_ptr, c->offsets.p, sizeof(int64_t) * (na + 1), k, c->side));
      if (fits && out->indices && n > 0) {
        int64_t* dst = on_device ? out->indices : ensure<int64_t>(c, c->i64_tmp, n);
        CU(lsm::launch_i32_to_i64(n, static_cast<int32_t*>(c->pair_b.p), dst, c->side));
        if (!on_device) CU(cudaMemcpyAsync(out->indices, dst, sizeof(int64_t) * n, k, c->side));
      }
      CU(cudaEventRecord(c->side_ev[1], c->side));
    }
    narrow(c, s);
    if (out->elem_measure && na > 0) {
      double* em = on_device ? out->elem_measure : ensure<double>(c, c->elem_measure, na);
      CU(lsm::launch_row_sums(na, static_cast<int64_t*>(c->offsets.p), static_cast<double*>(c->pair_measure.p), em,
                              s));
      if (!on_device) CU(cudaMemcpyAsync(out->elem_measure, em, sizeof(double) * na, cudaMemcpyDeviceToHost, s));
    }
    if (fits && out->pair_measure && n > 0)
      CU(cudaMemcpyAsync(out->pair_measure, c->pair_measure.p, sizeof(double) * n, k, s));
    if (fits && out->pair_n_out && n > 0)
      CU(cudaMemcpyAsync(out->pair_n_out, c->pair_nout.p, sizeof(int32_t) * n, k, s));
    if (csr) CU(cudaStreamWaitEvent(s, c->side_ev[1], 0));
    read_stats(c, stats, s);
    if (!fits && (out->indices || out->pair_measure || out->pair_n_out)) {
      set_error(c, "supermesh: %lld candidates do not fit the per-candidate arrays (capacity %lld)", (long long)n,
                (long long)out->cand_capacity);
      throw Fail{LSM_ERROR_CAPACITY};
    }
  });
}

int libsupermesh_gpu_supermesh_elements(lsm_gpu_context* ctx, const lsm_gpu_mesh* a, const lsm_gpu_mesh* b,
                                        int on_device, lsm_gpu_elem_out* out, lsm_gpu_stats* stats, void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    REQUIRE(out != nullptr, "NULL output descriptor");
    REQUIRE(a && (a->dim == 2 || a->dim == 3), "supermesh elements: meshes must be 2D triangles or 3D tets");
    REQUIRE(!on_device || (((uintptr_t)out->elems) & 15u) == 0, "device elems must be 16-byte aligned");
    cudaStream_t s = pick(c, stream);
    find_candidates(c, a, b, on_device, true, false, s);
    const int64_t n = c->ncand;
    const int dim = c->dim, per = dim == 2 ? 6 : 12;
    out->n_candidates = n;
    // counting pass: the narrow phase (3D: its survivor list kept whole for
    // the second pass), then the offsets of every pair's simplices
    narrow(c, s, nullptr, nullptr, true);
    c->surv_valid = false;  // the list is not the plain narrow phase's
    int64_t* off = ensure<int64_t>(c, c->elem_off, n + 1);
    int64_t* tmp = ensure<int64_t>(c, c->scan_tmp, lsm::scan_tmp_entries(n) + 1);
    CU(lsm::launch_scan(n, static_cast<int*>(c->pair_nout.p), off, tmp, s));
    int64_t* h = static_cast<int64_t*>(c->host_scalars) + 40;
    CU(cudaMemcpyAsync(h, off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    read_stats(c, stats, s);  // waits for the stream
    const int64_t ne = *h;
    out->n_elements = ne;
    if (n > out->cand_capacity && out->elem_offset) {
      set_error(c, "supermesh elements: %lld candidates do not fit elem_offset (capacity %lld)", (long long)n,
                (long long)out->cand_capacity);
      throw Fail{LSM_ERROR_CAPACITY};
    }
    if (ne > out->elem_capacity) {
      set_error(c, "supermesh elements: %lld simplices do not fit the element arrays (capacity %lld)",
                (long long)ne, (long long)out->elem_capacity);
      throw Fail{LSM_ERROR_CAPACITY};
    }
    REQUIRE(ne == 0 || out->elems, "NULL elems");
    const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (out->elem_offset) CU(cudaMemcpyAsync(out->elem_offset, off, sizeof(int64_t) * (n + 1), k, s));
    if (ne > 0) {
      double* de = on_device ? out->elems : ensure<double>(c, c->x_elems, ne * per);
      int64_t* dpa = !out->parent_a ? nullptr : (on_device ? out->parent_a : ensure<int64_t>(c, c->x_pa, ne));
      int64_t* dpb = !out->parent_b ? nullptr : (on_device ? out->parent_b : ensure<int64_t>(c, c->x_pb, ne));
      // the counting pass's survivor segments (3D)
      const lsm::SegList esg = dim == 3 ? lsm::SegList{static_cast<int*>(c->seg_cnt.p), static_cast<int4*>(c->seg_tab.p)}
                                        : lsm::SegList{};
      CU(lsm::launch_emit_elements(dim, n, static_cast<int32_t*>(c->pair_a.p), static_cast<int32_t*>(c->pair_b.p),
                                   static_cast<double*>(c->a_coords.p), static_cast<double*>(c->a_tol.p),
                                   static_cast<double*>(c->b_setup.p), static_cast<int32_t*>(c->ovf_list.p),
                                   reinterpret_cast<unsigned long long*>(bad_flag(c) + 8), off, de, dpa, dpb, s,
                                   &esg));
      if (!on_device) {
        CU(cudaMemcpyAsync(out->elems, de, sizeof(double) * ne * per, k, s));
        if (dpa) CU(cudaMemcpyAsync(out->parent_a, dpa, sizeof(int64_t) * ne, k, s));
        if (dpb) CU(cudaMemcpyAsync(out->parent_b, dpb, sizeof(int64_t) * ne, k, s));
      }
    }
    CU(cudaStreamSynchronize(s));
  });
}

int libsupermesh_gpu_clip_candidates(lsm_gpu_context* ctx, lsm_gpu_stats* stats, void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    if (c->ncand < 0 || !c->simplex_prep) {
      set_error(c, "no simplex candidate search has run on this context");
      throw Fail{LSM_ERROR_STATE};
    }
    cudaStream_t s = pick(c, stream);
    narrow(c, s);
    read_stats(c, stats, s);
  });
}

int libsupermesh_gpu_clip_candidates_ordered(lsm_gpu_context* ctx, const int32_t* order, int on_device,
                                              lsm_gpu_stats* stats, void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    if (c->ncand < 0 || !c->simplex_prep) {
      set_error(c, "no simplex candidate search has run on this context");
      throw Fail{LSM_ERROR_STATE};
    }
    cudaStream_t s = pick(c, stream);
    const int32_t* d = order;
    if (order && !on_device) {
      int32_t* t = ensure<int32_t>(c, c->x_nout, c->ncand);
      CU(cudaMemcpyAsync(t, order, sizeof(int32_t) * c->ncand, cudaMemcpyHostToDevice, s));
      d = t;
    }
    narrow(c, s, d);
    read_stats(c, stats, s);
  });
}

int libsupermesh_gpu_get_pair_results(lsm_gpu_context* ctx, double* measure, int32_t* n_out, int on_device,
                                      void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    if (!c->have_pairs) {
      set_error(c, "no supermesh has run on this context");
      throw Fail{LSM_ERROR_STATE};
    }
    cudaStream_t s = pick(c, stream);
    const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (measure && c->ncand > 0)
      CU(cudaMemcpyAsync(measure, c->pair_measure.p, sizeof(double) * c->ncand, k, s));
    if (n_out && c->ncand > 0) CU(cudaMemcpyAsync(n_out, c->pair_nout.p, sizeof(int32_t) * c->ncand, k, s));
    CU(cudaStreamSynchronize(s));
  });
}

int libsupermesh_gpu_intersect_pairs(lsm_gpu_context* ctx, int dim, int64_t n, const double* a, const double* b,
                                     double* measure, int32_t* n_out, double* elems, int on_device, void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    REQUIRE(dim == 2 || dim == 3, "Invalid dimension %d", dim);
    REQUIRE(n >= 0, "negative pair count");
    if (n == 0) return;
    REQUIRE(a && b, "NULL element arrays");
    REQUIRE(!on_device || dim == 2 || ((((uintptr_t)a | (uintptr_t)b) & 15u) == 0),
            "device tetrahedron arrays must be 16-byte aligned (a %p, b %p)", (const void*)a, (const void*)b);
    // output tets are written with 16-byte stores
    REQUIRE(!on_device || dim == 2 || ((uintptr_t)elems & 15u) == 0,
            "device elems must be 16-byte aligned (%p)", (const void*)elems);
    cudaStream_t s = pick(c, stream);
    const int per = dim == 2 ? 6 : 12;
    const int64_t cap = dim == 2 ? 22 : 81;
    const double *da = a, *db = b;
    double* dm = measure;
    int32_t* dn = n_out;
    double* de = elems;
    if (!on_device) {
      double* ta = ensure<double>(c, c->x_a, n * per);
      double* tb = ensure<double>(c, c->x_b, n * per);
      CU(cudaMemcpyAsync(ta, a, sizeof(double) * n * per, cudaMemcpyHostToDevice, s));
      CU(cudaMemcpyAsync(tb, b, sizeof(double) * n * per, cudaMemcpyHostToDevice, s));
      da = ta;
      db = tb;
      dm = measure ? ensure<double>(c, c->x_measure, n) : nullptr;
      dn = n_out ? ensure<int32_t>(c, c->x_nout, n) : nullptr;
      de = elems ? ensure<double>(c, c->x_elems, n * cap * per) : nullptr;
    }
    if (dim == 3 && n >= kPairsPipelineMin && n <= INT32_MAX) {
      // large batches: per-pair setup, the exact early-outs and the index
      // clipper (one launch per stage); small ones stay on the one-launch
      // register clipper below (identical results)
      double* setup = ensure<double>(c, c->x_setup, n * lsm::kSetup3);
      double* tol = ensure<double>(c, c->x_tol, n);
      int32_t* iota = ensure<int32_t>(c, c->x_iota, n);
      double* faces = g_tet_screen ? ensure<double>(c, c->x_faces, n * lsm::kScreen3) : nullptr;
      double* screen = g_tet_screen ? ensure<double>(c, c->x_screen, n * lsm::kScreen3) : nullptr;
      int32_t* list = ensure<int32_t>(c, c->x_list, 4 * n);
      double* pm = dm ? dm : ensure<double>(c, c->x_measure, n);
      int32_t* pn = dn ? dn : ensure<int32_t>(c, c->x_nout, n);
      unsigned long long* work = pairs_work(c);
      const lsm::SegList sg = seg_list(c, c->x_seg_cnt, c->x_seg_tab, n);
      CU(lsm::launch_setup_pairs3(n, da, db, setup, tol, iota, faces, screen, s));
      if (de)
        CU(lsm::launch_clip_elems(n, iota, iota, da, tol, setup, pm, pn, de, list, work, faces, screen, s, &sg));
      else
        CU(lsm::launch_clip(3, n, iota, iota, da, tol, setup, pm, pn, list, nullptr, work, s, nullptr, nullptr,
                            nullptr, faces, screen, nullptr, nullptr, &sg));
    } else {
      CU(lsm::launch_pairs_explicit(dim, n, da, db, dm, dn, de, s));
    }
    if (!on_device) {
      if (measure) CU(cudaMemcpyAsync(measure, dm, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      if (n_out) CU(cudaMemcpyAsync(n_out, dn, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
      if (elems) CU(cudaMemcpyAsync(elems, de, sizeof(double) * n * cap * per, cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
  });
}

int libsupermesh_gpu_intersect_pairs_mixed(lsm_gpu_context* ctx, int kind, int64_t n, const double* a,
                                           const double* b, double* measure, int32_t* n_out, double* elems,
                                           int on_device, void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    REQUIRE(kind >= LSM_PAIR_INTERVALS && kind <= LSM_PAIR_HEX_HEX, "unknown pair kind %d", kind);
    REQUIRE(n >= 0, "negative pair count");
    if (n == 0) return;
    REQUIRE(a && b, "NULL element arrays");
    REQUIRE(!on_device || kind != LSM_PAIR_TET_HEX || ((((uintptr_t)a | (uintptr_t)elems) & 15u) == 0),
            "device tetrahedron array a and elems must be 16-byte aligned (a %p, elems %p)", (const void*)a,
            (const void*)elems);
    cudaStream_t s = pick(c, stream);
    const MixedShape m = mixed_shape(kind);
    const double *da = a, *db = b;
    double* dm = measure;
    int32_t* dn = n_out;
    double* de = elems;
    if (!on_device) {
      double* ta = ensure<double>(c, c->x_a, n * m.per_a);
      double* tb = ensure<double>(c, c->x_b, n * m.per_b);
      CU(cudaMemcpyAsync(ta, a, sizeof(double) * n * m.per_a, cudaMemcpyHostToDevice, s));
      CU(cudaMemcpyAsync(tb, b, sizeof(double) * n * m.per_b, cudaMemcpyHostToDevice, s));
      da = ta;
      db = tb;
      dm = measure ? ensure<double>(c, c->x_measure, n) : nullptr;
      dn = n_out ? ensure<int32_t>(c, c->x_nout, n) : nullptr;
      de = elems ? ensure<double>(c, c->x_elems, n * m.cap * m.per_out) : nullptr;
    }
    if (kind == LSM_PAIR_TET_HEX && n >= kPairsPipelineMin && n <= INT32_MAX) {
      // large batches: per-pair setup, the exact early-out and the six-plane
      // index clipper; small ones stay on the one-launch clipper (same results)
      double* pm = dm ? dm : ensure<double>(c, c->x_measure, n);
      int32_t* pn = dn ? dn : ensure<int32_t>(c, c->x_nout, n);
      const lsm::SegList hsg = seg_list(c, c->x_seg_cnt, c->x_seg_tab, n);
      CU(lsm::launch_tet_hex_pairs(n, da, db, pm, pn, de, ensure<double>(c, c->x_setup, n * 28),
                                   ensure<double>(c, c->x_tol, n), ensure<int32_t>(c, c->x_iota, n),
                                   ensure<int32_t>(c, c->x_list, 4 * n), pairs_work(c), s, &hsg));
    } else if (kind == LSM_PAIR_HEX_HEX && n >= kPairsPipelineMin && n <= INT32_MAX / 5 &&
               (((uintptr_t)de) & 15u) == 0) {
      // large batches: A's five tets clipped by the six-plane index clipper,
      // one launch per tet, each pair's results carried in order (output tets
      // written with 16-byte stores: device elems off a 16-byte boundary
      // stay on the one-launch clipper below, same results)
      double* pm = dm ? dm : ensure<double>(c, c->x_measure, n);
      int32_t* pn = dn ? dn : ensure<int32_t>(c, c->x_nout, n);
      const lsm::SegList hsg = seg_list(c, c->x_seg_cnt, c->x_seg_tab, n);
      CU(lsm::launch_hex_hex_pairs(n, da, db, pm, pn, de, ensure<double>(c, c->x_setup, n * 28),
                                   ensure<double>(c, c->x_sub, 5 * n * 12), ensure<double>(c, c->x_tol, 5 * n),
                                   ensure<int32_t>(c, c->x_iota, n), ensure<int32_t>(c, c->x_list, 4 * n),
                                   pairs_work(c), s, &hsg));
    } else {
      CU(lsm::launch_pairs_mixed(kind, n, da, db, dm, dn, de, s));
    }
    if (!on_device) {
      if (measure) CU(cudaMemcpyAsync(measure, dm, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      if (n_out) CU(cudaMemcpyAsync(n_out, dn, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
      if (elems)
        CU(cudaMemcpyAsync(elems, de, sizeof(double) * n * m.cap * m.per_out, cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
  });
}

int libsupermesh_gpu_p1_mass(lsm_gpu_context* ctx, const lsm_gpu_mesh* a, const lsm_gpu_mesh* b, const double* u_a,
                             const double* v_b, double* blocks, double* integral, int on_device, void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    cudaStream_t s = pick(c, stream);
    REQUIRE(a && b && a->index_bytes == b->index_bytes, "A and B must use the same index width");
    REQUIRE(a->dim == 2 || a->dim == 3, "P1 mass matrix: Invalid dimension %d", a->dim);
    find_candidates(c, a, b, on_device, true, true, s);
    const int64_t nnz = c->ncand;
    require_pair_index(c, nnz);
    const int loc = c->dim + 1;
    const double *du = u_a, *dv = v_b;
    if (!on_device && u_a && v_b) {
      double* tu = ensure<double>(c, c->u_a, a->nnodes);
      double* tv = ensure<double>(c, c->v_b, b->nnodes);
      CU(cudaMemcpyAsync(tu, u_a, sizeof(double) * a->nnodes, cudaMemcpyHostToDevice, s));
      CU(cudaMemcpyAsync(tv, v_b, sizeof(double) * b->nnodes, cudaMemcpyHostToDevice, s));
      du = tu;
      dv = tv;
    }
    double* dbk = blocks;
    if (blocks && !on_device) dbk = ensure<double>(c, c->blocks, nnz * loc * loc);
    const int nblk = lsm::p1_grid_blocks(c->dim);
    lsm::Partial* part = ensure<lsm::Partial>(c, c->partials, nblk + 1);
    lsm::Partial* tot = ensure<lsm::Partial>(c, c->totals, 1);
    const void* en_a = on_device ? a->enlist : c->a_en.p;
    const void* en_b = on_device ? b->enlist : c->b_en.p;
    const lsm::SegList p1sg = p1_seg(c, c->dim, nnz);
    CU(lsm::launch_p1_mass(c->dim, nnz, static_cast<int32_t*>(c->pair_a.p), static_cast<int32_t*>(c->pair_b.p),
                           static_cast<double*>(c->a_coords.p), static_cast<double*>(c->a_tol.p),
                           static_cast<double*>(c->b_coords.p), static_cast<double*>(c->b_setup.p), en_a, en_b,
                           a->index_bytes, du, dv, dbk, part, s, p1_survivors(c, c->dim, nnz), p1_work(c),
                           c->dim == 3 && g_tet_screen ? static_cast<double*>(c->a_faces.p) : nullptr,
                           c->dim == 3 && g_tet_screen ? static_cast<double*>(c->b_screen.p) : nullptr,
                           c->dim == 3 && du && dv ? ensure<double>(c, c->x_measure, std::max<int64_t>(nnz, 1))
                                                   : nullptr,
                           &p1sg));
    CU(lsm::launch_finalize(part, nblk, tot, s));
    double* h = static_cast<double*>(c->host_scalars) + 64;
    CU(cudaMemcpyAsync(h, tot, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (blocks && !on_device && nnz > 0)
      CU(cudaMemcpyAsync(blocks, dbk, sizeof(double) * nnz * loc * loc, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (integral) *integral = h[0];
  });
}

int libsupermesh_gpu_p2_inner_product(lsm_gpu_context* ctx, const lsm_gpu_mesh* a, const lsm_gpu_mesh* b,
                                      const void* enlist_p2_a, const double* field_a, int64_t nnodes_p2_a,
                                      const void* enlist_p2_b, const double* field_b, int64_t nnodes_p2_b,
                                      double* pair_values, double* integral, double* area, int on_device,
                                      void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    cudaStream_t s = pick(c, stream);
    REQUIRE(a && b && a->index_bytes == b->index_bytes, "A and B must use the same index width");
    REQUIRE(a->dim == 2 && b->dim == 2, "P2 inner product: meshes must be 2D triangles");
    REQUIRE(enlist_p2_a && enlist_p2_b && field_a && field_b, "NULL P2 arrays");
    REQUIRE(nnodes_p2_a > 0 && nnodes_p2_b > 0, "empty P2 spaces");
    find_candidates(c, a, b, on_device, true, true, s);
    const int64_t nnz = c->ncand;
    const int ib = a->index_bytes;
    const void *e2a = enlist_p2_a, *e2b = enlist_p2_b;
    const double *fa = field_a, *fb = field_b;
    if (!on_device) {
      char* ta = ensure<char>(c, c->x_a, (a->nelements * 6 * ib + 7) / 8 * 8);
      char* tb = ensure<char>(c, c->x_b, (b->nelements * 6 * ib + 7) / 8 * 8);
      double* tfa = ensure<double>(c, c->u_a, nnodes_p2_a);
      double* tfb = ensure<double>(c, c->v_b, nnodes_p2_b);
      CU(cudaMemcpyAsync(ta, enlist_p2_a, (size_t)a->nelements * 6 * ib, cudaMemcpyHostToDevice, s));
      CU(cudaMemcpyAsync(tb, enlist_p2_b, (size_t)b->nelements * 6 * ib, cudaMemcpyHostToDevice, s));
      CU(cudaMemcpyAsync(tfa, field_a, sizeof(double) * nnodes_p2_a, cudaMemcpyHostToDevice, s));
      CU(cudaMemcpyAsync(tfb, field_b, sizeof(double) * nnodes_p2_b, cudaMemcpyHostToDevice, s));
      e2a = ta;
      e2b = tb;
      fa = tfa;
      fb = tfb;
    }
    int* bad = bad_flag(c);
    CU(cudaMemsetAsync(bad, 0, sizeof(int), s));
    CU(lsm::launch_check_index(a->nelements * 6, e2a, ib, nnodes_p2_a, bad, s));
    CU(lsm::launch_check_index(b->nelements * 6, e2b, ib, nnodes_p2_b, bad, s));
    double* pv = (pair_values && on_device) ? pair_values : ensure<double>(c, c->pair_measure, nnz);
    double* pa_ = ensure<double>(c, c->elem_measure, std::max<int64_t>(nnz, c->nel_a));
    int32_t* pn = ensure<int32_t>(c, c->pair_nout, nnz);
    int* hb = static_cast<int*>(c->host_scalars);
    CU(cudaMemcpyAsync(hb, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    REQUIRE(hb[0] == 0, "Invalid node index in a P2 element list");
    CU(lsm::launch_p2_inner(nnz, static_cast<int32_t*>(c->pair_a.p), static_cast<int32_t*>(c->pair_b.p),
                            static_cast<double*>(c->a_coords.p), static_cast<double*>(c->a_tol.p),
                            static_cast<double*>(c->b_coords.p), static_cast<double*>(c->b_setup.p), e2a, fa, e2b,
                            fb, ib, pv, pa_, pn, s));
    const int nred = lsm::reduce_pairs_blocks();
    lsm::Partial* part = ensure<lsm::Partial>(c, c->partials, 2 * nred);
    lsm::Partial* tot = ensure<lsm::Partial>(c, c->totals, 2);
    CU(lsm::launch_reduce_pairs(nnz, pv, pn, part, s));
    CU(lsm::launch_finalize(part, nred, tot, s));
    CU(lsm::launch_reduce_pairs(nnz, pa_, pn, part + nred, s));
    CU(lsm::launch_finalize(part + nred, nred, tot + 1, s));
    lsm::Partial* h = reinterpret_cast<lsm::Partial*>(static_cast<char*>(c->host_scalars) + 512);
    CU(cudaMemcpyAsync(h, tot, 2 * sizeof(lsm::Partial), cudaMemcpyDeviceToHost, s));
    if (pair_values && !on_device && nnz > 0)
      CU(cudaMemcpyAsync(pair_values, pv, sizeof(double) * nnz, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (integral) *integral = h[0].sum;
    if (area) *area = h[1].sum;
    c->have_pairs = false;  // pair_measure now holds P2 contributions
  });
}

int libsupermesh_gpu_sched_set_weights(lsm_gpu_context* ctx, const float* params, int on_device) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    REQUIRE(params != nullptr, "NULL parameters");
    cudaStream_t s = c->stream;
    const float* d = params;
    if (!on_device) {
      float* t = ensure<float>(c, c->sched_adam, 2 * lsm::kSchedParams);
      CU(cudaMemcpyAsync(t, params, sizeof(float) * lsm::kSchedParams, cudaMemcpyHostToDevice, s));
      d = t;
    }
    lsm::SchedWeights* w = reinterpret_cast<lsm::SchedWeights*>(ensure<char>(c, c->sched_w, sizeof(lsm::SchedWeights)));
    CU(lsm::launch_sched_pack(d, w, s));
    CU(cudaStreamSynchronize(s));
    c->have_sched = true;
  });
}

int libsupermesh_gpu_sched_samples(lsm_gpu_context* ctx, int64_t cap, void* features, int8_t* classes, int64_t* n,
                                   void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    REQUIRE(cap >= 0 && (cap == 0 || (features && classes)), "invalid sample buffers");
    REQUIRE((((uintptr_t)features) & 15u) == 0, "features must be 16-byte aligned");
    if (!c->surv_valid || !c->have_pairs || c->dim != 3) {
      set_error(c, "no 3D narrow phase since the last candidate search");
      throw Fail{LSM_ERROR_STATE};
    }
    cudaStream_t s = pick(c, stream);
    const unsigned long long* nl = reinterpret_cast<const unsigned long long*>(bad_flag(c) + 8);
    const int4* list = static_cast<const int4*>(c->ovf_list.p);
    if (c->surv_seg) {
      // the survivors in the clipper's order, as one list
      int4* flat = ensure<int4>(c, c->surv_list, std::max<int64_t>(c->surv_npairs, 1));
      CU(lsm::launch_seg_compact(c->surv_npairs, nl + 2, static_cast<const int4*>(c->seg_tab.p), list, flat, s));
      list = flat;
    }
    CU(lsm::launch_sched_samples(list, nl, cap, static_cast<double*>(c->a_coords.p),
                                 static_cast<double*>(c->b_screen.p), static_cast<int32_t*>(c->pair_nout.p), features,
                                 classes, s));
    unsigned long long* h = reinterpret_cast<unsigned long long*>(static_cast<char*>(c->host_scalars) + 512);
    CU(cudaMemcpyAsync(h, nl, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (n) *n = (int64_t)*h;
  });
}

int libsupermesh_gpu_sched_predict(lsm_gpu_context* ctx, int64_t n, const void* features, float* logits,
                                   int8_t* classes, void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    REQUIRE(n >= 0 && (n == 0 || (features && classes)), "invalid buffers");
    REQUIRE((((uintptr_t)features) & 15u) == 0, "features must be 16-byte aligned");
    if (!c->have_sched) {
      set_error(c, "no scheduler weights (libsupermesh_gpu_sched_set_weights)");
      throw Fail{LSM_ERROR_STATE};
    }
    cudaStream_t s = pick(c, stream);
    CU(lsm::launch_sched_predict(n, features, static_cast<const lsm::SchedWeights*>(c->sched_w.p), logits, classes, s));
    CU(cudaStreamSynchronize(s));
  });
}

int libsupermesh_gpu_sched_train(lsm_gpu_context* ctx, int64_t n, const void* features, const int8_t* classes,
                                 float* params, int steps, float lr, float* loss_trace, int trace_every,
                                 float* grad_first, void* stream) {
  Ctx* c = C(ctx);
  return guarded(c, [&] {
    REQUIRE(n > 0 && features && classes && params, "invalid training buffers");
    REQUIRE((((uintptr_t)features) & 15u) == 0, "features must be 16-byte aligned");
    REQUIRE(steps >= 0 && lr > 0.0f, "invalid steps or learning rate");
    cudaStream_t s = pick(c, stream);
    float* adam = ensure<float>(c, c->sched_adam, 2 * lsm::kSchedParams);
    CU(lsm::launch_sched_train(features, classes, n, params, adam, steps, lr, loss_trace, trace_every, grad_first, s));
    CU(cudaStreamSynchronize(s));
  });
}

int libsupermesh_gpu_supermesh_batched(lsm_gpu_context* ctx, int npairs, const lsm_gpu_mesh* a,
                                       const lsm_gpu_mesh* b, int on_device, double* totals,
                                       int64_t* n_candidates, int64_t* n_intersecting, void* stream) {
  return batched(C(ctx), npairs, a, b, on_device, totals, n_candidates, n_intersecting, nullptr, stream);
}

int libsupermesh_gpu_supermesh_batched_ex(lsm_gpu_context* ctx, int npairs, const lsm_gpu_mesh* a,
                                          const lsm_gpu_mesh* b, int on_device, lsm_gpu_batch_out* out,
                                          void* stream) {
  Ctx* c = C(ctx);
  if (!c) return LSM_ERROR_INVALID_ARGUMENT;
  if (!out) {
    set_error(c, "NULL output descriptor");
    return LSM_ERROR_INVALID_ARGUMENT;
  }
  // counts are needed to report the size a retry needs
  std::vector<int64_t> nc_local;
  int64_t* nc = out->n_candidates;
  if (!nc) {
    nc_local.assign(npairs > 0 ? npairs : 1, 0);
    nc = nc_local.data();
  }
  return batched(c, npairs, a, b, on_device, out->totals, nc, out->n_intersecting, out, stream);
}

}  // extern "C"
