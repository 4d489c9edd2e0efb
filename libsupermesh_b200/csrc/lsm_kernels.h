// Host-side launchers for the supermesh kernels (all asynchronous on the
// given stream).  Device buffers are owned by the caller (lsm_capi.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace lsm {

// Per-element records written by the prep kernels.
//   coords  [nel][loc*dim]  float64 vertex coordinates (gathered)
//   box64   [nel][2*dim]    float64 AABB (lo..., hi...)
//   box32   [nel][8]        float32 AABB rounded outwards (lo.xyz, pad, hi.xyz, pad)
//   setup   [nel][kSetup]   clip setup of a B element: 2D lines (12) or 3D
//                           planes (16), then tol = 10*spacing(measure)
//   tolv    [nel]           10*spacing(measure) (A elements)
constexpr int kSetup2 = 14;  // 3 lines x (nx, ny, px, py), tol, pad
constexpr int kSetup3 = 20;  // 4 planes x (nx, ny, nz, c), tol, pad (16-byte aligned rows)
// Separation screen of the tet clipper (3D simplices, optional):
//   faces   [nel][kScreen3]  A: 4 outward face planes (nx, ny, nz, h), h
//                            bounding n.x over every vertex clipping derives
//   screen  [nel][kScreen3]  B: 4 vertices, dilation factor g, residual tau,
//                            coordinate bound M, pad
constexpr int kScreen3 = 16;

// Per-block partial of a narrow-phase launch: compensated measure sum,
// intersecting pairs and output simplices.
struct Partial {
  double sum;
  double err;
  unsigned long long n_int;
  unsigned long long n_out;
};

// Process-wide count of kernel launches issued by this library (every
// launcher adds its launches with count_launch).
unsigned long long launches();
void count_launch(int n = 1);
// SMs of the current device; grid of at most per_sm blocks per SM for n items.
int sm_count();
int grid_for(int64_t n, int block, int per_sm);

// Grid of the 2D clipper (blocks per SM) and block size of the search.
int tri_blocks_per_sm();
void set_tri_blocks_per_sm(int v);
int query_block();
void set_query_block(int v);
// Leaves per bucket of the single-mesh hierarchy (1 = none; 2, 4 or 8):
// subtrees of at most this many leaves are scanned as contiguous leaf
// records instead of being walked.
int leaf_bucket();
void set_leaf_bucket(int v);
// The bucket size launch_bvh_build uses for n leaves (1 = none); BVH::bucket
// must carry it to the search.
int tree_bucket(int n, bool leaf_records);

struct BVH {
  int n = 0;                 // leaves
  // Node k (2n-1 nodes) is the 32-byte pair lo_left[2k], hi_esc[2k] of one
  // interleaved array (hi_esc = lo_left + 1), so a visit reads one sector.
  float4* lo_left = nullptr;  // lo.xyz, .w = left child / element (int bits)
  float4* hi_esc = nullptr;   // hi.xyz, .w = escape node (int bits), -1 = end
  // optional [n][8] f64 leaf records in sorted order: lo (3), hi (3),
  // {element, escape} as two ints, pad
  double* leaf = nullptr;
  // internal nodes of at most `bucket` leaves carry a leaf-bucket code in
  // place of their left child (1: none)
  int bucket = 1;
};

// Mesh prep: gather coordinates, boxes, measures/tolerances, B clip setup.
// idx_bytes selects the enlist element type (4 = int32, 8 = int64).
cudaError_t launch_prep(int dim, int loc, int64_t nel, const double* pos, const void* enlist, int idx_bytes,
                        double* coords, double* box64, float* box32, double* tolv, double* setup,
                        int* bad_index, int64_t nnodes, cudaStream_t s, double* faces = nullptr,
                        double* screen = nullptr);

// Root box (float64) of a set of element boxes: rootbox[2*dim].
cudaError_t launch_root_box(int dim, int64_t nel, const double* box64, double* partial,
                            int partial_cap, double* rootbox, cudaStream_t s);

cudaError_t launch_morton(int dim, int64_t nel, const double* box64, const double* rootbox,
                          uint32_t* keys, int32_t* vals, cudaStream_t s);

// Stable LSD radix sort of (key, val) pairs, 8 bits per pass over the low
// `bits` bits (at most 32), n < 2^30.  tmp buffers must hold n entries; hist
// (scratch: digit counts, block tickets, look-back status) must hold
// radix_hist_entries(n).  Result ends in keys/vals.  *err (optional) becomes
// nonzero if a look-back wait gave up (bounded; not expected to happen).
int64_t radix_hist_entries(int64_t n);
// Test hooks of the sort's bounded waits (process-wide): the number of
// polls before a look-back wait gives up (default 2^22), and a block (>= 1,
// -1 = none) that never publishes its digit counts, so that the waits of the
// blocks after it run out.  Only sorts given an err word take the stall.
void set_sort_spin_limit(int v);
int sort_spin_limit();
void set_sort_stall_block(int b);
int sort_stall_block();
cudaError_t radix_sort_pairs(int64_t n, int bits, uint32_t* keys, int32_t* vals, uint32_t* keys_tmp,
                             int32_t* vals_tmp, uint32_t* hist, cudaStream_t s, int* err = nullptr);

// LBVH over sorted Morton codes.  work_int needs 8*n ints.
cudaError_t launch_bvh_build(int dim, int n, const uint32_t* sorted_keys, const int32_t* sorted_vals,
                             const float* box32, BVH bvh, int* work_int, cudaStream_t s,
                             const double* box64 = nullptr);

// Spill pool of the count pass's row cache: rows longer than the cache
// continue in chunks of kSpillChunk candidates (pool[chunks][kSpillChunk]),
// chained per row (row_chunk[nel_a]: first chunk, or -2 for a row that
// could not keep all its candidates; written for every row longer than the
// cache; chunk_next[chunks]); *next (zeroed by the caller) counts the chunks
// handed out.
constexpr int kSpillChunk = 64;
struct Spill {
  int32_t* pool = nullptr;
  int* next = nullptr;
  int* chunk_next = nullptr;
  int* row_chunk = nullptr;
  int chunks = 0;
};

// Candidate search.  Pass 1 (fill=false) writes counts[nel_a]; pass 2 writes
// pair_a/pair_b at offsets[a].  With a cache ([nel_a][cap] int32) pass 1 also
// keeps each row's first cap candidates, the rest in spill chunks (sp), and
// lists the rows that could not keep them all in over_rows ({count,
// rows...}, count zeroed by the caller, nel_a + 1 ints); pass 2 then copies
// the kept rows and traverses only the listed ones.
// pair_cap: entries pair_a / pair_b hold; the fill writes no pair beyond it
// (the caller compares the count with it afterwards).
cudaError_t launch_query(int dim, bool fill, int64_t nel_a, const double* box64_a, BVH bvh,
                         const double* box64_b, int* counts, const int64_t* offsets, int32_t* pair_a,
                         int32_t* pair_b, cudaStream_t s, int32_t* cache = nullptr, int cap = 0,
                         int* over_rows = nullptr, Spill sp = Spill{}, int64_t pair_cap = INT64_MAX);

// Exclusive scan of int32 counts into int64 offsets[n+1] (offsets[n] = total).
int64_t scan_tmp_entries(int64_t n);
cudaError_t launch_scan(int64_t n, const int* counts, int64_t* offsets, int64_t* tmp, cudaStream_t s);

// Narrow phase over candidate pairs: pair_measure/pair_nout per pair.
// 2D: overflow_list collects pairs whose polygon outgrew the fast-path
// buffers; launch_clip_tris_wide re-runs them.  3D: overflow_list (npairs
// entries) receives the pairs that survive the exact early-out; `work`
// holds two counters (survivors, clipper progress), reset by the launch.
// `order` (optional, npairs entries) is the schedule: the pairs in the order
// in which the clipper takes them.  Results do not depend on it.
// faces_a / screen_b (3D, optional, kScreen3 rows from the prep) enable the
// second exact early-out (B beyond a face of A).
// bin (3D, optional): the learned scheduler's reordering of the survivors
// between the early-out pass and the clipper (lsm_sched.h).
// seg (3D, optional, ignored with bin): the survivors are written as
// per-block segments of overflow_list (no global counter) and the clipper
// takes them by chunks from seg->table; `work` then holds three counters
// (survivors, chunks taken, chunks).  launch_seg_compact gathers such a list
// into a compacted one.
struct SchedBin;
// Per-block survivor segments of the early-out pass over npairs pairs:
// count [seg_blocks(npairs)] segment lengths, table
// [seg_table_entries(npairs)] chunks {first, end, compacted position, 0}.
struct SegList {
  int* count = nullptr;
  int4* table = nullptr;
};
int clip_grid_blocks(int dim);
int seg_blocks(int64_t npairs);
int64_t seg_table_entries(int64_t npairs);
cudaError_t launch_seg_compact(int64_t npairs, const unsigned long long* nchunks, const int4* table,
                               const int4* seg, int4* out, cudaStream_t s);
cudaError_t launch_clip(int dim, int64_t npairs, const int32_t* pair_a, const int32_t* pair_b,
                        const double* coords_a, const double* tol_a, const double* setup_b,
                        double* pair_measure, int32_t* pair_nout, int32_t* overflow_list,
                        int* overflow_count, unsigned long long* work, cudaStream_t s,
                        const int32_t* order = nullptr, cudaEvent_t ev_begin = nullptr,
                        cudaEvent_t ev_end = nullptr, const double* faces_a = nullptr,
                        const double* screen_b = nullptr, const SchedBin* bin = nullptr,
                        const int64_t* n_dev = nullptr, const SegList* seg = nullptr);
// Opt-in shared-memory limits for the clip kernels on the current device.
cudaError_t init_device_attributes();
cudaError_t launch_clip_tris_wide(const int32_t* overflow_list, const int* overflow_count, int64_t cap,
                                  const int32_t* pair_a, const int32_t* pair_b,
                                  const double* coords_a, const double* tol_a,
                                  const double* setup_b, double* pair_measure, int32_t* pair_nout,
                                  cudaStream_t s);
// Per-block partials of the pair measures/counts in a fixed order
// (reduce_pairs_blocks() == kReduceBlocks entries; the block count is fixed
// because it sets the totals' summation order).
constexpr int kReduceBlocks = 1024;
int reduce_pairs_blocks();
// n_dev (optional): the pair count on the device; npairs is then its upper
// bound (the pair arrays' capacity).  The same holds for launch_clip.
cudaError_t launch_reduce_pairs(int64_t npairs, const double* pair_measure, const int32_t* pair_nout,
                                Partial* partials, cudaStream_t s, const int64_t* n_dev = nullptr);

// Totals: merge of the per-block partials into out[0] (in order).
cudaError_t launch_finalize(const Partial* partials, int npartials, Partial* out, cudaStream_t s);

// Per-A-element measure: sum of pair measures over each CSR row, in order.
cudaError_t launch_row_sums(int64_t nel_a, const int64_t* offsets, const double* pair_measure,
                            double* elem_measure, cudaStream_t s);

// Convert int32 CSR to int64 (C API output).
cudaError_t launch_i32_to_i64(int64_t n, const int32_t* in, int64_t* out, cudaStream_t s);

// Single-pair style batched intersections over explicit element arrays
// (tri: [n][3][2]; tet: [n][4][3]).  out_elems optional ([n][22][3][2] or
// [n][81][4][3]).
// Explicit tetrahedron pairs through the early-out pass and the index
// clipper: per-pair setup (setup [n][kSetup3], tol_a [n], iota [n]; faces_a /
// screen_b [n][kScreen3] optional, for the second early-out), then, for
// measures and counts, launch_clip(3, n, iota, iota, tet_a, ...), or, with
// the output tets, launch_clip_elems (elems [n][81][4][3]; survivors: 4 ints
// per pair; work: two counters, three with seg).  tet_a must be 16-byte
// aligned.
cudaError_t launch_setup_pairs3(int64_t n, const double* tet_a, const double* tet_b, double* setup, double* tol_a,
                                int32_t* iota, double* faces_a, double* screen_b, cudaStream_t s);
// launch_clip_elems: the 3D narrow phase whose survivor list also holds the
// pairs with every plane a no-op (so that a second pass over the list sees
// every pair with output tets); measure/nout for every pair, elems optional;
// seg (optional) as for launch_clip.
cudaError_t launch_clip_elems(int64_t n, const int32_t* pair_a, const int32_t* pair_b, const double* tet_a,
                              const double* tol_a, const double* setup, double* measure, int32_t* nout,
                              double* elems, int32_t* survivors, unsigned long long* work, const double* faces_a,
                              const double* screen_b, cudaStream_t s, const SegList* seg = nullptr);
// The supermesh's simplices: pair p's output simplices (reference order) at
// elems[pair_off[p] ..] ([3][2] or [4][3] doubles each), parents optional.
// 3D takes the survivor list, work counters and seg of a launch_clip_elems
// pass over the same pairs; 2D clips the pairs again.
cudaError_t launch_emit_elements(int dim, int64_t npairs, const int32_t* pair_a, const int32_t* pair_b,
                                 const double* coords_a, const double* tol_a, const double* setup_b,
                                 const int32_t* survivors, unsigned long long* work, const int64_t* pair_off,
                                 double* elems, int64_t* parent_a, int64_t* parent_b, cudaStream_t s,
                                 const SegList* seg = nullptr);
// Explicit tet-hexahedron pairs (a [n][4][3] 16-byte aligned, hex_b
// [n][8][3]) through per-pair setup (setup [n][28], tol_a [n], iota [n]), the
// first early-out with the no-op planes, and the six-plane index clipper:
// measure/nout per pair and, optionally, elems [n][729][4][3]; survivors 4
// ints per pair, work two counters (three with seg, as for launch_clip).
cudaError_t launch_tet_hex_pairs(int64_t n, const double* tet_a, const double* hex_b, double* measure, int32_t* nout,
                                 double* elems, double* setup, double* tol_a, int32_t* iota, int32_t* survivors,
                                 unsigned long long* work, cudaStream_t s, const SegList* seg = nullptr);
// Explicit hexahedron-hexahedron pairs (hex_a, hex_b [n][8][3]) through the
// six-plane index clipper: A sliced into its five tets (sub [5][n][12] and
// tol [5][n], 16-byte aligned scratch), each clipped against B's planes
// (setup [n][28]) in one launch per tet, every pair's measure, count and
// output tets (elems optional, [n][5*729][4][3]) carried from tet to tet in
// the reference's order; survivors 4 ints per pair, work and seg as for
// launch_tet_hex_pairs.
cudaError_t launch_hex_hex_pairs(int64_t n, const double* hex_a, const double* hex_b, double* measure, int32_t* nout,
                                 double* elems, double* setup, double* sub, double* tol, int32_t* iota,
                                 int32_t* survivors, unsigned long long* work, cudaStream_t s,
                                 const SegList* seg = nullptr);
cudaError_t launch_pairs_explicit(int dim, int64_t n, const double* a, const double* b,
                                  double* measure, int32_t* nout, double* out_elems,
                                  cudaStream_t s);
cudaError_t launch_measure_explicit(int dim, int64_t n, const double* elems, double* out,
                                    cudaStream_t s);
// Mixed pairs: kind 0 intervals ([n][2] x [n][2] -> [n][2]), 1 tri vs quad
// ([n][3][2] x [n][4][2] -> [n][46][3][2]), 2 tet vs hex ([n][4][3] x
// [n][8][3] -> [n][729][4][3]), 3 quad vs quad (-> [n][62][3][2]), 4 hex vs
// hex (-> [n][5*729][4][3]).
cudaError_t launch_pairs_mixed(int kind, int64_t n, const double* a, const double* b, double* measure,
                               int32_t* nout, double* out_elems, cudaStream_t s);
// 1D sort finder.  prep gathers the first coordinate of both nodes of each
// element (coords[2*nel]) and the 64-bit order key of its left end;
// sort_by_key64 is a stable sort of (key, val) pairs; the max tree over the
// sorted right ends of B holds 2*tree_leaves_1d(nb) doubles.
cudaError_t launch_prep_1d(int64_t nel, const double* pos, int stride, const void* en, int idx_bytes,
                           int64_t nnodes, double* coords, uint32_t* key_lo, uint32_t* key_hi, int32_t* vals,
                           int* bad, cudaStream_t s);
cudaError_t sort_by_key64(int64_t n, uint32_t* key_lo, const uint32_t* key_hi, int32_t* vals, uint32_t* keys_tmp,
                          int32_t* vals_tmp, uint32_t* hist, cudaStream_t s);
cudaError_t launch_sorted_ends_1d(int64_t n, const int32_t* perm, const double* coords, double* lo, double* hi,
                                  cudaStream_t s);
int64_t tree_leaves_1d(int64_t n);
cudaError_t launch_max_tree(int64_t n, const double* v, double* tree, cudaStream_t s);
cudaError_t launch_rows_1d(int64_t na, const double* lo_a, const double* hi_a, int64_t nb, const double* lo_b,
                           const double* tree, int32_t* E, int32_t* L, cudaStream_t s);
cudaError_t launch_sweep_1d(int64_t na, int64_t nb, const int32_t* E, const int32_t* L, const double* lo_a,
                            const double* hi_a, const double* hi_b, int32_t* JS, cudaStream_t s);
cudaError_t launch_emit_1d(bool fill, int64_t na, const int32_t* JS, const int32_t* E, const double* lo_a,
                           const double* hi_b, const int32_t* perm_a, const int32_t* perm_b, int* counts,
                           const int64_t* offsets, int32_t* pair_a, int32_t* pair_b, cudaStream_t s);
cudaError_t launch_clip_intervals(int64_t n, const int32_t* pa, const int32_t* pb, const double* ca,
                                  const double* cb, double* measure, int32_t* nout, cudaStream_t s);

// P1-P1 mixed mass blocks per candidate pair and u^T M v partials.
// P2 inner product over a 2D candidate list (per pair: contribution, area,
// supermesh triangles); P2 element-node lists [nel][6] with idx_bytes.
cudaError_t launch_p2_inner(int64_t npairs, const int32_t* pair_a, const int32_t* pair_b, const double* coords_a,
                            const double* tol_a, const double* coords_b, const double* setup_b,
                            const void* en_p2_a, const double* field_a, const void* en_p2_b,
                            const double* field_b, int idx_bytes, double* pair_value, double* pair_area,
                            int32_t* pair_n, cudaStream_t s);
// bad = 1 if any of en[0..n) lies outside [0, limit).
cudaError_t launch_check_index(int64_t n, const void* en, int idx_bytes, int64_t limit, int* bad, cudaStream_t s);
// P1-P1 mixed mass: 2D clips every pair; 3D runs the exact early-out pass
// (survivors: 4 ints per pair, work: two counters (three with seg),
// faces_a / screen_b / seg as for launch_clip) and the index clipper with the quadrature on the survivors,
// with blocks of the other pairs zero-filled; 3D with u_a and v_b also needs
// pair_uv [npairs] (u^T M v per pair, summed in pair order).  partials:
// p1_grid_blocks(dim) entries.
cudaError_t launch_p1_mass(int dim, int64_t npairs, const int32_t* pair_a, const int32_t* pair_b,
                           const double* coords_a, const double* tol_a, const double* coords_b,
                           const double* setup_b, const void* enlist_a, const void* enlist_b,
                           int idx_bytes, const double* u_a, const double* v_b, double* blocks,
                           Partial* partials, cudaStream_t s, int32_t* survivors, unsigned long long* work,
                           const double* faces_a, const double* screen_b, double* pair_uv = nullptr,
                           const SegList* seg = nullptr);
int p1_grid_blocks(int dim);

// ---- batched (many mesh pairs per launch) --------------------------------
cudaError_t launch_prep_batched(int dim, int64_t nel, int nm, const int64_t* elem_off,
                                const unsigned long long* pos_ptr, const unsigned long long* en_ptr,
                                const int64_t* nnodes, int idx_bytes, double* coords, double* box64,
                                float* box32, double* tolv, double* setup, int32_t* pair_of, int* bad,
                                cudaStream_t s, double* faces = nullptr, double* screen = nullptr);
// keys[i] = pair_of[vals[i]] (second sort pass: by mesh)
cudaError_t launch_pair_keys(int64_t n, const int32_t* vals, const int32_t* pair_of, uint32_t* keys,
                             cudaStream_t s);
// One LBVH over all B meshes (sorted by mesh, then Morton); roots/stops per
// mesh.  codes: n u64; work: 8n ints.
cudaError_t launch_batched_tree(int n, int nm, const int32_t* sorted_vals, const int32_t* pair_of_b,
                                const uint32_t* mort, unsigned long long* codes, const float* box32,
                                const int64_t* mesh_off_b, BVH bvh, int* work, int* roots, int* stops,
                                cudaStream_t s, int dim = 3,
                                const double* box64 = nullptr, const int* sort_err = nullptr);
cudaError_t launch_query_batched(int dim, bool fill, int64_t nel_a, const double* box64_a,
                                 const int32_t* pair_of_a, const int* roots, const int* stops, BVH bvh,
                                 const double* box64_b, int* counts, const int64_t* offsets, int32_t* pair_a,
                                 int32_t* pair_b, cudaStream_t s, int32_t* cache = nullptr, int cap = 0,
                                 int* over_rows = nullptr, Spill sp = Spill{}, int64_t pair_cap = INT64_MAX);
// Per-pair CSR of a batch group (get_output layout): ind_ptr rows of mesh
// pair k at rowbase[k] (optional), candidate B elements local to their pair
// as int64 (optional).
cudaError_t launch_batch_csr(int64_t na, int nm, const int32_t* pair_of_a, const int64_t* eoa, const int64_t* offsets,
                             const int64_t* rowbase, int64_t* ind_ptr, int64_t ncand, const int32_t* pair_b,
                             const int32_t* pair_of_b, const int64_t* eob, int64_t* indices, cudaStream_t s);
int64_t mesh_totals_pieces(int nm);  // Partial scratch entries for launch_mesh_totals
cudaError_t launch_mesh_totals(int nm, const int64_t* elem_off_a, const int64_t* offsets, const double* pm,
                               const int32_t* pn, Partial* pieces, Partial* out, int64_t* ncand, cudaStream_t s,
                               int64_t cap = INT64_MAX);

}  // namespace lsm
