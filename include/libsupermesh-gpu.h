/*
 * libsupermesh GPU extension: batched and device-resident entry points of
 * the B200 supermesh library, declared beside the drop-in C API of
 * libsupermesh-c.h.  None of these has a single counterpart in the
 * reference; each comment names the reference routines whose work it
 * performs (paths within firedrakeproject/libsupermesh).
 *
 * Conventions
 *   - meshes: positions [nnodes][dim] float64, enlist [nelements][loc]
 *     0-based (int32 or int64), row-major -- the layout of
 *     libsupermesh_tree_intersection_finder_set_input.
 *   - A is the target (query) mesh whose elements are the CSR rows; B is the
 *     source mesh the search structure is built on.
 *   - on_device = 0: every pointer of the call is host memory (pinned for
 *     asynchronous copies); on_device = 1: every pointer is device memory of
 *     the context's GPU.  Outputs follow the inputs' memory space.
 *   - every function returns an lsm_status; the context keeps the message
 *     of the last failure (libsupermesh_gpu_last_error).
 *   - stream: a cudaStream_t (NULL = the context's own stream).  Calls are
 *     synchronous with respect to the host unless stated otherwise.
 *   - a call that clips (supermesh, P1, elements, batched groups) takes at
 *     most 2^31-1 candidate pairs (per dimension group for the batched
 *     entries); beyond that it returns LSM_ERROR_CAPACITY before clipping
 *     (the candidate search alone has no such limit).
 */
#ifndef LIBSUPERMESH_GPU_H
#define LIBSUPERMESH_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  LSM_SUCCESS = 0,
  LSM_ERROR_INVALID_ARGUMENT = 1,
  LSM_ERROR_OUT_OF_MEMORY = 2,
  LSM_ERROR_CAPACITY = 3,
  LSM_ERROR_TIMEOUT = 4,
  LSM_ERROR_CUDA = 5,
  LSM_ERROR_STATE = 6
} lsm_status;

typedef struct lsm_gpu_context lsm_gpu_context;

typedef struct {
  int dim;               /* 1, 2 or 3 */
  int loc;               /* dim + 1 (simplices); 2 for 1D interval meshes */
  int64_t nnodes;
  int64_t nelements;
  const double *positions; /* [nnodes][dim] */
  const void *enlist;      /* [nelements][loc], 0-based */
  int index_bytes;         /* 4 (int32) or 8 (int64) */
} lsm_gpu_mesh;

typedef struct {
  int64_t n_candidates;    /* strict-AABB candidate pairs (tree finder set) */
  int64_t n_intersecting;  /* pairs with at least one output simplex */
  int64_t n_out_simplices; /* supermesh elements */
  double total_measure;    /* compensated sum of all supermesh measures */
  double total_measure_err;/* its compensation term */
} lsm_gpu_stats;

/* Context on one CUDA device.  Owns a stream and grow-only device buffers
 * that are reused by later calls. */
int libsupermesh_gpu_context_create(int device, lsm_gpu_context **ctx);
int libsupermesh_gpu_context_destroy(lsm_gpu_context *ctx);
const char *libsupermesh_gpu_status_string(int status);
const char *libsupermesh_gpu_last_error(const lsm_gpu_context *ctx);
/* Bytes of device memory currently held by the context. */
int64_t libsupermesh_gpu_context_bytes(const lsm_gpu_context *ctx);
/* Kernel launches issued by this library in this process so far. */
int64_t libsupermesh_gpu_kernel_launches(void);

/* Process-wide tuning options.  They change launch shapes and work order,
 * never results (the autotuner in libsupermesh_b200/autotune.py picks the
 * launch shapes per GPU and workload):
 *   "tri_blocks_per_sm"  4, 8 (default) or 16 blocks of 128 threads per SM (2D clipper)
 *   "query_block"        64, 128 (default) or 256 threads per block (candidate search)
 *   "leaf_bucket"        1 (default), 2, 4 or 8: subtrees of the single-mesh search hierarchy with
 *                        at most this many leaves are scanned as contiguous leaf records instead
 *                        of being walked (same candidates, same order)
 *   "time_kernels"       1: record CUDA events around the clip kernel of every
 *                        narrow phase (read with libsupermesh_gpu_clip_kernel_ms); 0 (default)
 *   "spill_chunks"       -1 (default, automatic), 0 or n > 0: chunks of 64 candidates that the
 *                        batched search's row cache may take for rows longer than 256 (rows
 *                        that find none are traversed a second time)
 *   "tet_screen"         1 (default): tet pairs whose B lies beyond a face plane of A by a
 *                        proven rounding margin skip the clipper (exact: the reference
 *                        returns no tets for them); 0: only the A-beyond-a-face-of-B test
 *   "tet_schedule"       order of the 3D clipper's work list (never changes results):
 *                        0 (default) plain: the early-out pass's survivors in candidate order;
 *                        1 learned: survivors binned by the scheduler MLP's predicted output-size
 *                          class within windows of sched_window survivors (needs weights,
 *                          libsupermesh_gpu_sched_set_weights);
 *                        2 true classes: binned by the output counts of the previous narrow phase
 *                          over the same candidates (the best a predictor could do; a measurement)
 *   "sched_window"       survivors per binning window: 256 .. 8192, a multiple of 256 (default 1024)
 *   "batch_graph"        0 (default) or 1: a device-resident libsupermesh_gpu_supermesh_batched
 *                        call is captured into a CUDA graph after its first (eager) run; later
 *                        calls with the same meshes (same arrays, sizes and options; coordinates
 *                        may change in place) replay it with one graph launch and one host wait.
 *                        Pair arrays are sized from the first run's counts plus 1/8; a batch whose
 *                        candidates outgrow them, or a context that reallocated its buffers since
 *                        the capture, runs eagerly and is captured again.  Results are identical.
 * Failure-injection hooks for tests (host side only; no GPU fault is made):
 *   "fail_alloc_after"   -1 (default) off; n >= 0: the next n device allocations of any
 *                        context succeed and the following one fails as cudaMalloc out of
 *                        memory would (LSM_ERROR_OUT_OF_MEMORY; the hook then turns itself
 *                        off and the context stays usable)
 *   "sort_spin_limit"    polls (1 .. 2^22, default 2^22) before a look-back wait of the
 *                        radix sort gives up
 *   "sort_stall_block"   -1 (default) or b >= 1: block b of every pass of the tree build's
 *                        sort never publishes its counts, so the waits after it give up;
 *                        the search then returns LSM_ERROR_TIMEOUT ("look-back wait gave up")
 * Unknown names or values return LSM_ERROR_INVALID_ARGUMENT. */
int libsupermesh_gpu_set_option(const char *name, int64_t value);
int libsupermesh_gpu_get_option(const char *name, int64_t *value);

/* Device time (ms) of the clipping kernels of the last narrow phase on ctx
 * (2D: the triangle clipper; 3D: the exact early-out pass and the tet
 * clipper, which together settle every candidate), from CUDA events recorded
 * on its stream (needs option time_kernels = 1 during that phase; waits for
 * the kernels to finish). */
int libsupermesh_gpu_clip_kernel_ms(lsm_gpu_context *ctx, double *ms);

/* Pairs of the last 3D narrow phase on ctx that the exact early-outs left
 * for the clipper (the others were proven to give no tets).  Waits for the
 * device.  LSM_ERROR_STATE if no 3D narrow phase ran since the last
 * candidate search. */
int libsupermesh_gpu_clip_survivors(lsm_gpu_context *ctx, int64_t *n);

/* Candidate search only (tree finder): the work of
 * tree_intersection_finder_set_input_c (C_bindings.F90:346-366) on the GPU.
 * 1D meshes (dim 1, loc 2) take the sort finder instead
 * (sort_intersection_finder_set_input_c, C_bindings.F90:66-86).
 * Results stay in the context; read them with
 * libsupermesh_gpu_get_candidates. */
int libsupermesh_gpu_find_candidates(lsm_gpu_context *ctx, const lsm_gpu_mesh *a,
                                     const lsm_gpu_mesh *b, int on_device,
                                     int64_t *n_candidates, void *stream);

/* Copy the last candidate CSR out: ind_ptr[nelements_a + 1] (0-based, starts
 * at 0) and indices[n_candidates] (0-based B elements; within a row in
 * LBVH traversal order).  on_device selects the destination memory. */
int libsupermesh_gpu_get_candidates(lsm_gpu_context *ctx, int64_t *ind_ptr,
                                    int64_t *indices, int on_device, void *stream);

/* Whole supermesh of one mesh pair: candidate search, intersect every
 * candidate (intersect_tris_real / intersect_tets_real semantics), and sum
 * the libsupermesh_triangle_area / tetrahedron_volume of every output
 * simplex.  elem_measure_a (optional, [nelements_a]) receives per A element
 * the supermesh measure inside it; stats (optional) the totals. */
int libsupermesh_gpu_supermesh(lsm_gpu_context *ctx, const lsm_gpu_mesh *a,
                               const lsm_gpu_mesh *b, int on_device,
                               double *elem_measure_a, lsm_gpu_stats *stats,
                               void *stream);

/* Whole supermesh of one mesh pair with everything a drop-in caller reads:
 * the work of set_input / get_output (C_bindings.F90:346-391) and of one
 * intersect_*_real + measure call per candidate, in one call.
 *   elem_measure    [nelements_a] (optional): supermesh measure inside each A element
 *   ind_ptr         [nelements_a + 1] (optional): CSR row pointers (0-based, start at 0)
 *   indices         [cand_capacity] (optional): 0-based B element of each candidate
 *   pair_measure    [cand_capacity] (optional): measure of each candidate pair
 *   pair_n_out      [cand_capacity] (optional): its number of output simplices
 *   n_candidates    set by the call
 * Arrays follow on_device (host arrays should be pinned: the CSR's copy runs
 * on the context's second stream while the candidates are clipped).  If the
 * candidates do not fit cand_capacity the call fills elem_measure, ind_ptr,
 * n_candidates and stats and returns LSM_ERROR_CAPACITY. */
typedef struct {
  double *elem_measure;
  int64_t *ind_ptr;
  int64_t *indices;
  double *pair_measure;
  int32_t *pair_n_out;
  int64_t cand_capacity;
  int64_t n_candidates;
} lsm_gpu_pair_out;
int libsupermesh_gpu_supermesh_out(lsm_gpu_context *ctx, const lsm_gpu_mesh *a,
                                   const lsm_gpu_mesh *b, int on_device, lsm_gpu_pair_out *out,
                                   lsm_gpu_stats *stats, void *stream);

/* The supermesh itself: every output simplex of every candidate pair of A
 * and B (what one intersect_tris_real / intersect_tets_real call per
 * candidate returns, C_bindings.F90:152-174), candidates in the get_output
 * CSR order and, within a pair, the reference's output order.
 *   elem_offset  [cand_capacity + 1] (optional): the simplices of candidate k
 *                are elems[elem_offset[k] .. elem_offset[k+1]-1]
 *   elems        [elem_capacity][3][2] (triangles) or [elem_capacity][4][3]
 *                (tets); device arrays 16-byte aligned
 *   parent_a, parent_b [elem_capacity] (optional): 0-based A and B element of
 *                each simplex
 *   n_candidates, n_elements  set by the call
 * Simplex meshes only.  A counting pass (the narrow phase) sizes the output,
 * a second pass writes it.  If the candidates do not fit cand_capacity
 * (with elem_offset given) or the simplices elem_capacity, the call sets both
 * counts and the stats, writes nothing else and returns LSM_ERROR_CAPACITY;
 * a retry with those capacities succeeds. */
typedef struct {
  int64_t *elem_offset;
  double *elems;
  int64_t *parent_a;
  int64_t *parent_b;
  int64_t cand_capacity;
  int64_t elem_capacity;
  int64_t n_candidates;
  int64_t n_elements;
} lsm_gpu_elem_out;
int libsupermesh_gpu_supermesh_elements(lsm_gpu_context *ctx, const lsm_gpu_mesh *a,
                                        const lsm_gpu_mesh *b, int on_device,
                                        lsm_gpu_elem_out *out, lsm_gpu_stats *stats,
                                        void *stream);

/* Narrow phase alone: intersect and measure every candidate of the last
 * libsupermesh_gpu_find_candidates / libsupermesh_gpu_supermesh call on
 * this context (simplex meshes), as libsupermesh_gpu_supermesh does after
 * its search.  Lets callers time or repeat the clipping without the
 * search. */
int libsupermesh_gpu_clip_candidates(lsm_gpu_context *ctx, lsm_gpu_stats *stats, void *stream);

/* As libsupermesh_gpu_clip_candidates, taking the candidates in the order
 * given by `order` (a permutation of 0 .. n_candidates-1, e.g. a schedule that
 * groups pairs of similar cost into the same warps).  The results, stored
 * per candidate, do not depend on the order. */
int libsupermesh_gpu_clip_candidates_ordered(lsm_gpu_context *ctx, const int32_t *order, int on_device,
                                             lsm_gpu_stats *stats, void *stream);

/* Per-pair results of the last libsupermesh_gpu_supermesh call, in CSR
 * order: measure[n_candidates] and n_out[n_candidates]. */
int libsupermesh_gpu_get_pair_results(lsm_gpu_context *ctx, double *measure,
                                      int32_t *n_out, int on_device, void *stream);

/* Batched form of the per-pair C API.  tri: a, b [n][3][2]; tet: a, b
 * [n][4][3].  measure[n] = sum of output simplex measures, n_out[n] = number
 * of output simplices; elems (optional) [n][22][3][2] or [n][81][4][3] in
 * the reference's output order (slots past a pair's n_out are left
 * unspecified).  Tet batches of 2048 pairs or more run through per-pair
 * setup, the exact early-out pass and the index clipper; smaller ones through
 * a one-launch clipper (same results).  With on_device = 1 and dim = 3, a, b
 * and elems must be 16-byte aligned (tetrahedra are read and written with
 * 16-byte accesses); other pointers return LSM_ERROR_INVALID_ARGUMENT before
 * any launch. */
int libsupermesh_gpu_intersect_pairs(lsm_gpu_context *ctx, int dim, int64_t n,
                                     const double *a, const double *b,
                                     double *measure, int32_t *n_out,
                                     double *elems, int on_device, void *stream);

/* Mixed element pairs, batched: the per-pair entries libsupermesh_intersect_
 * intervals, _tri_quad and _tet_hex (C_bindings.F90:42-64, :113-125).
 *   LSM_PAIR_INTERVALS  a, b [n][2]         elems [n][1][2]
 *   LSM_PAIR_TRI_QUAD   a [n][3][2], b [n][4][2]   elems [n][46][3][2]
 *   LSM_PAIR_TET_HEX    a [n][4][3], b [n][8][3] (Gmsh hexahedron node
 *                       order)          elems [n][729][4][3]
 *   LSM_PAIR_QUAD_QUAD  a, b [n][4][2]  elems [n][62][3][2]   (intersect_quads,
 *                       Supermesh.F90:230-246)
 *   LSM_PAIR_HEX_HEX    a, b [n][8][3]  elems [n][3645][4][3] (intersect_hexes,
 *                       Supermesh.F90:303-334: A sliced into five tets)
 * measure[n] = sum of output measures, n_out[n] = number of outputs, elems
 * optional, in the reference's output order.  With on_device = 1 and kind
 * LSM_PAIR_TET_HEX, a and elems must be 16-byte aligned (as for
 * libsupermesh_gpu_intersect_pairs).  Batches of 2048 pairs or more of
 * LSM_PAIR_TET_HEX and LSM_PAIR_HEX_HEX (the latter when elems is NULL or
 * 16-byte aligned) run through the exact early-out pass and the six-plane
 * index clipper; smaller ones through a one-launch clipper, with identical
 * results. */
enum {
  LSM_PAIR_INTERVALS = 0,
  LSM_PAIR_TRI_QUAD = 1,
  LSM_PAIR_TET_HEX = 2,
  LSM_PAIR_QUAD_QUAD = 3,
  LSM_PAIR_HEX_HEX = 4
};
int libsupermesh_gpu_intersect_pairs_mixed(lsm_gpu_context *ctx, int kind, int64_t n,
                                           const double *a, const double *b,
                                           double *measure, int32_t *n_out,
                                           double *elems, int on_device, void *stream);

/* P1-P1 mixed mass matrix over the supermesh of A and B: per candidate pair
 * the local block M[i][j] = sum_c |c| sum_q w_q phi_i^A(x_q) phi_j^B(x_q)
 * (blocks, optional, [n_candidates][loc][loc], device memory only when
 * on_device), and integral = u_a^T M v_b (u_a [nnodes_a], v_b [nnodes_b],
 * optional).  Quadrature as test_parallel_p1_inner_product_{2d,3d}.F90. */
int libsupermesh_gpu_p1_mass(lsm_gpu_context *ctx, const lsm_gpu_mesh *a,
                             const lsm_gpu_mesh *b, const double *u_a,
                             const double *v_b, double *blocks, double *integral,
                             int on_device, void *stream);

/* P2 inner product over the supermesh of two 2D triangle meshes, as
 * test_parallel_p2_inner_product_2d.F90:398-522: P2 fields f_a, f_b given by
 * element-node lists [nelements][6] (vertices 1-3, then the midpoints of edges
 * 1-2, 2-3, 1-3; same index width as the meshes) and node values; for every
 * supermesh triangle c both fields are interpolated at c's vertices and edge
 * midpoints with the P2 basis of their own element and 2 |c| f_b . (M f_a) is
 * added, M the P2 mass matrix of the unit triangle.  integral / area receive
 * the compensated totals; pair_values (optional, [n_candidates], CSR order)
 * each candidate pair's contribution. */
int libsupermesh_gpu_p2_inner_product(lsm_gpu_context *ctx, const lsm_gpu_mesh *a,
                                      const lsm_gpu_mesh *b, const void *enlist_p2_a,
                                      const double *field_a, int64_t nnodes_p2_a,
                                      const void *enlist_p2_b, const double *field_b,
                                      int64_t nnodes_p2_b, double *pair_values, double *integral,
                                      double *area, int on_device, void *stream);

/* Learned scheduler of the 3D clipper (north-star pattern: a small BF16 MLP
 * predicts each surviving candidate pair's output-size class -- 0: no tets,
 * 1: 1-3, 2: 4-7, 3: 8 or more, the n_tets_c of intersect_tets_real,
 * Tetrahedron_Intersection.F90:137-179 -- and is used only to order the
 * clipper's work; every pair is still clipped exactly).  No counterpart in
 * the reference.  Network 24 -> 64 -> 64 -> 4 (ReLU), BF16 weights, FP32
 * accumulation on the tensor cores.  Parameters: LSM_SCHED_PARAMS FP32
 * values, row-major [out][in] blocks W1 [64][32] (inputs 24..31 are padding),
 * b1 [64], W2 [64][64], b2 [64], W3 [8][64] (rows 4..7 padding), b3 [8].
 * Features: LSM_SCHED_FEATURES BF16 per pair, A's then B's four vertices
 * (x, y, z) minus the mean of the eight, divided by the longest of the
 * twelve edges; 24..31 zero.  All buffers below are device memory of the
 * context's GPU, features 16-byte aligned. */
#define LSM_SCHED_PARAMS 6792
#define LSM_SCHED_FEATURES 32
/* Load weights for tet_schedule 1 (params host or device memory). */
int libsupermesh_gpu_sched_set_weights(lsm_gpu_context *ctx, const float *params, int on_device);
/* Training samples from the last plain 3D narrow phase: the features of the
 * first min(cap, survivors) pairs the early-out pass left for the clipper
 * and the class of the clipper's output count; *n = survivors. */
int libsupermesh_gpu_sched_samples(lsm_gpu_context *ctx, int64_t cap, void *features, int8_t *classes,
                                   int64_t *n, void *stream);
/* Inference: logits[n][4] (optional) and classes[n] of feature rows. */
int libsupermesh_gpu_sched_predict(lsm_gpu_context *ctx, int64_t n, const void *features, float *logits,
                                   int8_t *classes, void *stream);
/* Training: `steps` Adam steps (betas 0.9 / 0.999; learning rate decayed
 * from lr to 0 along a half cosine) on the softmax
 * cross-entropy, minibatches of 128 consecutive rows (row (128 step + i) mod
 * n: shuffle the samples first).  params (in: initial, out: trained);
 * loss_trace (optional) the minibatch loss of every trace_every-th step;
 * grad_first (optional, LSM_SCHED_PARAMS) the gradient of the first
 * minibatch.  Forward and backward products run on the tensor cores. */
int libsupermesh_gpu_sched_train(lsm_gpu_context *ctx, int64_t n, const void *features,
                                 const int8_t *classes, float *params, int steps, float lr,
                                 float *loss_trace, int trace_every, float *grad_first, void *stream);

/* Many independent mesh pairs in one call.  totals[npairs] receives each
 * pair's supermesh measure
 * and n_candidates[npairs] / n_intersecting[npairs] (optional) its counts.
 * All meshes live in the memory space given by on_device.  Host meshes are
 * copied in per dimension group; the 3D group's copies run on the context's
 * second stream while the 2D group computes (pinned host memory lets them
 * overlap).  The call returns with all its work on the device done. */
int libsupermesh_gpu_supermesh_batched(lsm_gpu_context *ctx, int npairs,
                                       const lsm_gpu_mesh *a, const lsm_gpu_mesh *b,
                                       int on_device, double *totals,
                                       int64_t *n_candidates, int64_t *n_intersecting,
                                       void *stream);

/* Batched supermesh with per-pair outputs: what a caller of the drop-in C
 * API gets from one set_input / get_output round and the per-candidate
 * intersect_*_real + measure calls, for every mesh pair of the batch (the
 * loop of test_tri_intersector.F90:89-104 and C_bindings.F90:377-391, many
 * mesh pairs at once).  No counterpart in the reference.
 *   totals, n_candidates, n_intersecting  [npairs], host (optional)
 *   cand_offset     [npairs], host (optional): first entry of pair i in the
 *                   per-candidate arrays, or -1 if they could not hold it
 *   total_candidates host (optional): entries written to them
 *   ind_ptr         [sum_i (nelements_a(i) + 1)] (optional): pair i's CSR row
 *                   pointers at offset sum_{j<i} (nelements_a(j) + 1),
 *                   starting at 0 (get_output semantics)
 *   indices         [cand_capacity] (optional): 0-based B element of the pair
 *   pair_measure    [cand_capacity] (optional): measure of each candidate
 *   pair_n_out      [cand_capacity] (optional): its number of output simplices
 *   p1_blocks       [p1_capacity] doubles (optional): for every candidate its
 *                   P1-P1 mixed mass block (loc x loc, row-major, loc = dim + 1;
 *                   the integrand of test_parallel_p1_inner_product_{2d,3d}),
 *                   pair i's blocks from p1_offset[i] (host, [npairs]) on
 * ind_ptr, indices, pair_measure, pair_n_out and p1_blocks follow on_device.
 * Each pair's candidates are contiguous and in its CSR order; 2D pairs come
 * before 3D pairs in the arrays.  If they need more than cand_capacity
 * entries (or p1_capacity doubles) the call still fills totals, counts and
 * ind_ptr, sets cand_offset / p1_offset of the pairs that did not fit to -1
 * and returns LSM_ERROR_CAPACITY: retry with capacity >= the sum of
 * n_candidates (p1: the sum of n_candidates(i) * (dim(i) + 1)^2). */
typedef struct {
  double *totals;
  int64_t *n_candidates;
  int64_t *n_intersecting;
  int64_t *cand_offset;
  int64_t *total_candidates;
  int64_t cand_capacity;
  int64_t *ind_ptr;
  int64_t *indices;
  double *pair_measure;
  int32_t *pair_n_out;
  int64_t *p1_offset;
  int64_t p1_capacity;
  double *p1_blocks;
} lsm_gpu_batch_out;
int libsupermesh_gpu_supermesh_batched_ex(lsm_gpu_context *ctx, int npairs,
                                          const lsm_gpu_mesh *a, const lsm_gpu_mesh *b,
                                          int on_device, lsm_gpu_batch_out *out, void *stream);

/* Allocation-free clipping of explicit tetrahedron pairs (no counterpart in
 * the reference).  For callers that cannot let a library allocate device
 * memory: applications whose GPU memory is owned by another pool allocator,
 * and stream-overlapped loops where cudaFree's implicit device-wide
 * synchronisation would serialise other work.  Same results as
 * libsupermesh_gpu_intersect_pairs (dim 3) for measure[n] and n_out[n]; total
 * (host, optional) receives the compensated sum of measure; it makes the call
 * wait for its stream (cudaStreamSynchronize), so a call issued inside stream
 * capture must pass total = NULL and sum measure itself.  tet_a, tet_b
 * ([n][4][3], 16-byte aligned), measure and n_out are device memory;
 * n <= LSM_NOALLOC_MAX_PAIRS (larger n returns LSM_ERROR_CAPACITY, a
 * misaligned tet_a or tet_b LSM_ERROR_INVALID_ARGUMENT, each with a message
 * on stderr).
 * Scratch lives in one fixed device array of LSM_NOALLOC_SCRATCH_BYTES that
 * every GPU loading the library holds until exit; the first call on a device
 * looks up its address (make that first call before any stream capture).
 * All calls share the array, so calls that overlap on the GPU race. */
#define LSM_NOALLOC_MAX_PAIRS 32768
#define LSM_NOALLOC_SCRATCH_BYTES 6193664
int libsupermesh_gpu_intersect_tets_noalloc(int64_t n, const double *tet_a, const double *tet_b,
                                            double *measure, int32_t *n_out, double *total,
                                            void *stream);

#ifdef __cplusplus
}
#endif

#endif
