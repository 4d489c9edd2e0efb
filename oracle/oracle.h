/*
 * CPU oracle for the supermesh hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64, FMA-free restatement of libsupermesh's serial hot path,
 * used solely as the checker in tests/, in __graft_entry__.smoke() and as the
 * timed CPU baseline in bench.py.  Nothing in the shipped library links it.
 *
 * Restated reference code (paths within firedrakeproject/libsupermesh):
 *   src/Triangle_Intersection.F90     intersect_tris_tri (:144-185), clip_buf
 *                                     (:282-335), get_lines_tri (:395-420),
 *                                     triangle_area (:453-477)
 *   src/Tetrahedron_Intersection.F90  intersect_tets_planes (:137-179),
 *                                     clip_buf (:244-436), get_planes_tet
 *                                     (:634-667), unit_cross (:669-677),
 *                                     distances_to_plane (:679-688),
 *                                     tetrahedron_volume_{real,tet} (:690-725)
 *   src/Quadtree_Intersection_Finder.F90 / src/Octree_Intersection_Finder.F90
 *                                     max_nelist_degree, allocate_node,
 *                                     add_element, query_node_internal, bbox,
 *                                     bboxes_intersect
 *   src/Intersection_Finder.F90       brute_force finder (:989-1077), sort
 *                                     finder (:811-921)
 *   src/Triangle_Intersection.F90     intersect_polys / get_lines_poly
 *                                     (:187-239, :422-451) for tri vs quad
 *   src/Supermesh.F90                 intersect_tet_hex (:248-295),
 *                                     intersect_quads (:230-246),
 *                                     intersect_hexes (:303-334)
 *   src/Interval_Intersection.F90     intersect_intervals, interval_size
 *   src/Intersections.F90:48-71       ragged -> CSR
 *   src/Precision.F90:72-113          Kahan compensated sum
 *   src/tests/test_parallel_p1_inner_product_{2d,3d}.F90  P1 quadrature
 *   src/tests/test_parallel_p2_inner_product_2d.F90      P2 interpolation
 *
 * Parity is pinned against the reference's own known answers and fixtures
 * (tests/test_oracle_pins.py).  The reference itself is Fortran 2008 + MPI and
 * cannot be compiled in this environment (no Fortran compiler), so no
 * reference binary backs the pin.
 */
#ifndef SUPERMESH_ORACLE_H
#define SUPERMESH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_TRI_BUF 22
#define ORC_TET_BUF 81

/* Fortran intrinsics on real64 */
double orc_spacing(double x);
double orc_norm2_3(const double v[3]);

/* Element measures; tri = [3][2], tet = [4][3] (vertex-major). */
double orc_triangle_area(const double tri[6]);
double orc_tetrahedron_volume(const double tet[12]);    /* vertex-1 based */
double orc_tetrahedron_volume_v4(const double tet[12]); /* vertex-4 based */

/* Single-pair intersections (tris_c: [22][3][2]; tets_c: [81][4][3]). */
void orc_intersect_tris(const double tri_a[6], const double tri_b[6],
                        double *tris_c, int *n_tris_c);
void orc_intersect_tets(const double tet_a[12], const double tet_b[12],
                        double *tets_c, int *n_tets_c);

/* Mixed pairs: tri vs quad ([3][2] x [4][2] -> <= 46 tris [46][3][2]); tet
 * vs hex in Gmsh order ([4][3] x [8][3] -> <= 729 tets); quad vs quad (<= 62
 * tris); hex vs hex (<= 5 * 729 tets); intervals. */
void orc_intersect_tri_quad(const double tri_a[6], const double quad_b[8], double *tris_c, int *n_tris_c);
void orc_intersect_tet_hex(const double tet_a[12], const double hex_b[24], double *tets_c, int *n_tets_c);
void orc_intersect_quads(const double quad_a[8], const double quad_b[8], double *tris_c, int *n_tris_c);
void orc_intersect_hexes(const double hex_a[24], const double hex_b[24], double *tets_c, int *n_tets_c);
double orc_interval_size(const double iv[2]);
void orc_intersect_intervals(const double a[2], const double b[2], double *c, int *n);

/* Tree (quadtree/octree) intersection finder.  A = query mesh (CSR rows),
 * B = tree mesh.  enlist is 0-based int32.  On success *indices is malloc'd
 * (free with orc_free) and indptr[nel_a+1] is filled.  Returns 0 on success. */
int orc_tree_finder(int dim, long nnodes_a, const double *pos_a, long nel_a,
                    int loc_a, const int32_t *en_a, long nnodes_b,
                    const double *pos_b, long nel_b, int loc_b,
                    const int32_t *en_b, int max_size, int64_t *indptr,
                    int32_t **indices, int64_t *nnz);
int orc_brute_force_finder(int dim, long nnodes_a, const double *pos_a,
                           long nel_a, int loc_a, const int32_t *en_a,
                           long nnodes_b, const double *pos_b, long nel_b,
                           int loc_b, const int32_t *en_b, int64_t *indptr,
                           int32_t **indices, int64_t *nnz);
/* 1D sort finder over 2-node elements; the first coordinate of each node is
 * read with stride `stride_*`.  stable_leaf selects the stable sort instead
 * of the reference's merge sort leaf step (see oracle.c). */
int orc_sort_finder_1d(long nnodes_a, const double *pos_a, int stride_a, long nel_a, const int32_t *en_a,
                       long nnodes_b, const double *pos_b, int stride_b, long nel_b, const int32_t *en_b,
                       int stable_leaf, int64_t *indptr, int32_t **indices, int64_t *nnz);
void orc_free(void *p);

/* Narrow phase over a candidate CSR.  Per candidate pair p it writes the
 * number of output simplices (pair_nout) and the measure (pair_measure, the
 * sum of libsupermesh_triangle_area / tetrahedron_volume over the outputs in
 * output order).  elem_measure[nel_a] accumulates per A element (in CSR row
 * order).  Totals are Kahan-compensated over pairs in CSR order.
 * nthreads > 1 parallelises over A rows (OpenMP); totals then combine the
 * per-thread compensated sums.  Any output pointer may be NULL. */
typedef struct {
  int64_t n_candidates;
  int64_t n_intersecting;
  int64_t n_out_simplices;
  double total;
  double total_err;
  double flops; /* algorithmic FP64 operations executed (see oracle.c) */
} orc_stats;

int orc_narrow(int dim, const double *pos_a, int loc_a, const int32_t *en_a,
               long nel_a, const double *pos_b, int loc_b, const int32_t *en_b,
               long nel_b, const int64_t *indptr, const int32_t *indices,
               double *pair_measure, int32_t *pair_nout, double *elem_measure,
               int nthreads, int count_flops, orc_stats *st);

/* Full pipeline as a C-API caller would drive it: tree finder, then
 * intersect + measure for every candidate.  Used for CPU-baseline timing. */
int orc_supermesh(int dim, long nnodes_a, const double *pos_a, long nel_a,
                  int loc_a, const int32_t *en_a, long nnodes_b,
                  const double *pos_b, long nel_b, int loc_b,
                  const int32_t *en_b, int nthreads, orc_stats *st);

/* P1-P1 mixed inner product u_A^T M v_B over the supermesh, following
 * test_parallel_p1_inner_product_{2d,3d}.F90 (2D: Dunavant degree-2 3-point
 * rule; 3D: Stroud 4-point rule).  Also writes per-pair element blocks
 * blocks[nnz][loc_a][loc_b] if non-NULL.  Returns 0 on success. */
int orc_p1_mass(int dim, const double *pos_a, const int32_t *en_a, long nel_a,
                const double *pos_b, const int32_t *en_b, long nel_b,
                const int64_t *indptr, const int32_t *indices,
                const double *u_a, const double *v_b, double *blocks,
                double *integral, double *measure);

/* P2 inner product over the 2D supermesh (test_parallel_p2_inner_product_2d
 * .F90:398-522): P2 fields given by [nel][6] element-node lists (vertices
 * 1-3, then edge midpoints 1-2, 2-3, 1-3) and node values.  pair_values
 * [nnz] (optional) receives each candidate pair's contribution (summed over
 * its supermesh triangles in output order); totals are compensated sums. */
int orc_p2_inner_product(const double *pos_a, const int32_t *en_a, long nel_a, const double *pos_b,
                         const int32_t *en_b, const int64_t *indptr, const int32_t *indices,
                         const int32_t *en_p2_a, const double *field_a, const int32_t *en_p2_b,
                         const double *field_b, double *pair_values, double *integral, double *area);

/* Kahan compensated sum of an array (Precision.F90:72-113). */
double orc_kahan_sum(const double *x, long n);

int orc_num_threads_available(void);

#ifdef __cplusplus
}
#endif

#endif
