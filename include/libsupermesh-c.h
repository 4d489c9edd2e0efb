/*
 * Drop-in C API of the B200 supermesh library.  The declarations are those
 * of firedrakeproject/libsupermesh include/libsupermesh-c.h:1-46 (same
 * names, argument order, pointer-only Fortran bind(c) passing and buffer
 * sizes), so that existing C callers and ctypes loaders link unchanged.
 * Each entry runs on the GPU; see libsupermesh-gpu.h for batched and
 * device-resident entry points.
 *
 * Semantics kept from the reference (C_bindings.F90):
 *   - enlist arrays are 0-based `long`; positions are [nnodes][dim];
 *   - the tree finder is a set_input -> query_output -> get_output state
 *     machine over one global result (:346-391); get_output copies the
 *     0-based CSR over A rows into caller buffers and releases the state;
 *   - every entry returns void; invalid input and device failures print a
 *     message to stderr and terminate the process, as libsupermesh_abort
 *     does (Debug.F90:78-94);
 *   - calls are serialised by a process-wide lock (the reference keeps
 *     module-level state and is not reentrant).
 * Row order inside the CSR follows the GPU search structure, not the
 * reference's quadtree; the set of indices per row is the same.
 */
#ifndef LIBSUPERMESH_C_H
#define LIBSUPERMESH_C_H

#include "libsupermesh.h"

#define TRI_BUF_SIZE 22 /* Triangle_Intersection.F90:56 */
#define TET_BUF_SIZE 81 /* Tetrahedron_Intersection.F90:56 */

#ifdef LIBSUPERMESH_DOUBLE_PRECISION
typedef double c_kind;
#else
typedef float c_kind;
#endif

#ifdef __cplusplus
#include <cmath>
extern "C" {
#else
#include <math.h>
#endif

/* 1D sort finder (C_bindings.F90:66-111; Intersection_Finder.F90:811-921):
 * 2-node elements, first coordinate of each node, sort by left end then one
 * sweep, on the GPU.  Shares the tree finder's result state, as the
 * reference's module arrays do.  Rows list B elements in sweep order
 * (ascending left end, ties by element number).  The sort is the stable sort
 * by left end; the reference's merge sort gives the same order whenever each
 * block of at most 4 elements it sorts directly is already in order (true
 * for meshes numbered along the line); otherwise its output can repeat and
 * lose elements, which this build does not reproduce. */
void libsupermesh_sort_intersection_finder_set_input(long *nnodes_a, int *dim_a, long *nelements_a, int *loc_a,
                                                     long *nnodes_b, int *dim_b, long *nelements_b, int *loc_b,
                                                     c_kind *positions_a, long *enlist_a, c_kind *positions_b,
                                                     long *enlist_b);
void libsupermesh_sort_intersection_finder_query_output(long *nindices);
void libsupermesh_sort_intersection_finder_get_output(long *nelements, long *nindices, long *indices, long *ind_ptr);

/* Tree finder (C_bindings.F90:346-391): 2D quadtree / 3D octree candidate
 * set, computed on the GPU by an LBVH with the same strict box test. */
void libsupermesh_tree_intersection_finder_set_input(long *nnodes_a, int *dim_a, long *nelements_a, int *loc_a,
                                                     long *nnodes_b, int *dim_b, long *nelements_b, int *loc_b,
                                                     c_kind *positions_a, long *enlist_a, c_kind *positions_b,
                                                     long *enlist_b);
void libsupermesh_tree_intersection_finder_query_output(long *nindices);
void libsupermesh_tree_intersection_finder_get_output(long *nelements, long *nindices, long *indices, long *ind_ptr);

/* Single-pair intersections and measures (C_bindings.F90:134-174). */
void libsupermesh_intersect_tris_real(c_kind *tri_a, c_kind *tri_b, c_kind *tris_c, int *n_tris_c);
void libsupermesh_intersect_tets_real(c_kind *tet_a, c_kind *tet_b, c_kind *tets_c, int *n_tets_c);
void libsupermesh_triangle_area(c_kind *tri, c_kind *area);
void libsupermesh_tetrahedron_volume(c_kind *tet, c_kind *volume);

/* 1D and mixed-element entries (C_bindings.F90:42-64, 113-132), on the GPU:
 * intervals (Interval_Intersection.F90), triangle vs quadrilateral
 * (Supermesh.F90:211-228, <= 46 output triangles) and tetrahedron vs
 * Gmsh-ordered hexahedron (Supermesh.F90:248-295, <= 729 output tets). */
void libsupermesh_interval_size(c_kind *interval, c_kind *size);
void libsupermesh_intersect_intervals(c_kind *interval_a, c_kind *interval_b, c_kind *intervals_c, int *n_intervals_c);
void libsupermesh_intersect_tet_hex(c_kind *tet_a, c_kind *hex_b, c_kind *tets_c, int *n_tets_c);
void libsupermesh_intersect_tri_quad(c_kind *tri_a, c_kind *quad_b, c_kind *tris_c, int *n_tris_c);

#ifdef __cplusplus
}
#endif

/* Output-buffer bounds (libsupermesh-c.h:33-41 upstream). */
static int libsupermesh_max_n_tris_c(int n_lines_b, int n_lines_a) {
  int out = n_lines_a * pow(2, n_lines_b) - 2;
  return out;
}

static int libsupermesh_max_n_tets_c(int n_planes_b) {
  int out = pow(3, n_planes_b);
  return out;
}

#endif
