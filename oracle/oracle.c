/*
 * CPU oracle for the supermesh hot path -- TEST INFRASTRUCTURE ONLY (the
 * checker for tests/, smoke() and bench.py's cpu_baseline leg; never linked
 * into the product library).  See oracle.h for the list of restated
 * reference routines.  Build with -ffp-contract=off: the reference is built
 * by gfortran for baseline x86-64 (SSE2, no FMA), so every FP64 operation
 * here is a single IEEE-rounded add/sub/mul/div/sqrt in the reference's
 * evaluation order.
 *
 * Fortran semantics mirrored:
 *   dot_product(a, b)  -> ((a1*b1 + a2*b2) + a3*b3)  (left to right)
 *   spacing(x)         -> 2**(exponent(x) - 53), tiny(x) when x == 0
 *   epsilon(x)         -> 2**-52
 *   norm2(v)           -> gfortran's inline scaled sum of squares
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* FLOP accounting: every FP64 +, -, *, /, sqrt executed counts 1;      */
/* abs/min/max/compare/negation count 0.                                */
/* ------------------------------------------------------------------ */
static __thread int tl_count = 0;
static __thread double tl_flops = 0.0;
#define FL(n)                 \
  do {                        \
    if (tl_count) tl_flops += (n); \
  } while (0)

/* ------------------------------------------------------------------ */
/* Fortran intrinsics                                                   */
/* ------------------------------------------------------------------ */
double orc_spacing(double x) {
  /* Fortran SPACING for real64: b**(e-p) with x = f * 2**e, f in [0.5, 1),
   * p = 53; returns TINY (2**-1022) when x == 0 or the result would be
   * subnormal. */
  if (x == 0.0) return DBL_MIN;
  int e;
  (void)frexp(x, &e);
  double s = ldexp(1.0, e - 53);
  if (s < DBL_MIN) return DBL_MIN;
  return s;
}

double orc_norm2_3(const double v[3]) {
  /* gfortran expands NORM2 inline as a scaled sum of squares:
   *   scale = 0, result = 1
   *   for x /= 0: ax = |x|
   *     if (scale < ax) { val = scale/ax; result = 1 + result*(val*val);
   *                       scale = ax }
   *     else           { val = ax/scale; result = result + val*val }
   *   norm = sqrt(result) * scale                                       */
  double scale = 0.0, result = 1.0;
  for (int i = 0; i < 3; ++i) {
    if (v[i] != 0.0) {
      double ax = fabs(v[i]);
      if (scale < ax) {
        double val = scale / ax;
        result = 1.0 + result * (val * val);
        scale = ax;
        FL(4);
      } else {
        double val = ax / scale;
        result = result + val * val;
        FL(3);
      }
    }
  }
  FL(2);
  return sqrt(result) * scale;
}

static const double ORC_EPS = 2.220446049250313080847263336181640625e-16; /* 2**-52 */

/* ------------------------------------------------------------------ */
/* Measures                                                            */
/* ------------------------------------------------------------------ */
double orc_triangle_area(const double t[6]) {
  /* Triangle_Intersection.F90:453-464: u = v3 - v1, v = v2 - v1,
   * area = 0.5 * |u2 v1 - u1 v2| */
  double u0 = t[4] - t[0], u1 = t[5] - t[1];
  double w0 = t[2] - t[0], w1 = t[3] - t[1];
  FL(8);
  return 0.5 * fabs(u1 * w0 - u0 * w1);
}

double orc_tetrahedron_volume(const double t[12]) {
  /* Tetrahedron_Intersection.F90:690-706 (vertex-1 based, the C API). */
  double e1[3], e2[3], e3[3];
  for (int c = 0; c < 3; ++c) {
    e1[c] = t[3 + c] - t[c];
    e2[c] = t[6 + c] - t[c];
    e3[c] = t[9 + c] - t[c];
  }
  double s = e1[0] * (e2[1] * e3[2] - e2[2] * e3[1]) +
             e1[1] * (e2[2] * e3[0] - e2[0] * e3[2]);
  s = s + e1[2] * (e2[0] * e3[1] - e2[1] * e3[0]);
  FL(24);
  return (1.0 / 6.0) * fabs(s);
}

double orc_tetrahedron_volume_v4(const double t[12]) {
  /* Tetrahedron_Intersection.F90:708-725 (vertex-4 based; used inside the
   * clipping tolerance). */
  double a[3], b[3], c[3], x[3];
  for (int k = 0; k < 3; ++k) {
    a[k] = t[k] - t[9 + k];
    b[k] = t[3 + k] - t[9 + k];
    c[k] = t[6 + k] - t[9 + k];
  }
  x[0] = b[1] * c[2] - b[2] * c[1];
  x[1] = b[2] * c[0] - b[0] * c[2];
  x[2] = b[0] * c[1] - b[1] * c[0];
  double d = (a[0] * x[0] + a[1] * x[1]) + a[2] * x[2];
  FL(24);
  return fabs(d) / 6.0;
}

/* ------------------------------------------------------------------ */
/* Triangle clipping (Triangle_Intersection.F90:144-185, 282-335, 395-420) */
/* ------------------------------------------------------------------ */
typedef struct {
  double n[2];
  double p[2];
} orc_line;

static void get_lines_tri(const double v[6], orc_line L[3]) {
  L[0].n[0] = -(v[3] - v[1]);
  L[0].n[1] = (v[2] - v[0]);
  L[0].p[0] = v[0];
  L[0].p[1] = v[1];
  L[1].n[0] = -(v[5] - v[3]);
  L[1].n[1] = (v[4] - v[2]);
  L[1].p[0] = v[2];
  L[1].p[1] = v[3];
  L[2].n[0] = -(v[1] - v[5]);
  L[2].n[1] = (v[0] - v[4]);
  L[2].p[0] = v[4];
  L[2].p[1] = v[5];
  double dot = (v[2] - v[0]) * L[2].n[0] + (v[3] - v[1]) * L[2].n[1];
  FL(11);
  if (dot > 0.0) {
    for (int i = 0; i < 3; ++i) {
      L[i].n[0] = -L[i].n[0];
      L[i].n[1] = -L[i].n[1];
    }
  }
}

#define ORC_PBUF (ORC_TRI_BUF + 2)

/* One Sutherland-Hodgman pass; returns the output vertex count. */
static int clip_buf_tri(const orc_line *L, const double *pts, int n,
                        double *out) {
  double d[64]; /* polygons of up to 48 vertices (tri vs quad) */
  for (int i = 0; i < n; ++i) {
    d[i] = L->n[0] * (pts[2 * i] - L->p[0]) + L->n[1] * (pts[2 * i + 1] - L->p[1]);
  }
  FL(5 * n);
  int m = 0;
  for (int i = 0; i < n; ++i) {
    const double *p1 = pts + 2 * i;
    double d1 = d[i];
    const double *p2;
    double d2;
    if (i == n - 1) {
      p2 = pts;
      d2 = d[0];
    } else {
      p2 = pts + 2 * (i + 1);
      d2 = d[i + 1];
    }
    if (d1 < 0.0) {
      if (d2 <= 0.0) {
        out[2 * m] = p1[0];
        out[2 * m + 1] = p1[1];
        ++m;
      } else {
        out[2 * m] = p1[0];
        out[2 * m + 1] = p1[1];
        ++m;
        double f = fabs(d1) / (fabs(d1) + fabs(d2));
        f = fmax(fmin(f, 1.0), 0.0);
        out[2 * m] = p1[0] + f * (p2[0] - p1[0]);
        out[2 * m + 1] = p1[1] + f * (p2[1] - p1[1]);
        ++m;
        FL(8);
      }
    } else if (d1 == 0.0) {
      out[2 * m] = p1[0];
      out[2 * m + 1] = p1[1];
      ++m;
    } else if (d2 < 0.0) {
      double f = fabs(d1) / (fabs(d1) + fabs(d2));
      f = fmax(fmin(f, 1.0), 0.0);
      out[2 * m] = p1[0] + f * (p2[0] - p1[0]);
      out[2 * m + 1] = p1[1] + f * (p2[1] - p1[1]);
      ++m;
      FL(8);
    }
  }
  return m;
}

/* Clip with precomputed lines and tolerance; writes the fan triangles. */
static int intersect_tris_lines(const double tri_a[6], const orc_line L[3],
                                double tol, double *tris_c) {
  double pa[2 * ORC_PBUF], pb[2 * ORC_PBUF];
  memcpy(pa, tri_a, 6 * sizeof(double));
  int n = clip_buf_tri(&L[0], pa, 3, pb);
  if (n < 3) return 0;
  n = clip_buf_tri(&L[1], pb, n, pa);
  if (n < 3) return 0;
  n = clip_buf_tri(&L[2], pa, n, pb);
  if (n < 3) return 0;
  int nt = 0;
  for (int i = 0; i < n - 2; ++i) {
    double *t = tris_c + 6 * nt;
    t[0] = pb[0];
    t[1] = pb[1];
    t[2] = pb[2 * (i + 1)];
    t[3] = pb[2 * (i + 1) + 1];
    t[4] = pb[2 * (i + 2)];
    t[5] = pb[2 * (i + 2) + 1];
    if (!(orc_triangle_area(t) < tol)) ++nt;
  }
  return nt;
}

void orc_intersect_tris(const double tri_a[6], const double tri_b[6],
                        double *tris_c, int *n_tris_c) {
  orc_line L[3];
  get_lines_tri(tri_b, L);
  double tol = 10.0 * fmin(orc_spacing(orc_triangle_area(tri_a)),
                           orc_spacing(orc_triangle_area(tri_b)));
  *n_tris_c = intersect_tris_lines(tri_a, L, tol, tris_c);
}

/* ------------------------------------------------------------------ */
/* Tetrahedron clipping (Tetrahedron_Intersection.F90:137-179, 244-436,   */
/* 634-688)                                                             */
/* ------------------------------------------------------------------ */
typedef struct {
  double n[3];
  double c;
} orc_plane;

static void unit_cross(const double a[3], const double b[3], double out[3]) {
  out[0] = a[1] * b[2] - a[2] * b[1];
  out[1] = a[2] * b[0] - a[0] * b[2];
  out[2] = a[0] * b[1] - a[1] * b[0];
  FL(9);
  double nrm = orc_norm2_3(out);
  out[0] = out[0] / nrm;
  out[1] = out[1] / nrm;
  out[2] = out[2] / nrm;
  FL(3);
}

static void get_planes_tet(const double v[12], orc_plane P[4]) {
  double e10[3], e20[3], e30[3], e21[3], e31[3];
  for (int c = 0; c < 3; ++c) {
    e10[c] = v[3 + c] - v[c];
    e20[c] = v[6 + c] - v[c];
    e30[c] = v[9 + c] - v[c];
    e21[c] = v[6 + c] - v[3 + c];
    e31[c] = v[9 + c] - v[3 + c];
  }
  FL(15);
  unit_cross(e20, e10, P[0].n);
  unit_cross(e10, e30, P[1].n);
  unit_cross(e30, e20, P[2].n);
  unit_cross(e21, e31, P[3].n);
  double det = (e10[0] * P[3].n[0] + e10[1] * P[3].n[1]) + e10[2] * P[3].n[2];
  FL(5);
  if (det < 0.0) {
    for (int i = 0; i < 4; ++i)
      for (int c = 0; c < 3; ++c) P[i].n[c] = -P[i].n[c];
  }
  for (int i = 0; i < 4; ++i) {
    P[i].c = (v[3 * i] * P[i].n[0] + v[3 * i + 1] * P[i].n[1]) +
             v[3 * i + 2] * P[i].n[2];
  }
  FL(20);
}

/* w0 * v[pos] + w1 * v[neg] with invdiff = 1/(d_pos - d_neg),
 * w0 = -d_neg*invdiff, w1 = d_pos*invdiff. */
static void interp(const double *vp, const double *vn, double dp, double dn,
                   double *out) {
  double invdiff = 1.0 / (dp - dn);
  double w0 = -dn * invdiff;
  double w1 = dp * invdiff;
  for (int c = 0; c < 3; ++c) out[c] = w0 * vp[c] + w1 * vn[c];
  FL(13);
}

static void set_v(double *t, int k, const double *p) {
  t[3 * k] = p[0];
  t[3 * k + 1] = p[1];
  t[3 * k + 2] = p[2];
}

/* Clip one tet by one plane, appending 0..3 tets to out; returns count. */
static int clip_buf_tet(const orc_plane *P, const double *tet, double *out) {
  double d[4];
  int neg[4], pos[4], zer[4];
  int nn = 0, np = 0, nz = 0;
  for (int i = 0; i < 4; ++i) {
    d[i] = ((P->n[0] * tet[3 * i] + P->n[1] * tet[3 * i + 1]) +
            P->n[2] * tet[3 * i + 2]) - P->c;
  }
  FL(24);
  for (int i = 0; i < 4; ++i) {
    if (fabs(d[i]) < ORC_EPS)
      zer[nz++] = i;
    else if (d[i] < 0.0)
      neg[nn++] = i;
    else if (d[i] > 0.0)
      pos[np++] = i;
  }
  if (nn == 0) return 0;
  if (np == 0) {
    memcpy(out, tet, 12 * sizeof(double));
    return 1;
  }
  double tmp[4][3];
  if (np == 3) { /* +++- */
    memcpy(out, tet, 12 * sizeof(double));
    for (int i = 0; i < 3; ++i) {
      double p[3];
      interp(out + 3 * pos[i], out + 3 * neg[0], d[pos[i]], d[neg[0]], p);
      set_v(out, pos[i], p);
    }
    return 1;
  }
  if (np == 2) {
    if (nn == 2) { /* ++-- */
      for (int i = 0; i < 2; ++i)
        interp(tet + 3 * pos[i], tet + 3 * neg[0], d[pos[i]], d[neg[0]], tmp[i]);
      for (int i = 0; i < 2; ++i)
        interp(tet + 3 * pos[i], tet + 3 * neg[1], d[pos[i]], d[neg[1]],
               tmp[i + 2]);
      double *o1 = out, *o2 = out + 12, *o3 = out + 24;
      memcpy(o1, tet, 12 * sizeof(double));
      set_v(o1, pos[0], tmp[2]);
      set_v(o1, pos[1], tmp[1]);
      set_v(o2, 0, tet + 3 * neg[1]);
      set_v(o2, 1, tmp[3]);
      set_v(o2, 2, tmp[2]);
      set_v(o2, 3, tmp[1]);
      set_v(o3, 0, tet + 3 * neg[0]);
      set_v(o3, 1, tmp[0]);
      set_v(o3, 2, tmp[1]);
      set_v(o3, 3, tmp[2]);
      return 3;
    }
    /* ++-0 */
    memcpy(out, tet, 12 * sizeof(double));
    for (int i = 0; i < 2; ++i) {
      double p[3];
      interp(out + 3 * pos[i], out + 3 * neg[0], d[pos[i]], d[neg[0]], p);
      set_v(out, pos[i], p);
    }
    return 1;
  }
  /* np == 1 */
  if (nn == 3) { /* +--- */
    for (int i = 0; i < 3; ++i)
      interp(tet + 3 * pos[0], tet + 3 * neg[i], d[pos[0]], d[neg[i]], tmp[i]);
    double *o1 = out, *o2 = out + 12, *o3 = out + 24;
    memcpy(o1, tet, 12 * sizeof(double));
    set_v(o1, pos[0], tmp[0]);
    set_v(o2, 0, tmp[0]);
    set_v(o2, 1, tet + 3 * neg[1]);
    set_v(o2, 2, tet + 3 * neg[2]);
    set_v(o2, 3, tmp[1]);
    set_v(o3, 0, tet + 3 * neg[2]);
    set_v(o3, 1, tmp[1]);
    set_v(o3, 2, tmp[2]);
    set_v(o3, 3, tmp[0]);
    return 3;
  }
  if (nn == 2) { /* +--0 */
    for (int i = 0; i < 2; ++i)
      interp(tet + 3 * pos[0], tet + 3 * neg[i], d[pos[0]], d[neg[i]], tmp[i]);
    double *o1 = out, *o2 = out + 12;
    memcpy(o1, tet, 12 * sizeof(double));
    set_v(o1, pos[0], tmp[0]);
    set_v(o2, 0, tmp[1]);
    set_v(o2, 1, tet + 3 * zer[0]);
    set_v(o2, 2, tet + 3 * neg[1]);
    set_v(o2, 3, tmp[0]);
    return 2;
  }
  /* +-00 */
  {
    double p[3];
    interp(tet + 3 * pos[0], tet + 3 * neg[0], d[pos[0]], d[neg[0]], p);
    memcpy(out, tet, 12 * sizeof(double));
    set_v(out, pos[0], p);
    return 1;
  }
}

/* Breadth-first clip of tet_a by the 4 planes, exactly as
 * intersect_tets_planes; keeps final tets with vol_v4 >= tol. */
static int intersect_tets_planes(const double tet_a[12], const orc_plane P[4],
                                 double tol, double *tets_c) {
  double buf[ORC_TET_BUF * 12];
  int n = 1;
  memcpy(tets_c, tet_a, 12 * sizeof(double));
  for (int i = 0; i < 4; ++i) {
    int m = 0;
    for (int j = 0; j < n; ++j) m += clip_buf_tet(&P[i], tets_c + 12 * j, buf + 12 * m);
    if (i != 3) {
      n = m;
      memcpy(tets_c, buf, (size_t)n * 12 * sizeof(double));
    } else {
      n = 0;
      for (int j = 0; j < m; ++j) {
        double vol = orc_tetrahedron_volume_v4(buf + 12 * j);
        if (vol >= tol) {
          memcpy(tets_c + 12 * n, buf + 12 * j, 12 * sizeof(double));
          ++n;
        }
      }
    }
  }
  return n;
}

void orc_intersect_tets(const double tet_a[12], const double tet_b[12],
                        double *tets_c, int *n_tets_c) {
  orc_plane P[4];
  get_planes_tet(tet_b, P);
  double vol_b = orc_tetrahedron_volume_v4(tet_b);
  double tol = 10.0 * fmin(orc_spacing(orc_tetrahedron_volume_v4(tet_a)),
                           orc_spacing(vol_b));
  *n_tets_c = intersect_tets_planes(tet_a, P, tol, tets_c);
}

/* ------------------------------------------------------------------ */
/* Mixed element pairs and intervals (Supermesh.F90:211-301,            */
/* Triangle_Intersection.F90:216-276, 422-451,                          */
/* Tetrahedron_Intersection.F90:190-242, Interval_Intersection.F90)     */
/* ------------------------------------------------------------------ */
static void get_lines_poly(const double *v, int loc, orc_line *L) {
  /* get_lines_poly: normal (y_{i+1}-y_i, -(x_{i+1}-x_i)), point v_i;
   * flipped when (v_1 - p_2) . n_2 > 0 */
  for (int i = 0; i < loc; ++i) {
    int j = (i + 1) % loc;
    L[i].n[0] = (v[2 * j + 1] - v[2 * i + 1]);
    L[i].n[1] = -(v[2 * j] - v[2 * i]);
    L[i].p[0] = v[2 * i];
    L[i].p[1] = v[2 * i + 1];
  }
  FL(4 * loc);
  double dot = (v[0] - L[1].p[0]) * L[1].n[0] + (v[1] - L[1].p[1]) * L[1].n[1];
  FL(5);
  if (dot > 0.0)
    for (int i = 0; i < loc; ++i) {
      L[i].n[0] = -L[i].n[0];
      L[i].n[1] = -L[i].n[1];
    }
}

#define ORC_QBUF 48 /* 3 * 2**4 */

void orc_intersect_tri_quad(const double tri_a[6], const double quad_b[8], double *tris_c, int *n_tris_c) {
  /* intersect_polys_lines with area_a only: tol = 10*spacing(area(tri_a)) */
  orc_line L[4];
  get_lines_poly(quad_b, 4, L);
  double pa[2 * ORC_QBUF], pb[2 * ORC_QBUF];
  memcpy(pa, tri_a, 6 * sizeof(double));
  int n = 3;
  double *cur = pa, *nxt = pb;
  *n_tris_c = 0;
  for (int i = 0; i < 4; ++i) {
    n = clip_buf_tri(&L[i], cur, n, nxt);
    if (n < 3) return;
    double *t = cur;
    cur = nxt;
    nxt = t;
  }
  double tol = 10.0 * orc_spacing(orc_triangle_area(tri_a));
  int nt = 0;
  for (int i = 0; i < n - 2; ++i) {
    double *t = tris_c + 6 * nt;
    t[0] = cur[0];
    t[1] = cur[1];
    t[2] = cur[2 * (i + 1)];
    t[3] = cur[2 * (i + 1) + 1];
    t[4] = cur[2 * (i + 2)];
    t[5] = cur[2 * (i + 2) + 1];
    if (!(orc_triangle_area(t) < tol)) ++nt;
  }
  *n_tris_c = nt;
}

static void hex_planes(const double *h, orc_plane P[6]) {
  /* Supermesh.F90 intersect_tet_hex: Gmsh node order, no orientation flip */
  static const int F[6][4] = {{1, 0, 5, 0}, {5, 4, 6, 4}, {1, 5, 2, 5}, {0, 1, 3, 1}, {4, 0, 7, 0}, {6, 7, 2, 7}};
  for (int f = 0; f < 6; ++f) {
    /* unit_cross(h[a] - h[b], h[c] - h[d]); c = h[b] . n (point on the face) */
    double u[3], w[3];
    for (int k = 0; k < 3; ++k) {
      u[k] = h[3 * F[f][0] + k] - h[3 * F[f][1] + k];
      w[k] = h[3 * F[f][2] + k] - h[3 * F[f][3] + k];
    }
    FL(6);
    unit_cross(u, w, P[f].n);
    const double *q = h + 3 * F[f][1];
    P[f].c = (q[0] * P[f].n[0] + q[1] * P[f].n[1]) + q[2] * P[f].n[2];
    FL(5);
  }
}

#define ORC_HBUF 729 /* 3**6 */

void orc_intersect_tet_hex(const double tet_a[12], const double hex_b[24], double *tets_c, int *n_tets_c) {
  /* intersect_tet_planes over 6 planes, tol = 10*spacing(vol_v4(tet_a)) */
  orc_plane P[6];
  hex_planes(hex_b, P);
  double tol = 10.0 * orc_spacing(orc_tetrahedron_volume_v4(tet_a));
  double *cur = tets_c;
  double *buf = (double *)malloc(sizeof(double) * 12 * ORC_HBUF);
  int n = 1;
  memcpy(cur, tet_a, 12 * sizeof(double));
  for (int i = 0; i < 6; ++i) {
    int m = 0;
    for (int j = 0; j < n; ++j) m += clip_buf_tet(&P[i], cur + 12 * j, buf + 12 * m);
    if (i != 5) {
      n = m;
      memcpy(cur, buf, (size_t)n * 12 * sizeof(double));
    } else {
      n = 0;
      for (int j = 0; j < m; ++j) {
        if (orc_tetrahedron_volume_v4(buf + 12 * j) >= tol) {
          memcpy(cur + 12 * n, buf + 12 * j, 12 * sizeof(double));
          ++n;
        }
      }
    }
  }
  free(buf);
  *n_tets_c = n;
}

/* intersect_quads (Supermesh.F90:230-246): quad A clipped by quad B's four
 * edge lines (get_lines_poly), no element areas given, so the fan keeps
 * triangles with area >= 10*tiny (Triangle_Intersection.F90:255-264);
 * buffers 4 * 2**4 points. */
#define ORC_QQBUF 64
void orc_intersect_quads(const double quad_a[8], const double quad_b[8], double *tris_c, int *n_tris_c) {
  orc_line L[4];
  get_lines_poly(quad_b, 4, L);
  double pa[2 * ORC_QQBUF], pb[2 * ORC_QQBUF];
  memcpy(pa, quad_a, 8 * sizeof(double));
  int n = 4;
  double *cur = pa, *nxt = pb;
  *n_tris_c = 0;
  for (int i = 0; i < 4; ++i) {
    n = clip_buf_tri(&L[i], cur, n, nxt);
    if (n < 3) return;
    double *t = cur;
    cur = nxt;
    nxt = t;
  }
  const double tol = 10.0 * DBL_MIN;
  int nt = 0;
  for (int i = 0; i < n - 2; ++i) {
    double *t = tris_c + 6 * nt;
    t[0] = cur[0];
    t[1] = cur[1];
    t[2] = cur[2 * (i + 1)];
    t[3] = cur[2 * (i + 1) + 1];
    t[4] = cur[2 * (i + 2)];
    t[5] = cur[2 * (i + 2) + 1];
    if (!(orc_triangle_area(t) < tol)) ++nt;
  }
  *n_tris_c = nt;
}

/* intersect_hexes (Supermesh.F90:303-334): hex A sliced into five tets
 * (Gmsh corners (3,6,7,8), (1,3,4,8), (1,5,6,8), (1,2,3,6), (1,3,6,8)), each
 * clipped by hex B with intersect_tet_hex; outputs concatenated. */
static const int ORC_HEX_TETS[5][4] = {{2, 5, 6, 7}, {0, 2, 3, 7}, {0, 4, 5, 7}, {0, 1, 2, 5}, {0, 2, 5, 7}};

void orc_intersect_hexes(const double hex_a[24], const double hex_b[24], double *tets_c, int *n_tets_c) {
  int n = 0;
  for (int t = 0; t < 5; ++t) {
    double tet[12];
    for (int v = 0; v < 4; ++v)
      for (int c = 0; c < 3; ++c) tet[3 * v + c] = hex_a[3 * ORC_HEX_TETS[t][v] + c];
    int m = 0;
    orc_intersect_tet_hex(tet, hex_b, tets_c + 12 * n, &m);
    n += m;
  }
  *n_tets_c = n;
}

double orc_interval_size(const double iv[2]) { return fabs(iv[1] - iv[0]); }

void orc_intersect_intervals(const double a[2], const double b[2], double *c, int *n) {
  double min_a = fmin(a[0], a[1]), max_a = fmax(a[0], a[1]);
  double min_b = fmin(b[0], b[1]), max_b = fmax(b[0], b[1]);
  if (max_b <= min_a || min_b >= max_a) {
    *n = 0;
    return;
  }
  c[0] = fmax(min_a, min_b);
  c[1] = fmin(max_a, max_b);
  double tol = 10.0 * fmin(orc_spacing(orc_interval_size(a)), orc_spacing(orc_interval_size(b)));
  *n = orc_interval_size(c) < tol ? 0 : 1;
}

/* ------------------------------------------------------------------ */
/* Quadtree / octree intersection finder                               */
/* ------------------------------------------------------------------ */
typedef struct orc_node {
  int n;      /* stored elements; > max_n marks an internal node */
  int max_n;
  double lo[3], hi[3];
  int *ele;     /* leaf storage [max_n] */
  double *ebox; /* leaf storage [max_n][2*dim] (lo..., hi...) */
  struct orc_node *children;
} orc_node;

typedef struct {
  int dim;
  orc_node root;
} orc_tree;

static int boxes_intersect(int dim, const double *lo1, const double *hi1,
                           const double *lo2, const double *hi2) {
  /* bboxes_intersect(bbox_1, bbox_2): strict overlap in every dimension. */
  for (int c = 0; c < dim; ++c)
    if (!(hi2[c] > lo1[c] && lo2[c] < hi1[c])) return 0;
  return 1;
}

static void elem_bbox(int dim, int loc, const double *pos, const int32_t *en,
                      long e, double *lo, double *hi) {
  const int32_t *nodes = en + (size_t)e * loc;
  for (int c = 0; c < dim; ++c) lo[c] = hi[c] = pos[(size_t)nodes[0] * dim + c];
  for (int k = 1; k < loc; ++k)
    for (int c = 0; c < dim; ++c) {
      double x = pos[(size_t)nodes[k] * dim + c];
      lo[c] = fmin(lo[c], x);
      hi[c] = fmax(hi[c], x);
    }
}

static int node_alloc_leaf(orc_node *nd, int dim, int max_n) {
  nd->n = 0;
  nd->max_n = max_n;
  nd->children = NULL;
  nd->ele = (int *)malloc(sizeof(int) * (size_t)max_n);
  nd->ebox = (double *)malloc(sizeof(double) * 2 * dim * (size_t)max_n);
  return (nd->ele && nd->ebox) ? 0 : -1;
}

static void node_free(orc_node *nd, int dim) {
  int nch = 1 << dim;
  if (nd->n <= nd->max_n) {
    free(nd->ele);
    free(nd->ebox);
  } else {
    for (int i = 0; i < nch; ++i) node_free(&nd->children[i], dim);
    free(nd->children);
  }
}

/* Child box selectors in the reference's child order
 * (Quadtree...F90:293-300, Octree...F90:273-288). */
static const int CH_X[8] = {0, 0, 1, 1, 0, 0, 1, 1};
static const int CH_Y[8] = {0, 1, 1, 0, 0, 1, 1, 0};
static const int CH_Z[8] = {0, 0, 0, 0, 1, 1, 1, 1};

static int add_element(orc_node *nd, int dim, int ele, const double *lo,
                       const double *hi) {
  if (!boxes_intersect(dim, nd->lo, nd->hi, lo, hi)) return 0;
  int nch = 1 << dim;
  if (nd->n <= nd->max_n - 1) {
    int k = nd->n++;
    nd->ele[k] = ele;
    memcpy(nd->ebox + (size_t)k * 2 * dim, lo, sizeof(double) * dim);
    memcpy(nd->ebox + (size_t)k * 2 * dim + dim, hi, sizeof(double) * dim);
  } else if (nd->n == nd->max_n) {
    nd->children = (orc_node *)calloc((size_t)nch, sizeof(orc_node));
    if (!nd->children) return -1;
    double mid[3];
    for (int c = 0; c < dim; ++c) mid[c] = 0.5 * (nd->lo[c] + nd->hi[c]);
    for (int i = 0; i < nch; ++i) {
      orc_node *ch = &nd->children[i];
      const int sel[3] = {CH_X[i], CH_Y[i], CH_Z[i]};
      for (int c = 0; c < dim; ++c) {
        ch->lo[c] = sel[c] ? mid[c] : nd->lo[c];
        ch->hi[c] = sel[c] ? nd->hi[c] : mid[c];
      }
      if (node_alloc_leaf(ch, dim, nd->max_n)) return -1;
    }
    for (int i = 0; i < nd->max_n; ++i)
      for (int j = 0; j < nch; ++j)
        if (add_element(&nd->children[j], dim, nd->ele[i],
                        nd->ebox + (size_t)i * 2 * dim,
                        nd->ebox + (size_t)i * 2 * dim + dim))
          return -1;
    for (int j = 0; j < nch; ++j)
      if (add_element(&nd->children[j], dim, ele, lo, hi)) return -1;
    nd->n = 0x7fffffff; /* huge(n): internal node */
    free(nd->ele);
    free(nd->ebox);
    nd->ele = NULL;
    nd->ebox = NULL;
  } else {
    for (int j = 0; j < nch; ++j)
      if (add_element(&nd->children[j], dim, ele, lo, hi)) return -1;
  }
  return 0;
}

static int max_nelist_degree(long nnodes, int loc, const int32_t *en, long nel) {
  int *cnt = (int *)calloc((size_t)nnodes, sizeof(int));
  if (!cnt) return -1;
  for (long e = 0; e < nel; ++e)
    for (int k = 0; k < loc; ++k) cnt[en[(size_t)e * loc + k]]++;
  int m = 0;
  for (long i = 0; i < nnodes; ++i)
    if (cnt[i] > m) m = cnt[i];
  free(cnt);
  return m;
}

static int tree_build(orc_tree *t, int dim, long nnodes, const double *pos,
                      int loc, const int32_t *en, long nel, int max_size) {
  t->dim = dim;
  int max_n = max_size;
  if (max_n <= 0) {
    int deg = max_nelist_degree(nnodes, loc, en, nel);
    if (deg < 0) return -1;
    max_n = deg > 256 ? deg : 256;
  }
  orc_node *r = &t->root;
  if (node_alloc_leaf(r, dim, max_n)) return -1;
  for (int c = 0; c < dim; ++c) r->lo[c] = r->hi[c] = pos[c];
  for (long i = 1; i < nnodes; ++i)
    for (int c = 0; c < dim; ++c) {
      r->lo[c] = fmin(r->lo[c], pos[(size_t)i * dim + c]);
      r->hi[c] = fmax(r->hi[c], pos[(size_t)i * dim + c]);
    }
  for (long e = 0; e < nel; ++e) {
    double lo[3], hi[3];
    elem_bbox(dim, loc, pos, en, e, lo, hi);
    if (add_element(r, dim, (int)e, lo, hi)) return -1;
  }
  return 0;
}

static void tree_query(const orc_node *nd, int dim, const double *lo,
                       const double *hi, int32_t *out, int *nout,
                       unsigned char *seen) {
  if (nd->n == 0) return;
  if (!boxes_intersect(dim, nd->lo, nd->hi, lo, hi)) return;
  if (nd->n <= nd->max_n) {
    for (int i = 0; i < nd->n; ++i) {
      int e = nd->ele[i];
      if (!seen[e]) {
        const double *eb = nd->ebox + (size_t)i * 2 * dim;
        if (boxes_intersect(dim, eb, eb + dim, lo, hi)) {
          out[(*nout)++] = e;
          seen[e] = 1;
        }
      }
    }
  } else {
    int nch = 1 << dim;
    for (int i = 0; i < nch; ++i)
      tree_query(&nd->children[i], dim, lo, hi, out, nout, seen);
  }
}

typedef struct {
  int32_t *v;
  int n;
} orc_row;

static int rows_to_csr(orc_row *rows, long nel_a, int64_t *indptr,
                       int32_t **indices, int64_t *nnz) {
  int64_t tot = 0;
  indptr[0] = 0;
  for (long a = 0; a < nel_a; ++a) {
    tot += rows[a].n;
    indptr[a + 1] = tot;
  }
  int32_t *ind = (int32_t *)malloc(sizeof(int32_t) * (size_t)(tot > 0 ? tot : 1));
  if (!ind) return -1;
  for (long a = 0; a < nel_a; ++a) {
    if (rows[a].n) memcpy(ind + indptr[a], rows[a].v, sizeof(int32_t) * rows[a].n);
    free(rows[a].v);
  }
  *indices = ind;
  *nnz = tot;
  return 0;
}

int orc_tree_finder(int dim, long nnodes_a, const double *pos_a, long nel_a,
                    int loc_a, const int32_t *en_a, long nnodes_b,
                    const double *pos_b, long nel_b, int loc_b,
                    const int32_t *en_b, int max_size, int64_t *indptr,
                    int32_t **indices, int64_t *nnz) {
  (void)nnodes_a;
  if (dim != 2 && dim != 3) return -1;
  orc_row *rows = (orc_row *)calloc((size_t)(nel_a > 0 ? nel_a : 1), sizeof(orc_row));
  if (!rows) return -1;
  if (nel_a > 0 && nel_b > 0) {
    orc_tree t;
    if (tree_build(&t, dim, nnodes_b, pos_b, loc_b, en_b, nel_b, max_size)) return -1;
    unsigned char *seen = (unsigned char *)calloc((size_t)nel_b, 1);
    int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)nel_b);
    for (long a = 0; a < nel_a; ++a) {
      double lo[3], hi[3];
      elem_bbox(dim, loc_a, pos_a, en_a, a, lo, hi);
      int n = 0;
      tree_query(&t.root, dim, lo, hi, buf, &n, seen);
      for (int i = 0; i < n; ++i) seen[buf[i]] = 0;
      rows[a].n = n;
      rows[a].v = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
      memcpy(rows[a].v, buf, sizeof(int32_t) * (size_t)n);
    }
    free(seen);
    free(buf);
    node_free(&t.root, dim);
  }
  int rc = rows_to_csr(rows, nel_a, indptr, indices, nnz);
  free(rows);
  return rc;
}

int orc_brute_force_finder(int dim, long nnodes_a, const double *pos_a,
                           long nel_a, int loc_a, const int32_t *en_a,
                           long nnodes_b, const double *pos_b, long nel_b,
                           int loc_b, const int32_t *en_b, int64_t *indptr,
                           int32_t **indices, int64_t *nnz) {
  (void)nnodes_a;
  (void)nnodes_b;
  if (dim != 2 && dim != 3) return -1;
  double *bb = (double *)malloc(sizeof(double) * 2 * dim * (size_t)(nel_b > 0 ? nel_b : 1));
  orc_row *rows = (orc_row *)calloc((size_t)(nel_a > 0 ? nel_a : 1), sizeof(orc_row));
  int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nel_b > 0 ? nel_b : 1));
  if (!bb || !rows || !buf) return -1;
  for (long b = 0; b < nel_b; ++b)
    elem_bbox(dim, loc_b, pos_b, en_b, b, bb + 2 * dim * b, bb + 2 * dim * b + dim);
  for (long a = 0; a < nel_a; ++a) {
    double lo[3], hi[3];
    elem_bbox(dim, loc_a, pos_a, en_a, a, lo, hi);
    int n = 0;
    for (long b = 0; b < nel_b; ++b)
      if (boxes_intersect(dim, lo, hi, bb + 2 * dim * b, bb + 2 * dim * b + dim))
        buf[n++] = (int32_t)b;
    rows[a].n = n;
    rows[a].v = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    memcpy(rows[a].v, buf, sizeof(int32_t) * (size_t)n);
  }
  free(bb);
  free(buf);
  int rc = rows_to_csr(rows, nel_a, indptr, indices, nnz);
  free(rows);
  return rc;
}

/* 1D sort finder (Intersection_Finder.F90:811-921).  Elements are ordered
 * by their left end with the reference's merge sort, then one sweep pointer j
 * walks the sorted B elements for each sorted A element: B elements ending at
 * or before the A element's left end are passed for good, the sweep stops at
 * the first B element starting at or after the A element's right end, and
 * every other one is recorded; after a row with records j steps back by one.
 *
 * The reference's merge sort (Intersection_Finder.F90:871-910) handles blocks
 * of at most 4 elements with a selection loop that writes, for each i, the
 * position of the first strict minimum of v(i:n); that is a permutation only
 * when the block is already non-decreasing.  stable_leaf = 0 restates it as
 * written; stable_leaf = 1 replaces that step by a stable insertion sort, so
 * the whole sort is the stable sort by left end. */
static void ref_merge_sort(const double *v, int n, int *idx, int *work, int stable_leaf) {
  if (n <= 4) {
    if (stable_leaf) {
      for (int i = 0; i < n; ++i) idx[i] = i;
      for (int i = 1; i < n; ++i) {
        int t = idx[i], k = i;
        while (k > 0 && v[t] < v[idx[k - 1]]) {
          idx[k] = idx[k - 1];
          --k;
        }
        idx[k] = t;
      }
    } else {
      for (int i = 0; i < n; ++i) {
        idx[i] = i;
        for (int j = i + 1; j < n; ++j)
          if (v[j] < v[idx[i]]) idx[i] = j;
      }
    }
    return;
  }
  const int h = n / 2;
  ref_merge_sort(v, h, idx, work, stable_leaf);
  ref_merge_sort(v + h, n - h, idx + h, work + h, stable_leaf);
  for (int i = 0; i < h; ++i) work[i] = idx[i];
  for (int i = h; i < n; ++i) work[i] = idx[i] + h;
  int i1 = 0, i2 = h;
  for (int i = 0; i < n; ++i) {
    if (i1 >= h) {
      for (int k = i; k < n; ++k) idx[k] = work[i2++];
      break;
    } else if (i2 >= n) {
      for (int k = i; k < n; ++k) idx[k] = work[i1++];
      break;
    } else if (v[work[i1]] <= v[work[i2]]) {
      idx[i] = work[i1++];
    } else {
      idx[i] = work[i2++];
    }
  }
}

/* minval / maxval of a 2-node element's coordinates (first coordinate of
 * each node, positions stored with stride `stride`). */
static void interval_ends(const double *pos, int stride, const int32_t *en, long e, double *lo, double *hi) {
  const double x0 = pos[(size_t)en[2 * e] * stride], x1 = pos[(size_t)en[2 * e + 1] * stride];
  *lo = x1 < x0 ? x1 : x0;
  *hi = x1 > x0 ? x1 : x0;
}

int orc_sort_finder_1d(long nnodes_a, const double *pos_a, int stride_a, long nel_a, const int32_t *en_a,
                       long nnodes_b, const double *pos_b, int stride_b, long nel_b, const int32_t *en_b,
                       int stable_leaf, int64_t *indptr, int32_t **indices, int64_t *nnz) {
  (void)nnodes_a;
  (void)nnodes_b;
  const size_t na = (size_t)(nel_a > 0 ? nel_a : 1), nb = (size_t)(nel_b > 0 ? nel_b : 1);
  double *la = (double *)calloc(na, sizeof(double)), *ha = (double *)calloc(na, sizeof(double));
  double *lb = (double *)calloc(nb, sizeof(double)), *hb = (double *)calloc(nb, sizeof(double));
  int *ia = (int *)malloc(sizeof(int) * na), *ib = (int *)malloc(sizeof(int) * nb);
  int *work = (int *)malloc(sizeof(int) * (na > nb ? na : nb));
  int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * nb);
  orc_row *rows = (orc_row *)calloc(na, sizeof(orc_row));
  if (!la || !ha || !lb || !hb || !ia || !ib || !work || !buf || !rows) return -1;
  for (long e = 0; e < nel_a; ++e) interval_ends(pos_a, stride_a, en_a, e, la + e, ha + e);
  for (long e = 0; e < nel_b; ++e) interval_ends(pos_b, stride_b, en_b, e, lb + e, hb + e);
  ref_merge_sort(la, (int)nel_a, ia, work, stable_leaf);
  ref_merge_sort(lb, (int)nel_b, ib, work, stable_leaf);
  long j = 0;
  for (long i = 0; i < nel_a; ++i) {
    const int a = ia[i];
    int n = 0;
    while (j < nel_b) {
      const int b = ib[j];
      if (hb[b] <= la[a]) {
        ++j;
      } else if (lb[b] >= ha[a]) {
        break;
      } else {
        buf[n++] = (int32_t)b;
        ++j;
      }
    }
    if (n > 0) --j;
    /* with a non-permutation sort an element can come twice: the reference
     * then reallocates that row; the last write wins */
    free(rows[a].v);
    rows[a].n = n;
    rows[a].v = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    memcpy(rows[a].v, buf, sizeof(int32_t) * (size_t)n);
  }
  free(la);
  free(ha);
  free(lb);
  free(hb);
  free(ia);
  free(ib);
  free(work);
  free(buf);
  int rc = rows_to_csr(rows, nel_a, indptr, indices, nnz);
  free(rows);
  return rc;
}

void orc_free(void *p) { free(p); }


/* ------------------------------------------------------------------ */
/* Kahan compensated sum (Precision.F90:72-113)                         */
/* ------------------------------------------------------------------ */
typedef struct {
  double sum, err;
} orc_cs;

static inline void cs_add(orc_cs *cs, double x) {
  double cx = cs->err + x;
  double s = cs->sum + cx;
  cs->err = cs->sum - s;
  cs->err = cs->err + cx;
  cs->sum = s;
}

double orc_kahan_sum(const double *x, long n) {
  orc_cs cs = {0.0, 0.0};
  for (long i = 0; i < n; ++i) cs_add(&cs, x[i]);
  return cs.sum + cs.err;
}

/* ------------------------------------------------------------------ */
/* Narrow phase driver                                                 */
/* ------------------------------------------------------------------ */
static void gather(int dim, int loc, const double *pos, const int32_t *en,
                   long e, double *out) {
  const int32_t *nodes = en + (size_t)e * loc;
  for (int k = 0; k < loc; ++k)
    for (int c = 0; c < dim; ++c) out[k * dim + c] = pos[(size_t)nodes[k] * dim + c];
}

int orc_num_threads_available(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int orc_narrow(int dim, const double *pos_a, int loc_a, const int32_t *en_a,
               long nel_a, const double *pos_b, int loc_b, const int32_t *en_b,
               long nel_b, const int64_t *indptr, const int32_t *indices,
               double *pair_measure, int32_t *pair_nout, double *elem_measure,
               int nthreads, int count_flops, orc_stats *st) {
  if (dim == 2 && !(loc_a == 3 && loc_b == 3)) return -1;
  if (dim == 3 && !(loc_a == 4 && loc_b == 4)) return -1;
  if (dim != 2 && dim != 3) return -1;
  if (nthreads < 1) nthreads = 1;
  double setup_flops = 0.0;
  if (count_flops) {
    /* Per-element work the clipper needs once per element: measures and
     * tolerances of A and B, and B's lines/planes. */
    tl_count = 1;
    tl_flops = 0.0;
    double v[12];
    for (long a = 0; a < nel_a; ++a) {
      gather(dim, loc_a, pos_a, en_a, a, v);
      if (dim == 2) (void)orc_triangle_area(v); else (void)orc_tetrahedron_volume_v4(v);
      FL(1);
    }
    for (long b = 0; b < nel_b; ++b) {
      gather(dim, loc_b, pos_b, en_b, b, v);
      if (dim == 2) {
        orc_line L[3];
        (void)orc_triangle_area(v);
        get_lines_tri(v, L);
      } else {
        orc_plane P[4];
        (void)orc_tetrahedron_volume_v4(v);
        get_planes_tet(v, P);
      }
      FL(1);
    }
    setup_flops = tl_flops;
    tl_count = 0;
  }
  int64_t n_int = 0, n_out = 0;
  double flops = 0.0;
  orc_cs tot = {0.0, 0.0};
#pragma omp parallel num_threads(nthreads) reduction(+ : n_int, n_out, flops)
  {
    orc_cs local = {0.0, 0.0};
    double *buf = (double *)malloc(sizeof(double) * 12 * ORC_TET_BUF);
    double va[12], vb[12];
    tl_count = count_flops;
    tl_flops = 0.0;
#pragma omp for schedule(dynamic, 64)
    for (long a = 0; a < nel_a; ++a) {
      gather(dim, loc_a, pos_a, en_a, a, va);
      double ea = 0.0;
      for (int64_t p = indptr[a]; p < indptr[a + 1]; ++p) {
        long b = indices[p];
        gather(dim, loc_b, pos_b, en_b, b, vb);
        int n;
        double m = 0.0;
        if (dim == 2) {
          orc_line L[3];
          int save = tl_count;
          tl_count = 0; /* per-element setup is counted once above */
          get_lines_tri(vb, L);
          double tol = 10.0 * fmin(orc_spacing(orc_triangle_area(va)),
                                   orc_spacing(orc_triangle_area(vb)));
          tl_count = save;
          n = intersect_tris_lines(va, L, tol, buf);
          for (int k = 0; k < n; ++k) {
            double ar = orc_triangle_area(buf + 6 * k);
            m = m + ar;
            cs_add(&local, ar);
            FL(1);
          }
        } else {
          orc_plane P[4];
          int save = tl_count;
          tl_count = 0;
          get_planes_tet(vb, P);
          double tol = 10.0 * fmin(orc_spacing(orc_tetrahedron_volume_v4(va)),
                                   orc_spacing(orc_tetrahedron_volume_v4(vb)));
          tl_count = save;
          n = intersect_tets_planes(va, P, tol, buf);
          for (int k = 0; k < n; ++k) {
            double vo = orc_tetrahedron_volume(buf + 12 * k);
            m = m + vo;
            cs_add(&local, vo);
            FL(1);
          }
        }
        if (pair_measure) pair_measure[p] = m;
        if (pair_nout) pair_nout[p] = n;
        if (n > 0) n_int++;
        n_out += n;
        ea = ea + m;
      }
      if (elem_measure) elem_measure[a] = ea;
    }
    flops += tl_flops;
    tl_count = 0;
    free(buf);
#pragma omp critical
    {
      /* combine compensated partial sums */
      cs_add(&tot, local.sum);
      cs_add(&tot, local.err);
    }
  }
  if (st) {
    st->n_candidates = indptr[nel_a];
    st->n_intersecting = n_int;
    st->n_out_simplices = n_out;
    st->total = tot.sum + tot.err;
    st->total_err = tot.err;
    st->flops = flops + setup_flops;
  }
  return 0;
}

int orc_supermesh(int dim, long nnodes_a, const double *pos_a, long nel_a,
                  int loc_a, const int32_t *en_a, long nnodes_b,
                  const double *pos_b, long nel_b, int loc_b,
                  const int32_t *en_b, int nthreads, orc_stats *st) {
  int64_t *indptr = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nel_a + 1));
  int32_t *indices = NULL;
  int64_t nnz = 0;
  if (!indptr) return -1;
  int rc = orc_tree_finder(dim, nnodes_a, pos_a, nel_a, loc_a, en_a, nnodes_b,
                           pos_b, nel_b, loc_b, en_b, 0, indptr, &indices, &nnz);
  if (rc == 0)
    rc = orc_narrow(dim, pos_a, loc_a, en_a, nel_a, pos_b, loc_b, en_b, nel_b,
                    indptr, indices, NULL, NULL, NULL, nthreads, 0, st);
  free(indptr);
  free(indices);
  return rc;
}

/* ------------------------------------------------------------------ */
/* P1-P1 mixed inner product                                           */
/* ------------------------------------------------------------------ */
static void p1_basis_2d(const double *cc, const double *x, double fns[3]) {
  /* test_parallel_p1_inner_product_2d.F90:206-229 */
  double e1[2] = {cc[2] - cc[0], cc[3] - cc[1]};
  double e2[2] = {cc[4] - cc[0], cc[5] - cc[1]};
  double j11 = e2[1], j12 = -e2[0], j21 = -e1[1], j22 = e1[0];
  double det = j11 * j22 - j12 * j21;
  j11 /= det;
  j12 /= det;
  j21 /= det;
  j22 /= det;
  double dx = x[0] - cc[0], dy = x[1] - cc[1];
  fns[1] = j11 * dx + j12 * dy;
  fns[2] = j21 * dx + j22 * dy;
  fns[0] = 1.0 - fns[1] - fns[2];
}

static void p1_basis_3d(const double *cc, const double *x, double fns[4]) {
  /* test_parallel_p1_inner_product_3d.F90:215-250: solve
   * [v2-v1 v3-v1 v4-v1] l = x - v1 by Gaussian elimination with partial
   * pivoting (same elimination order). */
  double m[3][4];
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) m[r][c] = cc[3 * (c + 1) + r] - cc[r];
    m[r][3] = x[r] - cc[r];
  }
  for (int i = 0; i < 3; ++i) {
    int j = i;
    double best = fabs(m[i][i]);
    for (int k = i + 1; k < 3; ++k)
      if (fabs(m[k][i]) > best) {
        best = fabs(m[k][i]);
        j = k;
      }
    if (j != i)
      for (int c = 0; c < 4; ++c) {
        double t = m[i][c];
        m[i][c] = m[j][c];
        m[j][c] = t;
      }
    double piv = m[i][i];
    for (int c = 0; c < 4; ++c) m[i][c] = m[i][c] / piv;
    for (int k = i + 1; k < 3; ++k) {
      double f = m[k][i];
      for (int c = 0; c < 4; ++c) m[k][c] = m[k][c] - f * m[i][c];
    }
  }
  for (int i = 2; i >= 0; --i)
    for (int k = i - 1; k >= 0; --k) {
      double f = m[k][i];
      for (int c = 0; c < 4; ++c) m[k][c] = m[k][c] - f * m[i][c];
    }
  fns[1] = m[0][3];
  fns[2] = m[1][3];
  fns[3] = m[2][3];
  fns[0] = 1.0 - fns[1] - fns[2] - fns[3];
}

int orc_p1_mass(int dim, const double *pos_a, const int32_t *en_a, long nel_a,
                const double *pos_b, const int32_t *en_b, long nel_b,
                const int64_t *indptr, const int32_t *indices,
                const double *u_a, const double *v_b, double *blocks,
                double *integral, double *measure) {
  (void)nel_b;
  if (dim != 2 && dim != 3) return -1;
  const int loc = dim + 1;
  /* Quadrature: 2D Dunavant degree 2 (points (4,1,1)/6, weights 1/3);
   * 3D Stroud T3:2-1 (points a,b,b,b with a=0.58541019662496852,
   * b=0.13819660112501050, weights 1/4). */
  const double q2w = 1.0 / 3.0;
  const double q2p[3][3] = {{4.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0},
                            {1.0 / 6.0, 4.0 / 6.0, 1.0 / 6.0},
                            {1.0 / 6.0, 1.0 / 6.0, 4.0 / 6.0}};
  const double qa = 5.8541019662496852e-1, qb = 1.3819660112501050e-1;
  const double q3w = 0.25;
  const double q3p[4][4] = {{qa, qb, qb, qb}, {qb, qa, qb, qb}, {qb, qb, qa, qb}, {qb, qb, qb, qa}};
  orc_cs I = {0.0, 0.0}, V = {0.0, 0.0};
  double *buf = (double *)malloc(sizeof(double) * 12 * ORC_TET_BUF);
  if (!buf) return -1;
  double va[12], vb[12];
  for (long a = 0; a < nel_a; ++a) {
    gather(dim, loc, pos_a, en_a, a, va);
    for (int64_t p = indptr[a]; p < indptr[a + 1]; ++p) {
      long b = indices[p];
      gather(dim, loc, pos_b, en_b, b, vb);
      int n;
      double blk[16];
      memset(blk, 0, sizeof(blk));
      if (dim == 2)
        orc_intersect_tris(va, vb, buf, &n);
      else
        orc_intersect_tets(va, vb, buf, &n);
      for (int k = 0; k < n; ++k) {
        const double *c = buf + (size_t)k * loc * dim;
        double meas = dim == 2 ? orc_triangle_area(c) : orc_tetrahedron_volume(c);
        cs_add(&V, meas);
        int nq = dim == 2 ? 3 : 4;
        for (int q = 0; q < nq; ++q) {
          double x[3] = {0.0, 0.0, 0.0};
          for (int d = 0; d < dim; ++d) {
            double s = 0.0;
            for (int v = 0; v < loc; ++v)
              s = s + (dim == 2 ? q2p[q][v] : q3p[q][v]) * c[v * dim + d];
            x[d] = s;
          }
          double fa[4], fb[4];
          if (dim == 2) {
            p1_basis_2d(va, x, fa);
            p1_basis_2d(vb, x, fb);
          } else {
            p1_basis_3d(va, x, fa);
            p1_basis_3d(vb, x, fb);
          }
          double w = (dim == 2 ? q2w : q3w) * meas;
          for (int i = 0; i < loc; ++i)
            for (int j = 0; j < loc; ++j) blk[i * loc + j] += w * fa[i] * fb[j];
        }
      }
      if (blocks) memcpy(blocks + (size_t)p * loc * loc, blk, sizeof(double) * loc * loc);
      if (u_a && v_b) {
        const int32_t *na = en_a + (size_t)a * loc;
        const int32_t *nb = en_b + (size_t)b * loc;
        double s = 0.0;
        for (int i = 0; i < loc; ++i)
          for (int j = 0; j < loc; ++j) s += u_a[na[i]] * blk[i * loc + j] * v_b[nb[j]];
        cs_add(&I, s);
      }
    }
  }
  free(buf);
  if (integral) *integral = I.sum + I.err;
  if (measure) *measure = V.sum + V.err;
  return 0;
}

/* P2 inner product (test_parallel_p2_inner_product_2d.F90:398-522): per
 * supermesh triangle c of A x B, the P2 fields of A and B are interpolated
 * at c's 3 vertices and 3 edge midpoints with the P2 basis of their own
 * element (basis_functions_p2 :399-433, interpolate_p2 :436-451), and
 * 2 * |c| * f_b . (M_p2 f_a) is added (:515-519), M_p2 the reference P2 mass
 * matrix (:64-72) on the unit triangle. */
static void p2_basis(const double *cc, const double *x, double fns[6]) {
  const double e10 = cc[2] - cc[0], e11 = cc[3] - cc[1];
  const double e20 = cc[4] - cc[0], e21 = cc[5] - cc[1];
  double j11 = e21, j12 = -e20, j21 = -e11, j22 = e10;
  const double det = j11 * j22 - j12 * j21;
  j11 = j11 / det;
  j12 = j12 / det;
  j21 = j21 / det;
  j22 = j22 / det;
  const double d1 = x[0] - cc[0], d2 = x[1] - cc[1];
  const double lx = j11 * d1 + j12 * d2, ly = j21 * d1 + j22 * d2;
  fns[0] = ((1.0 - lx) - ly) * ((1.0 - 2.0 * lx) - 2.0 * ly);
  fns[1] = lx * (2.0 * lx - 1.0);
  fns[2] = ly * (2.0 * ly - 1.0);
  fns[3] = (4.0 * lx) * ((1.0 - lx) - ly);
  fns[4] = (4.0 * lx) * ly;
  fns[5] = (4.0 * ly) * ((1.0 - lx) - ly);
}

static double p2_interp(const double *cc, const double vals[6], const double *x) {
  double f[6];
  p2_basis(cc, x, f);
  double s = 0.0;
  for (int k = 0; k < 6; ++k) s = s + f[k] * vals[k];
  return s;
}

static const double ORC_MASS_P2[6][6] = {
    {6.0 / 360.0, -1.0 / 360.0, -1.0 / 360.0, 0.0 / 360.0, -4.0 / 360.0, 0.0 / 360.0},
    {-1.0 / 360.0, 6.0 / 360.0, -1.0 / 360.0, 0.0 / 360.0, 0.0 / 360.0, -4.0 / 360.0},
    {-1.0 / 360.0, -1.0 / 360.0, 6.0 / 360.0, -4.0 / 360.0, 0.0 / 360.0, 0.0 / 360.0},
    {0.0 / 360.0, 0.0 / 360.0, -4.0 / 360.0, 32.0 / 360.0, 16.0 / 360.0, 16.0 / 360.0},
    {-4.0 / 360.0, 0.0 / 360.0, 0.0 / 360.0, 16.0 / 360.0, 32.0 / 360.0, 16.0 / 360.0},
    {0.0 / 360.0, -4.0 / 360.0, 0.0 / 360.0, 16.0 / 360.0, 16.0 / 360.0, 32.0 / 360.0}};

int orc_p2_inner_product(const double *pos_a, const int32_t *en_a, long nel_a, const double *pos_b,
                         const int32_t *en_b, const int64_t *indptr, const int32_t *indices,
                         const int32_t *en_p2_a, const double *field_a, const int32_t *en_p2_b,
                         const double *field_b, double *pair_values, double *integral, double *area) {
  orc_cs I = {0.0, 0.0}, V = {0.0, 0.0};
  double buf[6 * ORC_TRI_BUF];
  double va[6], vb[6], fa_n[6], fb_n[6];
  for (long a = 0; a < nel_a; ++a) {
    gather(2, 3, pos_a, en_a, a, va);
    for (int k = 0; k < 6; ++k) fa_n[k] = field_a[en_p2_a[6 * a + k]];
    for (int64_t p = indptr[a]; p < indptr[a + 1]; ++p) {
      const long b = indices[p];
      gather(2, 3, pos_b, en_b, b, vb);
      for (int k = 0; k < 6; ++k) fb_n[k] = field_b[en_p2_b[6 * b + k]];
      int n;
      orc_intersect_tris(va, vb, buf, &n);
      double sp = 0.0;
      for (int t = 0; t < n; ++t) {
        const double *c = buf + 6 * t;
        const double ar = orc_triangle_area(c);
        cs_add(&V, ar);
        double pts[6][2];
        for (int d = 0; d < 2; ++d) {
          pts[0][d] = c[d];
          pts[1][d] = c[2 + d];
          pts[2][d] = c[4 + d];
          pts[3][d] = 0.5 * (c[d] + c[2 + d]);
          pts[4][d] = 0.5 * (c[2 + d] + c[4 + d]);
          pts[5][d] = 0.5 * (c[d] + c[4 + d]);
        }
        double fac[6], fbc[6];
        for (int l = 0; l < 6; ++l) {
          fbc[l] = p2_interp(vb, fb_n, pts[l]);
          fac[l] = p2_interp(va, fa_n, pts[l]);
        }
        double dot = 0.0;
        for (int i = 0; i < 6; ++i) {
          double mi = 0.0;
          for (int k = 0; k < 6; ++k) mi = mi + ORC_MASS_P2[i][k] * fac[k];
          dot = dot + fbc[i] * mi;
        }
        sp = sp + (2.0 * ar) * dot;
      }
      if (pair_values) pair_values[p] = sp;
      cs_add(&I, sp);
    }
  }
  if (integral) *integral = I.sum + I.err;
  if (area) *area = V.sum + V.err;
  return 0;
}
