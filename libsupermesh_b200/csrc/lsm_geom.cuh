// Device geometry for the supermesh narrow phase: FP64, FMA-free (the whole
// library is compiled with -fmad=false), evaluated in libsupermesh's order so
// that every clipped vertex, area and volume is bit-identical to the
// reference algorithm.
//
// Reference routines (firedrakeproject/libsupermesh):
//   src/Triangle_Intersection.F90   clip_buf :282-335, get_lines_tri
//                                   :395-420, triangle_area :453-477,
//                                   intersect_tris_tri :144-185
//   src/Tetrahedron_Intersection.F90 clip_buf :244-436, get_planes_tet
//                                   :634-667, unit_cross :669-677,
//                                   distances_to_plane :679-688,
//                                   tetrahedron_volume_{real,tet} :690-725,
//                                   intersect_tets_planes :137-179
#pragma once

#include <cstdint>

namespace lsm {

// Fortran EPSILON(1.0_real64) = 2**-52.
constexpr double kEps = 2.220446049250313080847263336181640625e-16;
constexpr double kTiny = 2.2250738585072013830902327173324040642e-308;  // 2**-1022

// Fortran SPACING for real64: 2**(exponent(x)-53), TINY when that is not a
// normal number (x == 0, subnormal x, or |x| < 2**-969).
__device__ __forceinline__ double spacing(double x) {
  const unsigned long long bits = (unsigned long long)__double_as_longlong(x) & 0x7fffffffffffffffULL;
  const int e = (int)(bits >> 52);  // biased exponent of |x|
  const int es = e - 52;            // biased exponent of the spacing
  if (e == 0 || es < 1) return kTiny;
  return __longlong_as_double((long long)es << 52);
}

// gfortran's inline NORM2 of a 3-vector (scaled sum of squares).
__device__ __forceinline__ double norm2_3(double a, double b, double c) {
  double scale = 0.0, result = 1.0;
  const double v[3] = {a, b, c};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (v[i] != 0.0) {
      const double ax = fabs(v[i]);
      if (scale < ax) {
        const double val = scale / ax;
        result = 1.0 + result * (val * val);
        scale = ax;
      } else {
        const double val = ax / scale;
        result = result + val * val;
      }
    }
  }
  return sqrt(result) * scale;
}

// ---------------------------------------------------------------- measures
// tri: vertices (x0,y0),(x1,y1),(x2,y2).  0.5*|u2 v1 - u1 v2| with u = v3-v1,
// v = v2-v1.
__device__ __forceinline__ double tri_area(double x0, double y0, double x1, double y1,
                                           double x2, double y2) {
  const double u0 = x2 - x0, u1 = y2 - y0;
  const double w0 = x1 - x0, w1 = y1 - y0;
  return 0.5 * fabs(u1 * w0 - u0 * w1);
}

struct Tet {
  double x[4], y[4], z[4];
};

// Vertex-1 based volume (the C API's libsupermesh_tetrahedron_volume).
__device__ __forceinline__ double tet_volume_v1(const Tet& t) {
  const double e1x = t.x[1] - t.x[0], e1y = t.y[1] - t.y[0], e1z = t.z[1] - t.z[0];
  const double e2x = t.x[2] - t.x[0], e2y = t.y[2] - t.y[0], e2z = t.z[2] - t.z[0];
  const double e3x = t.x[3] - t.x[0], e3y = t.y[3] - t.y[0], e3z = t.z[3] - t.z[0];
  double s = e1x * (e2y * e3z - e2z * e3y) + e1y * (e2z * e3x - e2x * e3z);
  s = s + e1z * (e2x * e3y - e2y * e3x);
  return (1.0 / 6.0) * fabs(s);
}

// Vertex-4 based volume (used for the clipping tolerance).
__device__ __forceinline__ double tet_volume_v4(const Tet& t) {
  const double ax = t.x[0] - t.x[3], ay = t.y[0] - t.y[3], az = t.z[0] - t.z[3];
  const double bx = t.x[1] - t.x[3], by = t.y[1] - t.y[3], bz = t.z[1] - t.z[3];
  const double cx = t.x[2] - t.x[3], cy = t.y[2] - t.y[3], cz = t.z[2] - t.z[3];
  const double xx = by * cz - bz * cy;
  const double xy = bz * cx - bx * cz;
  const double xz = bx * cy - by * cx;
  const double d = (ax * xx + ay * xy) + az * xz;
  return fabs(d) / 6.0;
}

// ------------------------------------------------------------- tri setup
// Three edge lines of triangle B: (normal, point), normals not normalised,
// orientation fixed so that the inside has negative distance.
struct Lines {
  double nx[3], ny[3], px[3], py[3];
};

__device__ __forceinline__ void tri_lines(const double* v, Lines& L) {
  L.nx[0] = -(v[3] - v[1]);
  L.ny[0] = (v[2] - v[0]);
  L.px[0] = v[0];
  L.py[0] = v[1];
  L.nx[1] = -(v[5] - v[3]);
  L.ny[1] = (v[4] - v[2]);
  L.px[1] = v[2];
  L.py[1] = v[3];
  L.nx[2] = -(v[1] - v[5]);
  L.ny[2] = (v[0] - v[4]);
  L.px[2] = v[4];
  L.py[2] = v[5];
  const double dot = (v[2] - v[0]) * L.nx[2] + (v[3] - v[1]) * L.ny[2];
  if (dot > 0.0) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      L.nx[i] = -L.nx[i];
      L.ny[i] = -L.ny[i];
    }
  }
}

// Edge lines of a convex polygon B with `loc` vertices
// (Triangle_Intersection.F90:422-451): normal (y_{i+1}-y_i, -(x_{i+1}-x_i)),
// point v_i, all flipped when (v_1 - p_2) . n_2 > 0.
template <int LOC>
__device__ __forceinline__ void poly_lines(const double* v, double* nx, double* ny, double* px, double* py) {
#pragma unroll
  for (int i = 0; i < LOC; ++i) {
    const int j = (i + 1) % LOC;
    nx[i] = (v[2 * j + 1] - v[2 * i + 1]);
    ny[i] = -(v[2 * j] - v[2 * i]);
    px[i] = v[2 * i];
    py[i] = v[2 * i + 1];
  }
  const double dot = (v[0] - px[1]) * nx[1] + (v[1] - py[1]) * ny[1];
  if (dot > 0.0) {
#pragma unroll
    for (int i = 0; i < LOC; ++i) {
      nx[i] = -nx[i];
      ny[i] = -ny[i];
    }
  }
}

// Keep test of a final tet (vol_v4 >= tol) and its vertex-1 volume, with
// the vertex-4 volume evaluated only when needed.  Both volumes are |det|/6
// of the same four points through different edges; each computed det is
// within 8u T of the exact one, T the sum of the absolute monomials, T <= L^3
// for the vertex-1 edges and <= 4 L^3 for the vertex-4 edges (L the largest
// L1 length of the vertex-1 edges, u = 2^-53), so |v1 - v4| <= 7.4u L^3 + 2u
// v1.  bnd = 64u L^3 (+ an absolute term for subnormal results) bounds it
// with room to spare: if v1 clears tol by bnd the outcome of v4 >= tol is
// known; otherwise v4 is computed and compared as the reference does.
// Overflow or NaN make both quick comparisons false and take the exact path.
__device__ __forceinline__ bool final_tet_keep(const Tet& t, double tol, double& v1) {
  const double e1x = t.x[1] - t.x[0], e1y = t.y[1] - t.y[0], e1z = t.z[1] - t.z[0];
  const double e2x = t.x[2] - t.x[0], e2y = t.y[2] - t.y[0], e2z = t.z[2] - t.z[0];
  const double e3x = t.x[3] - t.x[0], e3y = t.y[3] - t.y[0], e3z = t.z[3] - t.z[0];
  double s = e1x * (e2y * e3z - e2z * e3y) + e1y * (e2z * e3x - e2x * e3z);
  s = s + e1z * (e2x * e3y - e2y * e3x);
  v1 = (1.0 / 6.0) * fabs(s);
  const double l1 = (fabs(e1x) + fabs(e1y)) + fabs(e1z);
  const double l2 = (fabs(e2x) + fabs(e2y)) + fabs(e2z);
  const double l3 = (fabs(e3x) + fabs(e3y)) + fabs(e3z);
  const double L = fmax(l1, fmax(l2, l3));
  const double bnd = 0x1p-47 * (L * L * L) + 0x1p-1016;
  if (v1 >= tol + bnd) return true;
  if (v1 < tol - bnd) return false;
  return tet_volume_v4(t) >= tol;
}

// ------------------------------------------------------------- tet setup
struct Planes {
  double nx[4], ny[4], nz[4], c[4];
};

__device__ __forceinline__ void unit_cross(double ax, double ay, double az, double bx,
                                           double by, double bz, double& ox, double& oy,
                                           double& oz) {
  ox = ay * bz - az * by;
  oy = az * bx - ax * bz;
  oz = ax * by - ay * bx;
  const double n = norm2_3(ox, oy, oz);
  ox = ox / n;
  oy = oy / n;
  oz = oz / n;
}

__device__ __forceinline__ void tet_planes(const Tet& t, Planes& P) {
  const double e10x = t.x[1] - t.x[0], e10y = t.y[1] - t.y[0], e10z = t.z[1] - t.z[0];
  const double e20x = t.x[2] - t.x[0], e20y = t.y[2] - t.y[0], e20z = t.z[2] - t.z[0];
  const double e30x = t.x[3] - t.x[0], e30y = t.y[3] - t.y[0], e30z = t.z[3] - t.z[0];
  const double e21x = t.x[2] - t.x[1], e21y = t.y[2] - t.y[1], e21z = t.z[2] - t.z[1];
  const double e31x = t.x[3] - t.x[1], e31y = t.y[3] - t.y[1], e31z = t.z[3] - t.z[1];
  unit_cross(e20x, e20y, e20z, e10x, e10y, e10z, P.nx[0], P.ny[0], P.nz[0]);
  unit_cross(e10x, e10y, e10z, e30x, e30y, e30z, P.nx[1], P.ny[1], P.nz[1]);
  unit_cross(e30x, e30y, e30z, e20x, e20y, e20z, P.nx[2], P.ny[2], P.nz[2]);
  unit_cross(e21x, e21y, e21z, e31x, e31y, e31z, P.nx[3], P.ny[3], P.nz[3]);
  const double det = (e10x * P.nx[3] + e10y * P.ny[3]) + e10z * P.nz[3];
  if (det < 0.0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      P.nx[i] = -P.nx[i];
      P.ny[i] = -P.ny[i];
      P.nz[i] = -P.nz[i];
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) P.c[i] = (t.x[i] * P.nx[i] + t.y[i] * P.ny[i]) + t.z[i] * P.nz[i];
}

// ------------------------------------------------ separation screen (3D)
// Data for the second exact early-out of the tet clipper, which proves that
// B lies beyond a face plane of A (the first one, in the prefilter, proves
// that A lies beyond a face plane of B).  Notation: u = 2^-53, M bounds the
// coordinates of A and B and the plane offsets c of B.
//
// (1) Every vertex the reference's clipping of A creates is a rounded convex
//     combination of A's vertices: one interpolation w0*vp + w1*vn has
//     w0, w1 in [0, 1+3u], w0 + w1 = 1 +- 3u and 2u rounding per coordinate,
//     so it lies within 8.7u*M' of an exact convex combination; four nested
//     levels stay within 36u*M.  For any direction n (|n| <= 1 + 6u),
//     n.p <= max_k n.a_k + 40u*M.  faces_a keeps h = that maximum plus
//     128*eps*(1 + M) (eps = 2u), which also covers the rounding of n.a_k.
// (2) Every vertex of every tet left after B's four planes satisfies
//     n_L.v - c_L <= e for all four planes (exact arithmetic on the stored
//     plane coefficients) with e = 2^-52 + 48u(M + |c|): it was classified
//     non-positive (computed d < 2^-52), or created on plane L (exact d
//     within 19u(M+|c|) of 0), and later interpolations of such vertices add
//     at most 7u(M+|c|) each.  So those vertices lie in
//     B+ = {x : n_L.x <= c_L + e, L = 0..3}.
// (3) If the four stored normals positively span R^3 (the signed 3x3
//     cofactors D_k all share one sign), B+ is bounded, and each of its
//     vertices is some v+_k = M_k^-1 (c + e), M_k = the three normals through
//     vertex k; |v+_k - b_k| <= sqrt3 |M_k^-1| (e + tau)
//     <= 3.01 (e + tau) / |det M_k|, tau = the largest residual
//     |n_L.b_k - c_L| of a stored plane at one of its own vertices.
//     screen_b keeps g = 3.02 / (min|D_k| - 1e-14) (+inf when the sign test
//     or the margin fails) and tau plus its own rounding.
// (4) If min_j n.b_j - 1.01 g (tau + e) > h for a face n of A, B+ and the
//     derived vertices are disjoint: no tet survives B's four planes and the
//     reference returns 0 tets.  The prefilter applies this with e bounded
//     by 2^-52 + 128*eps*(1 + 2M) and an extra 16*eps*(1 + M) for the
//     rounding of n.b_j.
//
// faces_a [nel][16]: 4 x (nx, ny, nz, h) of A's outward face planes.
// screen_b [nel][16]: B's 4 vertices (x, y, z), g, tau, M_B, 0.
__device__ __forceinline__ double max_abs_tet(const Tet& t) {
  double M = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) M = fmax(M, fmax(fabs(t.x[k]), fmax(fabs(t.y[k]), fabs(t.z[k]))));
  return M;
}

__device__ __forceinline__ double pos_inf() { return __longlong_as_double(0x7ff0000000000000ll); }

// Two doubles in one 16-byte store (p 16-byte aligned: every per-element row
// the prep writes holds an even number of doubles).
__device__ __forceinline__ void st2(double* p, double a, double b) {
  *reinterpret_cast<double2*>(p) = make_double2(a, b);
}

__device__ __forceinline__ void tet_faces_screen(const Tet& t, double* o) {
  Planes P;
  tet_planes(t, P);
  const double drift = 128.0 * kEps * (1.0 + max_abs_tet(t));
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    // a face of a degenerate A (a repeated vertex: zero cross product, NaN
    // normal) proves nothing: (0, 0, 0, +inf) never rejects.  fmax would
    // skip the NaN products and leave h at -inf, which rejects every B.
    const bool ok = isfinite(P.nx[i]) && isfinite(P.ny[i]) && isfinite(P.nz[i]);
    double h = -pos_inf();
#pragma unroll
    for (int k = 0; k < 4; ++k) h = fmax(h, (P.nx[i] * t.x[k] + P.ny[i] * t.y[k]) + P.nz[i] * t.z[k]);
    st2(o + 4 * i, ok ? P.nx[i] : 0.0, ok ? P.ny[i] : 0.0);
    st2(o + 4 * i + 2, ok ? P.nz[i] : 0.0, ok && isfinite(h) ? h + drift : pos_inf());
  }
}

__device__ __forceinline__ double det3(double ax, double ay, double az, double bx, double by, double bz,
                                       double cx, double cy, double cz) {
  return (ax * (by * cz - bz * cy) + ay * (bz * cx - bx * cz)) + az * (bx * cy - by * cx);
}

__device__ __forceinline__ void tet_screen_b(const Tet& t, const Planes& P, double* o) {
  double M = max_abs_tet(t);
#pragma unroll
  for (int i = 0; i < 4; ++i) M = fmax(M, fabs(P.c[i]));
  // residuals of each plane at its three own vertices (plane f omits vertex 3-f)
  double tau = 0.0;
#pragma unroll
  for (int f = 0; f < 4; ++f)
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k != 3 - f)
        tau = fmax(tau, fabs(((P.nx[f] * t.x[k] + P.ny[f] * t.y[k]) + P.nz[f] * t.z[k]) - P.c[f]));
  // D_j = (-1)^j det(normals other than j, in index order); sum_j D_j n_j = 0
  double D[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int r0 = j == 0 ? 1 : 0;
    const int r1 = j <= 1 ? 2 : 1;
    const int r2 = j <= 2 ? 3 : 2;
    const double d = det3(P.nx[r0], P.ny[r0], P.nz[r0], P.nx[r1], P.ny[r1], P.nz[r1], P.nx[r2], P.ny[r2],
                          P.nz[r2]);
    D[j] = (j & 1) ? -d : d;
  }
  const double kDetErr = 1e-14;
  const bool pos = D[0] > kDetErr && D[1] > kDetErr && D[2] > kDetErr && D[3] > kDetErr;
  const bool neg = D[0] < -kDetErr && D[1] < -kDetErr && D[2] < -kDetErr && D[3] < -kDetErr;
  const double dmin = fmin(fmin(fabs(D[0]), fabs(D[1])), fmin(fabs(D[2]), fabs(D[3])));
  const double g = (pos || neg) ? 3.02 / (dmin - kDetErr) : pos_inf();
  st2(o + 0, t.x[0], t.y[0]);
  st2(o + 2, t.z[0], t.x[1]);
  st2(o + 4, t.y[1], t.z[1]);
  st2(o + 6, t.x[2], t.y[2]);
  st2(o + 8, t.z[2], t.x[3]);
  st2(o + 10, t.y[3], t.z[3]);
  st2(o + 12, g, tau + 16.0 * kEps * (1.0 + 2.0 * M));
  st2(o + 14, M, 0.0);
}

// Face planes of a hexahedron in Gmsh node order (Supermesh.F90:262-280):
// plane f = unit_cross(h[a] - h[b], h[c] - h[d]) with offset h[b] . n; no
// orientation fix-up.
__device__ __forceinline__ void hex_planes(const double* h, double* nx, double* ny, double* nz, double* c) {
  const int F[6][4] = {{1, 0, 5, 0}, {5, 4, 6, 4}, {1, 5, 2, 5}, {0, 1, 3, 1}, {4, 0, 7, 0}, {6, 7, 2, 7}};
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const double* a = h + 3 * F[f][0];
    const double* b = h + 3 * F[f][1];
    const double* cc = h + 3 * F[f][2];
    const double* d = h + 3 * F[f][3];
    unit_cross(a[0] - b[0], a[1] - b[1], a[2] - b[2], cc[0] - d[0], cc[1] - d[1], cc[2] - d[2], nx[f], ny[f],
               nz[f]);
    c[f] = (b[0] * nx[f] + b[1] * ny[f]) + b[2] * nz[f];
  }
}

// Interval length and intersection (Interval_Intersection.F90:45-110).
__device__ __forceinline__ double interval_size(double a0, double a1) { return fabs(a1 - a0); }

__device__ __forceinline__ int intersect_intervals(double a0, double a1, double b0, double b1, double& c0,
                                                   double& c1) {
  const double min_a = fmin(a0, a1), max_a = fmax(a0, a1);
  const double min_b = fmin(b0, b1), max_b = fmax(b0, b1);
  if (max_b <= min_a || min_b >= max_a) return 0;
  c0 = fmax(min_a, min_b);
  c1 = fmin(max_a, max_b);
  const double tol = 10.0 * fmin(spacing(interval_size(a0, a1)), spacing(interval_size(b0, b1)));
  return interval_size(c0, c1) < tol ? 0 : 1;
}

// ------------------------------------------------------------ tri clipping
// Polygon storage is supplied by the caller through an accessor so that the
// same code runs on shared-memory slots (fast path) or local arrays.
// clip_stage: one Sutherland-Hodgman pass of polygon `in` (n vertices)
// against line (nx,ny,px,py), writing to `out`; returns the output count or
// -1 when it would exceed `cap` slots.
template <class Poly>
__device__ __forceinline__ int clip_stage(const Poly& in, Poly& out, int n, int cap, double nx,
                                          double ny, double px, double py) {
  const double x0 = in.x(0), y0 = in.y(0);
  const double d0 = nx * (x0 - px) + ny * (y0 - py);
  double x1 = x0, y1 = y0, d1 = d0;
  int m = 0;
  for (int i = 0; i < n; ++i) {
    double x2, y2, d2;
    if (i == n - 1) {
      x2 = x0;
      y2 = y0;
      d2 = d0;
    } else {
      x2 = in.x(i + 1);
      y2 = in.y(i + 1);
      d2 = nx * (x2 - px) + ny * (y2 - py);
    }
    if (d1 < 0.0) {
      if (m + (d2 <= 0.0 ? 1 : 2) > cap) return -1;
      out.set(m++, x1, y1);
      if (!(d2 <= 0.0)) {
        double f = fabs(d1) / (fabs(d1) + fabs(d2));
        f = fmax(fmin(f, 1.0), 0.0);
        out.set(m++, x1 + f * (x2 - x1), y1 + f * (y2 - y1));
      }
    } else if (d1 == 0.0) {
      if (m + 1 > cap) return -1;
      out.set(m++, x1, y1);
    } else if (d2 < 0.0) {
      if (m + 1 > cap) return -1;
      double f = fabs(d1) / (fabs(d1) + fabs(d2));
      f = fmax(fmin(f, 1.0), 0.0);
      out.set(m++, x1 + f * (x2 - x1), y1 + f * (y2 - y1));
    }
    x1 = x2;
    y1 = y2;
    d1 = d2;
  }
  return m;
}

// Full tri-tri clip.  Returns the number of kept fan triangles, or -1 on
// buffer overflow (caller retries with larger buffers).  `measure` receives
// the sum of kept fan-triangle areas in fan order.  If `emit` is non-null
// it is called as emit(k, x0,y0, x1,y1, x2,y2) for each kept triangle.
template <class Poly, class Emit>
__device__ __forceinline__ int clip_tri(double ax0, double ay0, double ax1, double ay1,
                                        double ax2, double ay2, const Lines& L, double tol,
                                        Poly& p, Poly& q, int cap, double& measure,
                                        Emit emit) {
  measure = 0.0;
  p.set(0, ax0, ay0);
  p.set(1, ax1, ay1);
  p.set(2, ax2, ay2);
  int n = clip_stage(p, q, 3, cap, L.nx[0], L.ny[0], L.px[0], L.py[0]);
  if (n < 0) return -1;
  if (n < 3) return 0;
  n = clip_stage(q, p, n, cap, L.nx[1], L.ny[1], L.px[1], L.py[1]);
  if (n < 0) return -1;
  if (n < 3) return 0;
  n = clip_stage(p, q, n, cap, L.nx[2], L.ny[2], L.px[2], L.py[2]);
  if (n < 0) return -1;
  if (n < 3) return 0;
  const double x0 = q.x(0), y0 = q.y(0);
  int kept = 0;
  double xi = q.x(1), yi = q.y(1);
  for (int i = 1; i < n - 1; ++i) {
    const double xj = q.x(i + 1), yj = q.y(i + 1);
    const double ar = tri_area(x0, y0, xi, yi, xj, yj);
    if (!(ar < tol)) {
      measure = measure + ar;
      emit(kept, x0, y0, xi, yi, xj, yj);
      ++kept;
    }
    xi = xj;
    yi = yj;
  }
  return kept;
}

// ------------------------------------------------------------ tet clipping
// Dynamic-index helpers (selects keep the tet in registers).
__device__ __forceinline__ double sel4(int k, double a0, double a1, double a2, double a3) {
  double r = a3;
  r = (k == 2) ? a2 : r;
  r = (k == 1) ? a1 : r;
  r = (k == 0) ? a0 : r;
  return r;
}

struct V3 {
  double x, y, z;
};

__device__ __forceinline__ V3 vget(const Tet& t, int k) {
  return V3{sel4(k, t.x[0], t.x[1], t.x[2], t.x[3]), sel4(k, t.y[0], t.y[1], t.y[2], t.y[3]),
            sel4(k, t.z[0], t.z[1], t.z[2], t.z[3])};
}

__device__ __forceinline__ void vset(Tet& t, int k, const V3& v) {
  t.x[k] = v.x;
  t.y[k] = v.y;
  t.z[k] = v.z;
}

// w0 * vp + w1 * vn, invdiff = 1/(dp - dn), w0 = -dn*invdiff, w1 = dp*invdiff
__device__ __forceinline__ V3 interp(const V3& vp, const V3& vn, double dp, double dn) {
  const double invdiff = __drcp_rn(dp - dn);
  const double w0 = -dn * invdiff;
  const double w1 = dp * invdiff;
  return V3{w0 * vp.x + w1 * vn.x, w0 * vp.y + w1 * vn.y, w0 * vp.z + w1 * vn.z};
}

// Classification of a tet's vertices against one plane
// (Tetrahedron_Intersection.F90:257-276): zero if |d| < eps, else by sign.
// Index lists are packed 2 bits per entry in ascending vertex order.
struct TetClass {
  double d[4];
  unsigned negl, posl, zerl;
  int nn, np;
};

__device__ __forceinline__ void classify_tet(const Tet& t, double nx, double ny, double nz, double c,
                                             TetClass& k) {
#pragma unroll
  for (int i = 0; i < 4; ++i) k.d[i] = ((nx * t.x[i] + ny * t.y[i]) + nz * t.z[i]) - c;
  unsigned negl = 0, posl = 0, zerl = 0;
  int nn = 0, np = 0, nz0 = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const bool zero = fabs(k.d[i]) < kEps;
    const bool neg = !zero && k.d[i] < 0.0;
    const bool pos = !zero && k.d[i] > 0.0;
    zerl |= zero ? (unsigned)i << (2 * nz0) : 0u;
    negl |= neg ? (unsigned)i << (2 * nn) : 0u;
    posl |= pos ? (unsigned)i << (2 * np) : 0u;
    nz0 += zero;
    nn += neg;
    np += pos;
  }
  k.negl = negl;
  k.posl = posl;
  k.zerl = zerl;
  k.nn = nn;
  k.np = np;
}

// Split a tet that has both positive and negative vertices
// (Tetrahedron_Intersection.F90:290-434).  Returns the number of children
// (1..3); `t` becomes child 0 and c1, c2 children 1 and 2, in the
// reference's output order.
//
// Every case (+++-, ++-0, +-00, ++--, +---, +--0) creates its new vertices
// by the same interpolation between a positive and a negative vertex, so the
// interpolations run in one predicated loop shared by all cases (warp lanes
// in different cases stay converged for the FP64 work); the cases differ
// only in which (positive, negative) pairs they interpolate and in how the
// children are assembled from vertices, which is register moves.
__device__ __forceinline__ int split_tet(Tet& t, const TetClass& k, Tet& c1, Tet& c2) {
  const int nn = k.nn, np = k.np;
  const int n0 = k.negl & 3, n1 = (k.negl >> 2) & 3, n2 = (k.negl >> 4) & 3;
  const int p0 = k.posl & 3, p1 = (k.posl >> 2) & 3, p2 = (k.posl >> 4) & 3;
  // interpolation list: entry i = (positive vertex, negative vertex)
  int ni;
  unsigned pairs;
  if (nn == 1) {  // every positive vertex towards n0
    ni = np;
    pairs = (unsigned)(p0 | n0 << 2) | (unsigned)(p1 | n0 << 2) << 4 | (unsigned)(p2 | n0 << 2) << 8;
  } else if (np == 2) {  // ++--: t0 = (p0,n0), t1 = (p1,n0), t2 = (p0,n1), t3 = (p1,n1)
    ni = 4;
    pairs = (unsigned)(p0 | n0 << 2) | (unsigned)(p1 | n0 << 2) << 4 | (unsigned)(p0 | n1 << 2) << 8 |
            (unsigned)(p1 | n1 << 2) << 12;
  } else {  // +--- / +--0: p0 towards each negative vertex
    ni = nn;
    pairs = (unsigned)(p0 | n0 << 2) | (unsigned)(p0 | n1 << 2) << 4 | (unsigned)(p0 | n2 << 2) << 8;
  }
  V3 T[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (i < ni) {
      const int P = (pairs >> (4 * i)) & 3, N = (pairs >> (4 * i + 2)) & 3;
      T[i] = interp(vget(t, P), vget(t, N), sel4(P, k.d[0], k.d[1], k.d[2], k.d[3]),
                    sel4(N, k.d[0], k.d[1], k.d[2], k.d[3]));
    } else {
      T[i] = V3{0.0, 0.0, 0.0};
    }
  }
  if (nn == 1) {
    // +++-, ++-0, +-00: positive vertex of rank r becomes T[r]
    unsigned pm = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
      if (i < np) pm |= 1u << ((k.posl >> (2 * i)) & 3);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      if (pm & (1u << v)) {
        const int r = __popc(pm & ((1u << v) - 1u));
        const V3 q = r == 0 ? T[0] : (r == 1 ? T[1] : T[2]);
        t.x[v] = q.x;
        t.y[v] = q.y;
        t.z[v] = q.z;
      }
    }
    return 1;
  }
  const V3 vn0 = vget(t, n0), vn1 = vget(t, n1);
  if (np == 2) {
    // ++--: child 0 = tet with v[p0] = t2, v[p1] = t1;
    //       child 1 = (v[n1], t3, t2, t1); child 2 = (v[n0], t0, t1, t2)
    vset(c1, 0, vn1);
    vset(c1, 1, T[3]);
    vset(c1, 2, T[2]);
    vset(c1, 3, T[1]);
    vset(c2, 0, vn0);
    vset(c2, 1, T[0]);
    vset(c2, 2, T[1]);
    vset(c2, 3, T[2]);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      if (v == p0) {
        t.x[v] = T[2].x;
        t.y[v] = T[2].y;
        t.z[v] = T[2].z;
      } else if (v == p1) {
        t.x[v] = T[1].x;
        t.y[v] = T[1].y;
        t.z[v] = T[1].z;
      }
    }
    return 3;
  }
  int kk;
  if (nn == 3) {
    // +---: child 1 = (t0, v[n1], v[n2], t1); child 2 = (v[n2], t1, t2, t0)
    const V3 vn2 = vget(t, n2);
    vset(c1, 0, T[0]);
    vset(c1, 1, vn1);
    vset(c1, 2, vn2);
    vset(c1, 3, T[1]);
    vset(c2, 0, vn2);
    vset(c2, 1, T[1]);
    vset(c2, 2, T[2]);
    vset(c2, 3, T[0]);
    kk = 3;
  } else {
    // +--0: child 1 = (t1, v[z0], v[n1], t0)
    const V3 vz0 = vget(t, k.zerl & 3);
    vset(c1, 0, T[1]);
    vset(c1, 1, vz0);
    vset(c1, 2, vn1);
    vset(c1, 3, T[0]);
    kk = 2;
  }
  // child 0 = tet with v[p0] = t0
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    if (v == p0) {
      t.x[v] = T[0].x;
      t.y[v] = T[0].y;
      t.z[v] = T[0].z;
    }
  }
  return kk;
}

// Clip tet `t` by plane (nx,ny,nz,c) (Tetrahedron_Intersection.F90:244-436).
// Returns the number of children k (0..3); `t` holds child 0.  The children
// are handed to the sink in the reference's output order: emit.begin(k),
// emit.child(0, t), emit.child(1, c1), emit.child(2, c2).
template <class Emit>
__device__ __forceinline__ int clip_tet_plane(Tet& t, double nx, double ny, double nz, double c,
                                              Emit& emit) {
  TetClass k;
  classify_tet(t, nx, ny, nz, c, k);
  if (k.nn == 0) return 0;
  if (k.np == 0) {
    emit.begin(1);
    emit.child(0, t);
    return 1;
  }
  Tet c1, c2;
  const int n = split_tet(t, k, c1, c2);
  emit.begin(n);
  emit.child(0, t);
  if (n >= 2) emit.child(1, c1);
  if (n >= 3) emit.child(2, c2);
  return n;
}

}  // namespace lsm
