"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package; the product library never does.  The C sources
(oracle.c) restate libsupermesh's serial hot path; see oracle.h.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

_DIR = Path(__file__).resolve().parent
_LIB_PATH = _DIR / "_build" / "liboracle.so"
_lib = None

TRI_BUF = 22
TET_BUF = 81

_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_candidates", ctypes.c_int64),
        ("n_intersecting", ctypes.c_int64),
        ("n_out_simplices", ctypes.c_int64),
        ("total", ctypes.c_double),
        ("total_err", ctypes.c_double),
        ("flops", ctypes.c_double),
    ]


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(_DIR)], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(_LIB_PATH))
        L.orc_spacing.restype = ctypes.c_double
        L.orc_spacing.argtypes = [ctypes.c_double]
        L.orc_norm2_3.restype = ctypes.c_double
        L.orc_triangle_area.restype = ctypes.c_double
        L.orc_tetrahedron_volume.restype = ctypes.c_double
        L.orc_tetrahedron_volume_v4.restype = ctypes.c_double
        L.orc_kahan_sum.restype = ctypes.c_double
        L.orc_kahan_sum.argtypes = [_dp, ctypes.c_long]
        L.orc_num_threads_available.restype = ctypes.c_int
        L.orc_interval_size.restype = ctypes.c_double
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i32(a):
    return a.ctypes.data_as(_i32p)


def _i64(a):
    return a.ctypes.data_as(_i64p)


def spacing(x: float) -> float:
    return lib().orc_spacing(float(x))


def triangle_area(tri) -> float:
    t = np.ascontiguousarray(tri, dtype=np.float64).reshape(6)
    return lib().orc_triangle_area(_d(t))


def tetrahedron_volume(tet) -> float:
    t = np.ascontiguousarray(tet, dtype=np.float64).reshape(12)
    return lib().orc_tetrahedron_volume(_d(t))


def intersect_tris(tri_a, tri_b):
    a = np.ascontiguousarray(tri_a, dtype=np.float64).reshape(6)
    b = np.ascontiguousarray(tri_b, dtype=np.float64).reshape(6)
    out = np.zeros((TRI_BUF, 3, 2))
    n = ctypes.c_int(0)
    lib().orc_intersect_tris(_d(a), _d(b), _d(out), ctypes.byref(n))
    return out[: n.value].copy()


def intersect_tets(tet_a, tet_b):
    a = np.ascontiguousarray(tet_a, dtype=np.float64).reshape(12)
    b = np.ascontiguousarray(tet_b, dtype=np.float64).reshape(12)
    out = np.zeros((TET_BUF, 4, 3))
    n = ctypes.c_int(0)
    lib().orc_intersect_tets(_d(a), _d(b), _d(out), ctypes.byref(n))
    return out[: n.value].copy()


def intersect_tri_quad(tri_a, quad_b):
    a = np.ascontiguousarray(tri_a, dtype=np.float64).reshape(6)
    b = np.ascontiguousarray(quad_b, dtype=np.float64).reshape(8)
    out = np.zeros((46, 3, 2))
    n = ctypes.c_int(0)
    lib().orc_intersect_tri_quad(_d(a), _d(b), _d(out), ctypes.byref(n))
    return out[: n.value].copy()


def intersect_tet_hex(tet_a, hex_b):
    a = np.ascontiguousarray(tet_a, dtype=np.float64).reshape(12)
    b = np.ascontiguousarray(hex_b, dtype=np.float64).reshape(24)
    out = np.zeros((729, 4, 3))
    n = ctypes.c_int(0)
    lib().orc_intersect_tet_hex(_d(a), _d(b), _d(out), ctypes.byref(n))
    return out[: n.value].copy()


def intersect_quads(quad_a, quad_b):
    a = np.ascontiguousarray(quad_a, dtype=np.float64).reshape(8)
    b = np.ascontiguousarray(quad_b, dtype=np.float64).reshape(8)
    out = np.zeros((62, 3, 2))
    n = ctypes.c_int(0)
    lib().orc_intersect_quads(_d(a), _d(b), _d(out), ctypes.byref(n))
    return out[: n.value].copy()


def intersect_hexes(hex_a, hex_b):
    a = np.ascontiguousarray(hex_a, dtype=np.float64).reshape(24)
    b = np.ascontiguousarray(hex_b, dtype=np.float64).reshape(24)
    out = np.zeros((5 * 729, 4, 3))
    n = ctypes.c_int(0)
    lib().orc_intersect_hexes(_d(a), _d(b), _d(out), ctypes.byref(n))
    return out[: n.value].copy()


def intersect_intervals(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(2)
    b = np.ascontiguousarray(b, dtype=np.float64).reshape(2)
    out = np.zeros(2)
    n = ctypes.c_int(0)
    lib().orc_intersect_intervals(_d(a), _d(b), _d(out), ctypes.byref(n))
    return out.copy() if n.value else np.zeros(0)


def interval_size(iv) -> float:
    iv = np.ascontiguousarray(iv, dtype=np.float64).reshape(2)
    return lib().orc_interval_size(_d(iv))


def sort_finder_1d(mesh_a, mesh_b, stable: bool = True):
    """Sort-and-sweep finder for 2-node meshes (first coordinate of each
    node).  stable=False keeps the reference's merge sort leaf step as
    written; stable=True uses the stable sort by left end."""
    pa = np.ascontiguousarray(mesh_a[0], dtype=np.float64)
    pb = np.ascontiguousarray(mesh_b[0], dtype=np.float64)
    sa = 1 if pa.ndim == 1 else pa.shape[1]
    sb = 1 if pb.ndim == 1 else pb.shape[1]
    ea = np.ascontiguousarray(mesh_a[1], dtype=np.int32)
    eb = np.ascontiguousarray(mesh_b[1], dtype=np.int32)
    indptr = np.zeros(ea.shape[0] + 1, dtype=np.int64)
    ind = _i32p()
    nnz = ctypes.c_int64(0)
    rc = lib().orc_sort_finder_1d(ctypes.c_long(pa.shape[0]), _d(pa), ctypes.c_int(sa), ctypes.c_long(ea.shape[0]),
                                  _i32(ea), ctypes.c_long(pb.shape[0]), _d(pb), ctypes.c_int(sb),
                                  ctypes.c_long(eb.shape[0]), _i32(eb), ctypes.c_int(int(stable)),
                                  _i64(indptr), ctypes.byref(ind), ctypes.byref(nnz))
    if rc != 0:
        raise RuntimeError("oracle 1D finder failed")
    n = nnz.value
    indices = np.ctypeslib.as_array(ind, shape=(max(n, 1),))[:n].copy()
    lib().orc_free(ind)
    return indptr, indices


def _mesh_args(pos, en):
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    en = np.ascontiguousarray(en, dtype=np.int32)
    return pos, en


def _finder(fn, dim, mesh_a, mesh_b, *extra):
    pa, ea = _mesh_args(*mesh_a)
    pb, eb = _mesh_args(*mesh_b)
    indptr = np.zeros(ea.shape[0] + 1, dtype=np.int64)
    ind = _i32p()
    nnz = ctypes.c_int64(0)
    rc = fn(ctypes.c_int(dim), ctypes.c_long(pa.shape[0]), _d(pa), ctypes.c_long(ea.shape[0]),
            ctypes.c_int(ea.shape[1]), _i32(ea), ctypes.c_long(pb.shape[0]), _d(pb),
            ctypes.c_long(eb.shape[0]), ctypes.c_int(eb.shape[1]), _i32(eb), *extra,
            _i64(indptr), ctypes.byref(ind), ctypes.byref(nnz))
    if rc != 0:
        raise RuntimeError("oracle finder failed")
    n = nnz.value
    indices = np.ctypeslib.as_array(ind, shape=(max(n, 1),))[:n].copy()
    lib().orc_free(ind)
    return indptr, indices


def tree_finder(dim, mesh_a, mesh_b, max_size: int = 0):
    """Quadtree/octree finder: CSR (indptr[nel_a+1], indices) over A rows."""
    return _finder(lib().orc_tree_finder, dim, mesh_a, mesh_b, ctypes.c_int(max_size))


def brute_force_finder(dim, mesh_a, mesh_b):
    return _finder(lib().orc_brute_force_finder, dim, mesh_a, mesh_b)


def narrow(dim, mesh_a, mesh_b, indptr, indices, nthreads: int = 1, count_flops: bool = False):
    """Clip every candidate pair; returns (pair_measure, pair_nout,
    elem_measure, Stats)."""
    pa, ea = _mesh_args(*mesh_a)
    pb, eb = _mesh_args(*mesh_b)
    indptr = np.ascontiguousarray(indptr, dtype=np.int64)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    nnz = int(indptr[-1])
    pm = np.zeros(max(nnz, 1))
    pn = np.zeros(max(nnz, 1), dtype=np.int32)
    em = np.zeros(max(ea.shape[0], 1))
    st = Stats()
    rc = lib().orc_narrow(ctypes.c_int(dim), _d(pa), ctypes.c_int(ea.shape[1]), _i32(ea),
                          ctypes.c_long(ea.shape[0]), _d(pb), ctypes.c_int(eb.shape[1]), _i32(eb),
                          ctypes.c_long(eb.shape[0]), _i64(indptr), _i32(indices), _d(pm), _i32(pn),
                          _d(em), ctypes.c_int(nthreads), ctypes.c_int(int(count_flops)),
                          ctypes.byref(st))
    if rc != 0:
        raise RuntimeError("oracle narrow phase failed")
    return pm[:nnz], pn[:nnz], em[: ea.shape[0]], st


def supermesh(dim, mesh_a, mesh_b, nthreads: int = 1) -> Stats:
    pa, ea = _mesh_args(*mesh_a)
    pb, eb = _mesh_args(*mesh_b)
    st = Stats()
    rc = lib().orc_supermesh(ctypes.c_int(dim), ctypes.c_long(pa.shape[0]), _d(pa),
                             ctypes.c_long(ea.shape[0]), ctypes.c_int(ea.shape[1]), _i32(ea),
                             ctypes.c_long(pb.shape[0]), _d(pb), ctypes.c_long(eb.shape[0]),
                             ctypes.c_int(eb.shape[1]), _i32(eb), ctypes.c_int(nthreads),
                             ctypes.byref(st))
    if rc != 0:
        raise RuntimeError("oracle supermesh failed")
    return st


def p1_mass(dim, mesh_a, mesh_b, indptr, indices, u_a, v_b, want_blocks: bool = False):
    """Returns (integral u^T M v, supermesh measure, blocks or None)."""
    pa, ea = _mesh_args(*mesh_a)
    pb, eb = _mesh_args(*mesh_b)
    indptr = np.ascontiguousarray(indptr, dtype=np.int64)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    u = np.ascontiguousarray(u_a, dtype=np.float64)
    v = np.ascontiguousarray(v_b, dtype=np.float64)
    loc = dim + 1
    nnz = int(indptr[-1])
    blocks = np.zeros((max(nnz, 1), loc, loc)) if want_blocks else None
    integral = ctypes.c_double(0.0)
    measure = ctypes.c_double(0.0)
    rc = lib().orc_p1_mass(ctypes.c_int(dim), _d(pa), _i32(ea), ctypes.c_long(ea.shape[0]),
                           _d(pb), _i32(eb), ctypes.c_long(eb.shape[0]), _i64(indptr),
                           _i32(indices), _d(u), _d(v),
                           _d(blocks) if blocks is not None else None,
                           ctypes.byref(integral), ctypes.byref(measure))
    if rc != 0:
        raise RuntimeError("oracle p1 mass failed")
    return integral.value, measure.value, (blocks[:nnz] if blocks is not None else None)


def p2_inner_product(mesh_a, mesh_b, indptr, indices, en_p2_a, field_a, en_p2_b, field_b):
    """Returns (integral, area, per-pair contributions[nnz])."""
    pa, ea = _mesh_args(*mesh_a)
    pb, eb = _mesh_args(*mesh_b)
    indptr = np.ascontiguousarray(indptr, dtype=np.int64)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    e2a = np.ascontiguousarray(en_p2_a, dtype=np.int32)
    e2b = np.ascontiguousarray(en_p2_b, dtype=np.int32)
    fa = np.ascontiguousarray(field_a, dtype=np.float64)
    fb = np.ascontiguousarray(field_b, dtype=np.float64)
    nnz = int(indptr[-1])
    pv = np.zeros(max(nnz, 1))
    integral = ctypes.c_double(0.0)
    area = ctypes.c_double(0.0)
    rc = lib().orc_p2_inner_product(_d(pa), _i32(ea), ctypes.c_long(ea.shape[0]), _d(pb), _i32(eb), _i64(indptr),
                                    _i32(indices), _i32(e2a), _d(fa), _i32(e2b), _d(fb), _d(pv),
                                    ctypes.byref(integral), ctypes.byref(area))
    if rc != 0:
        raise RuntimeError("oracle p2 inner product failed")
    return integral.value, area.value, pv[:nnz]


def kahan_sum(x) -> float:
    x = np.ascontiguousarray(x, dtype=np.float64)
    return lib().orc_kahan_sum(_d(x), ctypes.c_long(x.size))


def fequals(a: float, b: float) -> bool:
    """Unittest_Tools.F90:179-195: |a-b| < 100*max(eps, spacing(a), spacing(b))."""
    eps = 100.0 * max(2.0 ** -52, spacing(a), spacing(b))
    return abs(a - b) < eps
