"""B200-native supermesh library: Python binding of lib/libsupermesh.so.

The shared library exports the drop-in C API of libsupermesh
(include/libsupermesh-c.h) and the GPU extension (include/libsupermesh-gpu.h).
``get_library`` / ``get_include`` / ``load`` mirror the loader of the
reference's Python package (src/supermesh/__init__.py:8-22 upstream).  The
classes below are thin ctypes wrappers over those C entry points; all work
runs on the GPU, and nothing here falls back to the CPU: if the CUDA library
is missing, ``load`` raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

__all__ = [
    "get_library", "get_include", "load", "Context", "LsmError", "Stats",
    "tree_intersection_finder", "intersect_tris_real", "intersect_tets_real",
    "triangle_area", "tetrahedron_volume", "TRI_BUF_SIZE", "TET_BUF_SIZE",
]

_PKG = Path(__file__).resolve().parent
_LIB = _PKG / "lib" / "libsupermesh.so"
TRI_BUF_SIZE = 22
TET_BUF_SIZE = 81
SCHED_PARAMS = 6792    # LSM_SCHED_PARAMS
SCHED_FEATURES = 32    # LSM_SCHED_FEATURES

_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_lp = ctypes.POINTER(ctypes.c_long)
_ip = ctypes.POINTER(ctypes.c_int)


def get_library() -> str:
    """Path of the shared library."""
    return str(_LIB)


def get_include() -> str:
    """Directory holding libsupermesh-c.h, libsupermesh.h, libsupermesh-gpu.h."""
    return str(_PKG.parent / "include")


class LsmError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"libsupermesh GPU call failed ({status}): {message}")
        self.status = status


class Mesh(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int),
        ("loc", ctypes.c_int),
        ("nnodes", ctypes.c_int64),
        ("nelements", ctypes.c_int64),
        ("positions", ctypes.c_void_p),
        ("enlist", ctypes.c_void_p),
        ("index_bytes", ctypes.c_int),
    ]


class BatchOut(ctypes.Structure):
    _fields_ = [
        ("totals", ctypes.c_void_p),
        ("n_candidates", ctypes.c_void_p),
        ("n_intersecting", ctypes.c_void_p),
        ("cand_offset", ctypes.c_void_p),
        ("total_candidates", ctypes.c_void_p),
        ("cand_capacity", ctypes.c_int64),
        ("ind_ptr", ctypes.c_void_p),
        ("indices", ctypes.c_void_p),
        ("pair_measure", ctypes.c_void_p),
        ("pair_n_out", ctypes.c_void_p),
        ("p1_offset", ctypes.c_void_p),
        ("p1_capacity", ctypes.c_int64),
        ("p1_blocks", ctypes.c_void_p),
    ]


class PairOut(ctypes.Structure):
    _fields_ = [
        ("elem_measure", ctypes.c_void_p),
        ("ind_ptr", ctypes.c_void_p),
        ("indices", ctypes.c_void_p),
        ("pair_measure", ctypes.c_void_p),
        ("pair_n_out", ctypes.c_void_p),
        ("cand_capacity", ctypes.c_int64),
        ("n_candidates", ctypes.c_int64),
    ]


class ElemOut(ctypes.Structure):
    _fields_ = [
        ("elem_offset", ctypes.c_void_p),
        ("elems", ctypes.c_void_p),
        ("parent_a", ctypes.c_void_p),
        ("parent_b", ctypes.c_void_p),
        ("cand_capacity", ctypes.c_int64),
        ("elem_capacity", ctypes.c_int64),
        ("n_candidates", ctypes.c_int64),
        ("n_elements", ctypes.c_int64),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_candidates", ctypes.c_int64),
        ("n_intersecting", ctypes.c_int64),
        ("n_out_simplices", ctypes.c_int64),
        ("total_measure", ctypes.c_double),
        ("total_measure_err", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load() -> ctypes.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB.exists():
        raise RuntimeError(
            f"{_LIB} is missing: build it with `python libsupermesh_b200/build.py` "
            "(there is no CPU implementation to fall back to)")
    L = ctypes.CDLL(str(_LIB))
    vp = ctypes.c_void_p
    L.libsupermesh_gpu_context_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    L.libsupermesh_gpu_context_destroy.argtypes = [vp]
    L.libsupermesh_gpu_status_string.restype = ctypes.c_char_p
    L.libsupermesh_gpu_status_string.argtypes = [ctypes.c_int]
    L.libsupermesh_gpu_last_error.restype = ctypes.c_char_p
    L.libsupermesh_gpu_last_error.argtypes = [vp]
    L.libsupermesh_gpu_context_bytes.restype = ctypes.c_int64
    L.libsupermesh_gpu_context_bytes.argtypes = [vp]
    L.libsupermesh_gpu_kernel_launches.restype = ctypes.c_int64
    L.libsupermesh_gpu_kernel_launches.argtypes = []
    L.libsupermesh_gpu_clip_kernel_ms.argtypes = [vp, _dp]
    L.libsupermesh_gpu_clip_kernel_ms.restype = ctypes.c_int
    L.libsupermesh_gpu_clip_survivors.argtypes = [vp, _i64p]
    L.libsupermesh_gpu_clip_survivors.restype = ctypes.c_int
    L.libsupermesh_gpu_set_option.argtypes = [ctypes.c_char_p, ctypes.c_int64]
    L.libsupermesh_gpu_set_option.restype = ctypes.c_int
    L.libsupermesh_gpu_get_option.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
    L.libsupermesh_gpu_get_option.restype = ctypes.c_int
    mp = ctypes.POINTER(Mesh)
    L.libsupermesh_gpu_find_candidates.argtypes = [vp, mp, mp, ctypes.c_int, _i64p, vp]
    L.libsupermesh_gpu_get_candidates.argtypes = [vp, vp, vp, ctypes.c_int, vp]
    L.libsupermesh_gpu_supermesh.argtypes = [vp, mp, mp, ctypes.c_int, vp, ctypes.POINTER(Stats), vp]
    L.libsupermesh_gpu_get_pair_results.argtypes = [vp, vp, vp, ctypes.c_int, vp]
    L.libsupermesh_gpu_clip_candidates.argtypes = [vp, ctypes.POINTER(Stats), vp]
    L.libsupermesh_gpu_supermesh_out.argtypes = [vp, mp, mp, ctypes.c_int, ctypes.POINTER(PairOut),
                                                 ctypes.POINTER(Stats), vp]
    L.libsupermesh_gpu_supermesh_out.restype = ctypes.c_int
    L.libsupermesh_gpu_supermesh_elements.argtypes = [vp, mp, mp, ctypes.c_int, ctypes.POINTER(ElemOut),
                                                      ctypes.POINTER(Stats), vp]
    L.libsupermesh_gpu_supermesh_elements.restype = ctypes.c_int
    L.libsupermesh_gpu_clip_candidates_ordered.argtypes = [vp, vp, ctypes.c_int, ctypes.POINTER(Stats), vp]
    L.libsupermesh_gpu_clip_candidates_ordered.restype = ctypes.c_int
    L.libsupermesh_gpu_intersect_pairs.argtypes = [vp, ctypes.c_int, ctypes.c_int64, vp, vp, vp, vp, vp,
                                                   ctypes.c_int, vp]
    L.libsupermesh_gpu_intersect_pairs_mixed.argtypes = [vp, ctypes.c_int, ctypes.c_int64, vp, vp, vp, vp, vp,
                                                         ctypes.c_int, vp]
    L.libsupermesh_gpu_p1_mass.argtypes = [vp, mp, mp, vp, vp, vp, _dp, ctypes.c_int, vp]
    L.libsupermesh_gpu_p2_inner_product.argtypes = [vp, mp, mp, vp, vp, ctypes.c_int64, vp, vp, ctypes.c_int64, vp,
                                                    _dp, _dp, ctypes.c_int, vp]
    L.libsupermesh_gpu_supermesh_batched.argtypes = [vp, ctypes.c_int, mp, mp, ctypes.c_int, vp, vp, vp, vp]
    L.libsupermesh_gpu_supermesh_batched_ex.argtypes = [vp, ctypes.c_int, mp, mp, ctypes.c_int,
                                                        ctypes.POINTER(BatchOut), vp]
    L.libsupermesh_gpu_sched_set_weights.argtypes = [vp, vp, ctypes.c_int]
    L.libsupermesh_gpu_sched_samples.argtypes = [vp, ctypes.c_int64, vp, vp, _i64p, vp]
    L.libsupermesh_gpu_sched_predict.argtypes = [vp, ctypes.c_int64, vp, vp, vp, vp]
    L.libsupermesh_gpu_sched_train.argtypes = [vp, ctypes.c_int64, vp, vp, vp, ctypes.c_int, ctypes.c_float, vp,
                                               ctypes.c_int, vp, vp]
    for name in ("libsupermesh_gpu_context_create", "libsupermesh_gpu_context_destroy",
                 "libsupermesh_gpu_find_candidates", "libsupermesh_gpu_get_candidates",
                 "libsupermesh_gpu_supermesh", "libsupermesh_gpu_get_pair_results",
                 "libsupermesh_gpu_clip_candidates",
                 "libsupermesh_gpu_intersect_pairs", "libsupermesh_gpu_intersect_pairs_mixed",
                 "libsupermesh_gpu_p1_mass", "libsupermesh_gpu_p2_inner_product",
                 "libsupermesh_gpu_supermesh_batched", "libsupermesh_gpu_supermesh_batched_ex",
                 "libsupermesh_gpu_sched_set_weights",
                 "libsupermesh_gpu_sched_samples", "libsupermesh_gpu_sched_predict",
                 "libsupermesh_gpu_sched_train"):
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


PAIR_INTERVALS, PAIR_TRI_QUAD, PAIR_TET_HEX, PAIR_QUAD_QUAD, PAIR_HEX_HEX = 0, 1, 2, 3, 4
_MIXED = {PAIR_INTERVALS: (2, 2, (1, 2)), PAIR_TRI_QUAD: (6, 8, (46, 3, 2)), PAIR_TET_HEX: (12, 24, (729, 4, 3)),
          PAIR_QUAD_QUAD: (8, 8, (62, 3, 2)), PAIR_HEX_HEX: (24, 24, (5 * 729, 4, 3))}


def _ptr(a) -> int | None:
    """Address of a numpy array or of anything exposing data_ptr() (torch)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def _mesh(pos, en, on_device: bool) -> Mesh:
    if on_device:
        nnodes, dim = pos.shape
        nel, loc = en.shape
        ib = en.element_size()
        return Mesh(dim, loc, nnodes, nel, _ptr(pos), _ptr(en), ib)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    if en.dtype not in (np.int32, np.int64):
        en = en.astype(np.int64)
    en = np.ascontiguousarray(en)
    m = Mesh(pos.shape[1], en.shape[1], pos.shape[0], en.shape[0], pos.ctypes.data, en.ctypes.data,
             en.dtype.itemsize)
    m._keep = (pos, en)  # keep the arrays alive with the struct
    return m


class Context:
    """A GPU context (one device, one stream, reusable device buffers)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        self._h = ctypes.c_void_p()
        st = self.lib.libsupermesh_gpu_context_create(device, ctypes.byref(self._h))
        if st != 0:
            raise LsmError(st, self.lib.libsupermesh_gpu_status_string(st).decode())

    def close(self):
        if self._h:
            self.lib.libsupermesh_gpu_context_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        if st != 0:
            msg = self.lib.libsupermesh_gpu_last_error(self._h).decode()
            raise LsmError(st, msg)

    @property
    def device_bytes(self) -> int:
        return self.lib.libsupermesh_gpu_context_bytes(self._h)

    # -- candidate search -------------------------------------------------
    def find_candidates(self, mesh_a, mesh_b, on_device: bool = False, stream: int | None = None):
        ma, mb = _mesh(*mesh_a, on_device), _mesh(*mesh_b, on_device)
        n = ctypes.c_int64(0)
        self._check(self.lib.libsupermesh_gpu_find_candidates(self._h, ctypes.byref(ma), ctypes.byref(mb),
                                                              int(on_device), ctypes.byref(n), stream))
        return n.value

    def get_candidates(self, nel_a: int, n: int, out=None, stream: int | None = None):
        """CSR of the last search: (ind_ptr[nel_a + 1], indices[n]), int64,
        into `out` = (ind_ptr, indices) host arrays when given (pinned
        arrays make the copies asynchronous DMA)."""
        if out is None:
            indptr = np.zeros(nel_a + 1, dtype=np.int64)
            indices = np.zeros(max(n, 1), dtype=np.int64)
        else:
            indptr, indices = out
        self._check(self.lib.libsupermesh_gpu_get_candidates(self._h, indptr.ctypes.data, indices.ctypes.data,
                                                             0, stream))
        return indptr, indices[:n]

    # -- whole supermesh --------------------------------------------------
    def supermesh(self, mesh_a, mesh_b, elem_measure: bool = False, on_device: bool = False,
                  out=None, stream: int | None = None):
        """Returns (Stats, elem_measure or None)."""
        ma, mb = _mesh(*mesh_a, on_device), _mesh(*mesh_b, on_device)
        em = None
        if elem_measure:
            em = out if out is not None else np.zeros(ma.nelements, dtype=np.float64)
        st = Stats()
        self._check(self.lib.libsupermesh_gpu_supermesh(self._h, ctypes.byref(ma), ctypes.byref(mb),
                                                        int(on_device), _ptr(em), ctypes.byref(st), stream))
        return st, em

    def supermesh_out(self, mesh_a, mesh_b, out: dict, on_device: bool = False, stream: int | None = None):
        """Whole supermesh plus the per-candidate outputs in one call
        (libsupermesh_gpu_supermesh_out).  out: dict with any of
        elem_measure, ind_ptr, indices, pair_measure, pair_n_out (arrays in
        the memory space of on_device; host arrays should be pinned) and
        capacity.  Returns (Stats, n_candidates)."""
        ma, mb = _mesh(*mesh_a, on_device), _mesh(*mesh_b, on_device)
        o = PairOut(_ptr(out.get("elem_measure")), _ptr(out.get("ind_ptr")), _ptr(out.get("indices")),
                    _ptr(out.get("pair_measure")), _ptr(out.get("pair_n_out")), int(out.get("capacity", 0)), 0)
        st = Stats()
        self._check(self.lib.libsupermesh_gpu_supermesh_out(self._h, ctypes.byref(ma), ctypes.byref(mb),
                                                            int(on_device), ctypes.byref(o), ctypes.byref(st),
                                                            stream))
        return st, o.n_candidates

    def supermesh_elements(self, mesh_a, mesh_b, parents: bool = True, stream: int | None = None):
        """The supermesh's simplices (libsupermesh_gpu_supermesh_elements),
        host meshes: returns (Stats, elem_offset [n_candidates + 1], elems
        [n][3][2] or [n][4][3], parent_a, parent_b or None).  A first call
        with no capacity reads the counts; the second fills the arrays."""
        ma, mb = _mesh(*mesh_a, False), _mesh(*mesh_b, False)
        dim = ma.dim
        st = Stats()
        o = ElemOut(None, None, None, None, 0, 0, 0, 0)
        r = self.lib.libsupermesh_gpu_supermesh_elements(self._h, ctypes.byref(ma), ctypes.byref(mb), 0,
                                                         ctypes.byref(o), ctypes.byref(st), stream)
        if r not in (0, 3):
            self._check(r)
        nc, ne = o.n_candidates, o.n_elements
        off = np.zeros(nc + 1, dtype=np.int64)
        el = np.zeros((max(ne, 1), 3, 2) if dim == 2 else (max(ne, 1), 4, 3))
        pa = np.zeros(max(ne, 1), dtype=np.int64) if parents else None
        pb = np.zeros(max(ne, 1), dtype=np.int64) if parents else None
        o = ElemOut(_ptr(off), _ptr(el), _ptr(pa), _ptr(pb), nc, ne, 0, 0)
        self._check(self.lib.libsupermesh_gpu_supermesh_elements(self._h, ctypes.byref(ma), ctypes.byref(mb), 0,
                                                                 ctypes.byref(o), ctypes.byref(st), stream))
        return st, off, el[:ne], (pa[:ne] if parents else None), (pb[:ne] if parents else None)

    def supermesh_elements_device(self, mesh_a, mesh_b, out: dict, stream: int | None = None):
        """Device-resident form: meshes and out's arrays (elem_offset, elems,
        parent_a, parent_b; CUDA tensors) in device memory, with
        cand_capacity and elem_capacity.  Returns (Stats, n_candidates,
        n_elements); raises LsmError (status 3) when the arrays are too small."""
        ma, mb = _mesh(*mesh_a, True), _mesh(*mesh_b, True)
        o = ElemOut(_ptr(out.get("elem_offset")), _ptr(out.get("elems")), _ptr(out.get("parent_a")),
                    _ptr(out.get("parent_b")), int(out.get("cand_capacity", 0)), int(out.get("elem_capacity", 0)),
                    0, 0)
        st = Stats()
        r = self.lib.libsupermesh_gpu_supermesh_elements(self._h, ctypes.byref(ma), ctypes.byref(mb), 1,
                                                         ctypes.byref(o), ctypes.byref(st), stream)
        out["n_candidates"], out["n_elements"] = o.n_candidates, o.n_elements
        self._check(r)
        return st, o.n_candidates, o.n_elements

    def clip_candidates(self, stream: int | None = None) -> Stats:
        """Re-run the narrow phase over the last candidate set."""
        st = Stats()
        self._check(self.lib.libsupermesh_gpu_clip_candidates(self._h, ctypes.byref(st), stream))
        return st

    def clip_candidates_ordered(self, order, on_device: bool = False, stream: int | None = None) -> Stats:
        """Narrow phase over the last candidates, taken in the given order."""
        st = Stats()
        if not on_device:
            order = np.ascontiguousarray(order, dtype=np.int32)
        self._check(self.lib.libsupermesh_gpu_clip_candidates_ordered(self._h, _ptr(order), int(on_device),
                                                                      ctypes.byref(st), stream))
        return st

    def clip_kernel_ms(self) -> float:
        """Device time of the last narrow phase's clip kernel (option
        time_kernels must have been on)."""
        r = ctypes.c_double(0.0)
        self._check(self.lib.libsupermesh_gpu_clip_kernel_ms(self._h, ctypes.byref(r)))
        return r.value

    def clip_survivors(self) -> int:
        """Pairs of the last 3D narrow phase that the exact early-outs left
        for the clipper."""
        r = ctypes.c_int64(0)
        self._check(self.lib.libsupermesh_gpu_clip_survivors(self._h, ctypes.byref(r)))
        return r.value

    def pair_results(self, n: int, out=None, stream: int | None = None):
        """Per-candidate (measure[n] float64, n_out[n] int32) of the last
        narrow phase, in CSR order, into `out` = (measure, n_out) when given."""
        if out is None:
            m = np.zeros(max(n, 1), dtype=np.float64)
            k = np.zeros(max(n, 1), dtype=np.int32)
        else:
            m, k = out
        self._check(self.lib.libsupermesh_gpu_get_pair_results(self._h, m.ctypes.data, k.ctypes.data, 0, stream))
        return m[:n], k[:n]

    def intersect_pairs(self, dim: int, a, b, want_elems: bool = False):
        per = 6 if dim == 2 else 12
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1, per)
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1, per)
        n = a.shape[0]
        m = np.zeros(max(n, 1))
        k = np.zeros(max(n, 1), dtype=np.int32)
        e = None
        if want_elems:
            e = np.zeros((max(n, 1), 22, 3, 2) if dim == 2 else (max(n, 1), 81, 4, 3))
        self._check(self.lib.libsupermesh_gpu_intersect_pairs(self._h, dim, n, a.ctypes.data, b.ctypes.data,
                                                              m.ctypes.data, k.ctypes.data, _ptr(e), 0, None))
        return m[:n], k[:n], (e[:n] if e is not None else None)

    def intersect_pairs_mixed(self, kind: int, a, b, want_elems: bool = False):
        """kind: PAIR_INTERVALS, PAIR_TRI_QUAD, PAIR_TET_HEX, PAIR_QUAD_QUAD or
        PAIR_HEX_HEX."""
        per_a, per_b, out_shape = _MIXED[kind]
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1, per_a)
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1, per_b)
        n = a.shape[0]
        m = np.zeros(max(n, 1))
        k = np.zeros(max(n, 1), dtype=np.int32)
        e = np.zeros((max(n, 1),) + out_shape) if want_elems else None
        self._check(self.lib.libsupermesh_gpu_intersect_pairs_mixed(self._h, kind, n, a.ctypes.data, b.ctypes.data,
                                                                    m.ctypes.data, k.ctypes.data, _ptr(e), 0,
                                                                    None))
        return m[:n], k[:n], (e[:n] if e is not None else None)

    def intersect_pairs_device(self, a, b, measure, n_out, elems=None, dim: int = 3, kind: int | None = None,
                               stream: int | None = None):
        """Explicit element pairs in device memory (CUDA tensors): simplex
        pairs of dimension dim (kind None) or a mixed kind (PAIR_*); measure
        [n] f64, n_out [n] int32 and elems (optional) are written on the
        stream; nothing is copied to the host."""
        n = int(measure.shape[0])
        if kind is None:
            st = self.lib.libsupermesh_gpu_intersect_pairs(self._h, dim, n, _ptr(a), _ptr(b), _ptr(measure),
                                                           _ptr(n_out), _ptr(elems), 1, stream)
        else:
            st = self.lib.libsupermesh_gpu_intersect_pairs_mixed(self._h, kind, n, _ptr(a), _ptr(b), _ptr(measure),
                                                                 _ptr(n_out), _ptr(elems), 1, stream)
        self._check(st)

    def p1_mass(self, mesh_a, mesh_b, u_a=None, v_b=None, want_blocks: bool = False,
                on_device: bool = False, stream: int | None = None):
        """Returns (u^T M v or None, blocks or None).  Host meshes and fields,
        or with on_device meshes and fields in device memory (torch tensors;
        blocks then not available)."""
        ma, mb = _mesh(*mesh_a, on_device), _mesh(*mesh_b, on_device)
        if ma.index_bytes != mb.index_bytes:
            raise ValueError("A and B must use the same index width")
        if on_device:
            if want_blocks:
                raise ValueError("want_blocks needs host meshes")
            integral = ctypes.c_double(0.0)
            self._check(self.lib.libsupermesh_gpu_p1_mass(self._h, ctypes.byref(ma), ctypes.byref(mb), _ptr(u_a),
                                                          _ptr(v_b), None, ctypes.byref(integral), 1, stream))
            return (integral.value if u_a is not None and v_b is not None else None), None
        u = np.ascontiguousarray(u_a, dtype=np.float64) if u_a is not None else None
        v = np.ascontiguousarray(v_b, dtype=np.float64) if v_b is not None else None
        blocks, n = None, 0
        if want_blocks:
            n = self.find_candidates(mesh_a, mesh_b)
            loc = ma.dim + 1
            blocks = np.zeros((max(n, 1), loc, loc))
        integral = ctypes.c_double(0.0)
        self._check(self.lib.libsupermesh_gpu_p1_mass(self._h, ctypes.byref(ma), ctypes.byref(mb), _ptr(u),
                                                      _ptr(v), _ptr(blocks), ctypes.byref(integral), 0, stream))
        return (integral.value if u is not None else None), (blocks[:n] if blocks is not None else None)

    def p2_inner_product(self, mesh_a, mesh_b, enlist_p2_a, field_a, enlist_p2_b, field_b,
                         want_pairs: bool = False):
        """2D P2 inner product over the supermesh.  Returns (integral, area,
        per-pair contributions or None); host arrays."""
        ma, mb = _mesh(*mesh_a, False), _mesh(*mesh_b, False)
        if ma.index_bytes != mb.index_bytes:
            raise ValueError("A and B must use the same index width")
        dt = np.int32 if ma.index_bytes == 4 else np.int64
        e2a = np.ascontiguousarray(enlist_p2_a, dtype=dt)
        e2b = np.ascontiguousarray(enlist_p2_b, dtype=dt)
        fa = np.ascontiguousarray(field_a, dtype=np.float64)
        fb = np.ascontiguousarray(field_b, dtype=np.float64)
        pv, n = None, 0
        if want_pairs:
            n = self.find_candidates(mesh_a, mesh_b)
            pv = np.zeros(max(n, 1))
        integral, area = ctypes.c_double(0.0), ctypes.c_double(0.0)
        self._check(self.lib.libsupermesh_gpu_p2_inner_product(
            self._h, ctypes.byref(ma), ctypes.byref(mb), e2a.ctypes.data, fa.ctypes.data, fa.size,
            e2b.ctypes.data, fb.ctypes.data, fb.size, _ptr(pv), ctypes.byref(integral), ctypes.byref(area), 0,
            None))
        return integral.value, area.value, (pv[:n] if pv is not None else None)

    def supermesh_batched_pairs(self, pairs, capacity: int | None = None, on_device: bool = False, out=None,
                                stream: int | None = None, p1_blocks: bool = False):
        """Batched supermesh with per-pair outputs (host meshes and arrays
        unless on_device).  Returns a dict with totals, n_candidates,
        n_intersecting, cand_offset, total_candidates, and the arrays ind_ptr
        (pair i's rows at row_offset[i]), indices, pair_measure, pair_n_out.
        With capacity None the call is made twice if needed: the first
        attempt's counts size the retry (LSM_ERROR_CAPACITY).  `out` (dict
        of preallocated arrays, optional) is used as is.  p1_blocks: also
        every candidate's P1-P1 mass block (p1_blocks from p1_offset[i])."""
        n = len(pairs)
        A = (Mesh * max(n, 1))()
        B = (Mesh * max(n, 1))()
        keep = []
        for i, (ma, mb) in enumerate(pairs):
            a, b = _mesh(*ma, on_device), _mesh(*mb, on_device)
            keep.append((a, b))
            A[i], B[i] = a, b
        rows = [int(ma[1].shape[0]) + 1 for ma, _ in pairs]
        row_offset = np.concatenate([[0], np.cumsum(rows)[:-1]]).astype(np.int64) if n else np.zeros(0, np.int64)
        cap = capacity if capacity is not None else (out["capacity"] if out else 0)
        dims = [int(ma[0].shape[1]) for ma, _ in pairs]
        p1cap = 16 * cap if p1_blocks else 0
        while True:
            if out is None:
                r = {"totals": np.zeros(max(n, 1)), "n_candidates": np.zeros(max(n, 1), dtype=np.int64),
                     "n_intersecting": np.zeros(max(n, 1), dtype=np.int64),
                     "cand_offset": np.zeros(max(n, 1), dtype=np.int64),
                     "total_candidates": np.zeros(1, dtype=np.int64)}
                if on_device:
                    import torch

                    dev = torch.device("cuda", torch.cuda.current_device())
                    r["ind_ptr"] = torch.zeros(max(sum(rows), 1), dtype=torch.int64, device=dev)
                    r["indices"] = torch.zeros(max(cap, 1), dtype=torch.int64, device=dev)
                    r["pair_measure"] = torch.zeros(max(cap, 1), dtype=torch.float64, device=dev)
                    r["pair_n_out"] = torch.zeros(max(cap, 1), dtype=torch.int32, device=dev)
                    r["p1_blocks"] = torch.zeros(max(p1cap, 1), dtype=torch.float64, device=dev) if p1_blocks else None
                else:
                    r["ind_ptr"] = np.zeros(max(sum(rows), 1), dtype=np.int64)
                    r["indices"] = np.zeros(max(cap, 1), dtype=np.int64)
                    r["pair_measure"] = np.zeros(max(cap, 1))
                    r["pair_n_out"] = np.zeros(max(cap, 1), dtype=np.int32)
                    r["p1_blocks"] = np.zeros(max(p1cap, 1)) if p1_blocks else None
                r["p1_offset"] = np.zeros(max(n, 1), dtype=np.int64)
            else:
                r = out
            o = BatchOut(_ptr(r["totals"]), _ptr(r["n_candidates"]), _ptr(r["n_intersecting"]),
                         _ptr(r["cand_offset"]), _ptr(r["total_candidates"]), cap, _ptr(r["ind_ptr"]),
                         _ptr(r["indices"]), _ptr(r["pair_measure"]), _ptr(r["pair_n_out"]),
                         _ptr(r.get("p1_offset")), p1cap, _ptr(r.get("p1_blocks")))
            st = self.lib.libsupermesh_gpu_supermesh_batched_ex(self._h, n, A, B, int(on_device), ctypes.byref(o),
                                                                stream)
            if st == 3 and capacity is None and out is None:  # LSM_ERROR_CAPACITY: size the retry
                nc = r["n_candidates"][:n]
                cap = int(nc.sum())
                p1cap = int(sum(int(k) * (d + 1) ** 2 for k, d in zip(nc, dims))) if p1_blocks else 0
                continue
            self._check(st)
            r["row_offset"] = row_offset
            return r

    # -- learned scheduler (device buffers: torch tensors) -------------------
    def sched_set_weights(self, params) -> None:
        """Weights for option tet_schedule = 1: LSM_SCHED_PARAMS float32
        values (numpy on the host, or a device tensor)."""
        if hasattr(params, "data_ptr"):
            self._check(self.lib.libsupermesh_gpu_sched_set_weights(self._h, params.data_ptr(), 1))
        else:
            p = np.ascontiguousarray(params, dtype=np.float32)
            assert p.size == SCHED_PARAMS
            self._check(self.lib.libsupermesh_gpu_sched_set_weights(self._h, p.ctypes.data, 0))

    def sched_samples(self, cap: int, features, classes, stream: int | None = None) -> int:
        """Features (device, [cap][32] 2-byte elements) and classes (device
        int8 [cap]) of the survivors of the last plain 3D narrow phase;
        returns the number of survivors."""
        n = ctypes.c_int64(0)
        self._check(self.lib.libsupermesh_gpu_sched_samples(self._h, cap, features.data_ptr(), classes.data_ptr(),
                                                            ctypes.byref(n), stream))
        return n.value

    def sched_predict(self, n: int, features, logits, classes, stream: int | None = None) -> None:
        self._check(self.lib.libsupermesh_gpu_sched_predict(
            self._h, n, features.data_ptr(), logits.data_ptr() if logits is not None else None,
            classes.data_ptr(), stream))

    def sched_train(self, n: int, features, classes, params, steps: int, lr: float, loss_trace=None,
                    trace_every: int = 0, grad_first=None, stream: int | None = None) -> None:
        """Adam steps on device tensors; params (float32 [LSM_SCHED_PARAMS],
        device) is updated in place."""
        self._check(self.lib.libsupermesh_gpu_sched_train(
            self._h, n, features.data_ptr(), classes.data_ptr(), params.data_ptr(), steps, lr,
            loss_trace.data_ptr() if loss_trace is not None else None, trace_every,
            grad_first.data_ptr() if grad_first is not None else None, stream))

    def supermesh_batched(self, pairs, on_device: bool = False, stream: int | None = None):
        """pairs: list of (mesh_a, mesh_b).  Returns (totals, n_candidates,
        n_intersecting) as numpy arrays."""
        n = len(pairs)
        A = (Mesh * max(n, 1))()
        B = (Mesh * max(n, 1))()
        keep = []
        for i, (ma, mb) in enumerate(pairs):
            a, b = _mesh(*ma, on_device), _mesh(*mb, on_device)
            keep.append((a, b))
            A[i], B[i] = a, b
        totals = np.zeros(max(n, 1))
        nc = np.zeros(max(n, 1), dtype=np.int64)
        ni = np.zeros(max(n, 1), dtype=np.int64)
        self._check(self.lib.libsupermesh_gpu_supermesh_batched(self._h, n, A, B, int(on_device), totals.ctypes.data,
                                                                nc.ctypes.data, ni.ctypes.data, stream))
        return totals[:n], nc[:n], ni[:n]


def set_option(name: str, value: int) -> None:
    """Set a process-wide tuning option (see libsupermesh-gpu.h)."""
    st = load().libsupermesh_gpu_set_option(name.encode(), int(value))
    if st != 0:
        raise LsmError(st, f"invalid option {name}={value}")


def get_option(name: str) -> int:
    v = ctypes.c_int64(0)
    st = load().libsupermesh_gpu_get_option(name.encode(), ctypes.byref(v))
    if st != 0:
        raise LsmError(st, f"unknown option {name}")
    return v.value


def kernel_launches() -> int:
    """Kernel launches this library has issued in this process."""
    return load().libsupermesh_gpu_kernel_launches()


# -- drop-in C API (libsupermesh-c.h) --------------------------------------

def _long(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def tree_intersection_finder(pos_a, en_a, pos_b, en_b):
    """set_input -> query_output -> get_output through the C API."""
    return _finder("tree", pos_a, en_a, pos_b, en_b)


def sort_intersection_finder(pos_a, en_a, pos_b, en_b):
    """1D sort finder through the C API (2-node elements, first coordinate)."""
    return _finder("sort", pos_a, en_a, pos_b, en_b)


def _finder(kind, pos_a, en_a, pos_b, en_b):
    L = load()
    pa = np.ascontiguousarray(pos_a, dtype=np.float64)
    pb = np.ascontiguousarray(pos_b, dtype=np.float64)
    if pa.ndim == 1:
        pa = pa.reshape(-1, 1)
    if pb.ndim == 1:
        pb = pb.reshape(-1, 1)
    ea, eb = _long(en_a), _long(en_b)
    c_long, c_int = ctypes.c_long, ctypes.c_int
    args = [c_long(pa.shape[0]), c_int(pa.shape[1]), c_long(ea.shape[0]), c_int(ea.shape[1]),
            c_long(pb.shape[0]), c_int(pb.shape[1]), c_long(eb.shape[0]), c_int(eb.shape[1])]
    getattr(L, f"libsupermesh_{kind}_intersection_finder_set_input")(
        *[ctypes.byref(x) for x in args], pa.ctypes.data_as(_dp), ea.ctypes.data_as(_lp),
        pb.ctypes.data_as(_dp), eb.ctypes.data_as(_lp))
    n = c_long(0)
    getattr(L, f"libsupermesh_{kind}_intersection_finder_query_output")(ctypes.byref(n))
    indices = np.zeros(max(n.value, 1), dtype=np.int64)
    indptr = np.zeros(ea.shape[0] + 1, dtype=np.int64)
    nel = c_long(ea.shape[0])
    getattr(L, f"libsupermesh_{kind}_intersection_finder_get_output")(
        ctypes.byref(nel), ctypes.byref(n), indices.ctypes.data_as(_lp), indptr.ctypes.data_as(_lp))
    return indptr, indices[: n.value]


def intersect_tris_real(tri_a, tri_b):
    L = load()
    a = np.ascontiguousarray(tri_a, dtype=np.float64).reshape(3, 2)
    b = np.ascontiguousarray(tri_b, dtype=np.float64).reshape(3, 2)
    out = np.zeros((TRI_BUF_SIZE, 3, 2))
    n = ctypes.c_int(0)
    L.libsupermesh_intersect_tris_real(a.ctypes.data_as(_dp), b.ctypes.data_as(_dp), out.ctypes.data_as(_dp),
                                       ctypes.byref(n))
    return out[: n.value].copy()


def intersect_tets_real(tet_a, tet_b):
    L = load()
    a = np.ascontiguousarray(tet_a, dtype=np.float64).reshape(4, 3)
    b = np.ascontiguousarray(tet_b, dtype=np.float64).reshape(4, 3)
    out = np.zeros((TET_BUF_SIZE, 4, 3))
    n = ctypes.c_int(0)
    L.libsupermesh_intersect_tets_real(a.ctypes.data_as(_dp), b.ctypes.data_as(_dp), out.ctypes.data_as(_dp),
                                       ctypes.byref(n))
    return out[: n.value].copy()


def triangle_area(tri) -> float:
    L = load()
    t = np.ascontiguousarray(tri, dtype=np.float64).reshape(6)
    r = ctypes.c_double(0.0)
    L.libsupermesh_triangle_area(t.ctypes.data_as(_dp), ctypes.byref(r))
    return r.value


def tetrahedron_volume(tet) -> float:
    L = load()
    t = np.ascontiguousarray(tet, dtype=np.float64).reshape(12)
    r = ctypes.c_double(0.0)
    L.libsupermesh_tetrahedron_volume(t.ctypes.data_as(_dp), ctypes.byref(r))
    return r.value


def _pair_call(fn, a, b, shape_a, shape_b, out_shape):
    L = load()
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(shape_a)
    b = np.ascontiguousarray(b, dtype=np.float64).reshape(shape_b)
    out = np.zeros(out_shape)
    n = ctypes.c_int(0)
    getattr(L, fn)(a.ctypes.data_as(_dp), b.ctypes.data_as(_dp), out.ctypes.data_as(_dp), ctypes.byref(n))
    return out[: n.value].copy()


def intersect_tri_quad(tri_a, quad_b):
    return _pair_call("libsupermesh_intersect_tri_quad", tri_a, quad_b, (3, 2), (4, 2), (46, 3, 2))


def intersect_tet_hex(tet_a, hex_b):
    return _pair_call("libsupermesh_intersect_tet_hex", tet_a, hex_b, (4, 3), (8, 3), (729, 4, 3))


def intersect_intervals(interval_a, interval_b):
    """Returns an array of shape (n, 2), n in {0, 1}."""
    return _pair_call("libsupermesh_intersect_intervals", interval_a, interval_b, (2,), (2,), (1, 2))


def interval_size(interval) -> float:
    L = load()
    t = np.ascontiguousarray(interval, dtype=np.float64).reshape(2)
    r = ctypes.c_double(0.0)
    L.libsupermesh_interval_size(t.ctypes.data_as(_dp), ctypes.byref(r))
    return r.value
