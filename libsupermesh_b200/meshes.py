"""Mesh inputs for the supermesh path: Triangle/TetGen file reading and the
seeded synthetic meshes the benchmarks and parity tests run on.

File format follows ``src/Read_Triangle.F90:92-225`` of libsupermesh:
``.node`` header ``nnodes dim nattrs nbm`` then rows ``i x y [z] ...``;
``.ele`` header ``nele loc nattrs`` then rows ``i n1 .. nloc [attr]``, with
1-based node numbers.  Arrays returned here are row-major
``positions[nnodes][dim]`` (float64) and 0-based ``enlist[nele][loc]``
(int32), the layout of the C API in ``include/libsupermesh-c.h``.

Synthetic meshes (all coordinates float64):

* ``grid2d(n, seed, jitter)``: the unit square as an n x n grid, each square
  split into (v00, v10, v11) and (v00, v11, v01); node (i, j) has index
  ``j*(n+1)+i``.  Interior nodes move by ``(2u-1)*jitter*h`` per axis, where
  u comes from splitmix64 draw ``2k`` (x) and ``2k+1`` (y) for node k.
* ``grid3d(n, seed, jitter)``: the unit cube as n^3 cubes, each split into
  the 6 Kuhn (Freudenthal) tetrahedra (v000, v000+e_a, v000+e_a+e_b, v111)
  over the 6 axis permutations (a, b, c); node (i, j, k) has index
  ``(k*(n+1)+j)*(n+1)+i``; draws ``3k..3k+2``.
* splitmix64: ``z = seed + (i+1)*0x9E3779B97F4A7C15``, then the standard
  xor-shift-multiply finaliser; ``u = (z >> 11) * 2**-53``.
* Validity: uniform per-axis jitter of +-0.3h (2D) or +-0.25h (3D) inverts a
  handful of elements (e.g. 1 of 20,000 triangles at 100x100, seed 0), which
  would make the meshes overlap themselves.  Interior vertices of any element
  whose signed measure changes sign (or vanishes) therefore take fresh draws
  from the next block of the same stream (round r uses draws
  ``[r*dim*N, (r+1)*dim*N)``), repeated until no element is inverted; after 16
  rounds any remaining offenders keep their unjittered position.  With this
  the jittered meshes tile the unit square/cube exactly.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64_uniform(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """``count`` uniform doubles in [0, 1) from draws offset..offset+count-1."""
    with np.errstate(over="ignore"):
        i = np.arange(offset + 1, offset + count + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + i * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _signed_measure(pos: np.ndarray, en: np.ndarray) -> np.ndarray:
    v = pos[en]
    if en.shape[1] == 3:
        return ((v[:, 1, 0] - v[:, 0, 0]) * (v[:, 2, 1] - v[:, 0, 1])
                - (v[:, 2, 0] - v[:, 0, 0]) * (v[:, 1, 1] - v[:, 0, 1]))
    a = v[:, 1] - v[:, 0]
    return np.einsum("ij,ij->i", a, np.cross(v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]))


def _jitter(pos0, interior, en, seed, amp, transform=None, rounds=16):
    """Per-axis uniform jitter of interior nodes, redrawn where it inverts."""
    n, dim = pos0.shape
    mapped0 = transform(pos0) if transform else pos0
    ref = np.sign(_signed_measure(mapped0, en))
    disp = np.zeros_like(pos0)
    redo = interior.copy()
    for r in range(rounds):
        u = splitmix64_uniform(seed, dim * n, offset=r * dim * n).reshape(n, dim)
        disp[redo] = (2.0 * u[redo] - 1.0) * amp
        pos = pos0 + disp
        if transform:
            pos = transform(pos)
        bad = np.sign(_signed_measure(pos, en)) != ref
        if not bad.any():
            return np.ascontiguousarray(pos)
        redo = np.zeros(n, dtype=bool)
        redo[en[bad].ravel()] = True
        redo &= interior
    disp[redo] = 0.0
    pos = pos0 + disp
    return np.ascontiguousarray(transform(pos) if transform else pos)


def grid2d(n: int, seed: int, jitter: float = 0.3, transform=None):
    h = 1.0 / n
    idx = np.arange(n + 1)
    jj, ii = np.meshgrid(idx, idx, indexing="ij")
    x = (ii / n).astype(np.float64).ravel()
    y = (jj / n).astype(np.float64).ravel()
    interior = ((ii > 0) & (ii < n) & (jj > 0) & (jj < n)).ravel()
    pos0 = np.stack([x, y], axis=1)
    cj, ci = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    v00 = (cj * (n + 1) + ci).ravel()
    v10 = v00 + 1
    v01 = v00 + (n + 1)
    v11 = v01 + 1
    t1 = np.stack([v00, v10, v11], axis=1)
    t2 = np.stack([v00, v11, v01], axis=1)
    en = np.ascontiguousarray(np.stack([t1, t2], axis=1).reshape(-1, 3).astype(np.int32))
    if jitter:
        pos = _jitter(pos0, interior, en, seed, jitter * h, transform)
    else:
        pos = np.ascontiguousarray(transform(pos0) if transform else pos0)
    return pos, en


_KUHN_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


def grid3d(n: int, seed: int, jitter: float = 0.25, transform=None):
    h = 1.0 / n
    m = n + 1
    idx = np.arange(m)
    kk, jj, ii = np.meshgrid(idx, idx, idx, indexing="ij")
    coords = [(ii / n).ravel(), (jj / n).ravel(), (kk / n).ravel()]
    interior = ((ii > 0) & (ii < n) & (jj > 0) & (jj < n) & (kk > 0) & (kk < n)).ravel()
    pos0 = np.stack(coords, axis=1).astype(np.float64)
    ck, cj, ci = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    base = ((ck * m + cj) * m + ci).ravel()
    step = (1, m, m * m)
    v111 = base + step[0] + step[1] + step[2]
    tets = []
    for a, b, _ in _KUHN_PERMS:
        v1 = base + step[a]
        v2 = v1 + step[b]
        tets.append(np.stack([base, v1, v2, v111], axis=1))
    en = np.ascontiguousarray(np.stack(tets, axis=1).reshape(-1, 4).astype(np.int32))
    if jitter:
        pos = _jitter(pos0, interior, en, seed, jitter * h, transform)
    else:
        pos = np.ascontiguousarray(transform(pos0) if transform else pos0)
    return pos, en


def rotate_clamp(pos: np.ndarray, degrees: float, centre=(0.5, 0.5)) -> np.ndarray:
    th = math.radians(degrees)
    c, s = math.cos(th), math.sin(th)
    x = pos[:, 0] - centre[0]
    y = pos[:, 1] - centre[1]
    out = np.stack([centre[0] + c * x - s * y, centre[1] + s * x + c * y], axis=1)
    return np.ascontiguousarray(np.clip(out, 0.0, 1.0))


def grade_square(pos: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(pos * pos)


def read_node(path) -> np.ndarray:
    with open(path) as f:
        header = f.readline().split()
        nnodes, dim, nattrs, nbm = (int(v) for v in header[:4])
        data = np.loadtxt(f, max_rows=nnodes, ndmin=2)
    if data.shape[0] != nnodes or not np.array_equal(data[:, 0], np.arange(1, nnodes + 1)):
        raise ValueError(f"{path}: invalid vertex numbering")
    return np.ascontiguousarray(data[:, 1:1 + dim], dtype=np.float64)


def read_ele(path) -> np.ndarray:
    with open(path) as f:
        header = f.readline().split()
        nele, loc, nattrs = (int(v) for v in header[:3])
        data = np.loadtxt(f, max_rows=nele, ndmin=2, dtype=np.int64)
    if data.shape[0] != nele or not np.array_equal(data[:, 0], np.arange(1, nele + 1)):
        raise ValueError(f"{path}: invalid element numbering")
    en = data[:, 1:1 + loc]
    if (en < 1).any():
        raise ValueError(f"{path}: invalid node")
    return np.ascontiguousarray(en - 1, dtype=np.int32)


def read_mesh(basename):
    base = Path(basename)
    return read_node(str(base) + ".node"), read_ele(str(base) + ".ele")


# --- named workloads -------------------------------------------------------

def config_meshes(name: str):
    """Return ``(dim, (pos_a, en_a), (pos_b, en_b))`` for a named workload.

    A is the target (query) mesh giving the CSR rows; B is the source mesh the
    tree is built on.
    """
    if name == "tri2d_73x100":      # 10,658 x 20,000 triangles, jitter 0.3h
        return 2, grid2d(73, 1, 0.3), grid2d(100, 0, 0.3)
    if name == "tet3d_27x32":       # 118,098 x 196,608 Kuhn tets, jitter 0.25h
        return 3, grid3d(27, 3, 0.25), grid3d(32, 2, 0.25)
    if name == "tri2d_777x1024_rot7":  # 1,207,458 x 2,097,152 triangles
        pa, ea = grid2d(777, 5, 0.3)
        return 2, (rotate_clamp(pa, 7.0), ea), grid2d(1024, 4, 0.3)
    if name == "tet3d_graded_55x51":  # ~1.0M x ~0.8M tets, x -> x^2 grading
        return 3, grid3d(55, 7, 0.2, grade_square), grid3d(51, 8, 0.2, grade_square)
    if name.startswith("small"):
        # small{2,3}d_<na>x<nb>: reduced-size versions for parity tests
        dim = int(name[5])
        na, nb = (int(v) for v in name.split("_")[1].split("x"))
        if dim == 2:
            return 2, grid2d(na, 1, 0.3), grid2d(nb, 0, 0.3)
        return 3, grid3d(na, 3, 0.25), grid3d(nb, 2, 0.25)
    raise KeyError(name)


def batched_pairs(count: int = 256, seed: int = 6, emin: float = 1e3, emax: float = 1e5):
    """Mesh pairs of uneven size: half 2D, half 3D; element counts
    log-uniform in [emin, emax] per mesh; grid n = round(sqrt(E/2)) (2D) or
    round(cbrt(E/6)) (3D); jitter 0.3h (2D) or 0.25h (3D)."""
    u = splitmix64_uniform(seed, 2 * count)
    lo, hi = math.log10(emin), math.log10(emax)
    pairs = []
    for p in range(count):
        dim = 2 if p < count // 2 else 3
        meshes = []
        for s in range(2):
            e = 10.0 ** (lo + (hi - lo) * u[2 * p + s])
            mseed = seed * 1000 + 2 * p + s
            if dim == 2:
                n = max(1, int(round(math.sqrt(e / 2.0))))
                meshes.append(grid2d(n, mseed, 0.3))
            else:
                n = max(1, int(round((e / 6.0) ** (1.0 / 3.0))))
                meshes.append(grid3d(n, mseed, 0.25))
        pairs.append((dim, meshes[0], meshes[1]))
    return pairs


def p2_space(enlist):
    """P2 element-node list of a triangle mesh: [nel][6] with the P1 vertices
    first (same numbers), then new nodes for the edge midpoints 1-2, 2-3,
    1-3, numbered in first-visit order.  Returns (enlist_p2, nnodes_p2,
    edges) with edges mapping (min, max) vertex pairs to midpoint nodes."""
    en = np.asarray(enlist, dtype=np.int64)
    nv = int(en.max()) + 1 if en.size else 0
    e2 = np.zeros((len(en), 6), dtype=np.int64)
    e2[:, :3] = en
    edges = {}
    nxt = nv
    for e in range(len(en)):
        for l, (i, j) in enumerate(((0, 1), (1, 2), (0, 2))):
            k = (min(en[e, i], en[e, j]), max(en[e, i], en[e, j]))
            if k not in edges:
                edges[k] = nxt
                nxt += 1
            e2[e, 3 + l] = edges[k]
    return e2, nxt, edges


def p1_to_p2(values_p1, nnodes_p2, edges):
    """Interpolate a P1 nodal field onto the P2 space of p2_space: vertex
    values copied, midpoint values 0.5 * (sum of the edge's end values)."""
    v = np.asarray(values_p1, dtype=np.float64)
    out = np.zeros(nnodes_p2)
    out[: len(v)] = v
    for (i, j), k in edges.items():
        out[k] = 0.5 * (v[i] + v[j])
    return out
