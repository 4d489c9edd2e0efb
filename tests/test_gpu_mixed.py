"""GPU parity of the 1D and mixed-element entries of the C API: the sort
finder, intervals, triangle vs quadrilateral and tetrahedron vs hexahedron,
and the quad-quad / hex-hex pairs of intersect_elements.

All integer results (candidate CSR, row order, output counts) and all FP64
outputs must equal the oracle's bit for bit: the kernels evaluate the
reference's operations in the reference's order without FMA contraction.
"""
import numpy as np
import pytest

import libsupermesh_b200 as lsm

pytestmark = pytest.mark.gpu


def _line_mesh(x, shuffle_seed=None):
    x = np.asarray(x, dtype=np.float64)
    en = np.stack([np.arange(len(x) - 1), np.arange(1, len(x))], axis=1).astype(np.int64)
    if shuffle_seed is not None:
        en = en[np.random.default_rng(shuffle_seed).permutation(len(en))]
    return x.reshape(-1, 1), en


def _check_finder(oracle, A, B):
    ip, ind = lsm.sort_intersection_finder(A[0], A[1], B[0], B[1])
    ip_o, ind_o = oracle.sort_finder_1d(A, B, stable=True)
    assert np.array_equal(ip, ip_o)
    assert np.array_equal(ind, ind_o)  # same rows in the same sweep order
    return ip, ind


def test_sort_finder_reference_meshes(oracle_mod, ref_meshes):
    A, B = ref_meshes("line.1"), ref_meshes("line.2")
    for X, Y in ((A, B), (B, A), (A, A)):
        ip, ind = _check_finder(oracle_mod, X, Y)
        # elements numbered along the line: the reference's own merge sort
        # gives the same rows
        ip_r, ind_r = oracle_mod.sort_finder_1d(X, Y, stable=False)
        assert np.array_equal(ip, ip_r) and np.array_equal(ind, ind_r)


def test_sort_finder_shares_state_with_tree_finder(ref_meshes):
    # set_input of one finder, query/get_output of the other (one result
    # state, C_bindings.F90:30-32)
    import ctypes

    L = lsm.load()
    A, B = ref_meshes("line.1"), ref_meshes("line.2")
    pa, pb = np.ascontiguousarray(A[0]), np.ascontiguousarray(B[0])
    ea, eb = A[1].astype(np.int64), B[1].astype(np.int64)
    args = [ctypes.c_long(len(pa)), ctypes.c_int(1), ctypes.c_long(len(ea)), ctypes.c_int(2),
            ctypes.c_long(len(pb)), ctypes.c_int(1), ctypes.c_long(len(eb)), ctypes.c_int(2)]
    dp, lp = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_long)
    L.libsupermesh_sort_intersection_finder_set_input(*[ctypes.byref(x) for x in args], pa.ctypes.data_as(dp),
                                                       ea.ctypes.data_as(lp), pb.ctypes.data_as(dp),
                                                       eb.ctypes.data_as(lp))
    n = ctypes.c_long(0)
    L.libsupermesh_tree_intersection_finder_query_output(ctypes.byref(n))
    ind = np.zeros(n.value, dtype=np.int64)
    ip = np.zeros(len(ea) + 1, dtype=np.int64)
    L.libsupermesh_tree_intersection_finder_get_output(ctypes.byref(ctypes.c_long(len(ea))), ctypes.byref(n),
                                                       ind.ctypes.data_as(lp), ip.ctypes.data_as(lp))
    ip2, ind2 = lsm.sort_intersection_finder(A[0], A[1], B[0], B[1])
    assert np.array_equal(ip, ip2) and np.array_equal(ind, ind2)


@pytest.mark.parametrize("seed", range(6))
def test_sort_finder_random_and_degenerate(oracle_mod, seed):
    rng = np.random.default_rng(100 + seed)
    if seed % 2 == 0:
        # shuffled numbering of two meshes of [0, 1], the second also
        # partly outside it
        A = _line_mesh(np.sort(np.r_[0.0, rng.random(300), 1.0]), shuffle_seed=seed)
        B = _line_mesh(np.sort(np.r_[-0.5, rng.random(250), 1.5]), shuffle_seed=seed + 1)
    else:
        # overlapping intervals, repeated end points, zero-length elements,
        # reversed node order and signed zeros
        vals = np.array([0.0, -0.0, 0.25, 0.5, 0.75, 1.0, -1.0, 0.5])
        xa = rng.choice(vals, size=(60, 1))
        xb = rng.choice(vals, size=(50, 1))
        A = (xa, rng.integers(0, 60, size=(70, 2)))
        B = (xb, rng.integers(0, 50, size=(40, 2)))
    _check_finder(oracle_mod, A, B)
    _check_finder(oracle_mod, B, A)


def test_sort_finder_positions_with_stride(oracle_mod):
    # dim > 1: the first coordinate of each node is used
    rng = np.random.default_rng(5)
    xa = np.c_[np.sort(rng.random(40)), rng.random(40)]
    xb = np.c_[np.sort(rng.random(30)), rng.random(30), rng.random(30)]
    ea = np.stack([np.arange(39), np.arange(1, 40)], 1)
    eb = np.stack([np.arange(29), np.arange(1, 30)], 1)
    _check_finder(oracle_mod, (xa, ea), (xb, eb))


def test_sort_finder_empty_meshes(oracle_mod):
    A = _line_mesh([0.0, 0.5, 1.0])
    E = (A[0], np.zeros((0, 2), dtype=np.int64))
    ip, ind = lsm.sort_intersection_finder(E[0], E[1], A[0], A[1])
    assert list(ip) == [0] and len(ind) == 0
    ip, ind = lsm.sort_intersection_finder(A[0], A[1], E[0], E[1])
    assert list(ip) == [0, 0, 0] and len(ind) == 0


def test_sort_finder_large_mesh(oracle_mod):
    # 1M and 0.8M intervals, shuffled numbering: the CSR equals the oracle's
    # and every A interval is covered exactly by its candidates
    rng = np.random.default_rng(9)
    xa = np.sort(np.r_[0.0, rng.random(1_000_000 - 1), 1.0])
    xb = np.sort(np.r_[0.0, rng.random(800_000 - 1), 1.0])
    A = _line_mesh(xa, shuffle_seed=1)
    B = _line_mesh(xb, shuffle_seed=2)
    ip, ind = _check_finder(oracle_mod, A, B)
    with lsm.Context(0) as ctx:
        st, em = ctx.supermesh(A, B, elem_measure=True)
    assert st.n_candidates == len(ind)
    ea = A[0][A[1], 0]
    own = np.abs(ea[:, 1] - ea[:, 0])
    assert np.max(np.abs(em - own)) <= 1e-15
    assert abs(st.total_measure - 1.0) <= 1e-12


def test_gpu_supermesh_1d_matches_oracle(oracle_mod, ref_meshes):
    A, B = ref_meshes("line.1"), ref_meshes("line.2")
    with lsm.Context(0) as ctx:
        st, em = ctx.supermesh(A, B, elem_measure=True)
        n = st.n_candidates
        pm, pn = ctx.pair_results(n)
    ip, ind = oracle_mod.sort_finder_1d(A, B)
    assert n == len(ind)
    k = 0
    for a in range(len(ip) - 1):
        for b in ind[ip[a]:ip[a + 1]]:
            c = oracle_mod.intersect_intervals(A[0][A[1][a], 0], B[0][B[1][b], 0])
            assert pn[k] == (1 if c.size else 0)
            assert pm[k] == (oracle_mod.interval_size(c) if c.size else 0.0)
            k += 1
    assert oracle_mod.fequals(st.total_measure, 1.0)


# -- single pairs ------------------------------------------------------------

def _random_intervals(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.random((n, 2))
    b = rng.random((n, 2))
    b[: n // 8] = a[: n // 8]                      # identical
    b[n // 8: n // 4, 0] = a[n // 8: n // 4, 1]    # touching
    b[n // 4: n // 3] = b[n // 4: n // 3, ::-1]    # reversed
    a[n // 3: n // 3 + 8, 1] = a[n // 3: n // 3 + 8, 0]  # zero length
    return a, b


def test_intervals_bitexact(gpu_ctx, oracle_mod):
    a, b = _random_intervals(4000, 1)
    m, k, e = gpu_ctx.intersect_pairs_mixed(lsm.PAIR_INTERVALS, a, b, want_elems=True)
    for i in range(len(a)):
        ref = oracle_mod.intersect_intervals(a[i], b[i])
        assert k[i] == (1 if ref.size else 0)
        if ref.size:
            assert np.array_equal(e[i, 0], ref)
            assert m[i] == oracle_mod.interval_size(ref)
        else:
            assert m[i] == 0.0
    for i in range(32):
        assert lsm.interval_size(a[i]) == oracle_mod.interval_size(a[i])
        assert np.array_equal(lsm.intersect_intervals(a[i], b[i]).reshape(-1),
                              oracle_mod.intersect_intervals(a[i], b[i]))


def _random_quads(rng, n):
    """Convex quadrilaterals, counter-clockwise and clockwise."""
    c = rng.random((n, 1, 2))
    ang = np.sort(rng.random((n, 4)) * 2 * np.pi, axis=1)
    r = 0.2 + 0.5 * rng.random((n, 4))
    q = c + np.stack([r * np.cos(ang), r * np.sin(ang)], axis=2)
    q[1::2] = q[1::2, ::-1]
    return q


def test_tri_quad_bitexact(gpu_ctx, oracle_mod):
    rng = np.random.default_rng(3)
    n = 3000
    t = rng.random((n, 3, 2))
    q = _random_quads(rng, n)
    # unit squares against grid-aligned triangles, touching edges included
    t[:64] = np.array([[0, 0], [1, 0], [0, 1]], dtype=np.float64) * rng.integers(1, 3, (64, 1, 1))
    q[:64] = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], dtype=np.float64) + rng.integers(-1, 2, (64, 1, 2))
    m, k, e = gpu_ctx.intersect_pairs_mixed(lsm.PAIR_TRI_QUAD, t, q, want_elems=True)
    for i in range(n):
        ref = oracle_mod.intersect_tri_quad(t[i], q[i])
        assert k[i] == len(ref), i
        assert np.array_equal(e[i, : k[i]], ref), i
        meas = 0.0
        for o in ref:
            meas += oracle_mod.triangle_area(o)
        assert m[i] == meas, i
    for i in range(16):
        assert np.array_equal(lsm.intersect_tri_quad(t[i], q[i]), oracle_mod.intersect_tri_quad(t[i], q[i]))


def _random_hexes(rng, n):
    """Jittered boxes in Gmsh node order (bottom 0-3, top 4-7)."""
    unit = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                     [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.float64)
    lo = rng.random((n, 1, 3)) * 0.5
    size = 0.2 + 0.6 * rng.random((n, 1, 3))
    return lo + unit[None] * size + 0.03 * (rng.random((n, 8, 3)) - 0.5)


def test_tet_hex_bitexact(gpu_ctx, oracle_mod):
    rng = np.random.default_rng(4)
    n = 1500
    t = rng.random((n, 4, 3))
    h = _random_hexes(rng, n)
    # axis-aligned unit cubes and Kuhn tets sharing their faces
    unit = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                     [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.float64)
    h[:32] = unit
    t[:32] = unit[[0, 1, 2, 6]]
    m, k, e = gpu_ctx.intersect_pairs_mixed(lsm.PAIR_TET_HEX, t, h, want_elems=True)
    for i in range(n):
        ref = oracle_mod.intersect_tet_hex(t[i], h[i])
        assert k[i] == len(ref), i
        assert np.array_equal(e[i, : k[i]], ref), i
        meas = 0.0
        for o in ref:
            meas += oracle_mod.tetrahedron_volume(o)
        assert m[i] == meas, i
    for i in range(8):
        assert np.array_equal(lsm.intersect_tet_hex(t[i], h[i]), oracle_mod.intersect_tet_hex(t[i], h[i]))


_ORACLE_FN = {lsm.PAIR_TRI_QUAD: "intersect_tri_quad", lsm.PAIR_TET_HEX: "intersect_tet_hex",
              lsm.PAIR_QUAD_QUAD: "intersect_quads", lsm.PAIR_HEX_HEX: "intersect_hexes"}


def test_quad_quad_bitexact(gpu_ctx, oracle_mod):
    rng = np.random.default_rng(13)
    n = 2000
    a = _random_quads(rng, n)
    b = _random_quads(rng, n)
    unit = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], dtype=np.float64)
    a[:64] = unit + rng.integers(-1, 2, (64, 1, 2))
    b[:64] = unit
    m, k, e = gpu_ctx.intersect_pairs_mixed(lsm.PAIR_QUAD_QUAD, a, b, want_elems=True)
    for i in range(n):
        ref = oracle_mod.intersect_quads(a[i], b[i])
        assert k[i] == len(ref), i
        assert np.array_equal(e[i, : k[i]], ref), i
        meas = 0.0
        for o in ref:
            meas += oracle_mod.triangle_area(o)
        assert m[i] == meas, i


def test_hex_hex_bitexact(gpu_ctx, oracle_mod):
    rng = np.random.default_rng(14)
    n = 300
    a = _random_hexes(rng, n)
    b = _random_hexes(rng, n)
    m, k, e = gpu_ctx.intersect_pairs_mixed(lsm.PAIR_HEX_HEX, a, b, want_elems=True)
    for i in range(n):
        ref = oracle_mod.intersect_hexes(a[i], b[i])
        assert k[i] == len(ref), i
        assert np.array_equal(e[i, : k[i]], ref), i
        meas = 0.0
        for o in ref:
            meas += oracle_mod.tetrahedron_volume(o)
        assert m[i] == meas, i


def _gpu_mixed_total(ctx, kind, A, B, swap=False):
    """Candidates from the GPU search, each element pair clipped on the GPU
    (simplex first when one side is a box element); sum of the per-pair
    measures."""
    n = ctx.find_candidates(A, B)
    ip, ind = ctx.get_candidates(len(A[1]), n)
    rows = np.repeat(np.arange(len(A[1])), np.diff(ip))
    ea, eb = A[0][A[1][rows]], B[0][B[1][ind]]
    s, q = (eb, ea) if swap else (ea, eb)
    m, k, _ = ctx.intersect_pairs_mixed(kind, s, q)
    return float(np.sum(m)), m, k, s, q


@pytest.mark.parametrize("kind,na,nb,swap,expect", [
    (lsm.PAIR_TRI_QUAD, "square.1", "square.4", False, 1.0),   # test_element_intersector.F90:134-158
    (lsm.PAIR_TRI_QUAD, "square.3", "square.2", True, 1.0),    # :163-187
    (lsm.PAIR_QUAD_QUAD, "square.3", "square.4", False, 1.0),  # :192-216
    (lsm.PAIR_TET_HEX, "cube.1", "cube.3", False, 0.5),        # :250-274
    (lsm.PAIR_TET_HEX, "cube.3", "cube.2", True, 0.5),         # :279-303
    (lsm.PAIR_HEX_HEX, "cube.3", "cube.4", False, 0.5),        # :308-332
])
def test_mixed_reference_known_answers(gpu_ctx, oracle_mod, ref_meshes, kind, na, nb, swap, expect):
    A, B = ref_meshes(na), ref_meshes(nb)
    total, m, k, s, q = _gpu_mixed_total(gpu_ctx, kind, A, B, swap)
    assert oracle_mod.fequals(total, expect)
    fn = getattr(oracle_mod, _ORACLE_FN[kind])
    for i in range(len(m)):
        assert k[i] == len(fn(s[i], q[i]))


def test_device_resident_pairs_equal_host_pairs(gpu_ctx):
    """The explicit-pair entries with device arrays (on_device = 1, outputs
    left in device memory) give the host call's measures and counts, simplex
    and mixed kinds."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(12)
    n = 4000
    cases = [(3, None, rng.random((n, 4, 3)), rng.random((n, 4, 3))),
             (2, None, rng.random((n, 3, 2)), rng.random((n, 3, 2))),
             (3, lsm.PAIR_TET_HEX, rng.random((n, 4, 3)), _random_hexes(rng, n)),
             (2, lsm.PAIR_TRI_QUAD, rng.random((n, 3, 2)), _random_quads(rng, n))]
    for dim, kind, a, b in cases:
        if kind is None:
            m, k, _ = gpu_ctx.intersect_pairs(dim, a, b)
        else:
            m, k, _ = gpu_ctx.intersect_pairs_mixed(kind, a, b)
        da = torch.from_numpy(a.reshape(n, -1)).cuda()
        db = torch.from_numpy(b.reshape(n, -1)).cuda()
        dm = torch.empty(n, dtype=torch.float64, device="cuda")
        dk = torch.empty(n, dtype=torch.int32, device="cuda")
        gpu_ctx.intersect_pairs_device(da, db, dm, dk, dim=dim, kind=kind)
        torch.cuda.synchronize()
        assert np.array_equal(dm.cpu().numpy(), m) and np.array_equal(dk.cpu().numpy(), k), (dim, kind)


def test_tet_hex_device_hexahedra_any_alignment(gpu_ctx):
    """Device hexahedra of a large tet-hex batch are read in 16-byte loads
    when the array is 16-byte aligned and in 8-byte loads otherwise (a view
    at an odd double offset): both give the host call's measures and
    counts."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(17)
    n = 3000
    a = rng.random((n, 4, 3))
    b = _random_hexes(rng, n)
    m, k, _ = gpu_ctx.intersect_pairs_mixed(lsm.PAIR_TET_HEX, a, b)
    da = torch.from_numpy(a.reshape(n, -1)).cuda()
    flat = torch.from_numpy(b.reshape(-1)).cuda()
    for off in (0, 1):
        buf = torch.zeros(flat.numel() + 2, dtype=torch.float64, device="cuda")
        buf[off:off + flat.numel()] = flat
        db = buf[off:off + flat.numel()].view(n, 24)
        assert (db.data_ptr() % 16 == 0) == (off == 0)
        dm = torch.empty(n, dtype=torch.float64, device="cuda")
        dk = torch.empty(n, dtype=torch.int32, device="cuda")
        gpu_ctx.intersect_pairs_device(da, db, dm, dk, kind=lsm.PAIR_TET_HEX)
        torch.cuda.synchronize()
        assert np.array_equal(dm.cpu().numpy(), m) and np.array_equal(dk.cpu().numpy(), k), off


def test_hex_hex_large_batch_bitexact(gpu_ctx, oracle_mod):
    """Hexahedron pairs in a batch large enough for the six-plane index
    clipper (A's five tets in five launches, each pair's sum, count and
    output tets carried from tet to tet): measures and counts bit-identical
    to the oracle and to small batches (one-launch clipper), output tets of
    a sample of pairs to the oracle's.  Includes identical unit cubes, A
    inside B, B inside A and far-apart pairs."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(43)
    n = 2300
    a = _random_hexes(rng, n)
    b = _random_hexes(rng, n)
    unit = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                     [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.float64)
    a[:40] = unit
    b[:40] = unit
    c = b[40:200].mean(axis=1, keepdims=True)
    a[40:120] = c[:80] + 0.1 * (a[40:120] - a[40:120].mean(axis=1, keepdims=True))  # A inside B
    b[120:200] = a[120:200].mean(axis=1, keepdims=True) + 0.1 * (b[120:200] - c[80:])  # B inside A
    a[200:260] += 3.0  # far apart
    m, k, _ = gpu_ctx.intersect_pairs_mixed(lsm.PAIR_HEX_HEX, a, b)
    parts = [gpu_ctx.intersect_pairs_mixed(lsm.PAIR_HEX_HEX, a[j:j + 500], b[j:j + 500]) for j in range(0, n, 500)]
    assert np.array_equal(np.concatenate([x[0] for x in parts]), m)
    assert np.array_equal(np.concatenate([x[1] for x in parts]), k)
    assert (k[200:260] == 0).all()
    for i in range(n):
        ref = oracle_mod.intersect_hexes(a[i], b[i])
        assert k[i] == len(ref), i
        meas = 0.0
        for o in ref:
            meas += oracle_mod.tetrahedron_volume(o)
        assert m[i] == meas, i
    # output tets (device arrays: [n][5*729][4][3] does not fit a host test)
    da = torch.from_numpy(a.reshape(n, -1)).cuda()
    db = torch.from_numpy(b.reshape(n, -1)).cuda()
    dm = torch.empty(n, dtype=torch.float64, device="cuda")
    dk = torch.empty(n, dtype=torch.int32, device="cuda")
    de = torch.empty((n, 5 * 729, 4, 3), dtype=torch.float64, device="cuda")
    gpu_ctx.intersect_pairs_device(da, db, dm, dk, de, kind=lsm.PAIR_HEX_HEX)
    torch.cuda.synchronize()
    assert np.array_equal(dm.cpu().numpy(), m) and np.array_equal(dk.cpu().numpy(), k)
    for i in list(range(0, 260, 7)) + list(range(260, n, 97)):
        ref = oracle_mod.intersect_hexes(a[i], b[i])
        assert np.array_equal(de[i, : k[i]].cpu().numpy(), ref), i
    del de


def test_tet_hex_large_batch_bitexact(gpu_ctx, oracle_mod):
    """Tet-hex batches large enough for the early-out pass + six-plane index
    clipper: output tets, counts and measures bit-identical to the oracle and
    to small batches (one-launch clipper), with and without the output
    tets.  Includes tets well inside their hexahedron (every plane a no-op),
    hexahedra inside tets, far-apart pairs and Kuhn tets of unit cubes."""
    rng = np.random.default_rng(41)
    n = 2600
    t = rng.random((n, 4, 3))
    h = _random_hexes(rng, n)
    unit = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                     [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.float64)
    h[:64] = unit
    t[:64] = unit[[0, 1, 2, 6]]
    ch = h[64:300].mean(axis=1, keepdims=True)
    t[64:300] = ch + 0.05 * (rng.random((236, 4, 3)) - 0.5)  # tet inside the hexahedron
    t[300:400] = rng.random((100, 4, 3)) * 4.0 - 1.5  # large tets around the hexahedron
    t[400:500] += 3.0  # far apart
    m, k, e = gpu_ctx.intersect_pairs_mixed(lsm.PAIR_TET_HEX, t, h, want_elems=True)
    for i in range(n):
        ref = oracle_mod.intersect_tet_hex(t[i], h[i])
        assert k[i] == len(ref), i
        assert np.array_equal(e[i, : k[i]], ref), i
        meas = 0.0
        for o in ref:
            meas += oracle_mod.tetrahedron_volume(o)
        assert m[i] == meas, i
    assert (k[400:500] == 0).all()
    m1, k1, _ = gpu_ctx.intersect_pairs_mixed(lsm.PAIR_TET_HEX, t, h)
    assert np.array_equal(m1, m) and np.array_equal(k1, k)
    parts = [gpu_ctx.intersect_pairs_mixed(lsm.PAIR_TET_HEX, t[j:j + 650], h[j:j + 650]) for j in range(0, n, 650)]
    assert np.array_equal(np.concatenate([x[0] for x in parts]), m)
    assert np.array_equal(np.concatenate([x[1] for x in parts]), k)
