"""GPU parity: the CUDA library against the CPU oracle and the reference's
known answers.  All calls go through the C-ABI (libsupermesh_b200 is a
ctypes binding of lib/libsupermesh.so).

Bars (from the path's correctness contract):
  * candidate sets per A element: identical to the oracle's quadtree/octree
    set (integer work: exact);
  * number of output simplices per pair and the intersecting-pair set:
    exact;
  * per-pair measure: relative difference <= 1e-12 (the clipped vertices
    are computed with the reference's FP64 operation order, so in practice
    they agree bit for bit);
  * totals: |total - oracle total| <= 1e-12 and, for meshes that tile the
    same domain, |total - domain measure| <= 1e-12.
"""
from pathlib import Path

import numpy as np
import pytest

import libsupermesh_b200 as lsm
from libsupermesh_b200 import meshes as M

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]

REL_TOL = 1e-12


def rows(ip, ind):
    return [np.sort(ind[ip[a]:ip[a + 1]]) for a in range(len(ip) - 1)]


def pair_table(ip, ind, *vals):
    """Sort pairs by (row, b) so GPU and oracle orders line up."""
    r = np.repeat(np.arange(len(ip) - 1), np.diff(ip))
    order = np.lexsort((ind, r))
    return (r[order], np.asarray(ind)[order]) + tuple(np.asarray(v)[order] for v in vals)


def check_pipeline(ctx, oracle, dim, A, B, domain=None):
    ip_o, ind_o = oracle.tree_finder(dim, A, B)
    pm_o, pn_o, em_o, st_o = oracle.narrow(dim, A, B, ip_o, ind_o, nthreads=oracle.lib().orc_num_threads_available())
    st, em = ctx.supermesh(A, B, elem_measure=True)
    n = st.n_candidates
    assert n == len(ind_o)
    ip_g, ind_g = ctx.get_candidates(len(A[1]), n)
    assert np.array_equal(ip_g, ip_o)
    pm_g, pn_g = ctx.pair_results(n)
    ro, bo, mo, no = pair_table(ip_o, ind_o, pm_o, pn_o)
    rg, bg, mg, ng = pair_table(ip_g, ind_g, pm_g, pn_g)
    assert np.array_equal(ro, rg) and np.array_equal(bo, bg), "candidate sets differ"
    assert np.array_equal(no, ng), "output simplex counts differ"
    scale = np.maximum(np.abs(mo), 1e-300)
    rel = np.abs(mg - mo) / scale
    assert rel.max(initial=0.0) <= REL_TOL
    # intersecting-pair set, with and without the 1e-14 element-measure filter
    assert np.array_equal(no > 0, ng > 0)
    assert st.n_intersecting == int((no > 0).sum())
    assert st.n_out_simplices == int(no.sum())
    assert abs(st.total_measure - st_o.total) <= REL_TOL
    if domain is not None:
        assert abs(st.total_measure - domain) <= REL_TOL
    assert np.abs(em - em_o).max(initial=0.0) <= REL_TOL * max(1.0, np.abs(em_o).max(initial=0.0))
    return st


@pytest.mark.parametrize("name", ["small2d_7x9", "small2d_40x31", "small3d_4x5", "small3d_9x7"])
def test_small_configs(gpu_ctx, oracle_mod, name):
    dim, A, B = M.config_meshes(name)
    check_pipeline(gpu_ctx, oracle_mod, dim, A, B, domain=1.0)


@pytest.mark.parametrize("name", ["small2d_20x17", "small3d_7x6"])
@pytest.mark.parametrize("scale,shift", [(1.0, 1.0e6), (1.0, -3.5e4), (1.0e-6, 0.0)])
def test_far_and_tiny_coordinates(gpu_ctx, oracle_mod, name, scale, shift):
    """Meshes far from the origin or scaled far below unit size: the
    rounding margins of the exact early-outs and of the final-tet test grow
    with the coordinates or are dominated by their absolute terms; per-pair
    results still match the oracle."""
    dim, (pa, ea), (pb, eb) = M.config_meshes(name)
    A = (pa * scale + shift, ea)
    B = (pb * scale + shift, eb)
    st = check_pipeline(gpu_ctx, oracle_mod, dim, A, B)
    assert st.n_intersecting > 0
    assert abs(st.total_measure - scale ** dim) <= 1e-9 * scale ** dim


def test_config_tri2d_73x100_full(gpu_ctx, oracle_mod):
    dim, A, B = M.config_meshes("tri2d_73x100")
    st = check_pipeline(gpu_ctx, oracle_mod, dim, A, B, domain=1.0)
    assert st.n_candidates > 100000


def test_config_tet3d_27x32_full(gpu_ctx, oracle_mod):
    dim, A, B = M.config_meshes("tet3d_27x32")
    st = check_pipeline(gpu_ctx, oracle_mod, dim, A, B, domain=1.0)
    assert st.n_candidates > 10_000_000


def test_config_tri2d_777x1024_rot7_full(gpu_ctx, oracle_mod):
    # 1.2M x 2.1M triangles, target rotated 7 degrees and clamped (it has
    # degenerate and folded elements, so the total is the oracle's, not 1)
    dim, A, B = M.config_meshes("tri2d_777x1024_rot7")
    st = check_pipeline(gpu_ctx, oracle_mod, dim, A, B)
    assert st.n_candidates > 10_000_000


def test_config_tet3d_graded_full(gpu_ctx, oracle_mod):
    # ~1.0M x ~0.8M graded tets (x -> x^2 per axis, 20x variation in element
    # size; 56M candidates) against the oracle pair by pair: CSR offsets, the
    # candidate set of every row, n_out per pair, per-pair volume, the
    # intersecting-pair set and the total.  The graded mesh stresses the
    # rounding margins of the exact early-outs most.
    dim, A, B = M.config_meshes("tet3d_graded_55x51")
    st = check_pipeline(gpu_ctx, oracle_mod, dim, A, B, domain=1.0)
    assert st.n_candidates > 50_000_000


def test_config_tet3d_graded_full_properties(gpu_ctx):
    # ~1.0M x ~0.8M graded tets (56M candidates): size-independent checks
    # instead of the oracle: the total is the cube's volume and every target
    # element is covered exactly once (its supermesh volume is its own)
    dim, A, B = M.config_meshes("tet3d_graded_55x51")
    st, em = gpu_ctx.supermesh(A, B, elem_measure=True)
    assert st.n_candidates > 50_000_000
    assert abs(st.total_measure - 1.0) <= REL_TOL
    v = A[0][A[1]]
    e1, e2, e3 = v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]
    own = np.abs(np.einsum("ij,ij->i", e1, np.cross(e2, e3))) / 6.0
    assert np.all(np.abs(em - own) <= 1e-12 * own)
    # the per-pair results do not depend on the work order (true-class bins)
    pm, pn = gpu_ctx.pair_results(st.n_candidates)
    lsm.set_option("tet_schedule", 2)
    try:
        st2 = gpu_ctx.clip_candidates()
        pm2, pn2 = gpu_ctx.pair_results(st.n_candidates)
    finally:
        lsm.set_option("tet_schedule", 0)
    assert np.array_equal(pm, pm2) and np.array_equal(pn, pn2) and st2.total_measure == st.total_measure


def test_config_tri2d_777x1024_rot7_p1_mass(gpu_ctx, oracle_mod):
    dim, A, B = M.config_meshes("tri2d_777x1024_rot7")
    u, v = A[0][:, 0], B[0][:, 1]
    integral, _ = gpu_ctx.p1_mass(A, B, u, v)
    ip, ind = oracle_mod.tree_finder(dim, A, B)
    i_o, meas_o, _ = oracle_mod.p1_mass(dim, A, B, ip, ind, u, v)
    assert abs(integral - i_o) <= 1e-12 * abs(i_o)


def test_autotuner_keeps_results(gpu_ctx, tmp_path, monkeypatch):
    from libsupermesh_b200 import autotune

    monkeypatch.setenv("LIBSUPERMESH_TUNING_CACHE", str(tmp_path / "tuning.json"))
    for name in ("small2d_60x70", "small3d_10x12"):
        dim, A, B = M.config_meshes(name)
        ref, em_ref = gpu_ctx.supermesh(A, B, elem_measure=True)
        res = autotune.tune(gpu_ctx, A, B, reps=1)
        assert res["tried"] == (27 if dim == 2 else 9)
        st, em = gpu_ctx.supermesh(A, B, elem_measure=True)
        assert st.as_dict() == ref.as_dict() and np.array_equal(em, em_ref)
        assert autotune.apply_cached(dim, len(A[1]), len(B[1])) == res["setting"]
    for n, v in {"tri_blocks_per_sm": 8, "query_block": 128, "leaf_bucket": 1}.items():
        lsm.set_option(n, v)


def test_clip_kernel_timing_option(gpu_ctx):
    """time_kernels records events around the clip kernel; without the
    option the timing entry reports a state error."""
    dim, A, B = M.config_meshes("small3d_8x9")
    lsm.set_option("time_kernels", 0)
    gpu_ctx.supermesh(A, B)
    with pytest.raises(lsm.LsmError) as e:
        gpu_ctx.clip_kernel_ms()
    assert e.value.status == 6  # LSM_ERROR_STATE
    lsm.set_option("time_kernels", 1)
    try:
        st = gpu_ctx.clip_candidates()
        ms = gpu_ctx.clip_kernel_ms()
    finally:
        lsm.set_option("time_kernels", 0)
    assert st.n_candidates > 0 and 0.0 < ms < 1000.0


def _near_touching_tets(gaps, per_gap, seed):
    """A: random tets spread over a box; B: for each A tet a tet whose tip
    sits at a signed gap beyond the centroid of one of A's faces (negative:
    it pokes into A) and whose base lies farther out, so that B's own face
    planes do not separate the pair and only the B-beyond-a-face-of-A test
    can.  Returns ((pos_a, en_a), (pos_b, en_b), gap per pair)."""
    rng = np.random.default_rng(seed)
    ta, tb, gs = [], [], []
    for gap in gaps:
        for _ in range(per_gap):
            while True:
                a = rng.random((4, 3)) + rng.random(3) * 40.0
                vol = abs(np.linalg.det(a[1:] - a[0])) / 6.0
                if vol > 0.02:
                    break
            f = int(rng.integers(4))
            face = [k for k in range(4) if k != f]
            q = a[face].mean(axis=0)
            n = np.cross(a[face[1]] - a[face[0]], a[face[2]] - a[face[0]])
            n /= np.linalg.norm(n)
            if np.dot(n, a[f] - q) > 0:
                n = -n
            u = np.cross(n, [1.0, 0.0, 0.0] if abs(n[0]) < 0.9 else [0.0, 1.0, 0.0])
            u /= np.linalg.norm(u)
            v = np.cross(n, u)
            size = vol ** (1.0 / 3.0)
            th = rng.random() * 2 * np.pi + np.arange(3) * 2 * np.pi / 3
            base = q + 0.6 * size * n + 0.7 * size * (np.cos(th)[:, None] * u + np.sin(th)[:, None] * v)
            b = np.vstack([q + gap * n, base])[rng.permutation(4)]
            ta.append(a)
            tb.append(b)
            gs.append(gap)
    ta, tb = np.array(ta), np.array(tb)
    en = np.arange(4 * len(ta), dtype=np.int64).reshape(-1, 4)
    return (ta.reshape(-1, 3), en), (tb.reshape(-1, 3), en.copy()), np.array(gs)


def test_separation_screen_near_touching(gpu_ctx, oracle_mod):
    """Pairs separated by a face plane of A by gaps from far below to far
    above the screen's rounding margin, and overlapping ones: per-pair
    results equal the oracle's (check_pipeline) with the screen on and off,
    and the screen takes pairs away from the clipper where the gap is wide."""
    gaps = [-1e-3, -1e-9, -1e-13, 0.0, 1e-300, 1e-17, 1e-15, 1e-13, 1e-11, 1e-9, 1e-6, 1e-3]
    A, B, g = _near_touching_tets(gaps, 24, 21)
    lsm.set_option("tet_screen", 1)
    st = check_pipeline(gpu_ctx, oracle_mod, 3, A, B)
    with_screen = gpu_ctx.clip_survivors()
    lsm.set_option("tet_screen", 0)
    try:
        st0 = check_pipeline(gpu_ctx, oracle_mod, 3, A, B)
        without = gpu_ctx.clip_survivors()
    finally:
        lsm.set_option("tet_screen", 1)
    assert st.as_dict() == st0.as_dict()
    # every pair with a gap >= 1e-9 is screened out; the overlapping ones stay
    assert without - with_screen >= int((g >= 1e-9).sum())
    assert with_screen >= int((g < 0).sum())


def test_separation_screen_keeps_results(gpu_ctx):
    """Screen on and off give bit-identical per-pair results on a mesh pair,
    and the screen removes pairs from the clipper."""
    dim, A, B = M.config_meshes("small3d_10x12")
    lsm.set_option("tet_screen", 0)
    try:
        st0, em0 = gpu_ctx.supermesh(A, B, elem_measure=True)
        pm0, pn0 = gpu_ctx.pair_results(st0.n_candidates)
        s0 = gpu_ctx.clip_survivors()
    finally:
        lsm.set_option("tet_screen", 1)
    st1, em1 = gpu_ctx.supermesh(A, B, elem_measure=True)
    pm1, pn1 = gpu_ctx.pair_results(st1.n_candidates)
    s1 = gpu_ctx.clip_survivors()
    assert st0.as_dict() == st1.as_dict()
    assert np.array_equal(pm0, pm1) and np.array_equal(pn0, pn1) and np.array_equal(em0, em1)
    assert st1.n_intersecting <= s1 < s0


@pytest.mark.parametrize("na,nb", [(12, 3), (3, 12)])
def test_nested_meshes_plane_skipping(gpu_ctx, oracle_mod, na, nb):
    """A fine mesh inside a coarse one (and the reverse): many pairs have
    planes of B that keep A whole, which the clipper skips, and pairs with A
    inside all four planes, which the prefilter settles; per-pair results
    match the oracle."""
    A = M.grid3d(na, 3, 0.25)
    B = M.grid3d(nb, 2, 0.25)
    st = check_pipeline(gpu_ctx, oracle_mod, 3, A, B, domain=1.0)
    assert st.n_intersecting > 0


def test_int64_and_int32_enlists_agree(gpu_ctx):
    dim, A, B = M.config_meshes("small3d_5x6")
    s32, _ = gpu_ctx.supermesh(A, B)
    A64 = (A[0], A[1].astype(np.int64))
    B64 = (B[0], B[1].astype(np.int64))
    s64, _ = gpu_ctx.supermesh(A64, B64)
    assert s32.as_dict() == s64.as_dict()


def test_reference_known_answers(gpu_ctx, oracle_mod, ref_meshes):
    # test_tri_intersector.F90:104 and test_tet_intersector.F90:104
    st, _ = gpu_ctx.supermesh(ref_meshes("triangle_0_01"), ref_meshes("square_0_01"))
    assert oracle_mod.fequals(st.total_measure, 0.5)
    st, _ = gpu_ctx.supermesh(ref_meshes("pyramid_0_05"), ref_meshes("cube_0_05"))
    assert oracle_mod.fequals(st.total_measure, 1.0 / 3.0)


@pytest.mark.parametrize("dim,na,nb", [(2, "square.1", "square.2"), (3, "cube.1", "cube.2")])
def test_reference_completeness(gpu_ctx, oracle_mod, ref_meshes, dim, na, nb):
    # test_intersection_finder_completeness_{2d,3d}.F90: rows are B elements
    MA, MB = ref_meshes(na), ref_meshes(nb)
    st, em = gpu_ctx.supermesh(MB, MA, elem_measure=True)
    for b in range(len(MB[1])):
        v = MB[0][MB[1][b]]
        own = oracle_mod.triangle_area(v) if dim == 2 else oracle_mod.tetrahedron_volume(v)
        assert oracle_mod.fequals(own, em[b])
    check_pipeline(gpu_ctx, oracle_mod, dim, MB, MA)


def test_reference_tiny_candidate_sets(gpu_ctx, ref_meshes):
    t1, t2, tet = ref_meshes("triangle.1"), ref_meshes("triangle.2"), ref_meshes("tet")
    ip, ind = lsm.tree_intersection_finder(*t1, *t1)
    assert list(ind) == [0] and list(ip) == [0, 1]
    ip, ind = lsm.tree_intersection_finder(*t1, *t2)
    assert sorted(ind) == [0, 1, 2]
    ip, ind = lsm.tree_intersection_finder(*t2, *t2)
    for i in range(3):
        assert i in set(ind[ip[i]:ip[i + 1]])
    ip, ind = lsm.tree_intersection_finder(*tet, *tet)
    assert list(ind) == [0]


def test_legacy_tree_finder_matches_oracle(oracle_mod):
    for name in ("small2d_11x13", "small3d_5x4"):
        dim, A, B = M.config_meshes(name)
        ip, ind = lsm.tree_intersection_finder(A[0], A[1], B[0], B[1])
        ip_o, ind_o = oracle_mod.tree_finder(dim, A, B)
        assert np.array_equal(ip, ip_o)
        for r_g, r_o in zip(rows(ip, ind), rows(ip_o, ind_o)):
            assert np.array_equal(r_g, r_o)


def test_legacy_tree_finder_quads(oracle_mod):
    # the tree finder accepts any element type (here quads, loc 4)
    n = 6
    idx = np.arange(n + 1)
    jj, ii = np.meshgrid(idx, idx, indexing="ij")
    pos = np.stack([ii.ravel() / n, jj.ravel() / n], axis=1).astype(np.float64)
    cj, ci = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    v00 = (cj * (n + 1) + ci).ravel()
    quads = np.stack([v00, v00 + 1, v00 + n + 2, v00 + n + 1], axis=1).astype(np.int32)
    B = M.grid2d(5, 0, 0.3)
    ip, ind = lsm.tree_intersection_finder(pos, quads, *B)
    ip_o, ind_o = oracle_mod.brute_force_finder(2, (pos, quads), B)
    assert np.array_equal(ip, ip_o)
    for r_g, r_o in zip(rows(ip, ind), rows(ip_o, ind_o)):
        assert np.array_equal(r_g, r_o)


def _random_pairs(dim, n, seed):
    rng = np.random.default_rng(seed)
    per = (3, 2) if dim == 2 else (4, 3)
    a = rng.random((n,) + per)
    b = rng.random((n,) + per) * 0.8 + 0.1
    # include identical and shared-vertex pairs
    b[: n // 8] = a[: n // 8]
    b[n // 8: n // 4, 0] = a[n // 8: n // 4, 0]
    return a, b


@pytest.mark.parametrize("dim", [2, 3])
def test_intersect_pairs_bitexact(gpu_ctx, oracle_mod, dim):
    a, b = _random_pairs(dim, 400, 7 + dim)
    m, k, e = gpu_ctx.intersect_pairs(dim, a, b, want_elems=True)
    for i in range(len(a)):
        ref = oracle_mod.intersect_tris(a[i], b[i]) if dim == 2 else oracle_mod.intersect_tets(a[i], b[i])
        assert k[i] == len(ref)
        assert np.array_equal(e[i, : k[i]], ref), i
        meas = 0.0
        for o in ref:
            meas += oracle_mod.triangle_area(o) if dim == 2 else oracle_mod.tetrahedron_volume(o)
        assert m[i] == meas


def test_intersect_pairs_large_batch_bitexact(gpu_ctx, oracle_mod):
    """Tet pair batches large enough for the early-out pass + index clipper
    (the small ones use the one-launch clipper): output tets, counts and
    measures bit-identical to the oracle and to small batches of the same
    pairs, with the output tets requested and without, the second early-out
    on and off.  The pairs include identical and shared-vertex pairs, A well
    inside B (every plane a no-op), B inside A and far-apart pairs."""
    a, b = _random_pairs(3, 3200, 31)
    c = a.mean(axis=1, keepdims=True)
    b[400:600] = c[400:600] + 3.0 * (a[400:600] - c[400:600])  # A inside B
    b[600:800] = c[600:800] + 0.2 * (a[600:800] - c[600:800])  # B inside A
    b[800:1000] += 2.0  # far apart
    b[1000:1100] = a[1000:1100, ::-1]  # identical, vertices reversed
    m, k, e = gpu_ctx.intersect_pairs(3, a, b, want_elems=True)
    for i in range(len(a)):
        ref = oracle_mod.intersect_tets(a[i], b[i])
        assert k[i] == len(ref), i
        assert np.array_equal(e[i, : k[i]], ref), i
        meas = 0.0
        for o in ref:
            meas += oracle_mod.tetrahedron_volume(o)
        assert m[i] == meas, i
    assert (k[400:600] == 1).all() and (k[800:1000] == 0).all()
    m1, k1, _ = gpu_ctx.intersect_pairs(3, a, b)
    assert np.array_equal(m1, m) and np.array_equal(k1, k)
    def same_outputs(m2, k2, e2):
        # slots past a pair's count are unspecified
        assert np.array_equal(m2, m) and np.array_equal(k2, k)
        for i in range(len(a)):
            assert np.array_equal(e2[i, : k[i]], e[i, : k[i]]), i

    small = [gpu_ctx.intersect_pairs(3, a[j:j + 800], b[j:j + 800], want_elems=True) for j in range(0, len(a), 800)]
    same_outputs(*(np.concatenate([x[q] for x in small]) for q in range(3)))
    lsm.set_option("tet_screen", 0)
    try:
        same_outputs(*gpu_ctx.intersect_pairs(3, a, b, want_elems=True))
    finally:
        lsm.set_option("tet_screen", 1)


@pytest.mark.parametrize("n", [2047, 2048, 2049, 70001])
def test_intersect_pairs_batch_sizes_agree(gpu_ctx, n):
    """Tet pair batches just below, at and above the size where the early-out
    pass + index clipper take over (its survivors go to per-block segments
    that the clipper takes by chunks; 70001 pairs give partial blocks and
    segments of every length), against the same pairs in batches of 1000
    (one-launch clipper): measures, counts and output tets identical."""
    a, b = _random_pairs(3, n, 100 + n % 97)
    m, k, e = gpu_ctx.intersect_pairs(3, a, b, want_elems=n < 10000)
    parts = [gpu_ctx.intersect_pairs(3, a[j:j + 1000], b[j:j + 1000], want_elems=n < 10000)
             for j in range(0, n, 1000)]
    assert np.array_equal(m, np.concatenate([x[0] for x in parts]))
    assert np.array_equal(k, np.concatenate([x[1] for x in parts]))
    if e is not None:
        e2 = np.concatenate([x[2] for x in parts])
        for i in range(n):
            assert np.array_equal(e[i, : k[i]], e2[i, : k[i]]), i


def test_legacy_single_pair_entries(oracle_mod):
    a, b = _random_pairs(2, 16, 3)
    for i in range(len(a)):
        assert np.array_equal(lsm.intersect_tris_real(a[i], b[i]), oracle_mod.intersect_tris(a[i], b[i]))
        assert lsm.triangle_area(a[i]) == oracle_mod.triangle_area(a[i])
    a, b = _random_pairs(3, 16, 4)
    for i in range(len(a)):
        assert np.array_equal(lsm.intersect_tets_real(a[i], b[i]), oracle_mod.intersect_tets(a[i], b[i]))
        assert lsm.tetrahedron_volume(a[i]) == oracle_mod.tetrahedron_volume(a[i])


@pytest.mark.parametrize("name", ["small2d_12x17", "small3d_4x5", "small3d_20x9"])
def test_p1_mass_device_inputs(gpu_ctx, name):
    """Device-resident meshes and fields give the host call's u^T M v, bit
    for bit, and repeated calls give the same value (the 3D lanes take pairs
    in a dynamic order; the sum runs in pair order)."""
    torch = pytest.importorskip("torch")
    dim, A, B = M.config_meshes(name)
    u = np.cos(3 * A[0][:, 0]) + A[0][:, 1]
    v = np.sin(2 * B[0][:, 1]) - B[0][:, 0]
    ref, _ = gpu_ctx.p1_mass(A, B, u, v)
    dev = torch.device("cuda:0")
    tA = tuple(torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in A)
    tB = tuple(torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in B)
    tu, tv = torch.from_numpy(u).to(dev), torch.from_numpy(v).to(dev)
    torch.cuda.synchronize()
    val, blocks = gpu_ctx.p1_mass(tA, tB, tu, tv, on_device=True)
    assert blocks is None and val == ref
    for _ in range(3):
        assert gpu_ctx.p1_mass(tA, tB, tu, tv, on_device=True)[0] == ref


def test_p1_mass_reference_answers(gpu_ctx, oracle_mod, ref_meshes):
    A, B = ref_meshes("triangle_0_01"), ref_meshes("square_0_01")
    integral, _ = gpu_ctx.p1_mass(A, B, A[0][:, 0], B[0][:, 1])
    assert oracle_mod.fequals(integral, 8.3333333333333398e-2)
    A, B = ref_meshes("pyramid_0_05"), ref_meshes("cube_0_05")
    integral, _ = gpu_ctx.p1_mass(A, B, A[0][:, 0] + A[0][:, 2], B[0][:, 1])
    assert oracle_mod.fequals(integral, 1.2499999999999989e-1)


@pytest.mark.parametrize("name", ["small2d_12x17", "small2d_40x9", "small3d_4x5", "small3d_12x3", "small3d_3x11"])
def test_p1_mass_blocks_match_oracle(gpu_ctx, oracle_mod, name):
    """Blocks per candidate bit for bit and u^T M v (summed in another order:
    1e-12) against the oracle; 12x3 puts most of A's tets inside one of B's
    (no plane clips them), 3x11 most of B's inside one of A's."""
    dim, A, B = M.config_meshes(name)
    u = np.cos(3 * A[0][:, 0]) + A[0][:, 1]
    v = np.sin(2 * B[0][:, 1]) - B[0][:, 0]
    integral, blocks = gpu_ctx.p1_mass(A, B, u, v, want_blocks=True)
    ip_g, ind_g = gpu_ctx.get_candidates(len(A[1]), len(blocks))
    ip_o, ind_o = oracle_mod.tree_finder(dim, A, B)
    i_o, _, blocks_o = oracle_mod.p1_mass(dim, A, B, ip_o, ind_o, u, v, want_blocks=True)
    assert abs(integral - i_o) <= 1e-12 * max(1.0, abs(i_o))
    ro, bo, ko = pair_table(ip_o, ind_o, np.arange(len(ind_o)))
    rg, bg, kg = pair_table(ip_g, ind_g, np.arange(len(ind_g)))
    assert np.array_equal(bo, bg)
    assert np.array_equal(blocks[kg], blocks_o[ko])


def _p2_fields(A, B):
    e2a, na, eda = M.p2_space(A[1])
    e2b, nb, edb = M.p2_space(B[1])
    fa = M.p1_to_p2(A[0][:, 0], na, eda) * M.p1_to_p2(A[0][:, 1], na, eda)
    fb = M.p1_to_p2(B[0][:, 0], nb, edb) ** 2
    return e2a, fa, e2b, fb


def test_p2_inner_product_reference_answer(gpu_ctx, oracle_mod, ref_meshes):
    # test_parallel_p2_inner_product_2d.F90:45-46: area 0.5, integral
    # 2.7083333333333272e-2; per-pair contributions bit-identical to the oracle
    A, B = ref_meshes("triangle_0_01"), ref_meshes("square_0_01")
    e2a, fa, e2b, fb = _p2_fields(A, B)
    integral, area, pv = gpu_ctx.p2_inner_product(A, B, e2a, fa, e2b, fb, want_pairs=True)
    assert oracle_mod.fequals(area, 0.5) and oracle_mod.fequals(integral, 2.7083333333333272e-2)
    n = len(pv)
    ip_g, ind_g = gpu_ctx.get_candidates(len(A[1]), n)
    ip_o, ind_o = oracle_mod.tree_finder(2, A, B)
    i_o, a_o, pv_o = oracle_mod.p2_inner_product(A, B, ip_g, ind_g, e2a, fa, e2b, fb)
    assert np.array_equal(pv, pv_o)
    assert abs(integral - i_o) <= 1e-15 * abs(i_o) and abs(area - a_o) <= 1e-15


@pytest.mark.parametrize("name", ["small2d_30x41", "tri2d_73x100"])
def test_p2_inner_product_matches_oracle(gpu_ctx, oracle_mod, name):
    dim, A, B = M.config_meshes(name)
    e2a, fa, e2b, fb = _p2_fields(A, B)
    integral, area, pv = gpu_ctx.p2_inner_product(A, B, e2a, fa, e2b, fb, want_pairs=True)
    ip_g, ind_g = gpu_ctx.get_candidates(len(A[1]), len(pv))
    i_o, a_o, pv_o = oracle_mod.p2_inner_product(A, B, ip_g, ind_g, e2a, fa, e2b, fb)
    assert np.array_equal(pv, pv_o)
    assert abs(integral - i_o) <= 1e-13 * abs(i_o)
    assert abs(area - 1.0) <= 1e-12
    # int_{[0,1]^2} x y x^2 = 1/8
    assert abs(integral - 0.125) <= 1e-12


def test_p2_inner_product_rejects_bad_nodes(gpu_ctx):
    dim, A, B = M.config_meshes("small2d_3x4")
    e2a, fa, e2b, fb = _p2_fields(A, B)
    e2a = e2a.copy()
    e2a[0, 4] = len(fa) + 3
    with pytest.raises(lsm.LsmError):
        gpu_ctx.p2_inner_product(A, B, e2a, fa, e2b, fb)


def test_empty_and_single_element_meshes(gpu_ctx):
    dim, A, B = M.config_meshes("small2d_3x4")
    empty = (A[0], np.zeros((0, 3), dtype=np.int32))
    st, em = gpu_ctx.supermesh(empty, B, elem_measure=True)
    assert st.n_candidates == 0 and st.total_measure == 0.0
    st, em = gpu_ctx.supermesh(A, (B[0], np.zeros((0, 3), dtype=np.int32)), elem_measure=True)
    assert st.n_candidates == 0 and (em == 0).all()
    one = (np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), np.array([[0, 1, 2]], dtype=np.int32))
    st, em = gpu_ctx.supermesh(one, one, elem_measure=True)
    assert st.n_candidates == 1 and st.n_intersecting == 1 and abs(st.total_measure - 0.5) < 1e-15


def test_touching_boxes_are_not_candidates(gpu_ctx):
    A = (np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), np.array([[0, 1, 2]], dtype=np.int32))
    B = (np.array([[1.0, 0.0], [2.0, 0.0], [1.0, 1.0]]), np.array([[0, 1, 2]], dtype=np.int32))
    assert gpu_ctx.find_candidates(A, B) == 0


def test_invalid_input_is_reported(gpu_ctx):
    dim, A, B = M.config_meshes("small2d_3x4")
    bad = (A[0], A[1].copy())
    bad[1][0, 0] = len(A[0]) + 5
    with pytest.raises(lsm.LsmError) as e:
        gpu_ctx.supermesh(bad, B)
    assert e.value.status == 1
    with pytest.raises(lsm.LsmError):
        gpu_ctx.supermesh(A, M.config_meshes("small3d_2x2")[1])
    # the context stays usable after an error
    st, _ = gpu_ctx.supermesh(A, B)
    assert abs(st.total_measure - 1.0) < 1e-12


def test_device_resident_inputs(gpu_ctx):
    torch = pytest.importorskip("torch")
    dim, A, B = M.config_meshes("small3d_6x7")
    ref, em_ref = gpu_ctx.supermesh(A, B, elem_measure=True)
    dev = torch.device("cuda:0")
    tA = (torch.from_numpy(A[0]).to(dev), torch.from_numpy(A[1]).to(dev))
    tB = (torch.from_numpy(B[0]).to(dev), torch.from_numpy(B[1]).to(dev))
    out = torch.zeros(len(A[1]), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    st, _ = gpu_ctx.supermesh(tA, tB, elem_measure=True, on_device=True, out=out)
    assert st.as_dict() == ref.as_dict()
    assert np.array_equal(out.cpu().numpy(), em_ref)


@pytest.mark.parametrize("name", ["small2d_30x41", "small3d_8x9"])
def test_ordered_clip_matches_unordered(gpu_ctx, name):
    # a schedule changes only the order in which pairs are clipped
    dim, A, B = M.config_meshes(name)
    st, _ = gpu_ctx.supermesh(A, B)
    pm, pn = gpu_ctx.pair_results(st.n_candidates)
    order = np.random.default_rng(3).permutation(st.n_candidates).astype(np.int32)
    st2 = gpu_ctx.clip_candidates_ordered(order)
    pm2, pn2 = gpu_ctx.pair_results(st.n_candidates)
    assert np.array_equal(pm, pm2) and np.array_equal(pn, pn2)
    assert st2.as_dict() == st.as_dict()


def test_batched_matches_single(gpu_ctx):
    pairs = M.batched_pairs(6, seed=6, emin=2e2, emax=2e3)
    totals, nc, ni = gpu_ctx.supermesh_batched([(A, B) for _, A, B in pairs])
    for i, (dim, A, B) in enumerate(pairs):
        st, _ = gpu_ctx.supermesh(A, B)
        assert nc[i] == st.n_candidates and ni[i] == st.n_intersecting
        assert abs(totals[i] - st.total_measure) <= 1e-14
        assert abs(totals[i] - 1.0) <= 1e-12


def test_batched_spill_chunks_keep_results(gpu_ctx):
    """Mesh pairs of unrelated resolutions give rows longer than the search's
    256-entry row cache: with spill chunks, with a pool too small for all of
    them (the rest traversed again) and with none, the candidate counts and
    totals are identical."""
    pairs = [(3, M.grid3d(3, 3, 0.25), M.grid3d(14, 2, 0.25)),
             (3, M.grid3d(4, 5, 0.25), M.grid3d(13, 4, 0.25)),
             (2, M.grid2d(4, 1, 0.3), M.grid2d(60, 0, 0.3)),
             (2, M.grid2d(5, 3, 0.3), M.grid2d(45, 2, 0.3))]
    results = []
    try:
        for chunks in (-1, 7, 0):
            lsm.set_option("spill_chunks", chunks)
            for dim in (2, 3):
                sub = [(A, B) for d, A, B in pairs if d == dim]
                results.append((chunks, dim, gpu_ctx.supermesh_batched(sub)))
    finally:
        lsm.set_option("spill_chunks", -1)
    ref = {dim: r for ch, dim, r in results if ch == -1}
    for ch, dim, (tot, nc, ni) in results:
        rt, rc, ri = ref[dim]
        assert list(nc) == list(rc) and list(ni) == list(ri)
        assert list(tot) == list(rt)
    for d, A, B in pairs:
        st, _ = gpu_ctx.supermesh(A, B)
        assert abs(st.total_measure - 1.0) <= 1e-12
        assert st.n_candidates > 256 * len(A[1]) // 2  # long rows


def test_batched_vs_oracle(gpu_ctx, oracle_mod):
    pairs = M.batched_pairs(24, seed=16, emin=1e2, emax=3e3)
    totals, nc, ni = gpu_ctx.supermesh_batched([(A, B) for _, A, B in pairs])
    for i, (dim, A, B) in enumerate(pairs):
        ip, ind = oracle_mod.tree_finder(dim, A, B)
        _, _, _, st = oracle_mod.narrow(dim, A, B, ip, ind)
        assert nc[i] == st.n_candidates and ni[i] == st.n_intersecting
        assert abs(totals[i] - st.total) <= REL_TOL


def test_batched_host_calls_back_to_back(gpu_ctx):
    """Host-buffer batches of both dimensions, called back to back with
    growing meshes (the 3D group's meshes are copied on a second stream
    while the 2D group computes, into staging buffers the previous call
    used), give exactly the results of device-resident inputs."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    for seed, emax in ((31, 1e3), (32, 4e3), (33, 2e3)):
        pairs = M.batched_pairs(10, seed=seed, emin=1e2, emax=emax)
        assert {d for d, _, _ in pairs} == {2, 3}
        host = [(A, B) for _, A, B in pairs]
        t_h, nc_h, ni_h = gpu_ctx.supermesh_batched(host)
        tdev = [tuple((torch.from_numpy(np.ascontiguousarray(x[0])).to(dev),
                       torch.from_numpy(np.ascontiguousarray(x[1])).to(dev)) for x in pr) for pr in host]
        torch.cuda.synchronize()
        t_d, nc_d, ni_d = gpu_ctx.supermesh_batched(tdev, on_device=True)
        assert np.array_equal(nc_h, nc_d) and np.array_equal(ni_h, ni_d) and np.array_equal(t_h, t_d)
        assert np.abs(t_h - 1.0).max() <= 1e-12


def test_batched_host_error_then_recovery(gpu_ctx):
    """An invalid node index in a 2D mesh fails the batch while the 3D
    group's copies may still be running on the second stream; the call
    reports it (the kernels' bounds checks turn it into a status), and the
    next batch on the same context gives the expected results."""
    pairs = M.batched_pairs(8, seed=41, emin=1e2, emax=2e3)
    host = [(A, B) for _, A, B in pairs]
    i2 = next(i for i, (d, _, _) in enumerate(pairs) if d == 2)
    assert any(d == 3 for d, _, _ in pairs)
    A0, B0 = host[i2]
    en = A0[1].copy()
    en[0, 0] = len(A0[0]) + 7
    bad = list(host)
    bad[i2] = ((A0[0], en), B0)
    with pytest.raises(lsm.LsmError) as e:
        gpu_ctx.supermesh_batched(bad)
    assert e.value.status == 1
    t, nc, ni = gpu_ctx.supermesh_batched(host)
    for i, (dim, A, B) in enumerate(pairs):
        st, _ = gpu_ctx.supermesh(A, B)
        assert nc[i] == st.n_candidates and ni[i] == st.n_intersecting
        assert abs(t[i] - 1.0) <= 1e-12


def test_batched_device_inputs_and_empty_mesh(gpu_ctx):
    torch = pytest.importorskip("torch")
    pairs = M.batched_pairs(8, seed=26, emin=1e2, emax=1e3)
    host = [(A, B) for _, A, B in pairs]
    # one pair with an empty target mesh
    A0, B0 = host[1]
    host[1] = ((A0[0], A0[1][:0]), B0)
    t_ref, nc_ref, ni_ref = gpu_ctx.supermesh_batched(host)
    assert nc_ref[1] == 0 and t_ref[1] == 0.0
    dev = torch.device("cuda:0")
    tdev = [tuple((torch.from_numpy(np.ascontiguousarray(x[0])).to(dev), torch.from_numpy(np.ascontiguousarray(x[1])).to(dev))
                  for x in pr) for pr in host]
    torch.cuda.synchronize()
    t, nc, ni = gpu_ctx.supermesh_batched(tdev, on_device=True)
    assert np.array_equal(nc, nc_ref) and np.array_equal(ni, ni_ref) and np.array_equal(t, t_ref)


def _with_degenerate(dim, mesh, seed, count=40):
    """The mesh plus `count` zero-measure elements over its nodes: half with
    a repeated node, half flat (the last node replaced by a new node at the
    midpoint of the first two)."""
    pos, en = mesh
    rng = np.random.default_rng(seed)
    extra = en[rng.choice(len(en), count, replace=False)].copy()
    h = count // 2
    extra[:h, 1] = extra[:h, 0]
    mid = 0.5 * (pos[extra[h:, 0]] + pos[extra[h:, 1]])
    extra[h:, -1] = np.arange(len(pos), len(pos) + len(mid))
    return np.vstack([pos, mid]), np.vstack([en, extra]).astype(en.dtype)


@pytest.mark.parametrize("name", ["small2d_9x11", "small3d_5x6"])
def test_identical_and_degenerate_meshes(gpu_ctx, oracle_mod, name):
    """A mesh against itself (every element meets its copy exactly, its
    neighbours along shared faces), and meshes with zero-measure elements
    (repeated or collinear/coplanar nodes: NaN planes and zero tolerances)
    on either side: per-pair results equal the oracle's."""
    dim, A, B = M.config_meshes(name)
    check_pipeline(gpu_ctx, oracle_mod, dim, A, A, domain=1.0)
    Ad, Bd = _with_degenerate(dim, A, 3), _with_degenerate(dim, B, 4)
    check_pipeline(gpu_ctx, oracle_mod, dim, Ad, B)
    check_pipeline(gpu_ctx, oracle_mod, dim, A, Bd)
    check_pipeline(gpu_ctx, oracle_mod, dim, Ad, Bd)
    # the supermesh's simplices of the degenerate pairs too
    st, off, el, pa, pb = gpu_ctx.supermesh_elements(Ad, Bd)
    ip, ind = gpu_ctx.get_candidates(len(Ad[1]), st.n_candidates)
    rws = np.repeat(np.arange(len(ip) - 1), np.diff(ip))
    for k in range(st.n_candidates):
        ea, eb = Ad[0][Ad[1][rws[k]]], Bd[0][Bd[1][ind[k]]]
        ref = oracle_mod.intersect_tris(ea, eb) if dim == 2 else oracle_mod.intersect_tets(ea, eb)
        assert np.array_equal(el[off[k]:off[k + 1]], np.asarray(ref).reshape((-1,) + el.shape[1:])), k


@pytest.mark.parametrize("name", ["small2d_3x4", "small3d_2x3"])
def test_empty_meshes_through_every_entry(gpu_ctx, name):
    """An empty A (or B) through the supermesh, its simplices, the P1-P1
    product and the per-candidate outputs: no candidates, zero results, no
    error; the context then serves a normal call."""
    dim, A, B = M.config_meshes(name)
    loc = dim + 1
    emptyA = (A[0], np.zeros((0, loc), dtype=A[1].dtype))
    emptyB = (B[0], np.zeros((0, loc), dtype=B[1].dtype))
    for X, Y in ((emptyA, B), (A, emptyB), (emptyA, emptyB)):
        st, off, el, pa, pb = gpu_ctx.supermesh_elements(X, Y)
        assert st.n_candidates == 0 and len(el) == 0 and np.array_equal(off, [0])
        val, blocks = gpu_ctx.p1_mass(X, Y, X[0][:, 0], Y[0][:, 1], want_blocks=True)
        assert val == 0.0 and len(blocks) == 0
        out = {"elem_measure": np.zeros(len(X[1])), "ind_ptr": np.zeros(len(X[1]) + 1, dtype=np.int64),
               "indices": np.zeros(1, dtype=np.int64), "pair_measure": np.zeros(1),
               "pair_n_out": np.zeros(1, dtype=np.int32), "capacity": 0}
        st2, n = gpu_ctx.supermesh_out(X, Y, out)
        assert n == 0 and st2.total_measure == 0.0 and (out["ind_ptr"] == 0).all()
    m, k, _ = gpu_ctx.intersect_pairs(dim, np.zeros((0, loc, dim)), np.zeros((0, loc, dim)))
    assert len(m) == 0 and len(k) == 0
    st, _ = gpu_ctx.supermesh(A, B)
    assert abs(st.total_measure - 1.0) <= REL_TOL
