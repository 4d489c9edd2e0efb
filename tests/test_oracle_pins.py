"""Pins the CPU oracle to libsupermesh's own known answers and fixtures.

Every expected value below is taken from the reference's test suite
(paths within firedrakeproject/libsupermesh); the meshes are the reference's
fixtures (tests/golden/ref_meshes.npz).  Float comparisons use the
reference's fequals tolerance 100*max(eps, spacing(a), spacing(b))
(src/Unittest_Tools.F90:179-195).
"""
import numpy as np
import pytest


def _narrow_total(oracle, dim, A, B):
    ip, ind = oracle.tree_finder(dim, A, B)
    pm, pn, em, st = oracle.narrow(dim, A, B, ip, ind)
    return ip, ind, pm, pn, em, st


def test_tri_intersector_area_half(oracle_mod, ref_meshes):
    # src/tests/test_tri_intersector.F90:84-104: total area 0.5
    A, B = ref_meshes("triangle_0_01"), ref_meshes("square_0_01")
    *_, st = _narrow_total(oracle_mod, 2, A, B)
    assert oracle_mod.fequals(st.total, 0.5)


def test_tet_intersector_volume_third(oracle_mod, ref_meshes):
    # src/tests/test_tet_intersector.F90:84-104: Kahan total volume 1/3
    A, B = ref_meshes("pyramid_0_05"), ref_meshes("cube_0_05")
    *_, st = _narrow_total(oracle_mod, 3, A, B)
    assert oracle_mod.fequals(st.total, 1.0 / 3.0)


@pytest.mark.parametrize("dim,na,nb", [(2, "square.1", "square.2"), (3, "cube.1", "cube.2")])
def test_completeness(oracle_mod, ref_meshes, dim, na, nb):
    # src/tests/test_intersection_finder_completeness_{2d,3d}.F90:95-136:
    # map_ba from the tree finder; for every B element the clipped measure
    # summed over its candidates equals its own measure.
    MA, MB = ref_meshes(na), ref_meshes(nb)
    ip, ind = oracle_mod.tree_finder(dim, MB, MA)
    pm, pn, em, st = oracle_mod.narrow(dim, MB, MA, ip, ind)
    for b in range(len(ip) - 1):
        v = MB[0][MB[1][b]]
        own = oracle_mod.triangle_area(v) if dim == 2 else oracle_mod.tetrahedron_volume(v)
        assert oracle_mod.fequals(own, em[b]), (b, own, em[b])


@pytest.mark.parametrize("dim,na,nb", [(2, "square.1", "square.2"), (3, "cube.1", "cube.2"),
                                       (2, "triangle_0_01", "square_0_01")])
def test_tree_equals_brute_force(oracle_mod, ref_meshes, dim, na, nb):
    # The quadtree/octree candidate set equals the strict-AABB brute-force set
    # (Intersection_Finder.F90:989-1077); both run on the reference fixtures.
    A, B = ref_meshes(na), ref_meshes(nb)
    ip, ind = oracle_mod.tree_finder(dim, A, B)
    bip, bind = oracle_mod.brute_force_finder(dim, A, B)
    assert np.array_equal(ip, bip)
    for a in range(len(ip) - 1):
        assert sorted(ind[ip[a]:ip[a + 1]]) == sorted(bind[bip[a]:bip[a + 1]])


def test_finder_tiny_sets(oracle_mod, ref_meshes):
    # src/tests/test_intersection_finder_2d.F90:77-118 and _3d.F90:76-90
    t1, t2, tet = ref_meshes("triangle.1"), ref_meshes("triangle.2"), ref_meshes("tet")
    assert list(oracle_mod.tree_finder(2, t1, t1)[1]) == [0]
    assert sorted(oracle_mod.tree_finder(2, t1, t2)[1]) == [0, 1, 2]
    ip, ind = oracle_mod.tree_finder(2, t2, t2)
    for i in range(3):
        assert i in set(ind[ip[i]:ip[i + 1]])
    assert list(oracle_mod.tree_finder(3, tet, tet)[1]) == [0]


def test_p1_inner_product_2d(oracle_mod, ref_meshes):
    # src/tests/test_parallel_p1_inner_product_2d.F90:42-43, run serially on
    # the unpartitioned meshes: area 0.5, integral of x_A * y_B 8.33...e-2
    A, B = ref_meshes("triangle_0_01"), ref_meshes("square_0_01")
    ip, ind = oracle_mod.tree_finder(2, A, B)
    integral, measure, _ = oracle_mod.p1_mass(2, A, B, ip, ind, A[0][:, 0], B[0][:, 1])
    assert oracle_mod.fequals(measure, 0.5)
    assert oracle_mod.fequals(integral, 8.3333333333333398e-2)


def test_p1_inner_product_3d(oracle_mod, ref_meshes):
    # src/tests/test_parallel_p1_inner_product_3d.F90:44-45: volume 1/3,
    # integral of (x+z)_A * y_B 1.2499999999999989e-1
    A, B = ref_meshes("pyramid_0_05"), ref_meshes("cube_0_05")
    ip, ind = oracle_mod.tree_finder(3, A, B)
    integral, measure, _ = oracle_mod.p1_mass(3, A, B, ip, ind, A[0][:, 0] + A[0][:, 2], B[0][:, 1])
    assert oracle_mod.fequals(measure, 3.3333333333333331e2 / 1.0e3)
    assert oracle_mod.fequals(integral, 1.2499999999999989e4 / 1.0e5)


def test_element_intersector_simplices(oracle_mod, ref_meshes):
    # src/tests/test_element_intersector.F90:102-129 (tri-tri on square.1/2)
    # and the tet-tet case on cube.1/2: total measure 1.
    for dim, na, nb in [(2, "square.1", "square.2"), (3, "cube.1", "cube.2")]:
        A, B = ref_meshes(na), ref_meshes(nb)
        *_, st = _narrow_total(oracle_mod, dim, A, B)
        assert oracle_mod.fequals(st.total, 1.0)


def test_spacing_and_norm2(oracle_mod):
    sp = oracle_mod.spacing
    assert sp(1.0) == 2.0 ** -52
    assert sp(1.5) == 2.0 ** -52
    assert sp(0.5) == 2.0 ** -53
    assert sp(0.0) == 2.0 ** -1022
    assert sp(2.0 ** -1030) == 2.0 ** -1022
    assert sp(-3.0) == 2.0 ** -51


def test_single_pair_cases(oracle_mod):
    # identical triangles: one output of the same area
    t = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]])
    out = oracle_mod.intersect_tris(t, t)
    assert abs(sum(oracle_mod.triangle_area(o) for o in out) - 0.5) < 1e-15
    # boxes touching along an edge: empty
    t2 = np.array([[1.0, 0.0], [2.0, 0.0], [1.0, 1.0]])
    assert len(oracle_mod.intersect_tris(t, t2)) == 0
    # unit tet with itself
    T = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
    out = oracle_mod.intersect_tets(T, T)
    assert abs(sum(oracle_mod.tetrahedron_volume(o) for o in out) - 1.0 / 6.0) < 1e-15


# -- mixed element pairs and 1D entries --------------------------------------

def _mixed_total(oracle, dim, A, B, swap=False):
    """Sum of output measures over the strict-AABB candidates, clipping each
    simplex of one mesh by the quad/hex of the other (Supermesh.F90:176-194
    passes (simplex, box element) whichever side the simplex is on)."""
    ip, ind = oracle.brute_force_finder(dim, A, B)
    total = 0.0
    for a in range(len(ip) - 1):
        ea = A[0][A[1][a]]
        for b in ind[ip[a]:ip[a + 1]]:
            eb = B[0][B[1][b]]
            s, q = (eb, ea) if swap else (ea, eb)
            if dim == 2:
                for t in oracle.intersect_tri_quad(s, q):
                    total += oracle.triangle_area(t)
            else:
                for t in oracle.intersect_tet_hex(s, q):
                    total += oracle.tetrahedron_volume(t)
    return total


def test_tri_quad_area_one(oracle_mod, ref_meshes):
    # src/tests/test_element_intersector.F90:134-158: tri-quad, total 1
    assert oracle_mod.fequals(_mixed_total(oracle_mod, 2, ref_meshes("square.1"), ref_meshes("square.4")), 1.0)


def test_quad_tri_area_one(oracle_mod, ref_meshes):
    # src/tests/test_element_intersector.F90:163-187: quad-tri, total 1
    assert oracle_mod.fequals(
        _mixed_total(oracle_mod, 2, ref_meshes("square.3"), ref_meshes("square.2"), swap=True), 1.0)


def test_tet_hex_volume_half(oracle_mod, ref_meshes):
    # src/tests/test_element_intersector.F90:250-274: tet-hex, total 0.5
    assert oracle_mod.fequals(_mixed_total(oracle_mod, 3, ref_meshes("cube.1"), ref_meshes("cube.3")), 0.5)


def test_hex_tet_volume_half(oracle_mod, ref_meshes):
    # src/tests/test_element_intersector.F90:279-303: hex-tet, total 0.5
    assert oracle_mod.fequals(
        _mixed_total(oracle_mod, 3, ref_meshes("cube.3"), ref_meshes("cube.2"), swap=True), 0.5)


def _same_type_total(oracle, dim, A, B):
    ip, ind = oracle.brute_force_finder(dim, A, B)
    fn = oracle.intersect_quads if dim == 2 else oracle.intersect_hexes
    meas = oracle.triangle_area if dim == 2 else oracle.tetrahedron_volume
    total = 0.0
    for a in range(len(ip) - 1):
        for b in ind[ip[a]:ip[a + 1]]:
            for o in fn(A[0][A[1][a]], B[0][B[1][b]]):
                total += meas(o)
    return total


def test_quad_quad_area_one(oracle_mod, ref_meshes):
    # src/tests/test_element_intersector.F90:192-216: quad-quad, total 1
    assert oracle_mod.fequals(_same_type_total(oracle_mod, 2, ref_meshes("square.3"), ref_meshes("square.4")), 1.0)


def test_hex_hex_volume_half(oracle_mod, ref_meshes):
    # src/tests/test_element_intersector.F90:308-332: hex-hex, total 0.5
    assert oracle_mod.fequals(_same_type_total(oracle_mod, 3, ref_meshes("cube.3"), ref_meshes("cube.4")), 0.5)


def _interval_total(oracle, A, B, ip, ind):
    total = 0.0
    for a in range(len(ip) - 1):
        for b in ind[ip[a]:ip[a + 1]]:
            c = oracle.intersect_intervals(A[0][A[1][a], 0], B[0][B[1][b], 0])
            if c.size:
                total += oracle.interval_size(c)
    return total


@pytest.mark.parametrize("stable", [False, True])
def test_intervals_size_one(oracle_mod, ref_meshes, stable):
    # src/tests/test_interval_intersector.F90:84-99: total size 1 over the
    # 1D finder's candidates (line.1 vs line.2)
    A, B = ref_meshes("line.1"), ref_meshes("line.2")
    ip, ind = oracle_mod.sort_finder_1d(A, B, stable=stable)
    assert oracle_mod.fequals(_interval_total(oracle_mod, A, B, ip, ind), 1.0)


@pytest.mark.parametrize("stable", [False, True])
def test_sort_finder_completeness_1d(oracle_mod, ref_meshes, stable):
    # src/tests/test_intersection_finder_completeness_1d.F90:94-121: map_ba
    # from the sort finder; every B interval is covered by its candidates.
    A, B = ref_meshes("line.1"), ref_meshes("line.2")
    ip, ind = oracle_mod.sort_finder_1d(B, A, stable=stable)
    for b in range(len(ip) - 1):
        own = oracle_mod.interval_size(B[0][B[1][b], 0])
        got = 0.0
        for a in ind[ip[b]:ip[b + 1]]:
            c = oracle_mod.intersect_intervals(A[0][A[1][a], 0], B[0][B[1][b], 0])
            if c.size:
                got += oracle_mod.interval_size(c)
        assert oracle_mod.fequals(own, got), b


def test_sort_finder_leaf_sort_on_shuffled_mesh(oracle_mod, ref_meshes):
    # The reference's merge sort orders blocks of <= 4 elements with a
    # selection loop (Intersection_Finder.F90:871-879) that is a permutation
    # only for blocks already in order.  On a shuffled numbering the faithful
    # restatement repeats and drops elements, so rows go missing; the stable
    # sort used by the GPU library keeps the finder complete.
    A, B = ref_meshes("line.1"), ref_meshes("line.2")
    perm = np.random.default_rng(0).permutation(B[1].shape[0])
    Bs = (B[0], B[1][perm])
    faithful = oracle_mod.sort_finder_1d(Bs, A, stable=False)
    stable = oracle_mod.sort_finder_1d(Bs, A, stable=True)
    brute = [sorted(a for a in range(A[1].shape[0])
                    if max(A[0][A[1][a], 0]) > min(Bs[0][Bs[1][b], 0])
                    and min(A[0][A[1][a], 0]) < max(Bs[0][Bs[1][b], 0])) for b in range(Bs[1].shape[0])]
    rows = lambda r: [sorted(r[1][r[0][b]:r[0][b + 1]]) for b in range(len(r[0]) - 1)]
    assert rows(stable) == brute
    assert rows(faithful) != brute


def test_interval_basics(oracle_mod):
    # Interval_Intersection.F90: |b - a|, open-overlap test, tolerance
    # 10*min(spacing(|a|), spacing(|b|))
    assert oracle_mod.interval_size([0.75, 0.25]) == 0.5
    assert np.array_equal(oracle_mod.intersect_intervals([0.0, 1.0], [1.0, 0.5]), [0.5, 1.0])
    assert oracle_mod.intersect_intervals([0.0, 1.0], [1.0, 2.0]).size == 0
    assert oracle_mod.intersect_intervals([0.0, 1.0], [1.0 - 2.0 ** -50, 2.0]).size == 0


def _p2_fields(A, B):
    from libsupermesh_b200 import meshes as M

    e2a, na, eda = M.p2_space(A[1])
    e2b, nb, edb = M.p2_space(B[1])
    fa = M.p1_to_p2(A[0][:, 0], na, eda) * M.p1_to_p2(A[0][:, 1], na, eda)  # x y on A
    fb = M.p1_to_p2(B[0][:, 0], nb, edb) ** 2                               # x^2 on B
    return e2a, fa, e2b, fb


def test_p2_inner_product_known_answer(oracle_mod, ref_meshes):
    # src/tests/test_parallel_p2_inner_product_2d.F90:45-46, :151-152:
    # area 0.5, integral 2.7083333333333272e-2 (run on the unpartitioned
    # meshes: the supermesh of the whole domain is the union of the ranks')
    A, B = ref_meshes("triangle_0_01"), ref_meshes("square_0_01")
    e2a, fa, e2b, fb = _p2_fields(A, B)
    ip, ind = oracle_mod.tree_finder(2, A, B)
    integral, area, _ = oracle_mod.p2_inner_product(A, B, ip, ind, e2a, fa, e2b, fb)
    assert oracle_mod.fequals(area, 0.5)
    assert oracle_mod.fequals(integral, 2.7083333333333272e-2)
