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
