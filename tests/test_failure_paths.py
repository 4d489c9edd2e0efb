"""Failure detection of the GPU extension, with every failure made on the
host side: no test here faults, traps or hangs the GPU.

The reference has one failure mode, a fatal abort (libsupermesh_abort,
src/Debug.F90:78-94).  The GPU extension instead returns an lsm_status and
keeps the context usable; these tests make each failure happen and then
check that the next call on the same context gives the right answer:

  * a device pointer that the kernels could not load from (a tetrahedron
    array off a 16-byte boundary): refused on the host before any launch;
  * a device allocation that fails (option fail_alloc_after makes the n-th
    allocation report out-of-memory without calling cudaMalloc);
  * a bounded device wait that runs out (option sort_stall_block keeps one
    block of the tree build's radix sort from publishing its counts, so the
    look-back waits of the blocks after it give up after sort_spin_limit
    polls; the kernels after the sort then read a repaired permutation).
"""
import ctypes

import numpy as np
import pytest

import libsupermesh_b200 as lsm
from libsupermesh_b200 import meshes as M

pytestmark = pytest.mark.gpu

LSM_ERROR_INVALID_ARGUMENT = 1
LSM_ERROR_OUT_OF_MEMORY = 2
LSM_ERROR_TIMEOUT = 4


def _tet_pairs(n, seed=0):
    rng = np.random.default_rng(seed)
    base = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)
    a = base[None] + rng.uniform(-0.3, 0.3, (n, 4, 3))
    b = base[None] * 0.9 + rng.uniform(-0.3, 0.3, (n, 4, 3)) + 0.1
    return a, b


def test_misaligned_device_tets_are_refused(gpu_ctx):
    torch = pytest.importorskip("torch")
    a, b = _tet_pairs(64)
    n = len(a)
    # one spare double in front: the view starting at element 1 is 8-byte
    # aligned but not 16-byte aligned
    da = torch.zeros(n * 12 + 1, dtype=torch.float64, device="cuda")
    db = torch.zeros(n * 12 + 1, dtype=torch.float64, device="cuda")
    da[1:] = torch.from_numpy(a.reshape(-1))
    db[1:] = torch.from_numpy(b.reshape(-1))
    meas = torch.zeros(n, dtype=torch.float64, device="cuda")
    nout = torch.zeros(n, dtype=torch.int32, device="cuda")
    L = gpu_ctx.lib
    odd_a, odd_b = da.data_ptr() + 8, db.data_ptr() + 8
    assert odd_a % 16 == 8
    st = L.libsupermesh_gpu_intersect_pairs(gpu_ctx._h, 3, n, ctypes.c_void_p(odd_a), ctypes.c_void_p(odd_b),
                                            ctypes.c_void_p(meas.data_ptr()), ctypes.c_void_p(nout.data_ptr()),
                                            None, 1, None)
    assert st == LSM_ERROR_INVALID_ARGUMENT
    assert b"16-byte" in L.libsupermesh_gpu_last_error(gpu_ctx._h)
    hexes = torch.zeros(n * 24 + 2, dtype=torch.float64, device="cuda")
    st = L.libsupermesh_gpu_intersect_pairs_mixed(gpu_ctx._h, lsm.PAIR_TET_HEX, n, ctypes.c_void_p(odd_a),
                                                  ctypes.c_void_p(hexes.data_ptr()),
                                                  ctypes.c_void_p(meas.data_ptr()),
                                                  ctypes.c_void_p(nout.data_ptr()), None, 1, None)
    assert st == LSM_ERROR_INVALID_ARGUMENT
    # aligned inputs, output tets at an odd double offset (16-byte stores)
    elems = torch.zeros(n * 81 * 12 + 2, dtype=torch.float64, device="cuda")
    st = L.libsupermesh_gpu_intersect_pairs(gpu_ctx._h, 3, n, ctypes.c_void_p(da.data_ptr()),
                                            ctypes.c_void_p(db.data_ptr()), ctypes.c_void_p(meas.data_ptr()),
                                            ctypes.c_void_p(nout.data_ptr()), ctypes.c_void_p(elems.data_ptr() + 8),
                                            1, None)
    assert st == LSM_ERROR_INVALID_ARGUMENT
    # the context is untouched: the aligned copies give the host results
    ga = da[1:].clone()
    gb = db[1:].clone()
    st = L.libsupermesh_gpu_intersect_pairs(gpu_ctx._h, 3, n, ctypes.c_void_p(ga.data_ptr()),
                                            ctypes.c_void_p(gb.data_ptr()), ctypes.c_void_p(meas.data_ptr()),
                                            ctypes.c_void_p(nout.data_ptr()), None, 1, None)
    assert st == 0
    torch.cuda.synchronize()
    m_h, k_h, _ = gpu_ctx.intersect_pairs(3, a, b)
    assert np.array_equal(meas.cpu().numpy(), m_h) and np.array_equal(nout.cpu().numpy(), k_h)


def test_allocation_failure_reports_oom_and_context_recovers(oracle_mod):
    dim, A, B = M.config_meshes("small3d_5x6")
    ip, ind = oracle_mod.tree_finder(dim, A, B)
    _, _, _, st_o = oracle_mod.narrow(dim, A, B, ip, ind)
    for after in (0, 3, 9):
        with lsm.Context(0) as ctx:  # fresh context: every buffer must be allocated
            lsm.set_option("fail_alloc_after", after)
            try:
                with pytest.raises(lsm.LsmError) as ei:
                    ctx.supermesh(A, B)
            finally:
                lsm.set_option("fail_alloc_after", -1)
            assert ei.value.status == LSM_ERROR_OUT_OF_MEMORY
            assert "fail_alloc_after" in str(ei.value)
            st, _ = ctx.supermesh(A, B)
            assert st.n_candidates == len(ind)
            assert st.n_intersecting == st_o.n_intersecting
            assert abs(st.total_measure - st_o.total) <= 1e-12


@pytest.mark.parametrize("name", ["small3d_7x9", "small2d_31x50"])
def test_sort_wait_gives_up_with_timeout_and_context_recovers(gpu_ctx, name):
    dim, A, B = M.config_meshes(name)
    assert len(B[1]) > 2 * 2048  # at least three blocks of 2048 keys in the sort
    ref, _ = gpu_ctx.supermesh(A, B)
    lsm.set_option("sort_spin_limit", 2000)
    lsm.set_option("sort_stall_block", 1)
    try:
        with pytest.raises(lsm.LsmError) as ei:
            gpu_ctx.supermesh(A, B)
    finally:
        lsm.set_option("sort_stall_block", -1)
        lsm.set_option("sort_spin_limit", 1 << 22)
    assert ei.value.status == LSM_ERROR_TIMEOUT
    assert "look-back" in str(ei.value)
    st, _ = gpu_ctx.supermesh(A, B)
    assert st.n_candidates == ref.n_candidates
    assert st.total_measure == ref.total_measure
    assert st.n_out_simplices == ref.n_out_simplices


def test_sort_wait_gives_up_in_batched_search(gpu_ctx):
    pairs = [M.config_meshes(n)[1:] for n in ("small3d_7x9", "small3d_5x6")]
    ref = gpu_ctx.supermesh_batched(pairs)
    lsm.set_option("sort_spin_limit", 2000)
    lsm.set_option("sort_stall_block", 1)
    try:
        with pytest.raises(lsm.LsmError) as ei:
            gpu_ctx.supermesh_batched(pairs)
    finally:
        lsm.set_option("sort_stall_block", -1)
        lsm.set_option("sort_spin_limit", 1 << 22)
    assert ei.value.status == LSM_ERROR_TIMEOUT
    again = gpu_ctx.supermesh_batched(pairs)
    for x, y in zip(ref, again):
        assert np.array_equal(x, y)
