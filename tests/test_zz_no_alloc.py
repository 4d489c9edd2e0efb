"""The allocation-free entry point libsupermesh_gpu_intersect_tets_noalloc.

It is meant for callers that cannot let the library allocate device memory
(memory owned by another pool allocator; loops that cannot afford cudaFree's
implicit device synchronisation).  Checked here through the C-ABI against the
context-based entry libsupermesh_gpu_intersect_pairs on the same device
inputs, on two calls in a row (the fixed scratch array keeps the previous
call's contents, so the second call checks that the counters are cleared),
plus the size limit.  This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import libsupermesh_b200 as lsm

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # same bar as the other parity tests


def _pairs(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.random((n, 4, 3))
    b = rng.random((n, 4, 3)) * 0.8 + 0.1
    b[: n // 8] = a[: n // 8]                    # identical tets
    b[n // 8: n // 4, 0] = a[n // 8: n // 4, 0]  # shared vertex
    return a, b


def _noalloc(L, n, da, db, dm, dk, stream=None):
    total = ctypes.c_double(0.0)
    st = L.libsupermesh_gpu_intersect_tets_noalloc(ctypes.c_int64(n), ctypes.c_void_p(da), ctypes.c_void_p(db),
                                                   ctypes.c_void_p(dm), ctypes.c_void_p(dk), ctypes.byref(total),
                                                   ctypes.c_void_p(stream))
    return st, total.value


def test_noalloc_matches_context_entry_twice():
    torch = pytest.importorskip("torch")
    L = lsm.load()
    L.libsupermesh_gpu_intersect_tets_noalloc.restype = ctypes.c_int
    dev = torch.device("cuda:0")
    ctx = lsm.Context(0)
    try:
        for call, (n, seed) in enumerate([(20000, 11), (7000, 12)]):
            a, b = _pairs(n, seed)
            ta = torch.from_numpy(a).to(dev)
            tb = torch.from_numpy(b).to(dev)
            # existing entry point, device inputs
            m_ref = torch.zeros(n, dtype=torch.float64, device=dev)
            k_ref = torch.zeros(n, dtype=torch.int32, device=dev)
            torch.cuda.synchronize()
            st = ctx.lib.libsupermesh_gpu_intersect_pairs(ctx._h, 3, n, ta.data_ptr(), tb.data_ptr(),
                                                          m_ref.data_ptr(), k_ref.data_ptr(), None, 1, None)
            assert st == 0
            # allocation-free entry point
            m = torch.full((n,), -1.0, dtype=torch.float64, device=dev)
            k = torch.full((n,), -1, dtype=torch.int32, device=dev)
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info(0)[0]
            st, total = _noalloc(L, n, ta.data_ptr(), tb.data_ptr(), m.data_ptr(), k.data_ptr())
            torch.cuda.synchronize()
            free_after = torch.cuda.mem_get_info(0)[0]
            assert st == 0
            if call > 0:  # after the first call's one-time set-up nothing is allocated
                assert free_after == free_before
            mr, kr = m_ref.cpu().numpy(), k_ref.cpu().numpy()
            mn, kn = m.cpu().numpy(), k.cpu().numpy()
            assert np.array_equal(kn, kr)
            rel = np.abs(mn - mr) / np.maximum(np.abs(mr), 1e-300)
            assert rel.max() <= REL_TOL
            assert abs(total - float(np.sum(mr))) <= REL_TOL * max(1.0, abs(float(np.sum(mr))))
            assert (kr > 0).sum() > n // 8  # the identical pairs at least
    finally:
        ctx.close()


def test_noalloc_rejects_oversize():
    L = lsm.load()
    L.libsupermesh_gpu_intersect_tets_noalloc.restype = ctypes.c_int
    st, _ = _noalloc(L, 32768 + 1, 0, 0, 0, 0)
    assert st == 3  # LSM_ERROR_CAPACITY


def test_noalloc_matches_oracle():
    """Pair by pair against the CPU oracle (the reference algorithm restated):
    output counts equal, and each measure equal to the oracle's sum of its
    output tets' volumes within the parity tolerance."""
    torch = pytest.importorskip("torch")
    import oracle

    L = lsm.load()
    L.libsupermesh_gpu_intersect_tets_noalloc.restype = ctypes.c_int
    n = 600
    a, b = _pairs(n, 13)
    dev = torch.device("cuda:0")
    ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    m = torch.zeros(n, dtype=torch.float64, device=dev)
    k = torch.zeros(n, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    st, total = _noalloc(L, n, ta.data_ptr(), tb.data_ptr(), m.data_ptr(), k.data_ptr())
    assert st == 0
    mn, kn = m.cpu().numpy(), k.cpu().numpy()
    want = np.zeros(n)
    for i in range(n):
        ref = oracle.intersect_tets(a[i], b[i])
        assert kn[i] == len(ref), i
        want[i] = sum(oracle.tetrahedron_volume(o) for o in ref)
    rel = np.abs(mn - want) / np.maximum(np.abs(want), 1e-300)
    assert rel.max() <= REL_TOL
    assert abs(total - oracle.kahan_sum(want)) <= REL_TOL * max(1.0, abs(total))


def test_noalloc_refuses_misaligned_pairs():
    """Tetrahedra are loaded 16 bytes at a time: an array that starts on an
    8-byte boundary only is refused on the host, before any launch."""
    torch = pytest.importorskip("torch")
    L = lsm.load()
    L.libsupermesh_gpu_intersect_tets_noalloc.restype = ctypes.c_int
    n = 64
    a, b = _pairs(n, 14)
    dev = torch.device("cuda:0")
    buf = torch.zeros(2 * n * 12 + 2, dtype=torch.float64, device=dev)
    m = torch.zeros(n, dtype=torch.float64, device=dev)
    k = torch.zeros(n, dtype=torch.int32, device=dev)
    base = buf.data_ptr()
    assert base % 16 == 0
    st, _ = _noalloc(L, n, base + 8, base + 8 + n * 96 + 8, m.data_ptr(), k.data_ptr())
    assert st == 1  # LSM_ERROR_INVALID_ARGUMENT
    # aligned views of the same buffer work
    buf[: n * 12] = torch.from_numpy(a.reshape(-1))
    buf[n * 12: 2 * n * 12] = torch.from_numpy(b.reshape(-1))
    torch.cuda.synchronize()
    st, _ = _noalloc(L, n, base, base + n * 96, m.data_ptr(), k.data_ptr())
    assert st == 0
