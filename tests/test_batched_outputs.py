"""Per-pair outputs of the batched entry (libsupermesh_gpu_supermesh_batched_ex):
for every mesh pair of a batch, the CSR of the candidate search in the
get_output layout (C_bindings.F90:377-391) and each candidate's measure and
output count, compared with the oracle restatement of the reference on the
batched256 workload (256 mesh pairs of 1e3-1e5 elements, half 2D, half 3D),
and with the single-pair entry on small batches; plus the capacity contract
(LSM_ERROR_CAPACITY with the counts a retry needs) and device-memory outputs.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import libsupermesh_b200 as lsm
from libsupermesh_b200 import meshes as M

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12


def _table(ip, ind, *vals):
    """Candidates sorted by (row, B element) with their values."""
    r = np.repeat(np.arange(len(ip) - 1), np.diff(ip))
    o = np.lexsort((ind, r))
    return (r[o], np.asarray(ind)[o]) + tuple(np.asarray(v)[o] for v in vals)


def _pair_view(res, pairs, i):
    na = len(pairs[i][0][1])
    r0 = res["row_offset"][i]
    ip = res["ind_ptr"][r0:r0 + na + 1]
    c0, nc = res["cand_offset"][i], res["n_candidates"][i]
    sl = slice(c0, c0 + nc)
    return ip, res["indices"][sl], res["pair_measure"][sl], res["pair_n_out"][sl]


def _small_batch():
    names = ["small3d_5x6", "small2d_12x17", "small3d_7x6", "small2d_31x50", "small3d_4x9", "small2d_7x9"]
    return [M.config_meshes(n)[1:] for n in names]


def test_batched_pairs_match_single_pair_entry(gpu_ctx):
    pairs = _small_batch()
    res = gpu_ctx.supermesh_batched_pairs(pairs)
    assert res["total_candidates"][0] == res["n_candidates"][: len(pairs)].sum()
    for i, (A, B) in enumerate(pairs):
        st, _ = gpu_ctx.supermesh(A, B)
        ip1, ind1 = gpu_ctx.get_candidates(len(A[1]), st.n_candidates)
        pm1, pn1 = gpu_ctx.pair_results(st.n_candidates)
        ip, ind, pm, pn = _pair_view(res, pairs, i)
        assert res["n_candidates"][i] == st.n_candidates
        assert np.array_equal(ip, ip1)
        a = _table(ip, ind, pm, pn)
        b = _table(ip1, ind1, pm1, pn1)
        for x, y in zip(a, b):
            assert np.array_equal(x, y), i
        assert res["totals"][i] == st.total_measure
        assert res["n_intersecting"][i] == st.n_intersecting


def test_batched_capacity_contract(gpu_ctx):
    pairs = _small_batch()
    with pytest.raises(lsm.LsmError) as ei:
        gpu_ctx.supermesh_batched_pairs(pairs, capacity=10)
    assert ei.value.status == 3  # LSM_ERROR_CAPACITY
    full = gpu_ctx.supermesh_batched_pairs(pairs)  # sizes the retry from the counts
    need = int(full["n_candidates"][: len(pairs)].sum())
    exact = gpu_ctx.supermesh_batched_pairs(pairs, capacity=need)
    for k in ("ind_ptr", "indices", "pair_measure", "pair_n_out", "cand_offset", "totals"):
        assert np.array_equal(full[k][: len(exact[k])], exact[k][: len(full[k])]), k


def test_batched_device_outputs_equal_host_outputs(gpu_ctx):
    torch = pytest.importorskip("torch")
    pairs = _small_batch()
    host = gpu_ctx.supermesh_batched_pairs(pairs)
    dpairs = [tuple((torch.from_numpy(m[0]).cuda(), torch.from_numpy(m[1]).cuda()) for m in p) for p in pairs]
    dev = gpu_ctx.supermesh_batched_pairs(dpairs, capacity=int(host["total_candidates"][0]), on_device=True)
    n = int(host["total_candidates"][0])
    assert np.array_equal(dev["cand_offset"], host["cand_offset"])
    assert np.array_equal(dev["ind_ptr"].cpu().numpy(), host["ind_ptr"])
    assert np.array_equal(dev["indices"].cpu().numpy()[:n], host["indices"][:n])
    assert np.array_equal(dev["pair_measure"].cpu().numpy()[:n], host["pair_measure"][:n])
    assert np.array_equal(dev["pair_n_out"].cpu().numpy()[:n], host["pair_n_out"][:n])


def test_config_batched256_per_pair_vs_oracle(gpu_ctx, oracle_mod):
    """The batched256 workload (162M candidates) pair by pair against the
    oracle: each mesh pair's CSR offsets and row sets, per-candidate output
    counts (exact) and measures (1e-12 relative), and each pair's total."""
    pairs = M.batched_pairs(256, seed=6)
    meshes = [(A, B) for _, A, B in pairs]
    res = gpu_ctx.supermesh_batched_pairs(meshes)

    def check(i):
        dim, A, B = pairs[i]
        ip_o, ind_o = oracle_mod.tree_finder(dim, A, B)
        pm_o, pn_o, _, st_o = oracle_mod.narrow(dim, A, B, ip_o, ind_o)
        ip, ind, pm, pn = _pair_view(res, meshes, i)
        assert res["n_candidates"][i] == len(ind_o), i
        assert np.array_equal(ip, ip_o), i
        ro, bo, mo, no = _table(ip_o, ind_o, pm_o, pn_o)
        rg, bg, mg, ng = _table(ip, ind, pm, pn)
        assert np.array_equal(ro, rg) and np.array_equal(bo, bg), i
        assert np.array_equal(no, ng), i
        rel = np.abs(mg - mo) / np.maximum(np.abs(mo), 1e-300)
        assert rel.max(initial=0.0) <= REL_TOL, i
        assert abs(res["totals"][i] - st_o.total) <= REL_TOL, i
        assert abs(res["totals"][i] - 1.0) <= REL_TOL, i
        return len(ind_o)

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        counts = list(ex.map(check, range(len(pairs))))
    assert sum(counts) == res["total_candidates"][0] > 100_000_000


def test_batched_p1_blocks_match_single_pair_entry(gpu_ctx):
    """P1-P1 mass blocks through the batched entry equal the blocks of the
    single-pair P1 entry, candidate by candidate (matched by (row, B
    element): the two searches order each row's candidates differently)."""
    pairs = _small_batch()
    res = gpu_ctx.supermesh_batched_pairs(pairs, p1_blocks=True)
    for i, (A, B) in enumerate(pairs):
        loc = A[1].shape[1]
        _, blk1 = gpu_ctx.p1_mass(A, B, want_blocks=True)
        st, _ = gpu_ctx.supermesh(A, B)
        ip1, ind1 = gpu_ctx.get_candidates(len(A[1]), st.n_candidates)
        ip, ind, _, _ = _pair_view(res, pairs, i)
        nc = int(res["n_candidates"][i])
        o = int(res["p1_offset"][i])
        blk = res["p1_blocks"][o:o + nc * loc * loc].reshape(nc, loc * loc)
        a = _table(ip, ind, blk)
        b = _table(ip1, ind1, blk1.reshape(-1, loc * loc))
        for x, y in zip(a, b):
            assert np.array_equal(x, y), i


def test_batched_with_empty_meshes_and_empty_batch(gpu_ctx):
    """Mesh pairs with an empty side give no candidates and a zero total; an
    empty batch is a no-op."""
    _, A, B = M.config_meshes("small3d_5x6")
    _, A2, B2 = M.config_meshes("small2d_12x17")
    empty3 = (np.zeros((0, 3)), np.zeros((0, 4), dtype=A[1].dtype))
    empty2 = (np.zeros((0, 2)), np.zeros((0, 3), dtype=A2[1].dtype))
    pairs = [(A, B), (A, empty3), (empty3, B), (A2, empty2), (A2, B2)]
    res = gpu_ctx.supermesh_batched_pairs(pairs)
    nc = res["n_candidates"][: len(pairs)]
    assert nc[1] == nc[2] == nc[3] == 0 and nc[0] > 0 and nc[4] > 0
    assert res["totals"][1] == res["totals"][2] == res["totals"][3] == 0.0
    for i in (0, 4):
        assert abs(res["totals"][i] - 1.0) <= REL_TOL
    assert np.all(res["ind_ptr"][res["row_offset"][1]:res["row_offset"][1] + len(A[1]) + 1] == 0)
    empty = gpu_ctx.supermesh_batched_pairs([])
    assert empty["total_candidates"][0] == 0
