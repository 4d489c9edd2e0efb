"""libsupermesh_gpu_supermesh_elements: the supermesh's simplices for every
candidate pair, in the get_output CSR order and, within a pair, the order of
intersect_tris_real / intersect_tets_real (C_bindings.F90:152-174).  Checked
against the oracle's per-pair intersection bit for bit, with the parents,
the counts of the narrow phase and the capacity contract, for host and
device outputs."""
import numpy as np
import pytest

import libsupermesh_b200 as lsm
from libsupermesh_b200 import meshes as M

pytestmark = pytest.mark.gpu


def _check_against_oracle(ctx, oracle_mod, dim, A, B, sample=None):
    st, off, el, pa, pb = ctx.supermesh_elements(A, B)
    nc = st.n_candidates
    ip, ind = ctx.get_candidates(len(A[1]), nc)
    assert len(off) == nc + 1 and off[0] == 0 and off[-1] == len(el) == st.n_out_simplices
    rows = np.repeat(np.arange(len(ip) - 1), np.diff(ip))
    ks = range(nc) if sample is None else sample
    for k in ks:
        a, b = rows[k], ind[k]
        ea, eb = A[0][A[1][a]], B[0][B[1][b]]
        ref = oracle_mod.intersect_tris(ea, eb) if dim == 2 else oracle_mod.intersect_tets(ea, eb)
        got = el[off[k]:off[k + 1]]
        assert len(got) == len(ref), k
        assert np.array_equal(got, np.asarray(ref).reshape(got.shape)), k
        assert (pa[off[k]:off[k + 1]] == a).all() and (pb[off[k]:off[k + 1]] == b).all(), k
    return st, off, el


@pytest.mark.parametrize("name", ["small3d_6x7", "small3d_12x3", "small3d_3x11", "small2d_12x17", "small2d_40x9"])
def test_elements_match_oracle(gpu_ctx, oracle_mod, name):
    """Every candidate's simplices equal the oracle's intersection of the
    pair; 12x3 puts most of A's tets inside one of B's, 3x11 the reverse."""
    dim, A, B = M.config_meshes(name)
    st, off, el = _check_against_oracle(gpu_ctx, oracle_mod, dim, A, B)
    # the counts are the narrow phase's
    pm, pn = gpu_ctx.pair_results(st.n_candidates)
    assert np.array_equal(np.diff(off), pn)
    st2, _ = gpu_ctx.supermesh(A, B)
    assert st2.as_dict() == st.as_dict()


def test_elements_large_workload_sampled(gpu_ctx, oracle_mod):
    """tet3d_27x32 (10M candidates): a sample of candidates against the
    oracle, counts against the narrow phase, the volumes' sum against the
    supermesh's total."""
    dim, A, B = M.config_meshes("tet3d_27x32")
    rng = np.random.default_rng(3)
    st0, _ = gpu_ctx.supermesh(A, B)
    sample = np.sort(rng.choice(st0.n_candidates, 3000, replace=False))
    st, off, el = _check_against_oracle(gpu_ctx, oracle_mod, dim, A, B, sample)
    assert st.as_dict() == st0.as_dict()
    v = el.reshape(-1, 4, 3)
    e1, e2, e3 = v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]
    vol = np.abs(np.einsum("ij,ij->i", e1, np.cross(e2, e3))) / 6.0
    assert abs(vol.sum() - 1.0) < 1e-9


def test_elements_device_outputs_and_capacity(gpu_ctx):
    torch = pytest.importorskip("torch")
    dim, A, B = M.config_meshes("small3d_8x9")
    st, off, el, pa, pb = gpu_ctx.supermesh_elements(A, B)
    tA = tuple(torch.from_numpy(x).cuda() for x in A)
    tB = tuple(torch.from_numpy(x).cuda() for x in B)
    nc, ne = st.n_candidates, len(el)
    small = {"elems": torch.zeros((ne - 1, 4, 3), dtype=torch.float64, device="cuda"),
             "elem_capacity": ne - 1}
    with pytest.raises(lsm.LsmError) as ei:
        gpu_ctx.supermesh_elements_device(tA, tB, small)
    assert ei.value.status == 3 and small["n_elements"] == ne and small["n_candidates"] == nc
    out = {"elem_offset": torch.zeros(nc + 1, dtype=torch.int64, device="cuda"),
           "elems": torch.zeros((ne, 4, 3), dtype=torch.float64, device="cuda"),
           "parent_a": torch.zeros(ne, dtype=torch.int64, device="cuda"),
           "parent_b": torch.zeros(ne, dtype=torch.int64, device="cuda"),
           "cand_capacity": nc, "elem_capacity": ne}
    st2, nc2, ne2 = gpu_ctx.supermesh_elements_device(tA, tB, out)
    torch.cuda.synchronize()
    assert (nc2, ne2) == (nc, ne) and st2.as_dict() == st.as_dict()
    assert np.array_equal(out["elem_offset"].cpu().numpy(), off)
    assert np.array_equal(out["elems"].cpu().numpy(), el)
    assert np.array_equal(out["parent_a"].cpu().numpy(), pa)
    assert np.array_equal(out["parent_b"].cpu().numpy(), pb)
