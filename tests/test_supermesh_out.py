"""libsupermesh_gpu_supermesh_out: one call returning the per-element
measures, the CSR (get_output layout) and the per-candidate measures and
counts, with the CSR copied while the candidates are clipped.  Checked
against the separate calls (supermesh, get_candidates, get_pair_results) and
the oracle, for host and device outputs, plus the capacity contract."""
import numpy as np
import pytest

import libsupermesh_b200 as lsm
from libsupermesh_b200 import meshes as M

pytestmark = pytest.mark.gpu


def _host_out(nel_a, cap):
    return {"elem_measure": np.zeros(nel_a), "ind_ptr": np.zeros(nel_a + 1, dtype=np.int64),
            "indices": np.zeros(max(cap, 1), dtype=np.int64), "pair_measure": np.zeros(max(cap, 1)),
            "pair_n_out": np.zeros(max(cap, 1), dtype=np.int32), "capacity": cap}


@pytest.mark.parametrize("name", ["small3d_9x7", "small2d_40x31", "tet3d_27x32"])
def test_supermesh_out_equals_separate_calls(gpu_ctx, oracle_mod, name):
    dim, A, B = M.config_meshes(name)
    st, em = gpu_ctx.supermesh(A, B, elem_measure=True)
    ip, ind = gpu_ctx.get_candidates(len(A[1]), st.n_candidates)
    pm, pn = gpu_ctx.pair_results(st.n_candidates)
    out = _host_out(len(A[1]), st.n_candidates)
    st2, n = gpu_ctx.supermesh_out(A, B, out)
    assert n == st.n_candidates and st2.as_dict() == st.as_dict()
    assert np.array_equal(out["elem_measure"], em)
    assert np.array_equal(out["ind_ptr"], ip)
    assert np.array_equal(out["indices"][:n], ind)
    assert np.array_equal(out["pair_measure"][:n], pm) and np.array_equal(out["pair_n_out"][:n], pn)
    if name.startswith("small"):
        ip_o, _ = oracle_mod.tree_finder(dim, A, B)
        assert np.array_equal(out["ind_ptr"], ip_o)


def test_supermesh_out_device_arrays(gpu_ctx):
    torch = pytest.importorskip("torch")
    dim, A, B = M.config_meshes("small3d_8x9")
    host = _host_out(len(A[1]), 1)
    with pytest.raises(lsm.LsmError) as ei:  # capacity 1: CSR and measures only
        gpu_ctx.supermesh_out(A, B, host)
    assert ei.value.status == 3
    n = int(host["ind_ptr"][-1])
    host = _host_out(len(A[1]), n)
    gpu_ctx.supermesh_out(A, B, host)
    tA = tuple(torch.from_numpy(x).cuda() for x in A)
    tB = tuple(torch.from_numpy(x).cuda() for x in B)
    dev = {"elem_measure": torch.zeros(len(A[1]), dtype=torch.float64, device="cuda"),
           "ind_ptr": torch.zeros(len(A[1]) + 1, dtype=torch.int64, device="cuda"),
           "indices": torch.zeros(n, dtype=torch.int64, device="cuda"),
           "pair_measure": torch.zeros(n, dtype=torch.float64, device="cuda"),
           "pair_n_out": torch.zeros(n, dtype=torch.int32, device="cuda"), "capacity": n}
    gpu_ctx.supermesh_out(tA, tB, dev, on_device=True)
    torch.cuda.synchronize()
    for k in ("elem_measure", "ind_ptr", "indices", "pair_measure", "pair_n_out"):
        assert np.array_equal(dev[k].cpu().numpy(), host[k][: len(dev[k])]), k
