"""Randomised parity: meshes of random resolution, jitter and affine
placement (rotated, scaled and shifted copies of the unit grids, so that the
two meshes cut each other at arbitrary angles and cover different regions),
through the whole pipeline against the oracle pair by pair, with the
supermesh's simplices and the P1-P1 blocks.  Seeds are
fixed, so a failure reproduces."""
import numpy as np
import pytest

from libsupermesh_b200 import meshes as M

pytestmark = pytest.mark.gpu


def _rotation(dim, rng):
    q, r = np.linalg.qr(rng.normal(size=(dim, dim)))
    return q * np.sign(np.diag(r))


def _case(dim, seed):
    rng = np.random.default_rng(seed)
    grid = M.grid2d if dim == 2 else M.grid3d
    if dim == 2:
        na, nb = rng.integers(6, 40, 2)
    else:
        na, nb = rng.integers(3, 11, 2)
    A = grid(int(na), 100 + seed, jitter=float(rng.uniform(0.0, 0.3)))
    pos, en = grid(int(nb), 200 + seed, jitter=float(rng.uniform(0.0, 0.3)))
    R = _rotation(dim, rng) * rng.uniform(0.6, 1.4)
    pos = (pos - 0.5) @ R.T + 0.5 + rng.uniform(-0.3, 0.3, dim)
    return A, (np.ascontiguousarray(pos), en)


@pytest.mark.parametrize("dim,seed", [(2, s) for s in range(16)] + [(3, s) for s in range(16)])
def test_random_affine_meshes_match_oracle(gpu_ctx, oracle_mod, dim, seed):
    from test_gpu_parity import check_pipeline

    A, B = _case(dim, seed)
    check_pipeline(gpu_ctx, oracle_mod, dim, A, B)
    # and the supermesh's simplices of a sample of candidates
    st, off, el, pa, pb = gpu_ctx.supermesh_elements(A, B)
    ip, ind = gpu_ctx.get_candidates(len(A[1]), st.n_candidates)
    rows = np.repeat(np.arange(len(ip) - 1), np.diff(ip))
    rng = np.random.default_rng(seed)
    for k in rng.choice(st.n_candidates, min(400, st.n_candidates), replace=False):
        ea, eb = A[0][A[1][rows[k]]], B[0][B[1][ind[k]]]
        ref = oracle_mod.intersect_tris(ea, eb) if dim == 2 else oracle_mod.intersect_tets(ea, eb)
        assert np.array_equal(el[off[k]:off[k + 1]], np.asarray(ref).reshape((-1,) + el.shape[1:])), k
    # the P1-P1 blocks, bit for bit
    u, v = np.cos(A[0][:, 0]) + A[0][:, 1], B[0][:, -1]
    val, blocks = gpu_ctx.p1_mass(A, B, u, v, want_blocks=True)
    ip_o, ind_o = oracle_mod.tree_finder(dim, A, B)
    val_o, _, blocks_o = oracle_mod.p1_mass(dim, A, B, ip_o, ind_o, u, v, want_blocks=True)
    ip_g, ind_g = gpu_ctx.get_candidates(len(A[1]), len(blocks))
    ko = np.lexsort((ind_o, np.repeat(np.arange(len(ip_o) - 1), np.diff(ip_o))))
    kg = np.lexsort((ind_g, np.repeat(np.arange(len(ip_g) - 1), np.diff(ip_g))))
    assert np.array_equal(blocks[kg], blocks_o[ko])
    assert abs(val - val_o) <= 1e-12 * max(1.0, abs(val_o))
