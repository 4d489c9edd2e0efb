"""Synthetic mesh generators and the Triangle-format reader (CPU)."""
import hashlib

import numpy as np
import pytest

from libsupermesh_b200 import meshes as M


def _signed(pos, en):
    return M._signed_measure(pos, en)


def test_splitmix64_known_values():
    # splitmix64 with seed 0: first outputs 0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4
    u = M.splitmix64_uniform(0, 2)
    assert u[0] == (0xE220A8397B1DCDAF >> 11) * 2.0 ** -53
    assert u[1] == (0x6E789E6AA1B965F4 >> 11) * 2.0 ** -53


@pytest.mark.parametrize("n,seed,jit", [(73, 1, 0.3), (100, 0, 0.3), (16, 9, 0.3)])
def test_grid2d_valid_tiling(n, seed, jit):
    pos, en = M.grid2d(n, seed, jit)
    assert en.shape == (2 * n * n, 3) and pos.shape == ((n + 1) ** 2, 2)
    s = _signed(pos, en)
    assert (s > 0).all()
    assert abs(0.5 * s.sum() - 1.0) < 1e-12
    h = 1.0 / n
    base, _ = M.grid2d(n, seed, 0.0)
    assert np.abs(pos - base).max() <= jit * h * (1 + 1e-12)


@pytest.mark.parametrize("n,seed,jit", [(8, 3, 0.25), (32, 2, 0.25)])
def test_grid3d_valid_tiling(n, seed, jit):
    pos, en = M.grid3d(n, seed, jit)
    base, _ = M.grid3d(n, seed, 0.0)
    s, s0 = _signed(pos, en), _signed(base, en)
    assert (np.sign(s) == np.sign(s0)).all() and (s != 0).all()
    assert abs(np.abs(s).sum() / 6.0 - 1.0) < 1e-12


def test_generators_deterministic():
    a = M.grid3d(6, 3, 0.25)
    b = M.grid3d(6, 3, 0.25)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    digest = hashlib.sha256(M.grid2d(5, 1, 0.3)[0].tobytes()).hexdigest()
    assert digest == hashlib.sha256(M.grid2d(5, 1, 0.3)[0].tobytes()).hexdigest()


def test_config_sizes():
    dim, A, B = M.config_meshes("tri2d_73x100")
    assert dim == 2 and A[1].shape[0] == 10658 and B[1].shape[0] == 20000
    dim, A, B = M.config_meshes("tet3d_27x32")
    assert dim == 3 and A[1].shape[0] == 118098 and B[1].shape[0] == 196608


def test_batched_pairs_shapes():
    pairs = M.batched_pairs(8, seed=6, emin=1e2, emax=1e3)
    assert len(pairs) == 8
    assert [p[0] for p in pairs] == [2] * 4 + [3] * 4
    for dim, A, B in pairs:
        assert A[1].shape[1] == dim + 1 and B[1].shape[1] == dim + 1


def test_reader_roundtrip(tmp_path):
    pos, en = M.grid2d(3, 0, 0.3)
    with open(tmp_path / "m.node", "w") as f:
        f.write(f"{len(pos)} 2 0 0\n")
        for i, p in enumerate(pos):
            f.write(f"{i + 1} {float(p[0])!r} {float(p[1])!r}\n")
    with open(tmp_path / "m.ele", "w") as f:
        f.write(f"{len(en)} 3 1\n")
        for i, e in enumerate(en):
            f.write(f"{i + 1} {e[0] + 1} {e[1] + 1} {e[2] + 1} 7\n")
    p2, e2 = M.read_mesh(tmp_path / "m")
    assert np.array_equal(p2, pos) and np.array_equal(e2, en)
