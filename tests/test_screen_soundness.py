"""The tet narrow phase's exact shortcuts, restated in numpy and checked
against the oracle on CPU.

The GPU early-out pass settles a pair without clipping when it proves one
of three things: A lies beyond a face plane of B (no tets), B lies beyond a
face plane of A (no tets), or every plane of B keeps A whole (A itself is the
one tet).  It also skips the planes of B that keep A whole.  Here the same
tests, with the same margins, pick pairs from mesh candidates, near-touching
constructions and nested meshes, and the oracle (the reference algorithm)
must agree with each verdict: no output for a rejected pair, exactly A for a
pair inside all four planes.  The GPU parity tests compare the kernels'
results (no-op planes skipped) with the oracle pair by pair; this file pins
the shortcuts' soundness on the CPU.
"""
import numpy as np
import pytest

from libsupermesh_b200 import meshes as M

EPS = 2.0 ** -52


def planes(t):
    """Outward unit face planes (n, c) of a tet in the order the clipper
    uses: faces (0,1,2), (0,1,3), (0,2,3), (1,2,3), c from vertex i."""
    e10, e20, e30 = t[1] - t[0], t[2] - t[0], t[3] - t[0]
    e21, e31 = t[2] - t[1], t[3] - t[1]
    n = np.array([np.cross(e20, e10), np.cross(e10, e30), np.cross(e30, e20), np.cross(e21, e31)])
    n /= np.linalg.norm(n, axis=1)[:, None]
    if np.dot(e10, n[3]) < 0:
        n = -n
    c = np.array([np.dot(t[i], n[i]) for i in range(4)])
    return n, c


def verdicts(ta, tb):
    """(reject_a_beyond_b, reject_b_beyond_a, noop_mask) with the kernel's
    margins."""
    nb, cb = planes(tb)
    M_a = np.abs(ta).max()
    d = ta @ nb.T - cb  # [vertex, plane]
    thr = EPS + 64 * EPS * (1 + 2 * np.maximum(M_a, np.abs(cb)))
    rej1 = bool((d.min(axis=0) >= thr).any())
    noop = sum(1 << L for L in range(4) if d[:, L].max() <= -thr[L])
    # B beyond a face of A: dilation bound of B's planes
    na, _ = planes(ta)
    h = (ta @ na.T).max(axis=0) + 128 * EPS * (1 + M_a)
    M_b = max(np.abs(tb).max(), np.abs(cb).max())
    tau = max(abs(np.dot(nb[f], tb[k]) - cb[f]) for f in range(4) for k in range(4) if k != 3 - f)
    tau += 16 * EPS * (1 + 2 * M_b)
    D = [(-1) ** j * np.linalg.det(np.delete(nb, j, axis=0)) for j in range(4)]
    same = all(x > 1e-14 for x in D) or all(x < -1e-14 for x in D)
    rej2 = False
    if same:
        g = 3.02 / (min(abs(x) for x in D) - 1e-14)
        Mp = max(M_a, M_b)
        e = EPS + 128 * EPS * (1 + 2 * Mp)
        slack = 1.01 * g * (tau + e) + 16 * EPS * (1 + Mp)
        m = (tb @ na.T).min(axis=0)
        rej2 = bool((m >= h + slack).any())
    return rej1, rej2, noop


def candidate_pairs(name, count, seed):
    import oracle

    dim, A, B = M.config_meshes(name)
    ip, ix = oracle.tree_finder(dim, A, B)
    rows = np.repeat(np.arange(len(A[1])), np.diff(ip))
    rng = np.random.default_rng(seed)
    k = rng.choice(len(ix), min(count, len(ix)), replace=False)
    return A[0][A[1][rows[k]]], B[0][B[1][ix[k]]]


def near_touching(count, seed):
    """B's tip at a small signed gap beyond a face of A, base farther out."""
    rng = np.random.default_rng(seed)
    ta, tb = [], []
    for gap in (-1e-9, 0.0, 1e-15, 1e-13, 1e-11, 1e-9, 1e-6):
        for _ in range(count):
            a = rng.random((4, 3)) + rng.random(3) * 10
            if abs(np.linalg.det(a[1:] - a[0])) < 0.05:
                continue
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
            th = rng.random() * 2 * np.pi + np.arange(3) * 2 * np.pi / 3
            base = q + 0.4 * n + 0.5 * (np.cos(th)[:, None] * u + np.sin(th)[:, None] * v)
            ta.append(a)
            tb.append(np.vstack([q + gap * n, base])[rng.permutation(4)])
    return np.array(ta), np.array(tb)


def nested_pairs(count, seed):
    import oracle

    A = M.grid3d(9, 3, 0.25)
    B = M.grid3d(3, 2, 0.25)
    ip, ix = oracle.tree_finder(3, A, B)
    rows = np.repeat(np.arange(len(A[1])), np.diff(ip))
    rng = np.random.default_rng(seed)
    k = rng.choice(len(ix), min(count, len(ix)), replace=False)
    return A[0][A[1][rows[k]]], B[0][B[1][ix[k]]]


def degenerate_pairs(count, seed):
    """Zero-volume A (a repeated vertex: NaN face normals; or a vertex at
    the midpoint of an edge: coplanar) against overlapping tets: no face of
    such an A proves anything."""
    rng = np.random.default_rng(seed)
    ta = rng.random((count, 4, 3))
    ta[: count // 2, 1] = ta[: count // 2, 0]
    ta[count // 2:, 3] = 0.5 * (ta[count // 2:, 0] + ta[count // 2:, 1])
    tb = rng.random((count, 4, 3)) * 0.8 + 0.1
    return ta, tb


@pytest.mark.parametrize("source", ["candidates", "near_touching", "nested", "degenerate"])
def test_shortcut_verdicts_agree_with_the_oracle(oracle_mod, source):
    if source == "candidates":
        TA, TB = candidate_pairs("small3d_8x9", 4000, 1)
    elif source == "near_touching":
        TA, TB = near_touching(40, 2)
    elif source == "nested":
        TA, TB = nested_pairs(3000, 3)
    else:
        TA, TB = degenerate_pairs(400, 4)
    seen = {"rej1": 0, "rej2": 0, "inside": 0, "noop": 0}
    for ta, tb in zip(TA, TB):
        with np.errstate(invalid="ignore", divide="ignore"):
            rej1, rej2, noop = verdicts(ta, tb)
        ref = oracle_mod.intersect_tets(ta, tb)
        if rej1 or rej2:
            assert len(ref) == 0
            seen["rej1" if rej1 else "rej2"] += 1
        elif noop == 15:
            assert len(ref) == 1 and np.array_equal(ref[0], ta)
            seen["inside"] += 1
        elif noop:
            # the no-op planes' skip is checked on the GPU, where the clipper
            # applies it and its per-pair results must equal the oracle's
            seen["noop"] += 1
    # each source exercises the shortcuts it was built for
    if source == "candidates":
        assert seen["rej1"] > 0 and seen["rej2"] > 0 and seen["noop"] > 0
    elif source == "near_touching":
        assert seen["rej2"] > 0
    elif source == "nested":
        assert seen["inside"] > 0
