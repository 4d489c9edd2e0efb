"""CUDA-graph replay of device-resident batched calls (option batch_graph).

The first call of a batch runs eagerly and captures the whole batch (both
dimension groups, every phase, no host wait inside); later calls with the
same meshes replay the graph with one launch and one host wait.  The tests
check that a replay gives exactly the eager results, also after the caller
changed the coordinates in place, that candidates outgrowing the graph's
arrays fall back to an eager run (and a new capture), and that a graph is not
replayed after the context reallocated its buffers.
"""
import numpy as np
import pytest

import libsupermesh_b200 as lsm
from libsupermesh_b200 import meshes as M

pytestmark = pytest.mark.gpu


def _device_pairs(names):
    import torch

    out = []
    for n in names:
        _, A, B = M.config_meshes(n)
        out.append(tuple((torch.from_numpy(m[0].copy()).cuda(), torch.from_numpy(m[1]).cuda()) for m in (A, B)))
    return out


def _eager(ctx, pairs):
    lsm.set_option("batch_graph", 0)
    return ctx.supermesh_batched(pairs, on_device=True)


def _graph(ctx, pairs):
    lsm.set_option("batch_graph", 1)
    try:
        return ctx.supermesh_batched(pairs, on_device=True)
    finally:
        lsm.set_option("batch_graph", 0)


def _same(x, y):
    for u, v in zip(x, y):
        assert np.array_equal(u, v)


@pytest.mark.parametrize("names", [["small3d_5x6", "small2d_12x17", "small3d_7x6", "small2d_31x50"],
                                   ["small3d_9x7", "small3d_4x5"], ["small2d_20x17"]])
def test_replay_equals_eager(names):
    with lsm.Context(0) as ctx:
        pairs = _device_pairs(names)
        ref = _eager(ctx, pairs)
        l0 = lsm.kernel_launches()
        first = _graph(ctx, pairs)  # eager run + capture
        _same(first, ref)
        for _ in range(3):
            _same(_graph(ctx, pairs), ref)
        assert lsm.kernel_launches() > l0


def test_replay_follows_coordinates_changed_in_place():
    with lsm.Context(0) as ctx:
        pairs = _device_pairs(["small3d_6x5", "small2d_15x19"])
        _graph(ctx, pairs)
        # translate every mesh in place: same candidates, new arithmetic
        for A, B in pairs:
            A[0].add_(0.25)
            B[0].add_(0.25)
        got = _graph(ctx, pairs)
        ref = _eager(ctx, pairs)
        _same(got, ref)
        assert np.all(np.abs(got[0] - 1.0) <= 1e-12)


def test_overflow_falls_back_to_eager_and_recaptures():
    import torch

    with lsm.Context(0) as ctx:
        pairs = _device_pairs(["small2d_5x6", "small3d_3x4"])
        _graph(ctx, pairs)
        # scatter A's nodes over the domain: elements become large and
        # overlapping, so the candidates far outgrow the captured arrays
        g = torch.Generator(device="cuda")
        g.manual_seed(5)
        for A, _ in pairs:
            A[0].copy_(torch.rand(A[0].shape, generator=g, device="cuda", dtype=torch.float64))
        got = _graph(ctx, pairs)
        ref = _eager(ctx, pairs)
        _same(got, ref)
        assert ref[1].sum() > 3000
        _same(_graph(ctx, pairs), ref)  # the recaptured graph


def test_no_replay_after_buffers_were_reallocated():
    with lsm.Context(0) as ctx:
        pairs = _device_pairs(["small3d_5x6", "small2d_12x17"])
        ref = _eager(ctx, pairs)
        _graph(ctx, pairs)
        # a much larger call on the same context reallocates its buffers
        _, A, B = M.config_meshes("small3d_20x22")
        ctx.supermesh(A, B)
        _same(_graph(ctx, pairs), ref)
        _same(_graph(ctx, pairs), ref)
