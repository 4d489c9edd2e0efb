"""The learned scheduler's tensor-core kernels and its schedules.

  * inference (libsupermesh_gpu_sched_predict) against a plain PyTorch FP32
    reference of the same network (same BF16 rounding of weights, inputs and
    activations; FP32 accumulation);
  * the training kernel's gradient of one minibatch against PyTorch
    autograd on that reference;
  * training on a task with known labels reaches high accuracy;
  * every schedule (plain, learned bins, true-class bins, any window) gives
    bit-identical per-pair results: the scheduler only orders work;
  * training samples: one per survivor of the early-out pass, labelled with
    the class of the clipper's own output count.
"""
import numpy as np
import pytest

import libsupermesh_b200 as lsm
from libsupermesh_b200 import meshes as M
from libsupermesh_b200 import scheduler as S

pytestmark = pytest.mark.gpu

LOGIT_RTOL = 2e-2  # BF16 operands: FP32 accumulation order and activation rounding ties


def _features(n, seed):
    import torch

    g = torch.Generator().manual_seed(seed)
    x = torch.zeros((n, 32), dtype=torch.float32)
    x[:, :24] = torch.randn((n, 24), generator=g) * 0.5
    return x.to(torch.bfloat16).cuda()


def test_predict_matches_torch_fp32_reference(gpu_ctx):
    import torch

    params = S.init_params(3)
    params[S.OFF_B1:S.OFF_W2] = np.linspace(-0.1, 0.1, 64)
    params[S.OFF_B3:S.OFF_B3 + 4] = [0.05, -0.02, 0.01, 0.0]
    x = _features(5000, 1)
    gpu_ctx.sched_set_weights(params)
    logits = torch.empty((len(x), 4), dtype=torch.float32, device="cuda")
    cls = torch.empty(len(x), dtype=torch.int8, device="cuda")
    gpu_ctx.sched_predict(len(x), x, logits, cls)
    ref = S.torch_forward(params, x.cpu())
    got = logits.cpu()
    scale = ref.abs().max()
    assert float((got - ref).abs().max()) <= LOGIT_RTOL * float(scale)
    agree = (cls.cpu().long() == ref.argmax(dim=1)).float().mean()
    assert float(agree) >= 0.99


def test_training_gradient_matches_autograd(gpu_ctx):
    import torch

    n = 128
    params = S.init_params(5)
    x = _features(n, 2)
    y = torch.randint(0, 4, (n,), generator=torch.Generator().manual_seed(4)).to(torch.int8)
    p_dev = torch.from_numpy(params.copy()).cuda()
    grad = torch.zeros(lsm.SCHED_PARAMS, dtype=torch.float32, device="cuda")
    gpu_ctx.sched_train(n, x, y.cuda(), p_dev, 1, 1e-3, grad_first=grad)
    # autograd on the FP32 reference (BF16-rounded weights and inputs)
    P = torch.from_numpy(params.copy()).requires_grad_(True)
    w1, b1, w2, b2, w3, b3 = (P[S.OFF_W1:S.OFF_B1].view(64, 32)[:, :24], P[S.OFF_B1:S.OFF_W2],
                              P[S.OFF_W2:S.OFF_B2].view(64, 64), P[S.OFF_B2:S.OFF_W3],
                              P[S.OFF_W3:S.OFF_B3].view(8, 64)[:4], P[S.OFF_B3:S.OFF_B3 + 4])
    bf = lambda t: t.to(torch.bfloat16).to(torch.float32)  # noqa: E731
    xf = bf(x.cpu().float())[:, :24]
    h1 = torch.relu(xf @ bf(w1).T + b1)
    h2 = torch.relu(bf(h1) @ bf(w2).T + b2)
    logits = bf(h2) @ bf(w3).T + b3
    loss = torch.nn.functional.cross_entropy(logits, y.long())
    loss.backward()
    g_ref = P.grad.numpy()
    g = grad.cpu().numpy()
    for lo, hi in ((S.OFF_W1, S.OFF_B1), (S.OFF_B1, S.OFF_W2), (S.OFF_W2, S.OFF_B2), (S.OFF_B2, S.OFF_W3),
                   (S.OFF_W3, S.OFF_B3), (S.OFF_B3, S.NPARAMS)):
        err = np.linalg.norm(g[lo:hi] - g_ref[lo:hi])
        assert err <= 3e-2 * np.linalg.norm(g_ref[lo:hi]) + 1e-7, (lo, err, np.linalg.norm(g_ref[lo:hi]))


def test_training_learns_known_labels(gpu_ctx):
    import torch

    n = 65536
    x = _features(n, 7)
    teacher = torch.randn((24, 4), generator=torch.Generator().manual_seed(8))
    y = (x.cpu().float()[:, :24] @ teacher).argmax(dim=1).to(torch.int8).cuda()
    params = torch.from_numpy(S.init_params(1)).cuda()
    trace = torch.zeros(10, dtype=torch.float32, device="cuda")
    gpu_ctx.sched_train(n, x, y, params, 3000, 3e-3, trace, 300)
    tr = trace.cpu().numpy()
    assert tr[-1] < 0.5 * tr[0]
    acc, _ = S.evaluate(gpu_ctx, params.cpu().numpy(), x, y)
    assert acc > 0.9


@pytest.mark.parametrize("name", ["small3d_12x14", "small3d_14x11"])
def test_every_schedule_gives_identical_results(gpu_ctx, name):
    dim, A, B = M.config_meshes(name)
    lsm.set_option("tet_schedule", 0)
    st, _ = gpu_ctx.supermesh(A, B)
    pm, pn = gpu_ctx.pair_results(st.n_candidates)
    gpu_ctx.sched_set_weights(S.init_params(2))
    try:
        for mode in (1, 2):
            for window in (256, 1024, 8192):
                lsm.set_option("tet_schedule", mode)
                lsm.set_option("sched_window", window)
                st2 = gpu_ctx.clip_candidates()
                pm2, pn2 = gpu_ctx.pair_results(st.n_candidates)
                assert np.array_equal(pm, pm2) and np.array_equal(pn, pn2), (mode, window)
                assert st2.total_measure == st.total_measure
    finally:
        lsm.set_option("tet_schedule", 0)
        lsm.set_option("sched_window", 1024)


def test_samples_are_the_survivors_with_their_classes(gpu_ctx):
    import torch

    dim, A, B = M.config_meshes("small3d_12x14")
    lsm.set_option("tet_schedule", 0)
    st, _ = gpu_ctx.supermesh(A, B)
    surv = gpu_ctx.clip_survivors()
    x = torch.empty((surv + 10, 32), dtype=torch.bfloat16, device="cuda")
    y = torch.empty(surv + 10, dtype=torch.int8, device="cuda")
    n = gpu_ctx.sched_samples(surv + 10, x, y)
    assert n == surv
    _, pn = gpu_ctx.pair_results(st.n_candidates)
    yc = np.bincount(y[:n].cpu().numpy(), minlength=4)
    # the early-out pass settles pairs with no tets and pairs whose A lies
    # inside all four planes of B (one tet, A itself): every pair with more
    # than 3 tets survives, so those classes agree with the clipper's counts
    full = np.bincount(S.size_class(pn), minlength=4)
    assert np.array_equal(yc[2:], full[2:])
    assert yc[0] <= full[0] and yc[1] <= full[1] and yc.sum() == n
    f = x[:n].float().cpu().numpy()
    assert np.all(np.isfinite(f)) and np.abs(f[:, :24]).max() <= 4.0 and np.all(f[:, 24:] == 0)


def test_schedule_needs_weights_and_a_previous_phase():
    with lsm.Context(0) as ctx:
        dim, A, B = M.config_meshes("small3d_5x6")
        ctx.find_candidates(A, B)
        lsm.set_option("tet_schedule", 1)
        try:
            with pytest.raises(lsm.LsmError):
                ctx.clip_candidates()
            lsm.set_option("tet_schedule", 2)
            ctx.find_candidates(A, B)
            with pytest.raises(lsm.LsmError):
                ctx.clip_candidates()
        finally:
            lsm.set_option("tet_schedule", 0)
        st = ctx.clip_candidates()
        assert abs(st.total_measure - 1.0) <= 1e-12
