"""Learned scheduler of the tet clipper: training data, training and weights.

The library's scheduler (include/libsupermesh-gpu.h, option tet_schedule)
orders the 3D clipper's work list by each surviving pair's predicted
output-size class (0: no tets, 1: 1-3, 2: 4-7, 3: 8 or more; the n_tets_c of
intersect_tets_real, Tetrahedron_Intersection.F90:137-179 upstream).  The
predictor is a BF16 MLP 24 -> 64 -> 64 -> 4 whose inference and training run
in the library's own tensor-core kernels; this module drives them:

  * labels come from the plain clipper itself: the survivors of the exact
    early-out pass on config-1-style meshes (target 27^3 x 6 tets, source
    32^3 x 6, jitter 0.25h) with seeds 9..20 (six mesh pairs), each labelled
    by its output count (libsupermesh_gpu_sched_samples);
  * training is minibatch Adam in one kernel launch
    (libsupermesh_gpu_sched_train) over the shuffled samples;
  * the trained FP32 parameters are stored in data/sched_mlp.npz with the
    training record (seeds, steps, loss, held-out accuracy).

Every pair is still clipped exactly whatever the prediction, so the weights
only ever change the speed of the narrow phase, never its results.
"""
from __future__ import annotations

import json
import time
from pathlib import Path

import numpy as np

import libsupermesh_b200 as lsm
from libsupermesh_b200 import meshes as M

DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "data" / "sched_mlp.npz"
TRAIN_SEEDS = tuple(range(9, 21))
IN, IN_PAD, HID, CLS = 24, 32, 64, 4
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * IN_PAD
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + 8 * HID
NPARAMS = OFF_B3 + 8
assert NPARAMS == lsm.SCHED_PARAMS


def size_class(n_out):
    """Output-size class of output counts (numpy)."""
    n = np.asarray(n_out)
    return np.where(n <= 0, 0, np.where(n <= 3, 1, np.where(n <= 7, 2, 3))).astype(np.int8)


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases, zero padding entries (FP32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, dtype=np.float32)
    w1 = np.zeros((HID, IN_PAD), dtype=np.float32)
    w1[:, :IN] = rng.uniform(-1, 1, (HID, IN)) * np.sqrt(6.0 / IN)
    p[OFF_W1:OFF_B1] = w1.ravel()
    p[OFF_W2:OFF_B2] = (rng.uniform(-1, 1, (HID, HID)) * np.sqrt(6.0 / HID)).ravel()
    w3 = np.zeros((8, HID), dtype=np.float32)
    w3[:CLS] = rng.uniform(-1, 1, (CLS, HID)) * np.sqrt(6.0 / HID)
    p[OFF_W3:OFF_B3] = w3.ravel()
    return p


def unpack(p):
    """(W1 [64][24], b1, W2, b2, W3 [4][64], b3 [4]) views of a parameter vector."""
    p = np.asarray(p, dtype=np.float32)
    return (p[OFF_W1:OFF_B1].reshape(HID, IN_PAD)[:, :IN], p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(HID, HID),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(8, HID)[:CLS], p[OFF_B3:OFF_B3 + CLS])


def torch_forward(params, x_bf16):
    """Plain PyTorch FP32 reference of the library's forward pass: weights and
    inputs rounded to BF16 as the kernel stores them, activations rounded to
    BF16 between layers (the kernel feeds each layer's output to the next
    layer's tensor-core operands as BF16), FP32 accumulation.  Returns
    logits [n][4]."""
    import torch

    w1, b1, w2, b2, w3, b3 = (torch.as_tensor(np.array(a)) for a in unpack(params))
    bf = lambda t: t.to(torch.bfloat16).to(torch.float32)  # noqa: E731
    x = bf(x_bf16.to(torch.float32))[:, :IN]
    h1 = bf(torch.relu(x @ bf(w1).T + b1))
    h2 = bf(torch.relu(h1 @ bf(w2).T + b2))
    return h2 @ bf(w3).T + b3


def training_pairs(seeds=TRAIN_SEEDS):
    """Config-1-style mesh pairs (target 27^3 x 6, source 32^3 x 6 tets,
    jitter 0.25h) with consecutive seeds (9, 10), (11, 12), ..."""
    return [(M.grid3d(27, a, 0.25), M.grid3d(32, b, 0.25)) for a, b in zip(seeds[0::2], seeds[1::2])]


def collect(ctx, pairs, cap_per_pair: int, device):
    """Run the plain narrow phase on each mesh pair and take its survivors'
    features and classes (device tensors, concatenated)."""
    import torch

    xs, ys = [], []
    lsm.set_option("tet_schedule", 0)
    for A, B in pairs:
        ctx.supermesh(A, B)
        x = torch.empty((cap_per_pair, IN_PAD), dtype=torch.bfloat16, device=device)
        y = torch.empty(cap_per_pair, dtype=torch.int8, device=device)
        n = ctx.sched_samples(cap_per_pair, x, y)
        k = min(n, cap_per_pair)
        xs.append(x[:k])
        ys.append(y[:k])
    return torch.cat(xs), torch.cat(ys)


def train(ctx, x, y, steps: int, lr: float = 2e-3, seed: int = 0, trace_every: int = 500):
    """Shuffle the samples and run `steps` Adam steps in the library's
    training kernel.  Returns (params numpy, loss trace numpy, seconds)."""
    import torch

    g = torch.Generator(device=x.device)
    g.manual_seed(seed)
    perm = torch.randperm(len(x), device=x.device, generator=g)
    xs, ys = x[perm].contiguous(), y[perm].contiguous()
    params = torch.from_numpy(init_params(seed)).to(x.device)
    trace = torch.zeros(max(1, steps // trace_every + 1), dtype=torch.float32, device=x.device)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.sched_train(len(xs), xs, ys, params, steps, lr, trace, trace_every)
    dt = time.perf_counter() - t0
    return params.cpu().numpy(), trace.cpu().numpy()[: (steps + trace_every - 1) // trace_every], dt


def evaluate(ctx, params, x, y):
    """Accuracy and per-class confusion of the library's inference kernel."""
    import torch

    ctx.sched_set_weights(params)
    cls = torch.empty(len(x), dtype=torch.int8, device=x.device)
    ctx.sched_predict(len(x), x, None, cls)
    p, t = cls.cpu().numpy(), y.cpu().numpy()
    conf = np.zeros((CLS, CLS), dtype=np.int64)
    np.add.at(conf, (t, p), 1)
    return float((p == t).mean()), conf


def save(params, meta: dict, path: Path = DEFAULT_WEIGHTS) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez(path, params=np.asarray(params, dtype=np.float32), meta=json.dumps(meta))


def load(path: Path = DEFAULT_WEIGHTS):
    """(params, meta) of stored weights, or (None, None)."""
    if not Path(path).exists():
        return None, None
    d = np.load(path)
    return d["params"].astype(np.float32), json.loads(str(d["meta"]))


def main():
    """Generate the labels, train, evaluate on the graded workload's
    survivors, and store the weights (run on a GPU)."""
    import argparse

    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=40000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--cap", type=int, default=2_000_000, help="samples per training mesh pair")
    ap.add_argument("--out", default=str(DEFAULT_WEIGHTS))
    a = ap.parse_args()
    dev = torch.device("cuda:0")
    with lsm.Context(0) as ctx:
        t0 = time.perf_counter()
        x, y = collect(ctx, training_pairs(), a.cap, dev)
        t_collect = time.perf_counter() - t0
        hist = np.bincount(y.cpu().numpy(), minlength=CLS)
        params, trace, t_train = train(ctx, x, y, a.steps, a.lr)
        acc_train, _ = evaluate(ctx, params, x[:1_000_000], y[:1_000_000])
        dim, A, B = M.config_meshes("tet3d_graded_55x51")
        xg, yg = collect(ctx, [(A, B)], 20_000_000, dev)
        acc_graded, conf = evaluate(ctx, params, xg, yg)
        meta = {"train_seeds": list(TRAIN_SEEDS), "train_meshes": "target 27^3 x 6, source 32^3 x 6 tets, jitter 0.25h",
                "samples": int(len(x)), "class_counts": hist.tolist(), "steps": a.steps, "batch": 128, "lr": a.lr,
                "optimizer": "Adam (0.9, 0.999)", "loss_first": float(trace[0]), "loss_last": float(trace[-1]),
                "train_accuracy": acc_train, "graded_survivors": int(len(xg)), "graded_accuracy": acc_graded,
                "graded_confusion": conf.tolist(), "seconds_collect": t_collect, "seconds_train": t_train}
        save(params, meta, Path(a.out))
        print(json.dumps(meta))


if __name__ == "__main__":
    main()
