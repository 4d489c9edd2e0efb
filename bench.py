"""Benchmark of the supermesh hot path: clipped element pairs per second.

One step = one pass of the hot path over one pair of meshes: candidate
search (LBVH build + traversal), intersection of every candidate pair, and
the compensated measure reduction, through libsupermesh_gpu_supermesh.

Workload (default): 3D graded supermesh, target 55^3 x 6 = 998,250 Kuhn tets
(seed 7) against source 51^3 x 6 = 795,906 tets (seed 8), coordinates graded
x -> x^2 per axis, jitter 0.2h, FP64 (56.1M candidate pairs).  The unit of
work is one candidate pair of the strict-AABB candidate set (the tree
finder's set); pairs/s = candidates / step time.

  value      device-resident inputs (positions/enlists already in HBM), L2
             flushed before every step
  e2e        the same call with host (pinned) inputs: H2D of positions and
             element lists and D2H of the per-element measure in the timed
             region
  e2e_with_pairs  as e2e, plus the D2H of what a drop-in caller of the C API
             reads per candidate: the CSR (ind_ptr, indices as int64, the
             get_output layout) and per-pair measure and output count
  roofline   narrow phase: the exact early-out pass and the tet clipper (3D;
             together they settle every candidate) or the triangle clipper
             (2D), timed by the library's CUDA events over the same
             candidates, with the reference algorithm's FLOP count for all
             candidates, against the measured FP64 DADD/DMUL issue rate;
             broad_phase: the candidate search's algorithmic bytes over its
             device time, against the measured HBM copy bandwidth
  schedule   (3D) the narrow phase with the learned scheduler's bins beside
             the plain order, when trained weights are present
  cpu_baseline  the oracle restatement of the reference algorithm
             (quadtree/octree + breadth-first clipping), one thread, on a
             bounded sample of the workload (every k-th target element)

Multi-GPU: the workload is replicated per rank (independent replicas, no
collective on the data path); value = all ranks' pairs / max step time.

`--impl reference` times the reference algorithm on the host CPU (the oracle
restatement, all host threads; the Fortran reference cannot be built here)
on a bounded sample of the same workload per step.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "clipped element-pairs/sec"
L2_FLUSH_BYTES = 256 << 20


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", default="tet3d_graded_55x51")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--kernel-only", action="store_true",
                   help="run only warm-up + timed steps of --op (for profiler launch lists and captures)")
    p.add_argument("--op", choices=["supermesh", "p1_mass", "p2_inner", "pairs", "pairs_mixed"], default="supermesh",
                   help="with --kernel-only: the operation each step runs")
    p.add_argument("--schedule", type=int, default=0,
                   help="with --kernel-only: tet_schedule of the 3D narrow phase (1 needs the trained weights)")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the default launch shapes instead of running the autotuner first")
    return p.parse_args()


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.lines = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(gpus: int):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def all_max(x: float, world: int) -> float:
    """Max over ranks (device tensor under NCCL, host tensor under gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, steps: int, world: int, max_ms: float) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return units_per_rank * steps * world / (max_ms * 1e-3)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def load_probe():
    from libsupermesh_b200 import build

    L = ctypes.CDLL(str(build.build_probe()))
    L.lsm_probe_fp64_rate.restype = ctypes.c_double
    L.lsm_probe_fp64_rate.argtypes = [ctypes.c_int, ctypes.c_int]
    L.lsm_probe_flush_l2.restype = ctypes.c_int
    L.lsm_probe_flush_l2.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
    return L


def profile_traffic(kernel: str, workload: str):
    """dram bytes per launch from the committed ncu summaries, if present
    (summed over the kernels of a 'k1+k2' span)."""
    total = 0.0
    for k in kernel.split("+"):
        f = ROOT / "profiles" / f"{k}_{workload}.md"
        if not f.exists():
            return None
        m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", f.read_text())
        if not m:
            return None
        total += float(m.group(1))
    return total


def measured_peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return json.loads(f.read_text())
        except ValueError:
            return {}
    return {}


def cpu_baseline(dim, A, B, threads: int = 1):
    """Oracle (reference algorithm) on this host: full pipeline as the C API
    caller drives it.  Returns (pairs/s, seconds, stats)."""
    import oracle

    t0 = time.perf_counter()
    st = oracle.supermesh(dim, A, B, nthreads=threads)
    dt = time.perf_counter() - t0
    return st.n_candidates / dt, dt, st


def corner_sample(dim, A, B, frac: float = 0.125):
    """Bounded CPU sample of a workload: both meshes cut to the same corner
    box [lo, X]^dim, X the per-axis quantile of A's element centroids that
    keeps about `frac` of A's elements (B keeps about the same share, the
    meshes being graded alike).  The octree build, the queries and the
    clipping then shrink together, so pairs/s keeps the full workload's mix
    of build, search and clipping cost."""
    q = frac ** (1.0 / dim)
    ca = A[0][A[1]].mean(axis=1)
    X = float(np.quantile(ca[:, 0], q))

    def cut(m):
        inside = np.all(m[0][m[1]].max(axis=1) <= X, axis=1)
        return (m[0], np.ascontiguousarray(m[1][inside]))

    As, Bs = cut(A), cut(B)
    desc = (f"corner box x,y,z <= {X:.4g}: {len(As[1])} of {len(A[1])} target and {len(Bs[1])} of {len(B[1])} "
            f"source elements")
    return As, Bs, desc


def algorithmic_flops(dim, A, B):
    """Algorithmic FP64 operations of the narrow phase (per-pair clipping and
    measures plus per-element setup), counted by the oracle."""
    import oracle

    ip, ind = oracle.tree_finder(dim, A, B)
    n = os.cpu_count() or 1
    _, _, _, st = oracle.narrow(dim, A, B, ip, ind, nthreads=n, count_flops=True)
    return st.flops, st


def workload_config(args, dim, A, B, n_cand, world):
    """The `config` object of both arms' lines (identical for the same workload)."""
    return {"workload": args.workload, "dim": dim, "elements_a": int(len(A[1])), "elements_b": int(len(B[1])),
            "candidates": int(n_cand), "parallelism": f"replicas x{world}",
            "l2": "GPU arm: flushed before every timed step (256 MiB write, outside the events)"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    import oracle

    from libsupermesh_b200 import meshes as M

    dim, A, B = M.config_meshes(args.workload)
    As, Bs, desc = corner_sample(dim, A, B) if len(A[1]) > 200_000 else (A, B, "full workload")
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_baseline(dim, As, Bs, threads)
    times, st = [], None
    for _ in range(args.steps):
        _, dt, st = cpu_baseline(dim, As, Bs, threads)
        times.append(dt)
    total = sum(times)
    value = st.n_candidates * args.steps / total
    ip, ind = oracle.tree_finder(dim, A, B) if desc != "full workload" else (None, np.zeros(st.n_candidates))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, dim, A, B, len(ind), world),
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": "port",
                         "sample": f"per step: {desc} ({st.n_candidates} candidates); oracle quadtree/octree "
                                   f"finder (1 thread) + breadth-first clipping (OpenMP over A rows)"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "sample_total_measure": st.total,
    }
    print(json.dumps(line), flush=True)


def run_batched(args, world, rank, local):
    """256 independent mesh pairs (half 2D, half 3D, element counts
    log-uniform in [1e3, 1e5]) per step through libsupermesh_gpu_supermesh_batched."""
    import torch

    import libsupermesh_b200 as lsm
    from libsupermesh_b200 import meshes as M

    pairs = M.batched_pairs(256, seed=6)
    dev = torch.device("cuda", local)
    ctx = lsm.Context(local)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    probe = load_probe()
    flush_buf = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    tdev = [tuple((torch.from_numpy(m[0]).to(dev), torch.from_numpy(m[1]).to(dev)) for m in (A, B))
            for _, A, B in pairs]
    host = []
    h2d = 0
    for _, A, B in pairs:
        pin = []
        for m in (A, B):
            pin.append((torch.from_numpy(m[0]).pin_memory().numpy(), torch.from_numpy(m[1]).pin_memory().numpy()))
            h2d += m[0].nbytes + m[1].nbytes
        host.append(tuple(pin))
    torch.cuda.synchronize()

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        barrier(world)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        out = None
        for e0, e1 in evs:
            probe.lsm_probe_flush_l2(flush_buf.data_ptr(), L2_FLUSH_BYTES, sp)
            e0.record(stream)
            out = fn()
            e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return sum(e0.elapsed_time(e1) for e0, e1 in evs), out

    if args.kernel_only:
        ms_k, _ = timed(lambda: ctx.supermesh_batched(tdev, on_device=True, stream=sp), args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"kernel_only": True, "workload": args.workload, "ms_per_step": ms_k / args.steps}),
                  flush=True)
        ctx.close()
        return
    # eager: every phase launched by the host, one host wait per dimension
    # group for the candidate count; graph: the whole batch replayed from a
    # CUDA graph captured on the first call (option batch_graph)
    ms_eager, (tot0, nc0, ni0) = timed(lambda: ctx.supermesh_batched(tdev, on_device=True, stream=sp), args.steps,
                                       args.warmup)
    ms_eager = all_max(ms_eager, world)
    lsm.set_option("batch_graph", 1)
    launches0 = lsm.kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    ms, (tot, nc, ni) = timed(lambda: ctx.supermesh_batched(tdev, on_device=True, stream=sp), args.steps, args.warmup)
    clock_rec = clocks.stop()
    launches = (lsm.kernel_launches() - launches0) // (args.steps + args.warmup)
    lsm.set_option("batch_graph", 0)
    assert np.array_equal(tot, tot0) and np.array_equal(nc, nc0) and np.array_equal(ni, ni0)
    ms = all_max(ms, world)
    ncand = int(nc.sum())
    value = ncand * args.steps * world / (ms * 1e-3)
    ms_e2e, (tot2, nc2, _) = timed(lambda: ctx.supermesh_batched(host, on_device=False, stream=sp), args.steps,
                                   max(3, args.warmup // 2))
    ms_e2e = all_max(ms_e2e, world)
    assert np.array_equal(nc2, nc) and np.array_equal(tot2, tot)
    line = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "mesh_pairs": len(pairs), "candidates": ncand,
                   "intersecting": int(ni.sum()), "max_total_err": float(np.abs(tot - 1.0).max()),
                   "l2": "flushed before every timed step (256 MiB write, outside the events)",
                   "parallelism": f"replicas x{world}",
                   "form": "device-resident meshes, batch replayed from its CUDA graph (option batch_graph)"},
        "eager": {"value": ncand * args.steps * world / (ms_eager * 1e-3), "unit": "pairs/s",
                  "ms_per_step": ms_eager / args.steps},
        "e2e": {"value": ncand * args.steps * world / (ms_e2e * 1e-3), "unit": "pairs/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": len(pairs) * 24,
                "ms_per_step": ms_e2e / args.steps},
        "gpu_launches": launches * args.steps,
        "clocks": clock_rec,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        sample = pairs[::16]
        t0 = time.perf_counter()
        cand = 0
        for dim, A, B in sample:
            cand += oracle.supermesh(dim, A, B, nthreads=1).n_candidates
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": cand / dt, "unit": "pairs/s", "cores": 1, "kind": "port",
                                "sample": f"every 16th mesh pair ({len(sample)} pairs, {cand} candidates), "
                                          f"oracle finder + clipping, 1 thread, {dt:.2f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


def kernel_only(args, ctx, dim, A, B, tA, tB, step_device, timed, rank):
    """Warm-up + timed steps of one operation and nothing else (no second
    leg, no CPU work): the command that profiler launch lists and captures
    run.  --op supermesh: the whole pipeline (with --schedule for 3D);
    p1_mass: the P1-P1 product u^T M v (u = x on A, v = y on B, device
    meshes and fields); p2_inner: the 2D P2 inner product of P1 fields
    lifted to P2 (host arrays); pairs: the batched explicit-pair entry
    (libsupermesh_gpu_intersect_pairs, device memory) on the workload's first
    2^22 candidate pairs as element coordinates; pairs_mixed: the same pairs
    with B's element replaced by its bounding box as a hexahedron (3D, tet-hex)
    or quadrilateral (2D, tri-quad)."""
    import libsupermesh_b200 as lsm
    from libsupermesh_b200 import meshes as M

    sp = None
    units = None  # element pairs per call, where the op has a fixed count
    if args.op == "supermesh":
        if args.schedule:
            from libsupermesh_b200 import scheduler

            params, _ = scheduler.load()
            if args.schedule == 1 and params is None:
                raise SystemExit("--schedule 1 needs trained weights (python -m libsupermesh_b200.scheduler)")
            if params is not None:
                ctx.sched_set_weights(params)
            step_device()  # a plain phase first: tet_schedule 2 takes its classes from it
            lsm.set_option("tet_schedule", args.schedule)
        fn = step_device
    elif args.op == "p1_mass":
        du, dv = tA[0][:, 0].contiguous(), tB[0][:, 1].contiguous()

        def fn():
            return ctx.p1_mass(tA, tB, du, dv, on_device=True, stream=sp)
    elif args.op in ("pairs", "pairs_mixed"):
        import torch

        n_all = ctx.find_candidates(A, B)
        ip, ind = ctx.get_candidates(len(A[1]), n_all)
        n = min(n_all, 1 << 22)
        rows = np.repeat(np.arange(len(ip) - 1), np.diff(ip))[:n]
        ea = np.ascontiguousarray(A[0][A[1][rows]].reshape(n, -1))
        eb = B[0][B[1][ind[:n]]]
        kind = None
        if args.op == "pairs_mixed":
            lo, hi = eb.min(axis=1), eb.max(axis=1)
            if dim == 3:  # Gmsh node order: bottom face 0-3, top face 4-7
                corner = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                                   [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.float64)
                kind = lsm.PAIR_TET_HEX
            else:  # counter-clockwise
                corner = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], dtype=np.float64)
                kind = lsm.PAIR_TRI_QUAD
            eb = lo[:, None, :] + corner[None] * (hi - lo)[:, None, :]
        eb = np.ascontiguousarray(eb.reshape(n, -1))
        dev = tA[0].device
        da, db = torch.from_numpy(ea).to(dev), torch.from_numpy(eb).to(dev)
        dm = torch.empty(n, dtype=torch.float64, device=dev)
        dk = torch.empty(n, dtype=torch.int32, device=dev)
        units = n

        def fn():
            return ctx.intersect_pairs_device(da, db, dm, dk, dim=dim, kind=kind, stream=sp)
    else:
        if dim != 2:
            raise SystemExit("--op p2_inner needs a 2D workload")
        e2a, na2, edges_a = M.p2_space(A[1])
        e2b, nb2, edges_b = M.p2_space(B[1])
        fa = M.p1_to_p2(A[0][:, 0], na2, edges_a)
        fb = M.p1_to_p2(B[0][:, 1], nb2, edges_b)

        def fn():
            return ctx.p2_inner_product(A, B, e2a, fa, e2b, fb)
    ms, _ = timed(fn, args.steps, args.warmup)
    lsm.set_option("tet_schedule", 0)
    if rank == 0:
        line = {"kernel_only": True, "workload": args.workload, "op": args.op, "schedule": args.schedule,
                "ms_per_step": ms / args.steps}
        if units:
            line.update(pairs=units, pairs_per_s=units / (ms / args.steps * 1e-3))
        print(json.dumps(line), flush=True)


def drop_in_per_pair(ctx, dim, A, B, n_cand, n: int = 2000):
    """Calls per second of the drop-in per-pair entry
    (libsupermesh_intersect_tets_real / _tris_real: one copy in, one kernel
    launch, one copy out and a host wait per call) against the oracle's
    per-pair call (the reference algorithm on the host), on the first n
    candidate pairs of the workload, both driven by the same ctypes loop with
    preallocated arguments; host wall clock."""
    import libsupermesh_b200 as lsm
    import oracle

    ip, ind = ctx.get_candidates(len(A[1]), n_cand)
    n = min(n, n_cand)
    rows = np.repeat(np.arange(len(ip) - 1), np.diff(ip))[:n]
    ea = np.ascontiguousarray(A[0][A[1][rows]].reshape(n, -1))
    eb = np.ascontiguousarray(B[0][B[1][ind[:n]]].reshape(n, -1))
    cap = (lsm.TET_BUF_SIZE * 12) if dim == 3 else (lsm.TRI_BUF_SIZE * 6)
    out = np.zeros(cap)
    k = ctypes.c_int(0)
    dp = ctypes.POINTER(ctypes.c_double)
    args = [(ea[i].ctypes.data_as(dp), eb[i].ctypes.data_as(dp)) for i in range(n)]
    po, pk = out.ctypes.data_as(dp), ctypes.byref(k)
    g = getattr(lsm.load(), "libsupermesh_intersect_tets_real" if dim == 3 else "libsupermesh_intersect_tris_real")
    o = getattr(oracle.lib(), "orc_intersect_tets" if dim == 3 else "orc_intersect_tris")

    def rate(fn):
        for a, b in args[:20]:
            fn(a, b, po, pk)
        t0 = time.perf_counter()
        for a, b in args:
            fn(a, b, po, pk)
        return n / (time.perf_counter() - t0)

    gpu, cpu = rate(g), rate(o)
    return {"pairs": n, "gpu_calls_per_s": gpu, "oracle_calls_per_s": cpu, "gpu_vs_oracle": gpu / cpu,
            "entry": "libsupermesh_intersect_tets_real" if dim == 3 else "libsupermesh_intersect_tris_real",
            "timing": "host wall clock of a ctypes loop over the first candidate pairs (1 thread each)"}


def broad_phase_bytes(dim, A, B, n_cand):
    """Algorithmic bytes of the candidate search: both meshes' positions and
    element lists read once, 8 B per candidate pair written, and the radix
    sort of B's Morton keys (4 passes x (4 B key + 4 B value) read and
    written per element)."""
    pos = A[0].nbytes + B[0].nbytes
    en = len(A[1]) * A[1].shape[1] * 8 + len(B[1]) * B[1].shape[1] * 8
    return pos + en + 8 * n_cand + 4 * 16 * len(B[1])


def run_ours(args, world, rank, local):
    import torch

    import libsupermesh_b200 as lsm
    from libsupermesh_b200 import meshes as M

    if args.workload == "batched256":
        return run_batched(args, world, rank, local)
    dim, A, B = M.config_meshes(args.workload)
    dev = torch.device("cuda", local)
    ctx = lsm.Context(local)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    probe = load_probe()
    flush_buf = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def flush():
        probe.lsm_probe_flush_l2(flush_buf.data_ptr(), L2_FLUSH_BYTES, sp)

    tA = (torch.from_numpy(A[0]).to(dev), torch.from_numpy(A[1]).to(dev))
    tB = (torch.from_numpy(B[0]).to(dev), torch.from_numpy(B[1]).to(dev))
    em_dev = torch.zeros(len(A[1]), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    tuning = None
    if not args.no_autotune and not args.kernel_only:
        from libsupermesh_b200 import autotune

        tuning = autotune.tune(ctx, A, B, reps=2, store=False)

    def step_device():
        return ctx.supermesh(tA, tB, elem_measure=True, on_device=True, out=em_dev, stream=sp)[0]

    # pinned host inputs and outputs for the end-to-end legs
    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        return t.numpy()

    hA = (pinned(A[0]), pinned(A[1]))
    hB = (pinned(B[0]), pinned(B[1]))
    em_host = pinned(np.zeros(len(A[1])))
    h2d = A[0].nbytes + A[1].nbytes + B[0].nbytes + B[1].nbytes
    d2h = em_host.nbytes + 32

    def step_e2e():
        return ctx.supermesh(hA, hB, elem_measure=True, on_device=False, out=em_host, stream=sp)[0]

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        st = None
        for e0, e1 in evs:
            flush()
            e0.record(stream)
            st = fn()
            e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        ms = sum(e0.elapsed_time(e1) for e0, e1 in evs)
        return ms, st

    if args.kernel_only:
        return kernel_only(args, ctx, dim, A, B, tA, tB, step_device, timed, rank)

    launches0 = lsm.kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    ms_dev, st = timed(step_device, args.steps, args.warmup)
    clock_rec = clocks.stop()
    launches = lsm.kernel_launches() - launches0
    per_step_launches = launches // (args.steps + args.warmup)
    ms_dev = all_max(ms_dev, world)
    n_cand = st.n_candidates
    value = whole_job_rate(n_cand, args.steps, world, ms_dev)

    ms_e2e, st_e2e = timed(step_e2e, args.steps, max(3, args.warmup // 2))
    ms_e2e = all_max(ms_e2e, world)
    e2e = whole_job_rate(n_cand, args.steps, world, ms_e2e)
    assert st_e2e.n_candidates == n_cand and st_e2e.total_measure == st.total_measure

    # e2e with the per-candidate outputs a drop-in caller reads: the CSR
    # (get_output layout, int64) and each pair's measure and output count
    nel_a = len(A[1])
    csr_out = (pinned(np.zeros(nel_a + 1, dtype=np.int64)), pinned(np.zeros(max(n_cand, 1), dtype=np.int64)))
    pair_out = (pinned(np.zeros(max(n_cand, 1))), pinned(np.zeros(max(n_cand, 1), dtype=np.int32)))

    outs = {"elem_measure": em_host, "ind_ptr": csr_out[0], "indices": csr_out[1], "pair_measure": pair_out[0],
            "pair_n_out": pair_out[1], "capacity": n_cand}

    def step_e2e_pairs():
        # one call returns what a drop-in caller reads; the CSR's copy
        # overlaps the narrow phase on the library's second stream
        return ctx.supermesh_out(hA, hB, outs, on_device=False, stream=sp)[0]

    pair_steps = max(3, args.steps // 4)
    ms_e2e_p, st_p = timed(step_e2e_pairs, pair_steps, 2)
    ms_e2e_p = all_max(ms_e2e_p, world)
    assert st_p.total_measure == st.total_measure
    d2h_pairs = d2h + (nel_a + 1) * 8 + n_cand * (8 + 8 + 4)

    # broad phase alone (device-resident meshes): search time with events
    ms_bp, _ = timed(lambda: ctx.find_candidates(tA, tB, on_device=True, stream=sp), args.steps, 2)
    ms_bp = all_max(ms_bp, world) / args.steps
    step_device()  # leave the full pipeline's candidates and per-pair results current

    # narrow phase alone: the clipping kernels over the same candidates,
    # timed by the library with CUDA events on its stream
    lsm.set_option("time_kernels", 1)
    for _ in range(3):
        ctx.clip_candidates(stream=sp)
    kernel_ms = []
    for _ in range(args.steps):
        flush()
        ctx.clip_candidates(stream=sp)
        kernel_ms.append(ctx.clip_kernel_ms())
    lsm.set_option("time_kernels", 0)
    clip_ms = all_max(sum(kernel_ms), world) / args.steps
    clip_kernel = "k_prefilter_tets+k_clip_tets_ix" if dim == 3 else "k_clip_tris"

    line = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, dim, A, B, n_cand, world),
        "results": {"intersecting": st.n_intersecting, "out_simplices": st.n_out_simplices,
                    "total_measure": st.total_measure, "measure_err_vs_domain": abs(st.total_measure - 1.0)},
        "tuning": (tuning or {}).get("setting"),
        "intersecting_pairs_per_s": whole_job_rate(st.n_intersecting, args.steps, world, ms_dev),
        "e2e": {"value": e2e, "unit": "pairs/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": ms_e2e / args.steps},
        "e2e_with_pairs": {"value": whole_job_rate(n_cand, pair_steps, world, ms_e2e_p), "unit": "pairs/s",
                           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h_pairs,
                           "ms_per_step": ms_e2e_p / pair_steps,
                           "outputs": "per-element measure + CSR ind_ptr/indices (int64) + per-pair measure "
                                      "(f64) and output count (i32), into pinned host arrays, one "
                                      "libsupermesh_gpu_supermesh_out call per step"},
        "gpu_launches": per_step_launches * args.steps,
        "clocks": clock_rec,
    }
    if dim == 3:
        pm0, pn0 = ctx.pair_results(n_cand)
        sched = schedule_legs(ctx, sp, flush, args.steps, world, clip_ms, n_cand, pm0, pn0)
        if sched:
            line["schedule"] = sched
    if rank == 0:
        peak_rate = probe.lsm_probe_fp64_rate(0, 5)
        fma_rate = probe.lsm_probe_fp64_rate(1, 5)
        flops = None
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            flops, _ = algorithmic_flops(dim, A, B)
            As, Bs, desc = corner_sample(dim, A, B) if len(A[1]) > 200_000 else (A, B, "full workload")
            v, dt, st_cpu = cpu_baseline(dim, As, Bs, 1)
            cpu = {"value": v, "unit": "pairs/s", "cores": 1, "kind": "port",
                   "sample": f"{desc} ({st_cpu.n_candidates} candidates), oracle quadtree/octree "
                             f"finder + breadth-first clipping, 1 thread, {dt:.2f} s"}
        achieved = flops / (clip_ms * 1e-3) / 1e12 if flops else None
        peak = peak_rate / 1e12 if peak_rate > 0 else None
        pk = measured_peaks()
        hbm = pk.get("hbm_gbs")
        bp_bytes = broad_phase_bytes(dim, A, B, n_cand)
        bp_gbs = bp_bytes / (ms_bp * 1e-3) / 1e9
        line["roofline"] = {
            "kernel": clip_kernel,
            "bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": (achieved / peak) if (achieved and peak) else None,
            "traffic": profile_traffic(clip_kernel, args.workload),
            "launch_ms": clip_ms,
            "flops_per_launch": flops,
            "peak_source": "measured in-run: DADD+DMUL issue rate, 1 op each (the clipper is FMA-free); "
                           f"DFMA rate for context {fma_rate / 1e12:.1f} TFLOP/s",
            "broad_phase": {"bound": "hbm", "achieved": bp_gbs, "peak": hbm, "unit": "GB/s",
                            "frac": (bp_gbs / hbm) if hbm else None, "ms": ms_bp, "bytes": bp_bytes,
                            "peak_source": "MEASURED_PEAKS.json hbm_gbs (copy bandwidth)",
                            "note": "search time includes the host read of the candidate count"},
        }
        line["cpu_baseline"] = cpu
        line["drop_in_per_pair"] = drop_in_per_pair(ctx, dim, A, B, n_cand)
        line["p1_mass"] = p1_mass_timing(ctx, tA, tB, hA, hB, n_cand, stream, flush)
        if not args.no_cpu_baseline:
            line["p1_mass"]["cpu_baseline"] = p1_mass_cpu(dim, A, B)
        line["supermesh_elements"] = elements_timing(ctx, dim, tA, tB, n_cand, stream, flush)
        print(json.dumps(line), flush=True)
    ctx.close()


def schedule_legs(ctx, sp, flush, steps, world, plain_ms, n_cand, pm0, pn0):
    """The metric's "chosen vs plain" comparison on the 3D narrow phase: the
    early-out pass + clipper span (library CUDA events, L2 flushed before
    each) with the plain work order, with the survivors binned by the learned
    scheduler's predicted output-size class (tet_schedule 1), and binned by
    the true classes (tet_schedule 2: a perfect predictor, the ceiling of
    any scheduler).  The chosen form is the learned schedule where it is
    faster than the plain one and the plain one otherwise.  Every form's
    per-pair results are checked bit-identical to the plain run's."""
    import libsupermesh_b200 as lsm
    from libsupermesh_b200 import scheduler

    params, meta = scheduler.load()
    if params is None:
        return None
    ctx.sched_set_weights(params)

    def span(mode):
        lsm.set_option("tet_schedule", mode)
        lsm.set_option("time_kernels", 1)
        try:
            ctx.clip_candidates(stream=sp)
            ms = []
            for _ in range(steps):
                flush()
                ctx.clip_candidates(stream=sp)
                ms.append(ctx.clip_kernel_ms())
            pm, pn = ctx.pair_results(n_cand)
            assert np.array_equal(pm, pm0) and np.array_equal(pn, pn0), f"schedule {mode} changed results"
        finally:
            lsm.set_option("time_kernels", 0)
            lsm.set_option("tet_schedule", 0)
        return all_max(sum(ms), world) / steps

    learned_ms = span(1)
    true_ms = span(2)
    chosen = "learned" if learned_ms < plain_ms else "plain"
    chosen_ms = min(learned_ms, plain_ms)
    return {"window": lsm.get_option("sched_window"),
            "plain_ms": plain_ms, "learned_ms": learned_ms, "true_class_ms": true_ms,
            "plain_pairs_per_s": n_cand / (plain_ms * 1e-3), "learned_pairs_per_s": n_cand / (learned_ms * 1e-3),
            "true_class_pairs_per_s": n_cand / (true_ms * 1e-3),
            "chosen": chosen, "chosen_pairs_per_s": n_cand / (chosen_ms * 1e-3),
            "chosen_vs_plain": plain_ms / chosen_ms, "learned_vs_plain": plain_ms / learned_ms,
            "true_class_vs_plain": plain_ms / true_ms,
            "results": "per-pair measures and counts bit-identical in every schedule",
            "model": {k: meta.get(k) for k in ("steps", "samples", "train_accuracy", "graded_accuracy",
                                               "loss_first", "loss_last")} if meta else None,
            "timing": "early-out pass + bin + clipper span, CUDA events on the library's stream, "
                      "L2 flushed before each, mean of the timed repetitions"}


def p1_mass_timing(ctx, tA, tB, hA, hB, n_cand, stream, flush):
    """The P1-P1 mixed mass product u^T M v over the supermesh (search,
    clipping and the quadrature blocks: 3-point rule per triangle, 4-point
    rule per tet), u = x on A, v = y on B, reported
    beside the main metric, not part of it: device-resident meshes and fields
    timed with CUDA events on the stream (L2 flushed before each call), and
    end to end from pinned host meshes and fields (copies inside the events).
    Median of 5 calls after 2 warm-up calls each."""
    import torch

    sp = stream.cuda_stream
    du, dv = tA[0][:, 0].contiguous(), tB[0][:, 1].contiguous()
    hu = torch.from_numpy(np.ascontiguousarray(hA[0][:, 0])).pin_memory().numpy()
    hv = torch.from_numpy(np.ascontiguousarray(hB[0][:, 1])).pin_memory().numpy()

    def timed(fn):
        for _ in range(2):
            fn()
        ms, val = [], None
        for _ in range(5):
            flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            val = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms)), val

    ms_dev, (val_dev, _) = timed(lambda: ctx.p1_mass(tA, tB, du, dv, on_device=True, stream=sp))
    ms_e2e, (val_e2e, _) = timed(lambda: ctx.p1_mass(hA, hB, hu, hv, stream=sp))
    assert val_dev == val_e2e
    return {"ms": ms_dev, "pairs_per_s": n_cand / (ms_dev * 1e-3), "uTMv": val_dev,
            "e2e_ms": ms_e2e, "e2e_pairs_per_s": n_cand / (ms_e2e * 1e-3),
            "timing": "CUDA events; device-resident meshes and fields, and (e2e) pinned host meshes and "
                      "fields with their copies"}


def p1_mass_cpu(dim, A, B):
    """The oracle's P1-P1 product (the reference's per-candidate clipping
    and quadrature, 1 host thread) on a corner-box sample of the workload
    with 1/64 of A's elements: candidate pairs per second, the search
    included."""
    import oracle

    As, Bs, desc = corner_sample(dim, A, B, frac=1.0 / 64)
    t0 = time.perf_counter()
    ip, ind = oracle.tree_finder(dim, As, Bs)
    oracle.p1_mass(dim, As, Bs, ip, ind, As[0][:, 0], Bs[0][:, 1])
    dt = time.perf_counter() - t0
    return {"value": len(ind) / dt, "unit": "pairs/s", "cores": 1, "kind": "port",
            "sample": f"{desc} ({len(ind)} candidates), oracle tree finder + P1 product, 1 thread, {dt:.2f} s"}


def elements_timing(ctx, dim, tA, tB, n_cand, stream, flush):
    """The supermesh's simplices themselves (libsupermesh_gpu_supermesh_elements:
    search, counting narrow phase, offsets, a second clipping pass writing
    every output simplex with its parents), device-resident meshes and
    outputs, reported beside the main metric.  CUDA events on the stream, L2
    flushed before each call, median of 5 after 2 warm-up calls."""
    import torch

    import libsupermesh_b200 as lsm

    sp = stream.cuda_stream
    probe = {}
    try:
        ctx.supermesh_elements_device(tA, tB, probe, stream=sp)
    except lsm.LsmError as e:
        if e.status != 3:
            raise
    nc, ne = probe["n_candidates"], probe["n_elements"]
    per = (3, 2) if dim == 2 else (4, 3)
    dev = tA[0].device
    out = {"elem_offset": torch.empty(nc + 1, dtype=torch.int64, device=dev),
           "elems": torch.empty((max(ne, 1),) + per, dtype=torch.float64, device=dev),
           "parent_a": torch.empty(max(ne, 1), dtype=torch.int64, device=dev),
           "parent_b": torch.empty(max(ne, 1), dtype=torch.int64, device=dev),
           "cand_capacity": nc, "elem_capacity": ne}
    for _ in range(2):
        ctx.supermesh_elements_device(tA, tB, out, stream=sp)
    ms = []
    for _ in range(5):
        flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.supermesh_elements_device(tA, tB, out, stream=sp)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = float(np.median(ms))
    nbytes = (nc + 1) * 8 + ne * (8 * per[0] * per[1] + 16)
    del out
    return {"ms": t, "n_elements": ne, "elements_per_s": ne / (t * 1e-3), "pairs_per_s": n_cand / (t * 1e-3),
            "output_bytes": nbytes,
            "timing": "CUDA events; device-resident meshes and outputs (simplices, per-candidate offsets, parents)"}


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
