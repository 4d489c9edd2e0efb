"""Autotuner for the supermesh library's launch shapes.

The tuning options (libsupermesh_gpu_set_option) change launch shapes and the
3D clipper variant, never results.  For a workload, `tune` times every
candidate setting of the relevant options on the GPU (CUDA events around the
full supermesh call, device-resident inputs, best of `reps` after a warm-up),
keeps the fastest, applies it, and stores it in a JSON cache keyed by GPU
name, dimension and problem size class, so later runs on the same kind of
workload apply the stored choice without timing (`apply_cached`).

Cache file: $LIBSUPERMESH_TUNING_CACHE, else
~/.cache/libsupermesh_b200/tuning.json.  Entries carry the library's kernel
source hash; a rebuilt library with different kernels ignores stale entries.
"""
from __future__ import annotations

import hashlib
import itertools
import json
import math
import os
from pathlib import Path

import libsupermesh_b200 as lsm

SPACE = {
    2: {"tri_blocks_per_sm": (4, 8, 16), "query_block": (64, 128, 256), "leaf_bucket": (1, 4, 8)},
    3: {"query_block": (64, 128, 256), "leaf_bucket": (1, 4, 8)},
}


def cache_path() -> Path:
    env = os.environ.get("LIBSUPERMESH_TUNING_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "libsupermesh_b200" / "tuning.json"


def _source_hash() -> str:
    h = hashlib.sha256()
    src = Path(__file__).resolve().parent / "csrc"
    for f in sorted(src.glob("*.cu*")) + sorted(src.glob("*.h")):
        h.update(f.read_bytes())
    return h.hexdigest()[:16]


def _key(dim: int, nel_a: int, nel_b: int) -> str:
    import torch

    gpu = torch.cuda.get_device_name(0) if torch.cuda.is_available() else "cpu"
    size_class = int(round(math.log2(max(1, nel_a + nel_b))))
    return f"{gpu}|dim{dim}|2^{size_class}"


def _load() -> dict:
    p = cache_path()
    if p.exists():
        try:
            return json.loads(p.read_text())
        except ValueError:
            return {}
    return {}


def _store(db: dict) -> None:
    p = cache_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_suffix(".tmp")
    tmp.write_text(json.dumps(db, indent=1, sort_keys=True))
    os.replace(tmp, p)


def apply(setting: dict) -> None:
    for k, v in setting.items():
        lsm.set_option(k, v)


def apply_cached(dim: int, nel_a: int, nel_b: int) -> dict | None:
    """Apply the stored choice for this kind of workload, if any."""
    entry = _load().get(_key(dim, nel_a, nel_b))
    if entry and entry.get("source") == _source_hash():
        apply(entry["setting"])
        return entry["setting"]
    return None


def tune(ctx, mesh_a, mesh_b, reps: int = 3, store: bool = True) -> dict:
    """Time every candidate setting on device-resident copies of the meshes
    (torch tensors on cuda:0); apply and return the fastest."""
    import torch

    dim = int(mesh_a[0].shape[1])
    dev = torch.device("cuda:0")
    ta = tuple(torch.as_tensor(x).to(dev) for x in mesh_a)
    tb = tuple(torch.as_tensor(x).to(dev) for x in mesh_b)
    stream = torch.cuda.current_stream()
    names = list(SPACE[dim])
    before = {n: lsm.get_option(n) for n in names}
    results = []
    ref = None
    for values in itertools.product(*(SPACE[dim][n] for n in names)):
        setting = dict(zip(names, values))
        apply(setting)
        ctx.supermesh(ta, tb, on_device=True, stream=stream.cuda_stream)  # warm-up
        best = math.inf
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st, _ = ctx.supermesh(ta, tb, on_device=True, stream=stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        sig = (st.n_candidates, st.n_intersecting, st.n_out_simplices)
        if ref is None:
            ref = sig
        elif sig != ref:  # settings must never change results
            apply(before)
            raise RuntimeError(f"setting {setting} changed the result: {sig} != {ref}")
        results.append((best, setting))
    results.sort(key=lambda r: r[0])
    best_ms, best_setting = results[0]
    apply(best_setting)
    if store:
        db = _load()
        db[_key(dim, len(mesh_a[1]), len(mesh_b[1]))] = {
            "setting": best_setting, "ms": best_ms, "source": _source_hash(),
            "tried": [{"ms": ms, "setting": s} for ms, s in results],
        }
        _store(db)
    return {"setting": best_setting, "ms": best_ms, "tried": len(results)}
