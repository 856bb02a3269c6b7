"""Autotuner for the batched seed->HSP launch.

The tunables are the screen kernel's block shape (warps per block) and
occupancy (blocks per SM, which also sets its register budget), the column cap
per side after which the lane screen hands a still-extending hit to the warp
extender, and the walk kernel's block shape.  The tuner times a sample of the
caller's units under each setting with the library's own CUDA-event counters,
keeps the fastest, applies it to the context and caches it in a JSON file
keyed by device, seed weight, transition count and workload class -- so the
one-transition and no-transition searches are tuned separately.
"""
from __future__ import annotations

import itertools
import json
import os
from typing import Optional

DEFAULT_SPACE = {
    "screen_warps": [8, 16],
    "screen_blocks_per_sm": [4, 3],
    "screen_cap": [192, 128, 64],
    "walk_warps": [8, 4],
}


def _cache_path(path: Optional[str]) -> str:
    if path:
        return path
    base = os.environ.get("XDG_CACHE_HOME", os.path.join(os.path.expanduser("~"), ".cache"))
    return os.path.join(base, "lastz_gxy_b200", "autotune.json")


def _device_name(ctx) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(ctx.device)
    except Exception:
        return f"cuda:{ctx.device}"


def tuning_key(ctx, pattern: str, transitions: int, workload: str) -> str:
    w = str(pattern).count("1")
    return f"{_device_name(ctx)}|w{w}|t{min(int(transitions), 2)}|{workload}"


def autotune(ctx, tables, queries, units, matrix, params, workload: str = "batch", space: Optional[dict] = None,
             sample_units: int = 512, reps: int = 2, cache: Optional[str] = None, use_cache: bool = True) -> dict:
    """Picks the fastest tuning for batch_search on (a sample of) these units and applies it."""
    from . import batch_search
    path = _cache_path(cache)
    key = tuning_key(ctx, tables[0].pattern, params.transitions, workload)
    store = {}
    if os.path.exists(path):
        try:
            with open(path) as f:
                store = json.load(f)
        except Exception:
            store = {}
    if use_cache and key in store:
        ctx.set_tuning(**store[key]["tuning"])
        return store[key]
    sp = space or DEFAULT_SPACE
    # A deterministic sample spread over the unit list.
    ul = list(units)
    step = max(1, len(ul) // max(1, sample_units))
    sample = ul[::step][:sample_units]
    names = list(sp)
    results = []
    ref = None
    for combo in itertools.product(*[sp[n] for n in names]):
        cfg = dict(zip(names, combo))
        ctx.set_tuning(**cfg)
        best = None
        for _ in range(reps):
            st = {}
            out = batch_search(tables, queries, sample, matrix, params, stats=st, ctx=ctx)
            best = st["device_ms"] if best is None else min(best, st["device_ms"])
        sig = [o.tobytes() for o in out]
        if ref is None:
            ref = sig
        elif sig != ref:
            raise RuntimeError(f"tuning {cfg} changed the HSPs; refusing to tune")
        results.append((best, cfg))
    results.sort(key=lambda x: x[0])
    best_ms, best_cfg = results[0]
    ctx.set_tuning(**best_cfg)
    entry = {"tuning": best_cfg, "device_ms": best_ms, "sample_units": len(sample),
             "tried": [{"ms": round(ms, 4), **cfg} for ms, cfg in results]}
    store[key] = entry
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(store, f, indent=1)
    except OSError:
        pass
    return entry
