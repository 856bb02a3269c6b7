"""Autotuner for the batched seed->HSP launch.

The tunables:

* filter_claim -- raw hits a warp of the upper-bound filter claims at a time
  (the hits-per-warp batch: larger claims cost fewer atomics, smaller ones
  balance the warps better at the end of a launch; 1 sizes it from each
  launch's hit count);
* filter_cap -- columns per side after which the filter passes a hit on to
  the exact screen unexamined;
* screen_cap -- columns per side after which the exact lane screen hands a
  still-extending hit to the warp extender of the diagonal walk;
* screen_warps / screen_blocks_per_sm -- the exact screen's block shape and
  occupancy (blocks per SM also sets its register budget);
* walk_warps -- the diagonal walk's block shape.

The tuner times a sample of the caller's units with the library's own
CUDA-event counters, one parameter at a time (coordinate descent from the
context's current setting, `sweeps` passes over the parameters), keeps the
fastest, applies it to the context and caches it in a JSON file keyed by
device, seed weight, transition count and workload class -- so the
one-transition and no-transition searches are tuned separately.  Every
setting must give the same HSPs as the first one timed; a setting that does
not is refused and the tuner raises.
"""
from __future__ import annotations

import json
import os
from typing import Optional

DEFAULT_SPACE = {
    "filter_claim": [1, 128, 512],
    "filter_cap": [96, 64, 160],
    "screen_cap": [192, 128],
    "screen_warps": [8, 16],
    "screen_blocks_per_sm": [4, 3],
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
             sample_units: int = 512, reps: int = 2, cache: Optional[str] = None, use_cache: bool = True,
             sweeps: int = 1) -> dict:
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
    cur = ctx.tuning()
    cfg = {n: cur[n] for n in sp}
    timed = {}
    ref = None

    def run(c: dict) -> float:
        nonlocal ref
        k = tuple(sorted(c.items()))
        if k in timed:
            return timed[k]
        ctx.set_tuning(**c)
        best = None
        out = None
        for _ in range(max(1, reps)):
            st = {}
            out = batch_search(tables, queries, sample, matrix, params, stats=st, ctx=ctx)
            best = st["device_ms"] if best is None else min(best, st["device_ms"])
        sig = [o.tobytes() for o in out]
        if ref is None:
            ref = sig
        elif sig != ref:
            raise RuntimeError(f"tuning {c} changed the HSPs; refusing to tune")
        timed[k] = best
        return best

    best_ms = run(cfg)
    for _ in range(max(1, sweeps)):
        for name in sp:
            for v in sp[name]:
                trial = dict(cfg, **{name: v})
                ms = run(trial)
                if ms < best_ms:
                    best_ms, cfg = ms, trial
    ctx.set_tuning(**cfg)
    entry = {"tuning": cfg, "device_ms": best_ms, "sample_units": len(sample),
             "tried": [{"ms": round(ms, 4), **dict(k)} for k, ms in sorted(timed.items(), key=lambda x: x[1])]}
    store[key] = entry
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(store, f, indent=1)
    except OSError:
        pass
    return entry
