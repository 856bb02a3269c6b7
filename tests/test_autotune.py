"""The autotuner's search, refusal rule and cache keying, on the host.

batch_search is replaced by a fake whose device time depends on the tuning
in force, so the test runs without a GPU: the tuner must pick the fastest
setting by coordinate descent, apply it to the context, cache it under a key
of (device, seed weight, transitions, workload), serve the next call from the
cache without timing anything, and refuse to tune when a setting changes the
HSPs."""
import json

import numpy as np
import pytest

P12 = "1110100110010101111"


class FakeCtx:
    device = 0

    def __init__(self):
        self.t = {"screen_warps": 8, "screen_cap": 192, "screen_blocks_per_sm": 4, "walk_warps": 8,
                  "max_hits_per_pass": 1 << 28, "initial_candidates": 0, "filter_cap": 96, "filter_claim": 256}
        self.applied = []

    def tuning(self):
        return dict(self.t)

    def set_tuning(self, **kw):
        self.t.update({k: v for k, v in kw.items() if v})
        self.applied.append(dict(kw))


class FakeTable:
    pattern = P12


class Params:
    def __init__(self, transitions=1):
        self.transitions = transitions


def fake_batch(ctx, cost, bad=None):
    calls = []

    def batch_search(tables, queries, units, matrix, params, stats=None, ctx=None):
        t = ctx.tuning()
        calls.append(dict(t))
        if stats is not None:
            stats["device_ms"] = cost(t)
        h = np.arange(8, dtype=np.uint32)
        if bad is not None and bad(t):
            h = h + 1
        return [h for _ in units]
    return batch_search, calls


def test_picks_fastest_and_caches(gxy, tmp_path, monkeypatch):
    from lastz_gxy_b200 import autotune as at
    ctx = FakeCtx()
    # Fastest at filter_claim 512, filter_cap 64, walk_warps 4.
    cost = lambda t: (10.0 - (t["filter_claim"] == 512) * 2 - (t["filter_cap"] == 64) - (t["walk_warps"] == 4) * 0.5)
    fn, calls = fake_batch(ctx, cost)
    monkeypatch.setattr(gxy, "batch_search", fn)
    cache = str(tmp_path / "tune.json")
    units = [(0, i, s) for i in range(40) for s in (0, 1)]
    e = at.autotune(ctx, [FakeTable()], [None], units, None, Params(1), workload="w", sample_units=16, reps=1,
                    cache=cache)
    assert e["tuning"]["filter_claim"] == 512 and e["tuning"]["filter_cap"] == 64 and e["tuning"]["walk_warps"] == 4
    assert ctx.t["filter_claim"] == 512 and ctx.t["filter_cap"] == 64
    assert e["sample_units"] == 16
    store = json.load(open(cache))
    key = at.tuning_key(ctx, P12, 1, "w")
    assert key.endswith("|w12|t1|w") and key in store
    # Second call: served from the cache, nothing timed.
    n = len(calls)
    ctx2 = FakeCtx()
    e2 = at.autotune(ctx2, [FakeTable()], [None], units, None, Params(1), workload="w", cache=cache)
    assert len(calls) == n and e2["tuning"] == e["tuning"] and ctx2.t["filter_claim"] == 512
    # Zero transitions is a different key: tuned afresh.
    at.autotune(FakeCtx(), [FakeTable()], [None], units, None, Params(0), workload="w", sample_units=16, reps=1,
                cache=cache)
    assert len(calls) > n
    assert at.tuning_key(ctx, P12, 0, "w") in json.load(open(cache))


def test_refuses_a_setting_that_changes_hsps(gxy, tmp_path, monkeypatch):
    from lastz_gxy_b200 import autotune as at
    ctx = FakeCtx()
    fn, _ = fake_batch(ctx, lambda t: 1.0, bad=lambda t: t["screen_cap"] == 128)
    monkeypatch.setattr(gxy, "batch_search", fn)
    with pytest.raises(RuntimeError, match="changed the HSPs"):
        at.autotune(ctx, [FakeTable()], [None], [(0, 0, 0)], None, Params(1), cache=str(tmp_path / "t.json"),
                    use_cache=False, reps=1)
