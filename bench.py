"""Seed->HSP throughput on B200 (Mbp^2/s), one JSON line on rank 0.

Workload (default): the 10 Mbp chromosome-scale plain configuration -- a 10 Mbp
target at 41% GC with 2,000 planted repeat families, 45% soft-masked, 20
N-blocks, against a query evolved from it to ~70% identity; seed 12of19 with
one transition, HOXD70, xdrop 910, hspthresh 3000, both strands.  One step is
the reference driver's per-(target, query) work: PosTable::build on the target,
the reverse complement of the query, and one search() launch per strand.

    Mbp^2 = (target Mbp) x (query Mbp) x (strands)

value: device-resident inputs, CUDA-event time of each step on the library's
primary stream, L2 flushed between steps (the step's working set, ~100 MB,
fits in the 126 MB L2).  e2e: the same step through the public C ABI from host
buffers (target and query PackedSeq copied in from pinned host memory each
step, the query from a second host thread while the table builds; HSPs
copied out).  The two strands' search() calls run concurrently
from two host threads, each on its own stream, as the reference's driver
runs its (chunk, query, strand) units in parallel on a shared table.

Multi-GPU (torchrun): every rank runs its own independent copy of the workload
(a different synthetic chromosome per rank, no collective on the data path);
value is all ranks' Mbp^2 over the slowest rank's time ("scaling": "weak").
--impl reference times the reference's CPU path (the oracle's AVX2 restatement
of seed_search / PosTable, src/hsp_simd.rs via src/hsp.rs:66-87) on host cores.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
P12 = "1110100110010101111"
L2_BYTES = 126 * 1024 * 1024


def _pkg():
    if "lastz_gxy_b200" in sys.modules:
        return sys.modules["lastz_gxy_b200"]
    d = os.path.join(ROOT, "lastz-gxy_b200")
    spec = importlib.util.spec_from_file_location("lastz_gxy_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["lastz_gxy_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM read + write bytes per launch of the search kernels, measured by
    ncu on the plain workload's plus-strand search (profiles/kernel_traffic.json,
    with the command that made it); None when the file is absent."""
    p = os.path.join(ROOT, "profiles", "kernel_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


def measured_traffic(tr, kernel: str, raw_by_strand):
    """(bytes, source) of `kernel` per launch, averaged over the strands'
    launches like the achieved rate: a strand whose launch is the one ncu
    captured (same raw hits: the plus strand of this workload) takes the
    measured bytes; any other takes them scaled by its raw hits."""
    if not tr or kernel not in tr.get("kernels", {}):
        return None, None
    k = tr["kernels"][kernel]
    b = k["dram_read_bytes"] + k["dram_write_bytes"]
    vals, exact = [], 0
    for raw in raw_by_strand:
        if tr.get("raw_hits") == int(round(raw)):
            vals.append(b)
            exact += 1
        else:
            vals.append(b * raw / tr["raw_hits"])
    src = "ncu dram__bytes_read.sum + dram__bytes_write.sum (profiles/kernel_traffic.json)"
    if exact == len(vals):
        return int(sum(vals) / len(vals)), f"measured: {src} of this launch ({tr['workload']})"
    if exact:
        return int(sum(vals) / len(vals)), (f"mean over the strands' launches: measured for the plus strand ({src}, "
                                            f"{tr['workload']}), the minus strand's scaled by its raw hits")
    return int(sum(vals) / len(vals)), f"ESTIMATE: {src} scaled by raw hits"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, nm in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def workload(rank: int):
    _pkg()
    from lastz_gxy_b200 import synth
    pr = synth.c2(seed=2 + rank)
    return pr.target.tobytes(), pr.query.tobytes()


def mbp2(lt: int, lq: int, strands: int = 2) -> float:
    return (lt / 1e6) * (lq / 1e6) * strands


def screen_bytes(st: dict, seed_len: int) -> float:
    """Algorithmic bytes of one exact-screen launch: 12 B per surviving hit
    read (t, q, unit), 3/8 B x 2 per examined column -- codes + valid bits of
    both sequences over the seed footprint and the columns both sides
    scanned, break columns included -- and 44 B per candidate written
    (record, key, index)."""
    cols = st["columns"] + seed_len * st["survivors"]
    return 12.0 * st["survivors"] + 0.75 * cols + 44.0 * st["candidates"]


def filter_bytes(st: dict) -> float:
    """Algorithmic bytes of one upper-bound filter launch: 12 B per raw hit
    read, 3/8 B x 2 per column it scanned on the two sides (codes + valid bits
    of both sequences), 12 B per survivor written."""
    return 12.0 * st["raw_hits"] + 0.75 * st["filter_columns"] + 12.0 * st["survivors"]


def enum_bytes(st: dict, lq: int, n_var: int) -> float:
    """Algorithmic bytes of one enumeration launch: 0.5 B/bp of query read,
    8 B of starts per (seedable window, variant), 4 B of positions per raw hit,
    12 B per raw hit written."""
    return 0.5 * lq + 8.0 * n_var * st["windows"] + 16.0 * st["raw_hits"]


def table_bytes(npos: int, lt: int, weight: int = 12) -> float:
    """Algorithmic bytes of PosTable::build over lt bases: the sequence read
    once (2-bit codes + valid + mask bits = 0.5 B/bp), the positions written
    (4 B each) and the bucket starts written (4 B x (4^w + 1)) with the
    occupancy bitmap (4^w / 8 B) -- what any build must move."""
    nw = 1 << (2 * weight)
    return 0.5 * lt + 4.0 * npos + 4.0 * (nw + 1) + nw / 8.0


def table_roofline(ms_list, npos, lt: int, peak: float, views: int = 1, workload: str = "", traffic=None) -> dict:
    """PosTable::build on the device (counts, scan, fill through atomic
    cursors, in-bucket sorts) against table_bytes; time = CUDA events around
    the whole build call (allocation and the host sync included).  For a
    multi-view build npos is a list of (positions, bp)."""
    ms = statistics.median(ms_list)
    b = sum(table_bytes(n, l) for n, l in npos) if views > 1 else table_bytes(npos if npos else lt, lt)
    ach = b / (ms / 1e3) / 1e9
    out = {"bound": "hbm", "kernel": "table build (k_count_words + scan + k_fill_buckets + "
                                     "k_sort_small_buckets / k_sort_block_buckets)",
           "achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
           "build_ms": round(ms, 3), "algorithmic_bytes": int(b)}
    if workload:
        out["workload"] = workload
    if traffic and "table_build" in traffic:
        tb = traffic["table_build"]
        out["traffic"] = int(sum(k["dram_read_bytes"] + k["dram_write_bytes"] for k in tb["kernels"].values()))
        out["traffic_source"] = "measured: ncu DRAM bytes of the build's count, scan, fill and bucket-pass kernels " \
                                "(profiles/kernel_traffic.json, %s)" % tb["workload"]
    return out


def run_ours(args, rank: int, world: int, device: int):
    import torch
    g = _pkg()
    torch.cuda.set_device(device)
    ctx = g.Context(device)
    tgt, qry = workload(rank)
    T = g.PackedSeq.from_ascii(tgt)
    Q = g.PackedSeq.from_ascii(qry)
    lt, lq = len(T), len(Q)
    m, sp = g.ScoringMatrix.hoxd70(), g.SearchParams()
    n_var = 1 + 12
    dT = T.to_device(ctx)
    dQ = Q.to_device(ctx)
    flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device=f"cuda:{device}")

    # The end-to-end leg reads its inputs from pinned host memory (page-locked
    # buffers, as a loader that feeds the device would hold them).
    keep = []

    def pinned(s):
        arrs = []
        for a in (s.codes, s.valid, s.mask):
            t = torch.empty(len(a), dtype=torch.uint8, pin_memory=True)
            keep.append(t)
            v = t.numpy()
            v[:] = a
            arrs.append(v)
        return g.PackedSeq(arrs[0], arrs[1], arrs[2], len(s))

    T, Q = pinned(T), pinned(Q)

    # The two strands' search() calls run concurrently, one per host thread
    # (each call on its own stream), as the reference's driver runs its
    # (chunk, query, strand) units in parallel on one shared table.
    from concurrent.futures import ThreadPoolExecutor
    pool = ThreadPoolExecutor(max_workers=1)

    def both_strands(tab, qs):
        def run(q):
            st = {}
            h = g.search_device(tab, q, m, sp, stats=st)
            return st, h
        f = pool.submit(run, qs[1])
        r0 = run(qs[0])
        return [r0, f.result()]

    def step_device(collect, concurrent=True):
        ctx.mark(2)
        tab = g.PosTable.build(dT, P12, 1, ctx=ctx)
        ctx.mark(3)
        if not table_npos:
            table_npos.append(tab.total_positions())
        dQr = dQ.reverse_complement()
        if concurrent:
            res = both_strands(tab, (dQ, dQr))
        else:
            res = []
            for q in (dQ, dQr):
                st = {}
                h = g.search_device(tab, q, m, sp, stats=st)
                res.append((st, h))
        for st, h in res:
            collect.append((st, len(h)))
        dQr.free()
        tab.free()
        table_ms.append(ctx.elapsed_ms(2, 3))   # read after the frees (which synchronise) so no extra wait

    def step_e2e(collect):
        fq = pool.submit(Q.to_device, ctx)                    # host query -> device (second thread)
        tab = g.PosTable.build(T, P12, 1, ctx=ctx)          # host target -> device, PosTable::build
        dq = fq.result()
        dqr = dq.reverse_complement()
        n = 0
        for _, h in both_strands(tab, (dq, dqr)):             # HSPs come back to host
            n += len(h)
        collect.append(n)
        dqr.free()
        dq.free()
        tab.free()

    def timed(fn, k, flush_l2=True):
        times, col = [], []
        for _ in range(k):
            if flush_l2:
                flush.zero_()
            torch.cuda.synchronize(device)
            ctx.mark(0)
            fn(col)
            ctx.mark(1)
            times.append(ctx.elapsed_ms(0, 1))
        return times, col

    table_ms, table_npos = [], []
    barrier = (lambda: torch.distributed.barrier()) if world > 1 else (lambda: None)
    for _ in range(args.warmup):
        step_device([])
        step_e2e([])
    launches0 = g.lib().gxy_kernel_launches()
    with ClockSampler(device) as clk:
        barrier()
        torch.cuda.synchronize(device)
        dev_times, dev_col = timed(step_device, args.steps)
        torch.cuda.synchronize(device)
        barrier()
        launches = (g.lib().gxy_kernel_launches() - launches0) // args.steps
        e2e_times, e2e_col = timed(step_e2e, args.steps)
        torch.cuda.synchronize(device)
        barrier()
    # Kernel durations with the strands one after the other (outside the
    # timed region): each kernel then has the device to itself.
    _, ser_col = timed(lambda c: step_device(c, concurrent=False), 3)
    total_ms = sum(dev_times)
    e2e_ms = sum(e2e_times)
    if world > 1:
        t = torch.tensor([total_ms, e2e_ms], dtype=torch.float64, device=f"cuda:{device}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms, e2e_ms = float(t[0]), float(t[1])
    per_step = mbp2(lt, lq)
    value = world * per_step * args.steps / (total_ms / 1e3)
    e2e_value = world * per_step * args.steps / (e2e_ms / 1e3)
    # Rooflines of the three search kernels from the timed steps (the two
    # strands share the device there) and alone (one launch at a time, after
    # the timed steps); the dominant kernel is the one with the most time alone.
    stats = [s for s, _ in dev_col]
    ser = [s for s, _ in ser_col]
    peak, peak_kind = peaks()
    tr = profiled_traffic()
    raw = statistics.mean(s["raw_hits"] for s in stats)
    kern = {}
    for name, key, fb in (("k_enumerate", "enum_ms", lambda s: enum_bytes(s, lq, n_var)),
                          ("k_filter_hits", "filter_ms", filter_bytes),
                          ("k_screen", "screen_ms", lambda s: screen_bytes(s, 19))):
        ms = statistics.mean(s[key] for s in stats)
        ms_alone = statistics.mean(s[key] for s in ser)
        if ms <= 0 or ms_alone <= 0:
            continue   # not timed (a multi-pass launch)
        byt = statistics.mean(fb(s) for s in stats)
        traffic, tsrc = measured_traffic(tr, name, [statistics.mean(x["raw_hits"] for x in stats[0::2]),
                                                    statistics.mean(x["raw_hits"] for x in stats[1::2])])
        kern[name] = {"bound": "hbm", "kernel": name, "achieved": round(byt / (ms / 1e3) / 1e9, 1),
                      "peak": peak, "unit": "GB/s", "frac": round(byt / (ms / 1e3) / 1e9 / peak, 4),
                      "traffic": traffic, "traffic_source": tsrc,
                      "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                      else "fallback 6.65 TB/s",
                      "kernel_ms": round(ms, 3), "algorithmic_bytes_per_launch": int(byt),
                      "timing": "CUDA events around each launch on its stream in the timed steps, where the other "
                                "strand's search shares the device",
                      "alone": {"kernel_ms": round(ms_alone, 3), "achieved": round(byt / (ms_alone / 1e3) / 1e9, 1),
                                "frac": round(byt / (ms_alone / 1e3) / 1e9 / peak, 4),
                                "timing": "the same launches one at a time after the timed steps"}}
    dominant = max(kern, key=lambda k: kern[k]["kernel_ms"])
    nh = sum(n for _, n in dev_col) / args.steps
    h2d = (T.codes.nbytes + T.valid.nbytes + T.mask.nbytes) + (Q.codes.nbytes + Q.valid.nbytes + Q.mask.nbytes)
    d2h = int(sum(e2e_col) / args.steps) * 16
    out = {
        "metric": "seed->HSP Mbp^2/s (12of19 + 1 transition, HOXD70 910/3000, both strands, bit-exact)",
        "value": round(value, 2), "unit": "Mbp^2/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator, lastz_gxy_b200/synth.py)",
        "config": {"workload": "plain 10 Mbp target x 10 Mbp query at ~70% identity, one launch per (target, strand)",
                   "target_bp": lt, "query_bp": lq, "strands": 2, "seed": "12of19", "transitions": 1,
                   "step": "PosTable::build + reverse complement + 2 search() launches, the two strands "
                           "concurrently from two host threads (the driver runs its units in parallel)",
                   "mbp2_per_step": round(per_step, 4), "l2": "flushed between timed steps (256 MB write)",
                   "parallelism": f"replicas x{world}"},
        "seed_hits_per_s": round(world * raw * 2 * args.steps / (total_ms / 1e3), 1),
        "hsps_per_s": round(world * nh * args.steps / (total_ms / 1e3), 1),
        "e2e": {"value": round(e2e_value, 2), "unit": "Mbp^2/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_ms / args.steps, 3),
                "host_buffers": "pinned PackedSeq arrays in, HSP arrays out"},
        "gpu_launches": int(launches * args.steps),
        "roofline": kern[dominant],
        "roofline_kernels": kern,
        "roofline_table": table_roofline(table_ms[-args.steps:], table_npos[-1], lt, peak, traffic=tr),
        "filter": {"survivors_per_raw_hit": round(statistics.mean(s["survivors"] / max(1, s["raw_hits"]) for s in stats), 5),
                   "candidates_per_survivor": round(statistics.mean(s["candidates"] / max(1, s["survivors"]) for s in stats), 4)},
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(tgt, qry)
    return out


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _cpu_run(O, T, tab, qry: bytes, sample_bp: int, threads: int, t_table: float, lt: int, lq: int) -> dict:
    """search() of the first sample_bp of the query on both strands: the
    sample is cut into one slice per thread (at least one), and every
    (slice, strand) pair is a unit on the thread pool; the table build is
    charged by the share of the query the sample covers."""
    n_slices = max(1, threads)
    step = (sample_bp + n_slices - 1) // n_slices
    units = []
    for lo in range(0, sample_bp, step):
        qs = O.pack_ascii(qry[lo:min(sample_bp, lo + step)])
        units += [(tab, T, qs), (tab, T, O.reverse_complement(qs))]
    p = O.params()
    t0 = time.perf_counter()
    O.search_units(units, p, avx2=True, threads=threads)
    t_search = time.perf_counter() - t0
    frac = sample_bp / lq
    secs = t_search + t_table * frac
    return {"value": round(mbp2(lt, sample_bp) / secs, 3), "unit": "Mbp^2/s", "cores": threads, "kind": "port",
            "sample": f"PosTable::build of the full {lt} bp target (1 thread, charged x{frac:.3f}) + search() of "
                      f"the first {sample_bp} bp of the query, both strands, in {len(units)} (slice, strand) units "
                      f"on {threads} thread(s); table {t_table:.2f}s, search {t_search:.2f}s"}


def cpu_baseline(tgt: bytes, qry: bytes, modes=("all_cores", "reference_faithful"), sample_1t: int = 2_000_000) -> dict:
    """The oracle's AVX2 restatement of the reference path (src/hsp_simd.rs
    through src/hsp.rs:66-87, seed_search / PosTable) on the host cores, on
    bounded samples of the workload, in two modes:

    reference_faithful: one thread.  The reference's driver parallelises over
      target chunks only (src/driver.rs:210, rayon par_iter over chunks), and
      this unchunked 10 Mbp target is one chunk, so its query strands run one
      after the other on one thread.  Sample: the first 2 Mbp of the query.
    all_cores: every host thread this process may use, over (query slice,
      strand) units.  Sample: max(2 Mbp, 0.5 Mbp per thread) of the query, up
      to all of it.

    The top-level fields are the all-cores mode (the stronger baseline)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    T = O.pack_ascii(tgt)
    t0 = time.perf_counter()
    tab = O.Table(T, P12, 1)
    t_table = time.perf_counter() - t0
    lt, lq = len(tgt), len(qry)
    out = {}
    nt = host_threads()
    if "all_cores" in modes:
        s = min(lq, max(2_000_000, 500_000 * nt))
        out["all_cores"] = _cpu_run(O, T, tab, qry, s, nt, t_table, lt, lq)
    if "reference_faithful" in modes:
        out["reference_faithful"] = _cpu_run(O, T, tab, qry, min(lq, sample_1t), 1, t_table, lt, lq)
    top = out.get("all_cores") or out["reference_faithful"]
    return {**top, "modes": out}


def run_reference(args):
    """--impl reference: the reference's CPU path (the oracle's AVX2 port) on
    the same workload, with every host thread; each step is the all-cores
    sample, and the one-thread reference-faithful mode is measured once."""
    tgt, qry = workload(0)
    vals = []
    faithful = None
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(tgt, qry, modes=("all_cores",))
        if i >= args.warmup:
            vals.append(r)
    faithful = cpu_baseline(tgt, qry, modes=("reference_faithful",))["modes"]["reference_faithful"]
    v = statistics.mean(x["value"] for x in vals)
    s = vals[0]["modes"]["all_cores"]
    return {
        "impl": "reference",
        "metric": "seed->HSP Mbp^2/s (12of19 + 1 transition, HOXD70 910/3000, both strands, bit-exact)",
        "value": round(v, 3), "unit": "Mbp^2/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(mbp2(len(tgt), len(qry)) / v * 1e3, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator, lastz_gxy_b200/synth.py)",
        "config": {"workload": "plain 10 Mbp target x 10 Mbp query at ~70% identity, one launch per (target, strand)",
                   "target_bp": len(tgt), "query_bp": len(qry), "strands": 2,
                   "ms_per_step": "the full workload's time at the measured rate"},
        "cpu_baseline": {"value": round(v, 3), "unit": "Mbp^2/s", "cores": s["cores"], "kind": "port",
                         "sample": s["sample"], "modes": {"all_cores": {**s, "value": round(v, 3)},
                                                          "reference_faithful": faithful}},
        "e2e": {"value": round(v, 3), "unit": "Mbp^2/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_batched(args):
    """Uneven batch: one 50 Mbp chromosome-style target and 4,096 log-normal query
    contigs (~200 Mbp), both strands -- one batched launch per pass against the
    plain per-(query, strand) search() loop on the same GPU; results must match."""
    import torch
    g = _pkg()
    from lastz_gxy_b200 import synth
    from lastz_gxy_b200.autotune import autotune
    s = args.scale
    t0 = time.time()
    tgt, queries = synth.c3(target_len=int(50_000_000 * s), n_queries=max(8, int(4096 * s)),
                            total=int(200_000_000 * s))
    gen_s = time.time() - t0
    ctx = g.Context(0)
    m, sp = g.ScoringMatrix.hoxd70(), g.SearchParams()
    dT = g.PackedSeq.from_ascii(tgt.tobytes()).to_device(ctx)
    ctx.mark(0)
    tab = g.PosTable.build(dT, P12, 1, ctx=ctx)
    ctx.mark(1)
    table_ms = ctx.elapsed_ms(0, 1)
    dq = [g.PackedSeq.from_ascii(q.tobytes()).to_device(ctx) for q in queries]
    units = [(0, qi, st) for qi in range(len(queries)) for st in (0, 1)]
    tune = autotune(ctx, [tab], dq, units, m, sp, workload="uneven-batch", sample_units=256, use_cache=False)
    # Batched: every unit in one call (graph-captured when it fits one pass).
    batched = None
    b_times = []
    b_steps, b_warm = max(1, min(args.steps, 5)), max(1, min(args.warmup, 3))
    for i in range(b_warm + b_steps):
        torch.cuda.synchronize()
        st = {}
        ctx.mark(2)
        out = g.batch_search([tab], dq, units, m, sp, use_graph=True, stats=st, ctx=ctx)
        ctx.mark(3)
        if i >= b_warm:
            b_times.append(ctx.elapsed_ms(2, 3))
        batched = (out, st)
    # Plain: the driver's loop, one search() per (query, strand), reverse complement per query.
    plain = []
    ctx.mark(4)
    for q in dq:
        qr = q.reverse_complement()
        plain.append(g.search_device(tab, q, m, sp))
        plain.append(g.search_device(tab, qr, m, sp))
        qr.free()
    ctx.mark(5)
    plain_ms = ctx.elapsed_ms(4, 5)
    same = all(a.tobytes() == b.tobytes() for a, b in zip(batched[0], plain))
    lt = len(tgt)
    mbp2_total = sum(mbp2(lt, len(q), 1) for q in queries) * 2
    b_ms = statistics.mean(b_times)
    st = batched[1]
    return {
        "workload": "uneven batch: %d bp target x %d query contigs (%d bp, log-normal), both strands"
                    % (lt, len(queries), sum(len(q) for q in queries)),
        "metric": "seed->HSP Mbp^2/s", "unit": "Mbp^2/s", "mbp2": round(mbp2_total, 2),
        "batched": {"value": round(mbp2_total / (b_ms / 1e3), 2), "ms": round(b_ms, 2), "steps": b_steps,
                    "passes": st.get("passes"), "raw_hits": st["raw_hits"], "candidates": st["candidates"],
                    "hsps": st["hsps"]},
        "plain": {"value": round(mbp2_total / (plain_ms / 1e3), 2), "ms": round(plain_ms, 2),
                  "launches": 2 * len(queries)},
        "speedup_batched_vs_plain": round(plain_ms / b_ms, 3),
        "bit_identical": same, "table_ms": round(table_ms, 3), "generate_s": round(gen_s, 1),
        "autotune": tune["tuning"],
    }


def batched_summary(r: dict) -> dict:
    """The uneven-batch leg of the default bench line."""
    return {"workload": r["workload"], "metric": "seed->HSP Mbp^2/s", "unit": "Mbp^2/s", "mbp2": r["mbp2"],
            "value": r["batched"]["value"], "ms": r["batched"]["ms"], "steps": r["batched"]["steps"],
            "passes": r["batched"]["passes"], "plain_loop": r["plain"],
            "ratio_batched_vs_plain": r["speedup_batched_vs_plain"], "same": r["bit_identical"],
            "same_means": "every unit's HSP array of the batched launch equals the plain search() of that unit",
            "autotune": r["autotune"]}


def served_summary(r: dict) -> dict:
    """The serving leg of the default bench line."""
    return {"workload": r["workload"], "mbp2": r["mbp2"], "served": r["served"], "serial_plain": r["serial_plain"],
            "p99_ratio_serial_vs_served": round(r["serial_plain"]["p99_ms"] / r["served"]["p99_ms"], 3)
            if r["served"]["p99_ms"] else None,
            "same": r["bit_identical"], "latency": r["latency"]}


def _pct(v, q):
    import numpy as np
    return round(float(np.percentile(np.asarray(v), q)), 2) if len(v) else None


def replay_served(g, srv, reqs, packed):
    """Replays the arrival trace in real time against a Server; returns
    (results, latencies_ms, makespan_s).  Latency = submit -> HSPs on the host."""
    ids = [None] * len(reqs)
    res = [None] * len(reqs)
    lat = [None] * len(reqs)
    done_t = [0.0] * len(reqs)
    cv = threading.Condition()

    def waiter():
        # Blocks (no polling) until request i is submitted, then on its result,
        # as the serial arm's worker does.
        for i in range(len(reqs)):
            with cv:
                cv.wait_for(lambda: ids[i] is not None)
            p, mi, l = srv.wait(ids[i], timeout_ms=600_000)
            res[i], lat[i] = (p, mi), l
            done_t[i] = time.perf_counter()
    w = threading.Thread(target=waiter)
    w.start()
    start = time.perf_counter()
    for i, r in enumerate(reqs):
        d = start + r.arrival_s - reqs[0].arrival_s - time.perf_counter()
        if d > 0:
            time.sleep(d)
        rid = srv.submit(r.target, packed[i])
        with cv:
            ids[i] = rid
            cv.notify()
    w.join()
    return res, lat, max(done_t) - start


def replay_serial(g, ctx, tabs, reqs, packed, m, sp):
    """The same trace served FIFO by plain per-pair launches, one request at a
    time, in real time: a worker thread takes each request once it has arrived
    and runs search() on both strands (host query in, HSPs out).  Returns
    (results, latencies_ms, makespan_s, device_service_ms)."""
    res = [None] * len(reqs)
    lat = [None] * len(reqs)
    service = [None] * len(reqs)
    arrive = [None] * len(reqs)
    cv = threading.Condition()

    def serve(i, r):
        dq = packed[i].to_device(ctx)
        dqr = dq.reverse_complement()
        p = g.search_device(tabs[r.target], dq, m, sp)
        mi = g.search_device(tabs[r.target], dqr, m, sp)
        dqr.free()
        dq.free()
        return p, mi

    # The same warm-up as the served arm: the trace's largest request, once.
    big = max(range(len(reqs)), key=lambda i: len(reqs[i].query))
    serve(big, reqs[big])

    def worker():
        for i, r in enumerate(reqs):
            with cv:
                cv.wait_for(lambda: arrive[i] is not None)
            ctx.mark(6)
            p, mi = serve(i, r)
            ctx.mark(7)
            res[i] = (p, mi)
            lat[i] = (time.perf_counter() - arrive[i]) * 1e3
            service[i] = ctx.elapsed_ms(6, 7)
    w = threading.Thread(target=worker)
    w.start()
    start = time.perf_counter()
    for i, r in enumerate(reqs):
        d = start + r.arrival_s - reqs[0].arrival_s - time.perf_counter()
        if d > 0:
            time.sleep(d)
        with cv:
            arrive[i] = time.perf_counter()
            cv.notify()
    w.join()
    return res, lat, max(arrive[i] + lat[i] / 1e3 for i in range(len(reqs))) - start, service


def served_setup(args):
    g = _pkg()
    from lastz_gxy_b200 import synth
    s = args.scale
    t0 = time.time()
    targets = synth.c5_targets(length=int(100_000_000 * s))
    reqs = synth.c5_requests(targets, n_requests=args.requests, hi=int(5_000_000 * min(1.0, s * 2)) or 10_001)
    gen_s = time.time() - t0
    ctx = g.Context(0)
    m, sp = g.ScoringMatrix.hoxd70(), g.SearchParams()
    tabs = [g.PosTable.build(g.PackedSeq.from_ascii(t.tobytes()).to_device(ctx), P12, 1, ctx=ctx) for t in targets]
    packed = [g.PackedSeq.from_ascii(r.query.tobytes()) for r in reqs]
    return g, ctx, targets, reqs, tabs, packed, m, sp, gen_s


def served_run(g, tabs, reqs, packed, m, sp, streams, batch_units, batch_bases):
    # Every dispatcher sizes its buffers for the trace's largest request at
    # start (warm_bases), then runs that request once.
    big = max(range(len(reqs)), key=lambda i: len(reqs[i].query))
    srv = g.Server(tabs, m, sp, max_streams=streams, max_batch_units=batch_units, max_batch_bases=batch_bases,
                   warm_bases=len(reqs[big].query))
    try:
        for rid in [srv.submit(reqs[big].target, packed[big]) for _ in range(streams)]:
            srv.wait(rid)
        res, lat, span = replay_served(g, srv, reqs, packed)
        return res, lat, span, srv.stats()
    finally:
        srv.close()


def run_served(args):
    """Serving: three resident chromosome-style targets; requests arrive as a
    Poisson process (50/s, seed 7), each a target slice of log-uniform length
    10 kbp-5 Mbp evolved to 60-95% identity, searched on both strands.  The
    arrival trace is replayed in real time against the serving loop, and again
    against serial plain launches (FIFO, one request at a time); both
    latencies are wall clock from arrival to HSPs on the host.  HSPs must match."""
    g, ctx, targets, reqs, tabs, packed, m, sp, gen_s = served_setup(args)
    mbp2_total = sum(mbp2(len(targets[r.target]), len(r.query), 2) for r in reqs)
    res, lat, makespan, st = served_run(g, tabs, reqs, packed, m, sp, args.streams, args.batch_units,
                                        args.batch_bases)
    sres, slat, sspan, service = replay_serial(g, ctx, tabs, reqs, packed, m, sp)
    same = all(a[0].tobytes() == b[0].tobytes() and a[1].tobytes() == b[1].tobytes() for a, b in zip(res, sres))
    return {
        "workload": "serving: %d resident targets of %d bp, %d requests, Poisson %.0f/s (seed 7), both strands"
                    % (len(targets), len(targets[0]), len(reqs), 50.0),
        "mbp2": round(mbp2_total, 2), "query_bp": sum(len(r.query) for r in reqs),
        "served": {"value": round(mbp2_total / makespan, 2), "unit": "Mbp^2/s", "makespan_s": round(makespan, 3),
                   "p50_ms": _pct(lat, 50), "p99_ms": _pct(lat, 99), "p999_ms": _pct(lat, 99.9),
                   "batches": st["batches"], "max_inflight_units": st["max_inflight_units"],
                   "streams": args.streams, "max_batch_units": args.batch_units, "max_batch_bases": args.batch_bases},
        "serial_plain": {"value": round(mbp2_total / sspan, 2), "unit": "Mbp^2/s",
                         "makespan_s": round(sspan, 3), "p50_ms": _pct(slat, 50),
                         "p99_ms": _pct(slat, 99), "p999_ms": _pct(slat, 99.9),
                         "mean_device_service_ms": round(statistics.mean(service), 2)},
        "bit_identical": same, "generate_s": round(gen_s, 1),
        "latency": "arrival -> HSPs back on the host, wall clock, both arms",
    }


def run_chunked(args):
    """Chunked single chromosome: a chromosome-style target and a query evolved
    to ~70% identity, split by --chunk-size 10,000,000 --halo 50,000 into chunks
    with resident tables; all (chunk, strand) units in batched launches, with the
    driver's primary-region filter, against plain per-(chunk, strand) launches.
    Transitions 1 and 0 are tuned and timed separately."""
    import numpy as np
    g = _pkg()
    from lastz_gxy_b200 import synth
    from lastz_gxy_b200.autotune import autotune
    s = args.scale
    t0 = time.time()
    pr = synth.c4(length=int(250_000_000 * s), families=max(1, int(30_000 * s)), nblocks=max(1, int(500 * s)))
    gen_s = time.time() - t0
    ctx = g.Context(0)
    m = g.ScoringMatrix.hoxd70()
    dT = g.PackedSeq.from_ascii(pr.target.tobytes()).to_device(ctx)
    dQ = g.PackedSeq.from_ascii(pr.query.tobytes()).to_device(ctx)
    chunks = g.chunk_target(len(pr.target), 10_000_000, 50_000)
    # One chunk's table alone (timed three times), then every chunk's table
    # from one build (one count, scan, fill and bucket sort over all chunks).
    mid = chunks[len(chunks) // 2]
    one_ms = []
    for _ in range(3):
        ctx.mark(8)
        t1 = g.PosTable.build_view(dT, mid[0], mid[1], P12, 1, ctx=ctx)
        ctx.mark(9)
        one_ms.append(ctx.elapsed_ms(8, 9))
        one_npos = t1.total_positions()
        t1.free()
    # The first build of all chunks also grows the device pool by the
    # gigabytes of its starts and counts; the second is the build itself.
    views_ms = []
    for rep in range(2):
        ctx.mark(8)
        tabs = g.PosTable.build_views(dT, [(lo, hi) for lo, hi, _, _ in chunks], P12, 1, ctx=ctx)
        ctx.mark(9)
        views_ms.append(ctx.elapsed_ms(8, 9))
        if rep == 0:
            for t in tabs:
                t.free()
    table_ms = views_ms[-1]
    pk = peaks()[0]
    tab_roof = {"one_chunk": table_roofline(one_ms, one_npos, mid[1] - mid[0], pk,
                                            workload="chunk %d..%d (%d bp)" % (mid[0], mid[1], mid[1] - mid[0])),
                "all_chunks": table_roofline([table_ms], [(t.total_positions(), hi - lo) for t, (lo, hi, _, _) in
                                                          zip(tabs, chunks)], 0, pk, views=len(chunks),
                                             workload="%d chunk tables from one build" % len(chunks))}
    units = [(ci, 0, st, chunks[ci][2], chunks[ci][3]) for ci in range(len(chunks)) for st in (0, 1)]
    mbp2_total = sum(mbp2(c[3] - c[2], len(pr.query), 1) for c in chunks) * 2
    out = {"workload": "chunked: %d bp target x %d bp query, %d chunks x 2 strands" % (
        len(pr.target), len(pr.query), len(chunks)), "mbp2": round(mbp2_total, 2), "table_build_ms": round(table_ms, 2),
        "table_build_first_ms": round(views_ms[0], 2),
        "roofline_table": tab_roof,
        "generate_s": round(gen_s, 1)}
    if args.max_hits_per_pass:
        ctx.set_tuning(max_hits_per_pass=args.max_hits_per_pass)
        out["max_hits_per_pass"] = args.max_hits_per_pass
    for tr in (1, 0):
        sp = g.SearchParams(transitions=tr)
        tune = autotune(ctx, tabs, [dQ], units, m, sp, workload="chunked", sample_units=4, reps=1, use_cache=False,
                        space={"screen_blocks_per_sm": [4, 3], "screen_cap": [192, 128]})
        st = {}
        ctx.mark(10)
        got = g.batch_search(tabs, [dQ], units, m, sp, stats=st, ctx=ctx)
        ctx.mark(11)
        b_ms = ctx.elapsed_ms(10, 11)
        ctx.mark(12)
        same = True
        dQr = dQ.reverse_complement()
        for u, (ci, _, strand, plo, phi) in enumerate(units):
            h = g.search_device(tabs[ci], dQr if strand else dQ, m, sp)
            h = h[(h["t_start"] >= plo) & (h["t_start"] < phi)]
            same = same and h.tobytes() == got[u].tobytes()
        dQr.free()
        ctx.mark(13)
        p_ms = ctx.elapsed_ms(12, 13)
        # The driver's --nogapped records of the same units (global t, one
        # group per strand, sorted, deduplicated) from one batch_records call.
        places = [(strand, chunks[ci][0]) for ci, _, strand, _, _ in units]
        ctx.mark(14)
        recs, offs = g.batch_records(tabs, [dQ], units, places, m, sp, ctx=ctx)
        ctx.mark(15)
        r_ms = ctx.elapsed_ms(14, 15)
        rdt = np.dtype([("t", "<u8"), ("q", "<u4"), ("l", "<u4"), ("s", "<i4")])
        rec_same = len(offs) == 3
        for strand in (0, 1):
            parts = []
            for u, (ci, _, sd, _, _) in enumerate(units):
                if sd != strand:
                    continue
                a = np.empty(len(got[u]), rdt)
                a["t"] = got[u]["t_start"].astype(np.uint64) + chunks[ci][0]
                a["q"], a["l"], a["s"] = got[u]["q_start"], got[u]["length"], got[u]["score"]
                parts.append(a)
            w = np.unique(np.concatenate(parts)) if parts else np.empty(0, rdt)
            r = recs[int(offs[strand]):int(offs[strand + 1])] if rec_same else recs[:0]
            rec_same = rec_same and len(r) == len(w) and bool(
                np.array_equal(r["t_start"].astype(np.uint64), w["t"]) and np.array_equal(r["q_start"], w["q"])
                and np.array_equal(r["span"], w["l"]) and np.array_equal(r["score"], w["s"]))
        out[f"transitions_{tr}"] = {
            "batched": {"value": round(mbp2_total / (b_ms / 1e3), 2), "ms": round(b_ms, 1), "raw_hits": st["raw_hits"],
                        "candidates": st["candidates"], "hsps": st["hsps"], "passes": st["passes"]},
            "plain": {"value": round(mbp2_total / (p_ms / 1e3), 2), "ms": round(p_ms, 1)},
            "records": {"value": round(mbp2_total / (r_ms / 1e3), 2), "ms": round(r_ms, 1), "n": int(len(recs)),
                        "same_as_host_postprocessing": rec_same},
            "bit_identical": same, "autotune": tune["tuning"]}
    return out


def run_input(args):
    """Input packing: one chromosome-style sequence of --length bp (default
    100 Mbp) as FASTA (60-column lines) and as UCSC 2bit, parsed into device
    sequences through the public API (host bytes in, device PackedSeq out,
    copies included), against the oracle's host packing of the same bases
    (PackedSeq::from_ascii restated in C; the reference also splits lines and
    pushes byte by byte, so this CPU figure is a lower bound on its cost).
    Result equality is checked on the downloaded sequences."""
    import numpy as np
    g = _pkg()
    from lastz_gxy_b200 import synth
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    L = args.length if args.length != 4_000_000 else 100_000_000
    t0 = time.time()
    seq = synth.c2(length=L).target.tobytes()
    fasta = b">chr1 synthetic\n" + b"\n".join(seq[i:i + 60] for i in range(0, len(seq), 60)) + b"\n"
    twobit = synth.to_2bit([("chr1", seq)])
    gen_s = time.time() - t0
    ctx = g.Context(0)
    out = {"workload": f"input: one {L} bp chromosome-style sequence (45% soft-masked, N blocks)",
           "fasta_bytes": len(fasta), "twobit_bytes": len(twobit), "generate_s": round(gen_s, 1)}
    for name, fn, data in (("fasta", g.parse_fasta, fasta), ("2bit", g.parse_2bit, twobit)):
        for _ in range(2):
            r = fn(data, ctx)
            del r
        times = []
        for _ in range(max(3, args.steps)):
            t = time.perf_counter()
            r = fn(data, ctx)
            times.append(time.perf_counter() - t)
            if len(times) < max(3, args.steps):
                del r
        best = statistics.median(times)
        h = r[0][1].to_host()
        o = O.pack_ascii(seq)
        nb = (o.len + 3) // 4
        same = bytes(h.codes[:nb]) == bytes(np.asarray(o.codes)[:nb]) and \
            bytes(h.valid[:(o.len + 7) // 8]) == bytes(np.asarray(o.valid)[:(o.len + 7) // 8]) and \
            bytes(h.mask[:(o.len + 7) // 8]) == bytes(np.asarray(o.mask)[:(o.len + 7) // 8])
        out[name] = {"ms": round(best * 1e3, 2), "mbp_per_s": round(L / 1e6 / best, 1),
                     "input_gb_per_s": round(len(data) / 1e9 / best, 2), "bit_identical": same}
        del r
    t = time.perf_counter()
    O.pack_ascii(seq)
    cpu = time.perf_counter() - t
    out["cpu_pack"] = {"ms": round(cpu * 1e3, 2), "mbp_per_s": round(L / 1e6 / cpu, 1), "cores": 1,
                       "kind": "port", "what": "oracle C PackedSeq::from_ascii of the bases (no line splitting)"}
    return out


def run_gapped(args, steps=None, warmup=None):
    """Gapped extension (src/gapped_extend.rs:78-460) of the plain workload's
    top-scoring anchors: the plus-strand HSPs of the 10 Mbp pair, their
    anchors (choose_anchor, window 31), the --anchors highest-scoring ones
    extended in one gxy_gapped_extend call.  Rate = DP cells (each side's band
    width summed over its rows) per second of the DP kernel, and anchors per
    second of the whole call.  The oracle extends a sample of the same anchors
    on the host cores (one thread, and every thread) and must agree with the
    device on every one of them."""
    import numpy as np
    g = _pkg()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    tgt, qry = workload(0)
    ctx = g.Context(0)
    if args.gapped_cells:
        ctx.set_tuning(gapped_cells=args.gapped_cells)
    m = g.ScoringMatrix.hoxd70()
    T, Q = g.PackedSeq.from_ascii(tgt), g.PackedSeq.from_ascii(qry)
    dT, dQ = T.to_device(ctx), Q.to_device(ctx)
    tab = g.PosTable.build(dT, P12, 1, ctx=ctx)
    hsps = g.search_device(tab, dQ, m, g.SearchParams())
    anchors = g.choose_anchors(dT, dQ, hsps, m, 31, ctx)
    order = np.argsort(-hsps["score"], kind="stable")[:args.anchors]
    A = np.ascontiguousarray(anchors[order])
    gp = g.GappedParams()
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    for _ in range(max(1, warmup)):
        g.gapped_extend(dT, dQ, A, m, gp, ctx=ctx)
    runs = []
    for _ in range(max(1, steps)):
        st = {}
        t0 = time.perf_counter()
        res = g.gapped_extend(dT, dQ, A, m, gp, ctx=ctx, stats=st)
        runs.append((time.perf_counter() - t0, st))
    wall = statistics.median(r[0] for r in runs)
    st = runs[len(runs) // 2][1]
    dev_s = statistics.median(r[1]["device_ms"] for r in runs) / 1e3
    cells = st["cells"]
    # The oracle on a sample of the anchors, spread over the ranked list.
    k = max(1, min(args.gapped_sample, len(A)))
    samp = np.linspace(0, len(A) - 1, k).astype(int)
    OT, OQ = O.pack_ascii(tgt), O.pack_ascii(qry)
    og = O.gapped_params()
    cells_samp, cells_one_l = [], []
    t0 = time.perf_counter()
    want = O.gapped_extend_many(OT, OQ, O.params(), og, A[samp, 0], A[samp, 1], threads=host_threads(),
                                cells=cells_samp)
    t_all = time.perf_counter() - t0
    one = samp[: max(1, k // 4)]
    t0 = time.perf_counter()
    O.gapped_extend_many(OT, OQ, O.params(), og, A[one, 0], A[one, 1], threads=1, cells=cells_one_l)
    t_one = time.perf_counter() - t0
    same = all((w is None and res[i] is None) or
               (w is not None and res[i] is not None and
                (res[i].t_start, res[i].q_start, res[i].t_len, res[i].q_len, res[i].score) ==
                (w["t_start"], w["q_start"], w["t_len"], w["q_len"], w["score"]) and
                [int(x) for x in res[i].script] == list(w["runs"]))
               for i, w in zip(samp, want))
    # The host rates count the DP cells the oracle computed for its sample.
    cells_all = sum(cells_samp)
    cells_one = sum(cells_one_l)
    return {
        "workload": f"gapped extension of the {len(A)} highest-scoring plus-strand anchors of the plain 10 Mbp pair "
                    f"(HOXD70, gap 400/30, y_drop 9400, gapped_threshold 3000)",
        "anchors": len(A), "passed": sum(r is not None for r in res), "rows": st["rows"], "cells": cells,
        "device_ms": round(dev_s * 1e3, 3), "call_ms": round(wall * 1e3, 3),
        "cells_per_s": round(cells / dev_s, 1), "anchors_per_s": round(len(A) / wall, 1),
        "warps_per_side": st["warps_per_side"], "reruns": st["reruns"],
        "max_side_rows": st["max_side_rows"], "second_pass_sides": st["second_pass_sides"],
        "cells_per_thread": st["cells_per_thread"], "second_pass_cells": st["second_pass_cells"],
        "us_per_row_of_longest_side": round(dev_s * 1e6 / max(1, st["max_side_rows"]), 3),
        "cpu_baseline": {"kind": "port", "all_cores": {"cores": host_threads(), "anchors": int(k), "s": round(t_all, 3),
                                                       "cells_per_s": round(cells_all / t_all, 1)},
                         "one_core": {"cores": 1, "anchors": int(len(one)), "s": round(t_one, 3),
                                      "cells_per_s": round(cells_one / t_one, 1)}},
        "same_as_oracle_on_sample": same,
    }


def run_gapped_case(args):
    """One long gapped extension, the small case the ncu captures use: a
    --length bp iid target and its 90%-identity copy (0.5% indels); the
    anchors of the three highest-scoring plus-strand HSPs."""
    import numpy as np
    g = _pkg()
    from lastz_gxy_b200 import synth
    rng = np.random.default_rng(5)
    t = synth.iid(rng, args.length, 0.41)
    q = synth.evolve(rng, t.copy(), 0.9, 0.005)
    ctx = g.Context(0)
    if args.gapped_cells:
        ctx.set_tuning(gapped_cells=args.gapped_cells)
    m = g.ScoringMatrix.hoxd70()
    dT = g.PackedSeq.from_ascii(t.tobytes()).to_device(ctx)
    dQ = g.PackedSeq.from_ascii(q.tobytes()).to_device(ctx)
    tab = g.PosTable.build(dT, P12, 1, ctx=ctx)
    hsps = g.search_device(tab, dQ, m, g.SearchParams())
    anchors = g.choose_anchors(dT, dQ, hsps, m, 31, ctx)
    A = np.ascontiguousarray(anchors[np.argsort(-hsps["score"], kind="stable")[:3]])
    out = []
    for _ in range(max(1, args.steps)):
        st = {}
        res = g.gapped_extend(dT, dQ, A, m, g.GappedParams(), ctx=ctx, stats=st)
        out.append({"device_ms": round(st["device_ms"], 3), "rows": st["rows"], "max_side_rows": st["max_side_rows"],
                    "cells_per_thread": st["cells_per_thread"], "warps_per_side": st["warps_per_side"],
                    "us_per_row_of_longest_side": round(st["device_ms"] * 1e3 / max(1, st["max_side_rows"]), 3),
                    "passed": sum(r is not None for r in res)})
    return {"workload": f"gapped case {args.length} bp", "runs": out}


def run_case(args):
    """One plus-strand search on the chromosome-style workload of --length bp
    (target and query both that long): the small case the ncu captures use."""
    g = _pkg()
    from lastz_gxy_b200 import synth
    pr = synth.c2(length=args.length)
    ctx = g.Context(0)
    dT = g.PackedSeq.from_ascii(pr.target.tobytes()).to_device(ctx)
    dQ = g.PackedSeq.from_ascii(pr.query.tobytes()).to_device(ctx)
    tab = g.PosTable.build(dT, P12, 1, ctx=ctx)
    out = []
    for _ in range(max(1, args.steps)):
        st = {}
        h = g.search_device(tab, dQ, g.ScoringMatrix.hoxd70(), g.SearchParams(), stats=st)
        out.append({"hsps": len(h), **st})
    return {"workload": f"case {args.length} bp", "runs": out}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--plain-only", action="store_true",
                    help="default workload: skip the batched and served legs of the line")
    ap.add_argument("--workload", default="plain",
                    choices=["plain", "batched", "served", "chunked", "case", "input", "gapped", "gapped_case"])
    ap.add_argument("--anchors", type=int, default=512, help="gapped workload: anchors extended per call")
    ap.add_argument("--gapped-sample", type=int, default=16, help="gapped workload: anchors the oracle extends")
    ap.add_argument("--gapped-cells", type=int, default=0, help="gapped workloads: DP cells per thread (4 or 8)")
    ap.add_argument("--requests", type=int, default=200, help="served workload: requests in the trace")
    ap.add_argument("--streams", type=int, default=2, help="served workload: dispatcher streams")
    ap.add_argument("--batch-units", type=int, default=64, help="served workload: units per batch at most")
    ap.add_argument("--batch-bases", type=int, default=16 << 20,
                    help="served workload: query bases (per strand) per batch at most")
    ap.add_argument("--length", type=int, default=4_000_000, help="case workload length (bp)")
    ap.add_argument("--scale", type=float, default=1.0, help="batched workload size factor")
    ap.add_argument("--max-hits-per-pass", type=int, default=0,
                    help="chunked workload: raw-hit buffer of the batched launches (0: the library default)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if args.workload == "batched":
        print(json.dumps(run_batched(args)), flush=True)
        return
    if args.workload == "served":
        print(json.dumps(run_served(args)), flush=True)
        return
    if args.workload == "chunked":
        print(json.dumps(run_chunked(args)), flush=True)
        return
    if args.workload == "case":
        print(json.dumps(run_case(args)), flush=True)
        return
    if args.workload == "input":
        print(json.dumps(run_input(args)), flush=True)
        return
    if args.workload == "gapped":
        print(json.dumps(run_gapped(args)), flush=True)
        return
    if args.workload == "gapped_case":
        print(json.dumps(run_gapped_case(args)), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out = run_ours(args, rank, world, local)
    if rank == 0 and world == 1 and not args.plain_only:
        # The headline's other two legs, measured in the same run: the uneven
        # batch (one batched launch vs the plain per-pair loop) and the
        # serving trace (served vs serial plain launches, latency quantiles).
        out["batched"] = batched_summary(run_batched(args))
        out["served"] = served_summary(run_served(args))
        # Gapped extension (src/gapped_extend.rs:78-460) of the workload's top
        # anchors, checked against the oracle on a sample in the same run.
        out["gapped"] = run_gapped(args, steps=3, warmup=1)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
