#!/usr/bin/env python3
"""Benchmark: hash-join probe throughput on one B200 (and N replicas).

Workload (the join configuration): build side 2^22 unique int32 keys (a
seeded permutation of 0..2^22-1) with int32 payload uniform [0, 2^20);
probe side 2^26 int32 keys, 90% drawn uniformly from the build keys and 10%
uniform in [2^22, 2^31), with int32 payload uniform [0, 2^20).  One step is
one probe pass: open -> consume(2^26 rows) -> close through the operator API,
producing COUNT(matches) and int64 SUM(build payload + probe payload).  The
hash table is built once, outside the timed steps.

  value : probe tuples/s with the probe columns resident in HBM
  e2e   : the same through the C ABI from pinned HOST memory: per step
          mgv_op_consume_host slices the host probe columns into pool
          buffers, the copy of slice k+1 overlapping the probe of slice k,
          and close() reads the result back

The default run (N = 1) adds the other configurations' figures to the same
line: select + aggregate, the select -> join -> group-by pipeline, the
batched and served query mixes and the result delivery channel, each
checked against the oracle or the plain path before it is printed.

Multi-GPU: one process per GPU, each an independent replica of the
workload (the probe shards with no exchange); value = all ranks' tuples /
the slowest rank's time.  `--impl reference` times the CPU restatement of
the reference's chained-table join (src/main8.cu:84-103) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "multigpu-vector_b200"))

BUILD_ROWS = 1 << 22
PROBE_ROWS = 1 << 26
HIT = 3865470566  # 0.9 * 2^32
SEED_B, SEED_P = 0x5EED0002, 0x5EED0003
METRIC = "join-probe tuples/s, % of HBM peak; batched queries/s & p99 vs plain"
BYTES_PER_TUPLE = 8  # probe key + probe payload, read once
WORKLOAD = ("hash join probe: build 2^22 unique int32 keys (seeded permutation) + int32 payload "
            "U[0,2^20); probe 2^26 int32 keys (90% build keys, 10% U[2^22,2^31)) + int32 payload "
            "U[0,2^20); COUNT + int64 SUM(build_payload + probe_payload)")


def measured_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measure_build(torch, bhead, bk, bp, nb, stream, args):
    """The build side on its own: open -> consume(all build rows) -> close of the
    hash_build operator, rebuilt from scratch each time, L2 flushed before each
    build by reading 1 GiB; device time with events on the launching stream.
    Algorithmic bytes: 8 B read (key + payload) + 8 B table write per build tuple."""
    with torch.cuda.stream(stream):
        flush = torch.ones(1 << 27, dtype=torch.int64, device="cuda")
        flush_out = torch.empty((), dtype=torch.int64, device="cuda")
    reps = max(10, min(args.steps, 50))
    times = []
    for i in range(3 + reps):
        with torch.cuda.stream(stream):
            torch.sum(flush, dim=0, out=flush_out)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bhead.open(stream)
        bhead.consume_columns([bk, bp], nb, stream)
        bhead.close(stream)
        e1.record(stream)
        stream.synchronize()
        if i >= 3:
            times.append(e0.elapsed_time(e1) / 1000.0)
    del flush, flush_out
    t = statistics.median(times)
    peak, kind = measured_peaks()
    achieved = 16 * nb / t / 1e9
    return {"value": nb / t, "unit": "build tuples/s", "ms": 1000 * t,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": kind, "algorithmic_bytes_per_build": 16 * nb},
            "workload": f"hash_build of {nb} unique keys + payloads (open -> consume -> close, region build), "
                        f"median of {reps}, L2 flushed before each build by reading 1 GiB",
            "note": "8 B read + 8 B table write per build tuple; the table's empty slots are written too, and "
                    "the rows are staged by table region once (read and written) before the regions are built",
            "checked": "the probe steps after it run against the table built last and are checked against the "
                       "oracle"}


def probe_traffic_per_launch():
    """DRAM bytes per probe launch from the committed ncu summary, if any."""
    p = os.path.join(HERE, "profiles", "join_probe_traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("dram_bytes_per_launch")
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, t0, t1):
        """Host-clock window of the timed region."""
        self.window = (t0, t1)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        w = getattr(self, "window", None)
        inside = [ln for t, ln in self.lines if w and w[0] <= t <= w[1]]
        scope = "timed region"
        if not inside:  # region shorter than the sampling period: use the whole run
            inside = [ln for _, ln in self.lines]
            scope = "warm-up + timed region"
        for ln in inside:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "scope": scope}


def oracle_chain(bk, bp):
    """The oracle's chained table (src/main8.cu:84-103 restated) on the build side."""
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import pyoracle as po

    return po.Chain(bk, bp)


def cpu_probe_baseline(chain, pk, pp, sample, threads):
    """The oracle's chained-table probe on host cores, the table built once and
    untimed (the GPU table is built untimed too): one core on a 2^22-row
    sample (the reference's single-thread loop), all threads on `sample` rows."""
    s1 = min(pk.size, 1 << 22)
    t0 = time.perf_counter()
    chain.probe_agg(pk[:s1], pp[:s1])
    t1 = time.perf_counter() - t0
    sa = min(pk.size, sample)
    t0 = time.perf_counter()
    chain.probe_agg_mt(pk[:sa], pp[:sa], threads)
    ta = time.perf_counter() - t0
    return {"value": s1 / t1, "unit": "tuples/s", "cores": 1, "kind": "port",
            "sample": f"first {s1} probe rows against the full 2^22-key chained table (built once, untimed); "
                      f"{t1:.2f} s on 1 core (the reference's single-thread probe loop, restated)",
            "all_cores": {"value": sa / ta, "unit": "tuples/s", "cores": threads, "kind": "port",
                          "sample": f"first {sa} probe rows, the same table; {ta:.2f} s on {threads} threads "
                                    "(ours: the loop split over the host's threads)"}}


def run_gather(args, mgv):
    """Random-read ceilings of this GPU (include/mgv_diag.h), one JSON line."""
    ctx = mgv.Context(int(os.environ.get("LOCAL_RANK", "0")))
    if args.gather_once:
        ms = ctx.diag_gather(args.gather_once << 20, 1 << 24, line_bytes=32, method=0, ctas_per_sm=2, reps=1,
                             inflight=4, lsu_warps=8)
        print(json.dumps({"gather_once": {"table_mib": args.gather_once, "lookups": 1 << 24, "ms": ms}}), flush=True)
        ctx.close()
        return 0
    n = 1 << 26
    out = []

    def one(**kw):
        try:
            ms = ctx.diag_gather(lookups=n, reps=10, **kw)
            out.append(dict(kw, ms=ms, g_lookups_per_s=n / ms / 1e6))
        except mgv.MgvError as e:
            out.append(dict(kw, error=str(e)))

    for mib in (40, 80):
        for lb in (32, 64, 128):
            for c in (2, 4):
                one(table_bytes=mib << 20, line_bytes=lb, method=0, ctas_per_sm=c, inflight=4, lsu_warps=8)
    for lb in (32, 64):
        for tw in (1, 2, 4):
            one(table_bytes=40 << 20, line_bytes=lb, method=1, ctas_per_sm=2, inflight=2, tma_warps=tw)
    for sh in (0.1, 0.2, 0.35):
        one(table_bytes=40 << 20, line_bytes=32, method=2, ctas_per_sm=2, inflight=4, lsu_warps=8, tma_warps=1,
            tma_share=sh)
    print(json.dumps({"gather_ceiling": out, "lookups": n}), flush=True)
    ctx.close()
    return 0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import numpy as np
    import pyoracle as po

    nb, npb = BUILD_ROWS, PROBE_ROWS
    bk = po.gen_perm(nb, SEED_B)
    bp = po.gen_uniform(nb, SEED_B, 1, 0, 1 << 20)
    sample = min(npb, args.cpu_sample)
    pk, _ = po.gen_probe_keys(sample, SEED_P, SEED_B, nb, HIT, nb, (1 << 31) - nb)
    pp = po.gen_uniform(sample, SEED_P, 2, 0, 1 << 20)
    threads = os.cpu_count() or 1
    chain = po.Chain(bk, bp)
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        chain.probe_agg_mt(pk, pp, threads)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    ms = 1000.0 * statistics.median(times)
    v = sample / (ms / 1000.0)
    s1 = min(sample, 1 << 22)  # the reference's own single-thread loop, for context
    t0 = time.perf_counter()
    chain.probe_agg(pk[:s1], pp[:s1])
    one_core = s1 / (time.perf_counter() - t0)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "tuples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "build_rows": nb, "probe_rows": npb, "probe_rows_per_step_sample": sample},
        "cpu_baseline": {"value": v, "unit": "tuples/s", "cores": threads, "kind": "port",
                         "sample": f"probe of {sample} rows per step against the full 2^22-key chained table "
                                   f"(built once, untimed), {threads} threads",
                         "single_core": {"value": one_core, "unit": "tuples/s", "cores": 1,
                                         "sample": f"first {s1} probe rows, 1 core"}},
        "e2e": {"value": v, "unit": "tuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mgv", choices=["mgv", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=1 << 24)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched and served summaries added to the join line (N = 1)")
    ap.add_argument("--load-factor", type=float, default=0.45,
                    help="join table load factor; 0.45 (a 71 MiB table for 2^22 keys) measured fastest under sustained "
                         "load (0.4 reads more of the table from DRAM and draws the GPU into its power cap; 0.5 and "
                         "up continue more runs into a second bucket)")
    ap.add_argument("--pipeline-load-factor", type=float, default=0.5,
                    help="pipeline: load factor of the 2^24-key radix-partitioned key-only table (0.5 and 0.6 "
                         "measured fastest, 0.4 about 4 %% slower: 8 keys per bucket keep runs short at 0.5, and "
                         "the smaller table stays in L2 more)")
    ap.add_argument("--build-rows", type=int, default=BUILD_ROWS)
    ap.add_argument("--probe-rows", type=int, default=PROBE_ROWS)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--probe-kernel", type=int, default=None, help="0 auto, 1 register prefetch, 2 staged")
    ap.add_argument("--rows-per-thread", type=int, default=None)
    ap.add_argument("--stages", type=int, default=None)
    ap.add_argument("--ctas-per-sm", type=int, default=None)
    ap.add_argument("--workload", default="join", choices=["join", "select", "pipeline", "batched", "served", "delivery"],
                    help="join: the headline probe; the others are the remaining configurations")
    ap.add_argument("--queries", type=int, default=512, help="batched: queries in the mix")
    ap.add_argument("--batch-config", default=None,
                    help="batched: 'load_factor,probe_item_rows,item_order' instead of autotuning")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="served: arrival window per rate")
    ap.add_argument("--rates", default="200,1000,5000", help="served: arrival rates (queries/s)")
    ap.add_argument("--served-plain-first", action="store_true",
                    help="served: run the plain server before the batched one at each rate")
    ap.add_argument("--saturate", type=int, default=5000, help="served: requests in the closing burst")
    ap.add_argument("--served-mix", default="sizes", choices=["sizes", "config3"],
                    help="served: the batched mix's sizes over 16 tables, or config-3 queries over one table")
    ap.add_argument("--served-burst-only", action="store_true",
                    help="served: only the batched server's closing burst (no rates, no plain server)")
    ap.add_argument("--serve-seconds-config3", type=float, default=0.5,
                    help="served config-3 mix: arrival window per rate")
    ap.add_argument("--saturate-config3", type=int, default=1000,
                    help="served config-3 mix: requests in the closing burst")
    ap.add_argument("--gather-ceiling", action="store_true",
                    help="measure the random bucket-read ceilings (line widths 32/64/128 B, LSU and TMA gather4, "
                         "40 and 80 MiB tables) instead of the join")
    ap.add_argument("--gather-once", type=int, default=0, metavar="MIB",
                    help="one 32-byte LSU gather pass set over a table of MIB MiB (2^24 lookups; for ncu captures)")
    ap.add_argument("--settle-s", type=float, default=1.0, help="untimed steps before timing, in seconds")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import mgv

    if args.workload != "join":
        import workloads

        return workloads.run(args)
    if args.gather_ceiling or args.gather_once:
        return run_gather(args, mgv)

    import replicas

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dist, world, rank, local = replicas.init("nccl")
    torch.cuda.set_device(local)
    ctx = mgv.Context(local)
    tune = {k: v for k, v in (("probe_kernel", args.probe_kernel), ("probe_rows_per_thread", args.rows_per_thread),
                              ("probe_stages", args.stages), ("probe_ctas_per_sm", args.ctas_per_sm)) if v is not None}
    if tune:
        ctx.set_tuning(**tune)
    tuning = ctx.tuning()
    stream = torch.cuda.Stream()
    nb, npb = args.build_rows, args.probe_rows

    with torch.cuda.stream(stream):
        bk = torch.empty(nb, dtype=torch.int32, device="cuda")
        bp = torch.empty(nb, dtype=torch.int32, device="cuda")
        pk = torch.empty(npb, dtype=torch.int32, device="cuda")
        pp = torch.empty(npb, dtype=torch.int32, device="cuda")
    ctx.gen_perm(bk, nb, SEED_B, stream=stream)
    ctx.gen_uniform(bp, nb, SEED_B, 1, 0, 1 << 20, stream=stream)
    hits = ctx.gen_probe_keys(pk, npb, SEED_P, SEED_B, nb, HIT, nb, (1 << 31) - nb, stream=stream)
    ctx.gen_uniform(pp, npb, SEED_P, 2, 0, 1 << 20, stream=stream)

    bhead, hb, probe, agg = mgv.create_count_join_1G_pipeline(ctx, nb, args.load_factor)
    tb0 = torch.cuda.Event(enable_timing=True)
    tb1 = torch.cuda.Event(enable_timing=True)
    tb0.record(stream)
    bhead.open(stream)
    bhead.consume_columns([bk, bp], nb, stream)
    bhead.close(stream)
    tb1.record(stream)
    stream.synchronize()
    build_ms = tb0.elapsed_time(tb1)
    build = None
    if not args.no_extras:
        build = measure_build(torch, bhead, bk, bp, nb, stream, args)
    info = hb.result()

    def step():
        probe.open(stream)
        probe.consume_columns([pk, pp], npb, stream)
        probe.close(stream)

    for _ in range(args.warmup):
        step()
    cnt, s = agg.result()
    assert cnt == hits, f"match count {cnt} != generated hits {hits}"

    # per-launch probe kernel time (events bracket the single probe launch)
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        # settle clocks (and let the sampler start) before the timed region
        t_settle = time.time()
        while time.time() - t_settle < args.settle_s:
            step()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        launches0 = ctx.launches
        h0 = time.time()
        start.record(stream)
        for i in range(args.steps):
            probe.open(stream)
            kev[i][0].record(stream)
            probe.consume_columns([pk, pp], npb, stream)
            kev[i][1].record(stream)
            probe.close(stream)
        end.record(stream)
        torch.cuda.synchronize()
        clk.mark(h0, time.time())
    launches = ctx.launches - launches0
    if dist:
        dist.barrier()
    elapsed = start.elapsed_time(end) / 1000.0
    kernel_s = statistics.mean(a.elapsed_time(b) for a, b in kev) / 1000.0
    elapsed = replicas.max_over_ranks(dist, elapsed, "cuda")
    assert replicas.same_on_all_ranks(dist, (cnt, s)), "replicas disagree"
    # ---- end to end through the C ABI from pinned host memory -------------
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(mgv, torch, ctx, probe, agg, pk, pp, npb, stream, args, dist, world, (cnt, s))

    # ---- oracle check of the timed run over every probe row, and the CPU baseline (rank 0, N = 1) ----
    checked = None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        hbk, hbp, hpk, hpp = (t.cpu().numpy() for t in (bk, bp, pk, pp))
        chain = oracle_chain(hbk, hbp)
        want = chain.probe_agg_mt(hpk, hpp, threads)
        assert want == (cnt, s), f"join result {(cnt, s)} differs from the oracle's {want}"
        checked = f"oracle: COUNT and SUM equal the oracle's chained-table join over all {npb} probe rows"
        cpu = cpu_probe_baseline(chain, hpk, hpp, args.cpu_sample, threads)
    # ---- the probe's own ceiling: random 32-byte reads of a table this size (N = 1) ----
    ceiling = None
    if world == 1 and not args.no_extras:
        ms = ctx.diag_gather(int(info.table_bytes), npb, line_bytes=32, method=0, ctas_per_sm=2, reps=5, inflight=4,
                             lsu_warps=8)
        ceiling = {"what": "random 32-byte bucket reads of a table of this size with nothing else in the kernel "
                           "(mgv_diag_gather, LSU, 2 CTAs x 8 warps per SM, 4 reads in flight per lane)",
                   "lookups_per_s": npb / (ms / 1e3), "probe_tuples_per_s": npb / kernel_s,
                   "frac": (npb / kernel_s) / (npb / (ms / 1e3))}
    # ---- the metric's other half: batched and served queries vs plain (N = 1) ----
    extras = {}
    if world == 1 and not args.no_extras:
        extras = run_extras(args, mgv, torch, ctx)
    if build is not None:
        extras["build"] = build
    return finish(args, ctx, info, build_ms, elapsed, kernel_s, launches, clk, cnt, s, e2e, cpu, world, rank,
                  dist, (probe, agg, bhead, hb), nb, npb, tuning, extras, checked, ceiling)


def run_extras(args, mgv, torch, ctx):
    """The 512-query batched mix (autotuned) and the served mix, as in
    `--workload batched` / `--workload served`, summarised for the join line."""
    import workloads

    class NoClock:
        def mark(self, *a):
            pass

    if os.path.join(HERE, "oracle") not in sys.path:
        sys.path.insert(0, os.path.join(HERE, "oracle"))  # the workloads check their results against the oracle
    sub = argparse.Namespace(**vars(args))
    sub.steps, sub.warmup, sub.batch_config = 5, 3, None
    t0 = time.time()
    sys.modules.setdefault("bench", sys.modules[__name__])
    select = workloads.run_select(sub, mgv, torch, ctx, sys.modules[__name__], NoClock(), emit=False)
    torch.cuda.empty_cache()
    pipeline = workloads.run_pipeline(sub, mgv, torch, ctx, sys.modules[__name__], NoClock(), emit=False)
    torch.cuda.empty_cache()
    batched = workloads.run_batched(sub, mgv, torch, ctx, None, NoClock(), emit=False)
    served = workloads.run_served(sub, mgv, torch, ctx, None, NoClock(), emit=False)
    torch.cuda.empty_cache()
    served3 = workloads.run_served(sub, mgv, torch, ctx, None, NoClock(), emit=False, mix="config3")
    torch.cuda.empty_cache()
    delivery = workloads.run_delivery(sub, mgv, torch, ctx, None, NoClock(), emit=False)
    torch.cuda.empty_cache()
    at = {r["rate"]: r for r in served["rates"]}
    keep = ("value", "unit", "ms", "workload", "roofline", "e2e", "cpu_baseline", "checked", "result", "gpu_launches",
            "phases_ms")
    return {
        "select": {k: select[k] for k in keep if k in select},
        "pipeline": {k: pipeline[k] for k in keep if k in pipeline},
        "batched": {"value": batched["value"], "unit": "queries/s", "ms_per_batch": batched["ms"],
                    "plain_value": batched["plain"]["value"], "speedup_vs_plain": batched["speedup_vs_plain"],
                    "workload": batched["workload"], "batch_config": batched["batch_config"],
                    "checked": batched["checked"]},
        "served": {"saturated_qps": served["value"], "saturated_plain_qps": served["saturated"]["plain"]["throughput_qps"],
                   "saturated_speedup_vs_plain": served["saturated_speedup_vs_plain"],
                   "saturated_detail": served["saturated"],
                   "p50_p99_ms": {str(r): {"batched": [at[r]["batched"]["p50_ms"], at[r]["batched"]["p99_ms"]],
                                           "plain": [at[r]["plain"]["p50_ms"], at[r]["plain"]["p99_ms"]]}
                                  for r in at},
                   "workload": served["workload"], "checked": served["checked"]},
        "served_config3": served_summary(served3),
        "delivery": {"value": delivery["value"], "unit": "rows/s", "host_gbs": delivery["host_gbs"],
                     "workload": delivery["workload"]},
        "extras_wall_s": time.time() - t0,
    }


def served_summary(served):
    """The served figures of one mix for the join line."""
    at = {r["rate"]: r for r in served["rates"]}
    pick = ("throughput_qps", "p50_ms", "p99_ms", "mean_ms", "mean_batch", "shared_scans")
    return {"saturated_qps": served["value"], "saturated_plain_qps": served["saturated"]["plain"]["throughput_qps"],
            "saturated_speedup_vs_plain": served["saturated_speedup_vs_plain"],
            "saturated_detail": served["saturated"],
            "rates": {str(r): {"batched": {k: at[r]["batched"][k] for k in pick},
                               "plain": {k: at[r]["plain"][k] for k in pick}} for r in at},
            "workload": served["workload"], "checked": served["checked"]}


def run_e2e(mgv, torch, ctx, probe, agg, pk, pp, npb, stream, args, dist, world, want):
    """The same probe through the C ABI from pinned HOST columns: per step,
    open -> mgv_op_consume_host (4 Mi-row slices through 3 pool buffers, the
    copy of slice k+1 overlapping the probe of slice k) -> close."""
    cap = mgv.DEFAULT_BUFFER_ROWS
    pool = mgv.Pool(ctx, 3, cap, 2)
    hpk = pk.cpu().pin_memory()
    hpp = pp.cpu().pin_memory()
    e2e_steps = max(1, args.e2e_steps)

    def e2e_step():
        probe.open(stream)
        probe.consume_host(pool, [hpk.data_ptr(), hpp.data_ptr()], npb, stream)
        probe.close(stream)

    e2e_step()
    assert agg.result() == want
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    import replicas

    e2e_s = replicas.max_over_ranks(dist, e0.elapsed_time(e1) / 1000.0, "cuda")
    e2e_value = replicas.job_rate(world, npb * e2e_steps, e2e_s)
    # the host link's plain copy rate for the same bytes (pinned -> device), for context
    h2d = 0.0
    for _ in range(3):
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        with torch.cuda.stream(stream):
            pk.copy_(hpk, non_blocking=True)
            pp.copy_(hpp, non_blocking=True)
        c1.record(stream)
        stream.synchronize()
        h2d = max(h2d, 8 * npb / (c0.elapsed_time(c1) / 1000.0) / 1e9)
    pool.destroy()
    e2e_gbs = 8 * npb * e2e_steps / e2e_s / 1e9 / world
    return {"value": e2e_value, "unit": "tuples/s", "h2d_bytes_per_step": 8 * npb, "d2h_bytes_per_step": 16,
            "h2d_gbs": e2e_gbs, "h2d_peak_gbs": h2d, "frac_of_h2d": e2e_gbs / h2d if h2d else None,
            "path": "mgv_op_consume_host (pinned host columns -> 4 Mi-row slices through 3 pool buffers, "
                    "copies overlapped with the probe) + mgv_op_close"}


def finish(args, ctx, info, build_ms, elapsed, kernel_s, launches, clk, cnt, s, e2e, cpu, world, rank, dist,
           ops, nb, npb, tuning, extras=None, checked=None, ceiling=None):
    import replicas

    value = replicas.job_rate(world, npb * args.steps, elapsed)
    peak, peak_kind = measured_peaks()
    achieved = BYTES_PER_TUPLE * npb / kernel_s / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "tuples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * elapsed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {
            "workload": WORKLOAD, "build_rows": nb, "probe_rows": npb, "load_factor": args.load_factor,
            "table_bytes": int(info.table_bytes), "build_ms": build_ms, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2: 512 MiB of probe columns streamed per step (evict-first); the hash "
                  "table is read at random and about half to two thirds of its sectors hit in L2",
            "step": "open -> consume(2^26 rows) -> close (COUNT + SUM read back)",
            "tuning": {"probe_kernel": tuning.probe_kernel, "rows_per_thread": tuning.probe_rows_per_thread,
                       "stages": tuning.probe_stages, "ctas_per_sm": tuning.probe_ctas_per_sm},
        },
        "hbm_peak_frac": achieved / peak,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "kernel_ms": kernel_s * 1000.0,
                     "algorithmic_bytes_per_launch": BYTES_PER_TUPLE * npb,
                     "traffic": probe_traffic_per_launch(), "lookup_ceiling": ceiling},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "result": {"count": cnt, "sum": s},
        "checked": checked or "count equals the generator's known hit count (oracle check skipped)",
    }
    line.update(extras or {})
    if rank == 0:
        print(json.dumps(line), flush=True)
    for o in ops:
        o.destroy()
    ctx.close()
    replicas.finish(dist)
    return 0


if __name__ == "__main__":
    sys.exit(main())
