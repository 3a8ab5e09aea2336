"""Benchmark workloads beside the headline join probe (run by bench.py --workload).

  select    select + aggregate: 2^22 rows, c0 U[0,2^31) with c0 < 2^30, COUNT and
            int64 SUM of c1 U[0,2^20); 8 B/row; the L2 is flushed between steps
  pipeline  select -> join -> group-by: probe 2^27 rows (key over 2^24 build keys,
            filter U[0,1000) <= 99, group Zipf(1) over 4096, value U[0,2^16)), build
            2^24 keys radix-partitioned on 8 bits; 16 B/probe row + 4 B/build key
  batched   512 select -> join -> group-by queries (build 2^U(10,22), probe
            2^U(12,24), selectivity U(1%,90%), groups 2^U(4,16), join-style value
            distributions) in one batch (CUDA graph replay) against the same queries
            one at a time through the plain pipeline
  served    open-loop Poisson arrivals of that mix at 200 / 1000 / 5000 queries/s
            over 16 resident tables, 40 GB budget, continuous batching vs the plain
            one-at-a-time server; p50 / p99 latency
  delivery  the join's full match multiset streamed to pinned host memory through
            a bounded sink (mgv_sink_drain between 4 Mi-row probe slices)

Every line is one JSON object; results are checked (batched against plain, the
pipeline against the oracle on its known total) before anything is printed.
"""
from __future__ import annotations

import json
import math
import os
import statistics
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "multigpu-vector_b200")
HIT = 3865470566


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _line(args, metric, value, unit, ms, workload, extra, clk, higher=True):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
         "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": higher, "scaling": "weak",
         "vs_baseline": None, "dtype": "int32", "data": "synthetic", "config": {"workload": workload}}
    d.update(extra)
    d["clocks"] = clk.summary()
    if int(os.environ.get("RANK", "0")) == 0:  # under torchrun every rank runs its own replica
        print(json.dumps(d), flush=True)


def _h2d_gbs(torch, host, dev, stream, reps=3):
    """Plain pinned host -> device copy rate of `host` (GB/s, best of reps)."""
    best = 0.0
    for _ in range(reps):
        e0, e1 = _events(torch)
        e0.record(stream)
        with torch.cuda.stream(stream):
            dev.copy_(host, non_blocking=True)
        e1.record(stream)
        stream.synchronize()
        best = max(best, host.numel() * host.element_size() / (e0.elapsed_time(e1) / 1000.0) / 1e9)
    return best


def _cpu_pair(one_fn, one_rows, all_fn, all_rows, total_rows, unit, what_one, what_all):
    """1-core reference-style loop and all-core port, each timed on a sample and
    scaled to the workload's rows; returns the cpu_baseline object (1 core)
    with the all-core figure beside it, labelled."""
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    one_fn()
    t1 = time.perf_counter() - t0
    t0 = time.perf_counter()
    all_fn(threads)
    ta = time.perf_counter() - t0
    return {"value": one_rows / t1, "unit": unit, "cores": 1, "kind": "port",
            "sample": f"{what_one}: {one_rows} rows in {t1:.3f} s on 1 core (the reference's own single-thread "
                      f"CPU loop, restated)",
            "all_cores": {"value": all_rows / ta, "unit": unit, "cores": threads, "kind": "port",
                          "sample": f"{what_all}: {all_rows} rows in {ta:.3f} s on {threads} threads (ours: "
                                    "the same loop split over the host's threads)"}}


def run_select(args, mgv, torch, ctx, bench, clk, emit=True):
    """Select + aggregate (c0 <= 2^30 - 1 -> COUNT, SUM(c1)) over 2^22 rows."""
    import pyoracle as po

    n = 1 << 22
    bound = (1 << 30) - 1
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        c0 = torch.empty(n, dtype=torch.int32, device="cuda")
        c1 = torch.empty(n, dtype=torch.int32, device="cuda")
        # 1 GiB > L2, read (not written) between steps: a written flush would
        # leave the L2 full of dirty lines whose write-back the next kernel
        # pays for; the read also outlasts the host's enqueueing of open and
        # consume, so the kernel's events see the kernel, not a launch gap
        flush = torch.ones(1 << 27, dtype=torch.int64, device="cuda")
        flush_out = torch.empty((), dtype=torch.int64, device="cuda")
    ctx.gen_uniform(c0, n, 0x5EED0001, 0, 0, 1 << 31, stream=stream)
    ctx.gen_uniform(c1, n, 0x5EED0001, 1, 0, 1 << 20, stream=stream)
    head, agg = mgv.create_sum_select_pipeline(ctx, bound, 0, 1)

    def timed_steps(steps):
        times, ktimes = [], []
        for i in range(args.warmup + steps):
            with torch.cuda.stream(stream):
                torch.sum(flush, dim=0, out=flush_out)  # inputs come from HBM every step
            e0, e1 = _events(torch)
            k0, k1 = _events(torch)
            e0.record(stream)
            head.open(stream)
            k0.record(stream)  # enqueued while the flush still runs: the kernel follows it directly
            head.consume_columns([c0, c1], n, stream)
            k1.record(stream)
            head.close(stream)
            e1.record(stream)
            stream.synchronize()
            if i >= args.warmup:
                times.append(e0.elapsed_time(e1) / 1000.0)
                ktimes.append(k0.elapsed_time(k1) / 1000.0)
        return times, ktimes

    launches0 = ctx.launches
    h0 = time.time()
    times, ktimes = timed_steps(args.steps)
    clk.mark(h0, time.time())
    launches = (ctx.launches - launches0) * args.steps // (args.warmup + args.steps)
    cnt, s = agg.result()
    # the same select through the warp-ballot compaction (qualifying rows packed
    # into 128-row vectors that the aggregate reads): untimed for the headline
    tuning0 = ctx.tuning()
    ctx.set_tuning(select_compact=1)
    try:
        _, ballot_kt = timed_steps(max(10, args.steps))
        ballot_res = agg.result()
    finally:
        ctx.set_tuning(select_compact=tuning0.select_compact)
    assert ballot_res == (cnt, s), "the warp-ballot select differs from the masked fold"
    bkt = statistics.median(ballot_kt)
    del flush, flush_out
    t = statistics.median(times)
    kt = statistics.median(ktimes)
    peak, kind = bench.measured_peaks()
    hc0, hc1 = c0.cpu().numpy(), c1.cpu().numpy()
    assert po.select_agg_mt(hc0, hc1, bound, os.cpu_count() or 1) == (cnt, s), "select result differs from the oracle"
    cpu = _cpu_pair(lambda: po.select_agg(hc0, hc1, bound), n, lambda th: po.select_agg_mt(hc0, hc1, bound, th), n,
                    n, "rows/s", "sum_select_cpu-style loop over all 2^22 rows", "the same over all 2^22 rows")
    # end to end: pinned host columns through mgv_op_consume_host into pool buffers of the
    # reference's size (4 Mi rows), so the 2^22 rows are one slice: the consume kernel takes
    # microseconds against the copy's 0.6 ms, and 1 Mi-row slices only added per-copy overhead
    h0c, h1c = c0.cpu().pin_memory(), c1.cpu().pin_memory()
    pool = mgv.Pool(ctx, 3, mgv.DEFAULT_BUFFER_ROWS, 2)
    et = []
    for i in range(3 + max(10, args.steps)):
        e0, e1 = _events(torch)
        e0.record(stream)
        head.open(stream)
        head.consume_host(pool, [h0c.data_ptr(), h1c.data_ptr()], n, stream)
        head.close(stream)
        e1.record(stream)
        stream.synchronize()
        if i >= 3:
            et.append(e0.elapsed_time(e1) / 1000.0)
    assert agg.result() == (cnt, s)
    e2e_t = statistics.median(et)
    with torch.cuda.stream(stream):
        both = torch.empty(2 * n, dtype=torch.int32, device="cuda")
    hb = torch.cat([h0c, h1c]).pin_memory()
    h2d = _h2d_gbs(torch, hb, both, stream)
    pool.destroy()
    workload = ("select c0 < 2^30 over 2^22 rows (c0 U[0,2^31)), COUNT + int64 SUM(c1 U[0,2^20)); L2 flushed between "
                "steps by reading 1 GiB")
    extra = {"roofline": {"bound": "hbm", "achieved": 8 * n / kt / 1e9, "peak": peak, "unit": "GB/s",
                          "frac": 8 * n / kt / 1e9 / peak, "peak_kind": kind, "kernel_ms": 1000 * kt,
                          "algorithmic_bytes_per_launch": 8 * n, "kernel": "k_select_agg"},
             "ballot_path": {"kernel": "k_chain<select, aggregate> (warp-ballot compaction into 128-row vectors; "
                                       "mgv_tuning.select_compact = 1)", "kernel_ms": 1000 * bkt,
                             "achieved_gbs": 8 * n / bkt / 1e9, "frac": 8 * n / bkt / 1e9 / peak,
                             "checked": "COUNT and SUM equal the masked fold's (and so the oracle's)"},
             "step_gbs": 8 * n / t / 1e9,
             "e2e": {"value": n / e2e_t, "unit": "rows/s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 16,
                     "ms_per_step": 1000 * e2e_t, "h2d_gbs": 8 * n / e2e_t / 1e9, "h2d_peak_gbs": h2d,
                     "frac_of_h2d": 8 * n / e2e_t / 1e9 / h2d,
                     "path": "mgv_op_consume_host (pinned host columns through a 4 Mi-row pool buffer: one slice) "
                             "+ close"},
             "result": {"count": cnt, "sum": s}, "cpu_baseline": cpu, "gpu_launches": launches,
             "checked": "oracle: COUNT and SUM equal the oracle's select + aggregate over all 2^22 rows",
             "note": "step = open -> consume -> close incl. the host read-back; 33.5 MB per step; the roofline is "
                     "the consume's kernel (k_select_agg), timed with events around it"}
    if emit:
        _line(args, "select+aggregate rows/s", n / t, "rows/s", 1000 * t, workload, extra, clk)
    head.destroy()
    agg.destroy()
    return {"value": n / t, "unit": "rows/s", "ms": 1000 * t, "workload": workload, **extra}


def run_pipeline(args, mgv, torch, ctx, bench, clk, emit=True):
    """select -> join -> group-by over 2^27 probe rows with a 2^24-key radix-partitioned build."""
    import numpy as np
    import pyoracle as po

    nb, npb = 1 << 24, 1 << 27
    lf = args.pipeline_load_factor
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        bk = torch.empty(nb, dtype=torch.int32, device="cuda")
        cols = [torch.empty(npb, dtype=torch.int32, device="cuda") for _ in range(4)]
    seed = 0x5EED0003
    ctx.gen_perm(bk, nb, seed, stream=stream)
    ctx.gen_uniform(cols[0], npb, seed, 1, 0, nb, stream=stream)
    ctx.gen_uniform(cols[1], npb, seed, 2, 0, 1000, stream=stream)
    ctx.gen_zipf(cols[2], npb, seed, 3, 4096, stream=stream)
    ctx.gen_uniform(cols[3], npb, seed, 4, 0, 1 << 16, stream=stream)
    part, hb, sel, gb = mgv.create_join_groupby_pipeline(ctx, nb, 4096, 99, 8, lf)
    bt, pt = [], []
    launches0 = ctx.launches
    h0 = time.time()
    for i in range(args.warmup + args.steps):
        e0, e1, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True), \
            torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        part.open(stream); part.consume_columns([bk], nb, stream); part.close(stream)
        e1.record(stream)
        sel.open(stream); sel.consume_columns(cols, npb, stream); sel.close(stream)
        e2.record(stream)
        stream.synchronize()
        if i >= args.warmup:
            bt.append(e0.elapsed_time(e1) / 1000.0)
            pt.append(e1.elapsed_time(e2) / 1000.0)
    clk.mark(h0, time.time())
    launches = (ctx.launches - launches0) * args.steps // (args.warmup + args.steps)
    res = gb.result()
    b, p_ = statistics.median(bt), statistics.median(pt)
    peak, kind = bench.measured_peaks()
    alg = 16 * npb + 4 * nb
    # the oracle over every row (select + probe on all host threads)
    threads = os.cpu_count() or 1
    hb_keys = bk.cpu().numpy()
    hcols = [c.cpu().numpy() for c in cols]
    want, _, _ = po.run_query(hb_keys, *hcols, 99, threads=threads)
    assert res == [(int(w["group"]), int(w["sum"]), int(w["count"])) for w in want], "pipeline differs from the oracle"
    total = sum(c for _, _, c in res)
    # CPU baselines: the full 2^24-key chained-table build timed once, the probe side on a sample, scaled
    ct = time.perf_counter()
    po.run_query(hb_keys, hcols[0][:0], hcols[1][:0], hcols[2][:0], hcols[3][:0], 99)
    t_build = time.perf_counter() - ct
    s1, sa = 1 << 22, 1 << 24
    ct = time.perf_counter()
    po.run_query(hb_keys, *[c[:s1] for c in hcols], 99)
    t1 = time.perf_counter() - ct - t_build
    ct = time.perf_counter()
    po.run_query(hb_keys, *[c[:sa] for c in hcols], 99, threads=threads)
    ta = time.perf_counter() - ct - t_build
    cpu1 = t_build + t1 * npb / s1
    cpua = t_build + ta * npb / sa
    cpu = {"value": npb / cpu1, "unit": "rows/s", "cores": 1, "kind": "port",
           "sample": f"full 2^24-key chained-table build ({t_build:.2f} s) + select/probe/group-by of the first "
                     f"2^22 probe rows ({t1:.2f} s) on 1 core, scaled to 2^27 rows",
           "all_cores": {"value": npb / cpua, "unit": "rows/s", "cores": threads, "kind": "port",
                         "sample": f"the same build (1 core) + the first 2^24 probe rows with the select/probe "
                                   f"split over {threads} threads ({ta:.2f} s), scaled to 2^27 rows (ours)"}}
    # end to end: pinned host build keys and probe columns through mgv_op_consume_host
    hbk = bk.cpu().pin_memory()
    hpc = [c.cpu().pin_memory() for c in cols]
    pool1 = mgv.Pool(ctx, 3, mgv.DEFAULT_BUFFER_ROWS, 1)
    pool4 = mgv.Pool(ctx, 3, mgv.DEFAULT_BUFFER_ROWS, 4)
    et = []
    for i in range(1 + max(2, args.steps // 10)):
        e0, e1 = _events(torch)
        e0.record(stream)
        part.open(stream); part.consume_host(pool1, [hbk.data_ptr()], nb, stream); part.close(stream)
        sel.open(stream); sel.consume_host(pool4, [c.data_ptr() for c in hpc], npb, stream); sel.close(stream)
        e1.record(stream)
        stream.synchronize()
        if i >= 1:
            et.append(e0.elapsed_time(e1) / 1000.0)
    assert gb.result() == res
    e2e_t = statistics.median(et)
    h2d = _h2d_gbs(torch, hpc[0], cols[0], stream)
    pool1.destroy(); pool4.destroy()
    del hpc, hbk
    workload = ("select (filter <= 99 of U[0,1000)) -> join (2^27 probe rows, key over 2^24 build keys) -> group-by "
                "(Zipf(1) over 4096 groups, int64 SUM(value U[0,2^16)) + COUNT); build radix-partitioned on 8 key "
                f"bits, table load factor {lf}")
    extra = {"roofline": {"bound": "hbm", "achieved": alg / (b + p_) / 1e9, "peak": peak, "unit": "GB/s",
                          "frac": alg / (b + p_) / 1e9 / peak, "peak_kind": kind,
                          "algorithmic_bytes_per_step": alg, "scope": "whole step (partition + build + probe)"},
             "phases_ms": {"partition+build": 1000 * b, "select+probe+groupby": 1000 * p_},
             "e2e": {"value": npb / e2e_t, "unit": "rows/s", "h2d_bytes_per_step": alg,
                     "d2h_bytes_per_step": 24 * len(res), "ms_per_step": 1000 * e2e_t, "h2d_gbs": alg / e2e_t / 1e9,
                     "h2d_peak_gbs": h2d, "frac_of_h2d": alg / e2e_t / 1e9 / h2d,
                     "path": "mgv_op_consume_host of the pinned build keys (partition -> build) and of the four "
                             "pinned probe columns (select -> probe -> group-by), 4 Mi-row slices through 3 pool "
                             "buffers, copies overlapped with the consumes"},
             "result": {"groups": len(res), "count": total}, "cpu_baseline": cpu, "gpu_launches": launches,
             "checked": "oracle: every group's SUM and COUNT equal the oracle's select -> chained-table join -> "
                        "group-by over all 2^27 probe rows"}
    if emit:
        _line(args, "select->join->group-by probe rows/s", npb / (b + p_), "rows/s", 1000 * (b + p_), workload,
              extra, clk)
    for o in (sel, gb, hb, part):
        o.destroy()
    return {"value": npb / (b + p_), "unit": "rows/s", "ms": 1000 * (b + p_), "workload": workload, **extra}


def run_delivery(args, mgv, torch, ctx, bench, clk, emit=True):
    """The join's full match multiset delivered to pinned host memory: the
    2^22-key / 2^26-probe join, consumed in 16 slices of 4 Mi probe rows, each
    drained from the sink (a pool of 8 buffers x 4 Mi rows x 3 columns) with
    mgv_sink_drain.  Unit: delivered match rows / s."""
    nb, npb, step = 1 << 22, 1 << 26, 1 << 22
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        bk = torch.empty(nb, dtype=torch.int32, device="cuda")
        bp = torch.empty(nb, dtype=torch.int32, device="cuda")
        pk = torch.empty(npb, dtype=torch.int32, device="cuda")
        pp = torch.empty(npb, dtype=torch.int32, device="cuda")
    ctx.gen_perm(bk, nb, 0x5EED0002, stream=stream)
    ctx.gen_uniform(bp, nb, 0x5EED0002, 1, 0, 1 << 20, stream=stream)
    hits = ctx.gen_probe_keys(pk, npb, 0x5EED0003, 0x5EED0002, nb, HIT, nb, (1 << 31) - nb, stream=stream)
    ctx.gen_uniform(pp, npb, 0x5EED0003, 2, 0, 1 << 20, stream=stream)
    hb = mgv.Op.hash_build(ctx, 0, 1, nb)
    hb.open(stream); hb.consume_columns([bk, bp], nb, stream); hb.close(stream)
    pool = mgv.Pool(ctx, 8, step, 3)
    sink = mgv.Op.sink(ctx, pool)
    probe = mgv.Op.hash_probe(ctx, 0, hb, sink)
    out = [torch.empty(hits, dtype=torch.int32).pin_memory() for _ in range(3)]

    def one_pass():
        probe.open(stream)
        total = 0
        for lo in range(0, npb, step):
            probe.consume_columns([pk[lo:lo + step], pp[lo:lo + step]], step, stream)
            total += sink.sink_drain([o.data_ptr() + 4 * total for o in out], hits - total, stream)
        probe.close(stream)
        return total

    for _ in range(max(1, args.warmup)):
        assert one_pass() == hits
    times = []
    h0 = time.time()
    for _ in range(args.steps):
        e0, e1 = _events(torch)
        e0.record(stream)
        one_pass()
        e1.record(stream)
        stream.synchronize()
        times.append(e0.elapsed_time(e1) / 1000.0)
    clk.mark(h0, time.time())
    # spot check against the build side: every delivered row's key is a build key with its payload
    k = out[0][:1 << 16].numpy()
    assert (k >= 0).all() and (k < nb).all()
    t = statistics.median(times)
    bytes_out = 12 * hits
    workload = ("full match multiset of the 2^22-key / 2^26-probe join (60.4 M rows of key, probe payload, "
                "build payload) delivered to pinned host memory through a sink of 8 x 4 Mi-row buffers, "
                "drained after each 4 Mi-row probe slice")
    extra = {"matches": hits, "bytes_to_host": bytes_out, "host_gbs": bytes_out / t / 1e9,
             "probe_rows_per_s": npb / t}
    if emit:
        _line(args, "delivered join rows/s", hits / t, "rows/s", 1000 * t, workload, extra, clk)
    for o in (probe, sink, hb):
        o.destroy()
    pool.destroy()
    return {"value": hits / t, "unit": "rows/s", "ms": 1000 * t, "workload": workload, **extra}


def _mix(ctx, torch, mgv, nq, seed, stream):
    """The batched configuration: per query, build 2^U(10,22) unique keys,
    probe 2^U(12,24) rows (key 90% from the build keys, filter U[0,1000),
    group Zipf(1) over 2^U(4,16) groups, value U[0,2^20)), selectivity U(1%,90%)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    spec = []
    for i in range(nq):
        nb = int(2 ** rng.uniform(10, 22))
        npr = int(2 ** rng.uniform(12, 24))
        bound = int(round(rng.uniform(0.01, 0.90) * 1000)) - 1
        g = int(2 ** rng.uniform(4, 16))
        spec.append((nb, npr, bound, g))
    tb, tp = sum(x[0] for x in spec), sum(x[1] for x in spec)
    with torch.cuda.stream(stream):
        B = torch.empty(tb, dtype=torch.int32, device="cuda")
        P = [torch.empty(tp, dtype=torch.int32, device="cuda") for _ in range(4)]
    descs = []
    ob = op = 0
    for i, (nb, npr, bound, g) in enumerate(spec):
        s = seed * 100000 + i
        bkey = B[ob:ob + nb]
        pk, pf, pg, pv = [c[op:op + npr] for c in P]
        ctx.gen_perm(bkey, nb, s, stream=stream)
        ctx.gen_probe_keys(pk, npr, s + 1, s, nb, HIT, nb, (1 << 31) - nb, stream=stream)
        ctx.gen_uniform(pf, npr, s + 1, 2, 0, 1000, stream=stream)
        ctx.gen_zipf(pg, npr, s + 1, 3, g, stream=stream)
        ctx.gen_uniform(pv, npr, s + 1, 4, 0, 1 << 20, stream=stream)
        descs.append(mgv.query_desc(bkey, nb, pk, pf, pg, pv, npr, bound, g))
        ob += nb
        op += npr
    stream.synchronize()
    return spec, descs, (B, P)


def run_batched(args, mgv, torch, ctx, bench, clk, emit=True):
    """Batched vs one-at-a-time queries/s; prints its line when emit, returns its figures."""
    stream = torch.cuda.Stream()
    nq = args.queries
    spec, descs, keep = _mix(ctx, torch, mgv, nq, 0x5EED0004, stream)
    t0 = time.perf_counter()
    if args.batch_config:
        lf, items, order = args.batch_config.split(",")
        cfg = mgv.BatchConfig(float(lf), 0, int(items), 0, 1, int(order))
    else:
        cfg = mgv.batch_autotune(ctx, descs)
    tune_s = time.perf_counter() - t0
    b = mgv.Batch(ctx, descs, cfg, keep)
    bt, pt = [], []
    h0 = time.time()
    for i in range(args.warmup + args.steps):
        e0, e1 = _events(torch)
        e0.record(stream)
        b.run(stream)
        e1.record(stream)
        stream.synchronize()
        if i >= args.warmup:
            bt.append(e0.elapsed_time(e1) / 1000.0)
    clk.mark(h0, time.time())
    plain_steps = max(1, min(args.steps, 3))
    for i in range(1 + plain_steps):
        e0, e1 = _events(torch)
        e0.record(stream)
        b.run_plain(stream)
        e1.record(stream)
        stream.synchronize()
        if i >= 1:
            pt.append(e0.elapsed_time(e1) / 1000.0)
    mism = sum(1 for q in range(nq) if b.result(q) != b.result(q, plain=True))
    assert mism == 0, f"{mism} queries differ between batched and plain"
    # and three queries -- the smallest, a median and the largest probe side --
    # against the oracle's select -> join -> group-by (all host threads)
    import pyoracle as po

    by_rows = sorted(range(nq), key=lambda q: spec[q][1])
    picked = [by_rows[0], by_rows[nq // 2], by_rows[-1]]
    B, P = keep
    ob = [0]
    op = [0]
    for nb_q, npr_q, _, _ in spec:
        ob.append(ob[-1] + nb_q)
        op.append(op[-1] + npr_q)
    for q in picked:
        nb_q, npr_q, bound_q, _ = spec[q]
        hb = B[ob[q]:ob[q] + nb_q].cpu().numpy()
        hp = [c[op[q]:op[q] + npr_q].cpu().numpy() for c in P]
        want, _, _ = po.run_query(hb, hp[0], hp[1], hp[2], hp[3], bound_q, os.cpu_count() or 1)
        assert b.result(q) == [(int(w["group"]), int(w["sum"]), int(w["count"])) for w in want], \
            f"batched query {q} differs from the oracle"
    tb, tp = statistics.median(bt), statistics.median(pt)
    rows = sum(x[1] for x in spec)
    st = b.stats()
    workload = (f"{nq} select->join->group-by queries, build 2^U(10,22), probe 2^U(12,24) rows (total {rows}), "
                "selectivity U(1%,90%), groups 2^U(4,16); one batch (CUDA graph replay) incl. results to host")
    extra = {"plain": {"value": nq / tp, "unit": "queries/s", "ms": 1000 * tp,
                       "how": "the same queries one at a time: hash_build open/consume/close, then "
                              "select->hash_probe->groupby open/consume/close, operators created once"},
             "speedup_vs_plain": tp / tb,
             "batch_config": {"load_factor": cfg.load_factor, "probe_item_rows": cfg.probe_item_rows,
                              "item_order": cfg.item_order, "autotuned": not args.batch_config, "tune_s": tune_s},
             "arena_bytes": st.arena_bytes, "probe_rows": rows,
             "probe_rows_per_s": rows / tb,
             "checked": "all queries equal between batched and plain; the smallest, a median and the largest "
                        "query (by probe rows) equal the oracle's select -> join -> group-by"}
    if emit:
        _line(args, "batched queries/s vs plain", nq / tb, "queries/s", 1000 * tb, workload, extra, clk)
    b.destroy()
    del keep
    return {"value": nq / tb, "unit": "queries/s", "ms": 1000 * tb, "workload": workload, **extra}


def run_served(args, mgv, torch, ctx, bench, clk, emit=True, mix="sizes"):
    """Served throughput and p50 / p99 vs the plain server; prints its line when emit, returns its figures.

    mix "sizes": requests of the batched mix's sizes over 16 resident tables.
    mix "config3": the config-3 query (select filter <= b -> join on 2^24
    build keys -> group-by Zipf(1) over 4096 groups, 2^27 probe rows) with
    the bound b uniform in [9, 199] (selectivity 1 % to 20 %, 10 % on
    average) over the one resident config-3 table, so that the requests of a
    batch share their scan."""
    import numpy as np

    stream = torch.cuda.Stream()
    tables = []
    if mix == "config3":
        ntab = 1
        nb, prows, g, seed = 1 << 24, 1 << 27, 4096, 0x5EED0003
        with torch.cuda.stream(stream):
            bk = torch.empty(nb, dtype=torch.int32, device="cuda")
            cols = [torch.empty(prows, dtype=torch.int32, device="cuda") for _ in range(4)]
        ctx.gen_perm(bk, nb, seed, stream=stream)
        ctx.gen_uniform(cols[0], prows, seed, 1, 0, nb, stream=stream)
        ctx.gen_uniform(cols[1], prows, seed, 2, 0, 1000, stream=stream)
        ctx.gen_zipf(cols[2], prows, seed, 3, g, stream=stream)
        ctx.gen_uniform(cols[3], prows, seed, 4, 0, 1 << 16, stream=stream)
        tables.append((nb, g, bk, cols))
        seconds, burst = args.serve_seconds_config3, args.saturate_config3
    else:
        ntab = 16
        rng = np.random.default_rng(0x5EED0005)
        prows = 1 << 24
        for t in range(ntab):
            nb = int(2 ** rng.uniform(10, 22))
            g = int(2 ** rng.uniform(4, 16))
            with torch.cuda.stream(stream):
                bk = torch.empty(nb, dtype=torch.int32, device="cuda")
                cols = [torch.empty(prows, dtype=torch.int32, device="cuda") for _ in range(4)]
            s = 0x5EED0005 * 100 + t
            ctx.gen_perm(bk, nb, s, stream=stream)
            ctx.gen_probe_keys(cols[0], prows, s + 1, s, nb, HIT, nb, (1 << 31) - nb, stream=stream)
            ctx.gen_uniform(cols[1], prows, s + 1, 2, 0, 1000, stream=stream)
            ctx.gen_zipf(cols[2], prows, s + 1, 3, g, stream=stream)
            ctx.gen_uniform(cols[3], prows, s + 1, 4, 0, 1 << 20, stream=stream)
            tables.append((nb, g, bk, cols))
        seconds, burst = args.serve_seconds, args.saturate
    stream.synchronize()
    rates = [float(r) for r in args.rates.split(",")]

    def trace(rate, seed):
        """Arrival times and requests; rate 0 = a burst of `burst` requests at once."""
        r = np.random.default_rng(seed)
        n = max(1, int(rate * seconds)) if rate else burst
        gaps = r.exponential(1.0 / rate, n) if rate else np.zeros(n)
        reqs = []
        for i in range(n):
            if mix == "config3":
                reqs.append((0, prows, int(r.integers(9, 200))))
                continue
            t = int(r.integers(ntab))
            rows = int(2 ** r.uniform(12, 24))
            bound = int(round(r.uniform(0.01, 0.90) * 1000)) - 1
            reqs.append((t, rows, bound))
        return np.cumsum(gaps), reqs

    def serve(plain, rate, seed):
        import ctypes
        import queue
        import threading

        srv = mgv.Server(ctx, 40 << 30, max_batch=256, max_inflight=2, plain=plain)
        tids = [srv.add_table(bk, nb) for nb, g, bk, cols in tables]
        def run_trace(at, reqs):
            """Submits `reqs` at their arrival times while a second thread waits
            for each and lands its rows (the ctypes wait releases the GIL).  The
            drain only waits: request i's rows land in its own slice of one
            preallocated array (its max_groups rows), so it keeps up with the
            server, and digests are computed after the timed region."""
            caps = [tables[t][1] for t, _, _ in reqs]
            offs = np.concatenate([[0], np.cumsum(caps)]).astype(np.int64)
            res = np.empty((int(offs[-1]), 3), dtype=np.uint64)  # mgv_group_row = 3 x 64 bits
            res.fill(0)  # its pages are faulted in here, not by the draining thread while timed
            got = [0] * len(reqs)
            tq: "queue.Queue[tuple[int, int] | None]" = queue.Queue()
            errs = []

            def drain():
                n, lat = ctypes.c_uint64(), ctypes.c_double()
                base = res.ctypes.data
                while True:
                    item = tq.get()
                    if item is None:
                        return
                    i, tk = item
                    st = mgv.load().mgv_server_wait(srv.h, tk, 600000, ctypes.c_void_p(base + 24 * int(offs[i])),
                                                    caps[i], ctypes.byref(n), ctypes.byref(lat))
                    if st != mgv.OK:
                        errs.append(st)
                    got[i] = min(n.value, caps[i])

            th = threading.Thread(target=drain)
            th.start()
            k_sub = 0
            t0 = time.perf_counter()
            for a, (t, rows, bound) in zip(at, reqs):
                wait = a - (time.perf_counter() - t0)
                if wait > 1e-4:
                    time.sleep(wait - 5e-5)  # releases the GIL for the draining thread
                while time.perf_counter() - t0 < a:
                    pass
                nb_, g_, bk_, cols_ = tables[t]
                tq.put((k_sub, srv.submit(tids[t], *cols_, rows, bound, g_)))
                k_sub += 1
            t_sub = time.perf_counter() - t0
            tq.put(None)
            th.join()
            wall = time.perf_counter() - t0
            return t_sub, wall, got, res, offs, errs

        # warm-up: a burst of the mix (four full batches), run the way the timed
        # burst runs (a draining thread), so the server's device regions and
        # pinned landing zones have grown to their steady-state sizes and number
        # before anything is timed (pinning a zone for a full batch's rows
        # takes 10-60 ms, and a burst keeps three or four zones in use: two
        # batches in flight, one or two whose requests are still being waited for)
        _, warm = trace(0.0, seed + 777)
        nwarm = 1024
        while len(warm) < nwarm:
            warm = warm + warm
        assert not run_trace(np.zeros(nwarm), warm[:nwarm])[5]
        srv.reset_stats()
        # both servers start their timed window from an idle GPU: the batched
        # warm-up burst runs the GPU flat out, and its power-capped clocks
        # would otherwise still be recovering at the first timed requests
        time.sleep(0.5)
        at, reqs = trace(rate, seed)
        t_sub, wall, got, res, offs, errs = run_trace(at, reqs)
        assert not errs, errs
        # order-independent digest of each request's rows (the server returns groups unordered)
        digests = []
        for i in range(len(reqs)):
            rows = res[offs[i]:offs[i] + got[i]]
            hsh = rows[:, 0] * np.uint64(0x9E3779B97F4A7C15) ^ rows[:, 1] * np.uint64(0xC2B2AE3D27D4EB4F) \
                ^ rows[:, 2] * np.uint64(0x165667B19E3779F9)
            digests.append((got[i], int(hsh.sum(dtype=np.uint64)), int(np.bitwise_xor.reduce(hsh)) if got[i] else 0))
        stats = srv.stats()
        srv.destroy()
        return {"offered_qps": rate or None, "arrived_qps": len(reqs) / t_sub, "requests": len(reqs),
                "throughput_qps": len(reqs) / wall, "p50_ms": stats.p50_ms, "p99_ms": stats.p99_ms,
                "mean_ms": stats.mean_ms, "max_ms": stats.max_ms, "batches": stats.batches,
                "mean_batch": stats.mean_batch, "shared_scans": stats.shared_scans,
                "scan_queries": stats.scan_queries, "peak_device_bytes": stats.peak_bytes}, digests, reqs, res, offs, got

    sys.setswitchinterval(2e-4)  # the submitting and draining threads share the GIL
    out = []
    h0 = time.time()
    burst_only = getattr(args, "served_burst_only", False)
    if burst_only:
        rates = []
    for k, rate in enumerate(rates + [0.0]):
        if burst_only:  # the batched server's burst alone (for launch lists), checked against the oracle below
            b, rb, breqs, bres, boffs, bgot = serve(False, rate, 1000 + k)
            out.append({"rate": "saturated", "batched": b, "plain": b})
            continue
        if getattr(args, "served_plain_first", False):
            p, rp, *_ = serve(True, rate, 1000 + k)
            b, rb, breqs, bres, boffs, bgot = serve(False, rate, 1000 + k)
        else:
            b, rb, breqs, bres, boffs, bgot = serve(False, rate, 1000 + k)
            p, rp, *_ = serve(True, rate, 1000 + k)
        assert rb == rp, "served results differ from the plain server"
        out.append({"rate": rate if rate else "saturated", "batched": b, "plain": p})
    clk.mark(h0, time.time())
    checked = "every request's result equals the plain server's"
    if mix == "config3":
        # two requests of the burst against the oracle as well (all host threads)
        import pyoracle as po

        nb, g, bk, cols = tables[0]
        hb = bk.cpu().numpy()
        hc = [c.cpu().numpy() for c in cols]
        for i in (0, len(breqs) - 1):
            _, rows, bound = breqs[i]
            want, _, _ = po.run_query(hb, hc[0][:rows], hc[1][:rows], hc[2][:rows], hc[3][:rows], bound,
                                      os.cpu_count() or 1)
            rws = bres[boffs[i]:boffs[i] + bgot[i]].view(np.int64)  # mgv_group_row: group (+ pad), sum, count
            gotr = [(((int(a) & 0xFFFFFFFF) ^ 0x80000000) - 0x80000000, int(b_), int(c)) for a, b_, c in rws]
            assert sorted(gotr) == [(int(w["group"]), int(w["sum"]), int(w["count"])) for w in want], \
                "served config-3 request differs from the oracle"
        checked += "; two requests of the burst equal the oracle's select -> join -> group-by over 2^27 rows"
    sat = out[-1]
    if mix == "config3":
        workload = ("open-loop Poisson arrivals of config-3 queries (select filter <= b, b uniform in [9, 199]: "
                    "selectivity 1-20 %, 10 % on average -> join on 2^24 resident build keys -> group-by Zipf(1) "
                    "over 4096 groups, 2^27 probe rows each) for "
                    f"{seconds} s at each rate, then a burst of {burst} requests (saturated); 40 GB budget; "
                    "continuous batching with shared scans")
    else:
        workload = ("open-loop Poisson arrivals of the batched mix over 16 resident tables (build 2^U(10,22), probe "
                    "2^U(12,24) rows, selectivity U(1%,90%), groups 2^U(4,16)) at each rate, then a burst of "
                    f"{burst} requests (saturated); 40 GB budget; continuous batching")
    extra = {"rates": out[:-1], "saturated": sat,
             "saturated_speedup_vs_plain": sat["batched"]["throughput_qps"] / sat["plain"]["throughput_qps"],
             "checked": checked}
    if emit:
        _line(args, "served queries/s & p99 latency vs plain", sat["batched"]["throughput_qps"], "queries/s",
              sat["batched"]["mean_ms"], workload, extra, clk)
    del tables
    return {"value": sat["batched"]["throughput_qps"], "unit": "queries/s", "workload": workload, **extra}


def run(args) -> int:
    sys.path.insert(0, PKG)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))  # the CPU baselines time the oracle
    import torch

    import bench  # the repo-root benchmark script: peaks and clock sampling
    import mgv

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    ctx = mgv.Context(int(os.environ.get("LOCAL_RANK", "0")))
    fn = {"select": run_select, "pipeline": run_pipeline, "batched": run_batched, "served": run_served,
          "delivery": run_delivery}[args.workload]
    kw = {"mix": args.served_mix} if args.workload == "served" else {}
    with bench.ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        fn(args, mgv, torch, ctx, bench, clk, **kw)
    ctx.close()
    return 0
