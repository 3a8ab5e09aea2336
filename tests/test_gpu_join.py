"""Hash build + probe on the GPU against the oracle's chained-table join.

The oracle restates sum_hashjoin_select_cpu (src/main8.cu:84-103), itself
pinned to the reference's compiled CPU code by tests/test_oracle_golden.py.
Cases follow the reference's join checks (src/main8.cu:322-355: match count
against the CPU join) plus the configurations' known answers.
"""
import json
import os

import numpy as np
import pytest

import mgv
import pyoracle as po
from gpu_util import dev, i32

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))
HIT = 3865470566  # 0.9 * 2^32


def join_count_sum(ctx, torch, bk, bp, pk, pp, load_factor=0.0, build_filter=None, expected=None):
    """Run build + probe -> aggregate(COUNT, SUM(bp + pp)); returns (count, sum, info)."""
    n, m = bk.size, pk.size
    bhead, hb, probe, agg = mgv.create_count_join_1G_pipeline(ctx, expected or max(n, 1), load_factor, build_filter)
    bhead.open()
    if n:
        bhead.consume_columns([dev(torch, bk), dev(torch, bp)], n)
    bhead.close()
    info = hb.result()
    probe.open()
    if m:
        probe.consume_columns([dev(torch, pk), dev(torch, pp)], m)
    probe.close()
    r = agg.result()
    for o in (probe, agg, bhead, hb):
        o.destroy()
    return r[0], r[1], info


def config2_inputs(nb, npb, seed=0x5EED0002):
    bk = po.gen_perm(nb, seed)
    bp = po.gen_uniform(nb, seed, 1, 0, 1 << 20)
    pk, hits = po.gen_probe_keys(npb, 0x5EED0003, seed, nb, HIT, nb, (1 << 31) - nb)
    pp = po.gen_uniform(npb, 0x5EED0003, 2, 0, 1 << 20)
    return bk, bp, pk, pp, hits


PROBE_VARIANTS = [dict(probe_kernel=0), dict(probe_kernel=1), dict(probe_kernel=2, probe_rows_per_thread=8, probe_stages=2),
                  dict(probe_kernel=2, probe_rows_per_thread=4, probe_stages=6),
                  dict(probe_kernel=2, probe_rows_per_thread=4, probe_stages=4, probe_ctas_per_sm=3),
                  dict(probe_kernel=2, probe_rows_per_thread=8, probe_stages=4, probe_ctas_per_sm=1),
                  dict(probe_kernel=3, probe_rows_per_thread=4, probe_stages=4, probe_ctas_per_sm=3),
                  dict(probe_kernel=3, probe_rows_per_thread=4, probe_stages=2, probe_ctas_per_sm=3)]


@pytest.fixture
def tuned(ctx, request):
    """Apply a probe tuning for one test and restore the default after it."""
    old = ctx.tuning()
    keep = {k: getattr(old, k) for k in ("probe_kernel", "probe_rows_per_thread", "probe_stages", "probe_ctas_per_sm")}
    ctx.set_tuning(**request.param)
    yield request.param
    ctx.set_tuning(**keep)


@pytest.mark.parametrize("tuned", PROBE_VARIANTS, indirect=True, ids=lambda v: "_".join(f"{k[6:]}{x}" for k, x in v.items()))
@pytest.mark.parametrize("nb,npb", [(1 << 10, 1 << 12), (1 << 16, 1 << 20), (1000003, 3000017), (77, 1000)])
def test_config2_shape(ctx, torch_cuda, tuned, nb, npb):
    bk, bp, pk, pp, hits = config2_inputs(nb, npb)
    cnt, s, info = join_count_sum(ctx, torch_cuda, bk, bp, pk, pp)
    want = po.Chain(bk, bp).probe_agg(pk, pp)
    assert (cnt, s) == want
    assert cnt == hits  # known answer: every hit row matches exactly one unique key
    assert info.rows == nb and info.has_duplicates == 0


@pytest.mark.parametrize("offset", [1, 2, 3])
def test_unaligned_probe_columns(ctx, torch_cuda, offset):
    """Columns that are not 16-byte aligned take the register-prefetch kernel."""
    torch = torch_cuda
    bk, bp, pk, pp, hits = config2_inputs(1 << 12, 50001)
    bhead, hb, probe, agg = mgv.create_count_join_1G_pipeline(ctx, bk.size)
    bhead.open(); bhead.consume_columns([dev(torch, bk), dev(torch, bp)], bk.size); bhead.close()
    dpk = dev(torch, np.concatenate([np.zeros(offset, np.int32), pk]))
    dpp = dev(torch, np.concatenate([np.zeros(offset, np.int32), pp]))
    probe.open()
    probe.consume_columns([dpk.data_ptr() + 4 * offset, dpp.data_ptr() + 4 * offset], pk.size)
    probe.close()
    assert agg.result() == po.Chain(bk, bp).probe_agg(pk, pp)
    for o in (probe, agg, hb):
        o.destroy()


@pytest.mark.parametrize("tuned", PROBE_VARIANTS[1:4], indirect=True, ids=lambda v: "_".join(f"{k[6:]}{x}" for k, x in v.items()))
@pytest.mark.parametrize("mode", [(-1, -1), (2, -1), (1, -1), (1, 2)])
def test_sum_modes(ctx, torch_cuda, tuned, mode):
    """COUNT with SUM of nothing, build payload, probe payload, or both."""
    torch = torch_cuda
    bk = po.gen_uniform(5000, 0x5EED0604, 0, 0, 4000)
    bp = po.gen_uniform(5000, 0x5EED0604, 1, -(1 << 31), 1 << 32)
    pk = po.gen_uniform(70001, 0x5EED0604, 2, 0, 4500)
    pp = po.gen_uniform(70001, 0x5EED0604, 3, -(1 << 31), 1 << 32)
    hb = mgv.Op.hash_build(ctx, 0, 1, bk.size)
    hb.open(); hb.consume_columns([dev(torch, bk), dev(torch, bp)], bk.size); hb.close()
    agg = mgv.Op.aggregate(ctx, *mode)
    pr = mgv.Op.hash_probe(ctx, 0, hb, agg)
    pr.open(); pr.consume_columns([dev(torch, pk), dev(torch, pp)], pk.size); pr.close()
    add_b = 2 in mode
    add_p = 1 in mode
    assert agg.result() == po.Chain(bk, bp).probe_agg(pk, pp, add_b, add_p)
    for o in (pr, agg, hb):
        o.destroy()


@pytest.mark.parametrize("lf", [0.4, 0.5])
def test_config2_full_size(ctx, torch_cuda, lf):
    """Build 2^22 unique keys, probe 2^26 (the headline configuration), at the
    benchmark's load factor (0.4) and the context default (0.5)."""
    torch = torch_cuda
    nb, npb = 1 << 22, 1 << 26
    bk = torch.empty(nb, dtype=torch.int32, device="cuda")
    bp = torch.empty(nb, dtype=torch.int32, device="cuda")
    pk = torch.empty(npb, dtype=torch.int32, device="cuda")
    pp = torch.empty(npb, dtype=torch.int32, device="cuda")
    ctx.gen_perm(bk, nb, 0x5EED0002)
    ctx.gen_uniform(bp, nb, 0x5EED0002, 1, 0, 1 << 20)
    hits = ctx.gen_probe_keys(pk, npb, 0x5EED0003, 0x5EED0002, nb, HIT, nb, (1 << 31) - nb)
    ctx.gen_uniform(pp, npb, 0x5EED0003, 2, 0, 1 << 20)
    bhead, hb, probe, agg = mgv.create_count_join_1G_pipeline(ctx, nb, lf)
    bhead.open(); bhead.consume_columns([bk, bp], nb); bhead.close()
    assert hb.result().rows == nb
    probe.open(); probe.consume_columns([pk, pp], npb); probe.close()
    cnt, s = agg.result()
    hbk, hbp = bk.cpu().numpy(), bp.cpu().numpy()
    hpk, hpp = pk.cpu().numpy(), pp.cpu().numpy()
    want = po.Chain(hbk, hbp).probe_agg_mt(hpk, hpp, os.cpu_count() or 1)
    assert cnt == hits
    assert (cnt, s) == want
    # sorted match multiset on the first 2^16 probe rows
    pool = mgv.Pool(ctx, 8, 1 << 16, 3)
    sink = mgv.Op.sink(ctx, pool)
    pe = mgv.Op.hash_probe(ctx, 0, hb, sink)
    pe.open(); pe.consume_columns([pk, pp], 1 << 16); pe.close()
    rows = sink.result()
    out = [torch.empty(rows, dtype=torch.int32, device="cuda") for _ in range(3)]
    for c in range(3):
        sink.sink_read(c, out[c].data_ptr(), rows)
    got = np.stack([out[0].cpu().numpy(), out[2].cpu().numpy(), out[1].cpu().numpy()], 1)  # key, bp, pp
    got = got[np.lexsort((got[:, 2], got[:, 1], got[:, 0]))]
    want_ms = po.Chain(hbk, hbp).probe_emit(hpk[:1 << 16], hpp[:1 << 16])
    assert np.array_equal(got, want_ms)
    for o in (pe, sink, probe, agg, bhead, hb):
        o.destroy()
    pool.destroy()


@pytest.mark.parametrize("lf", [0.25, 0.5, 0.75, 0.95])
def test_duplicates_and_load_factors(ctx, torch_cuda, lf):
    """Duplicate build keys: every duplicate matches (hashjoin.cu:148-162)."""
    nb, npb = 20000, 50000
    bk = po.gen_uniform(nb, 0x5EED0601, 0, 0, 3000)
    bp = po.gen_uniform(nb, 0x5EED0601, 1, -(1 << 31), 1 << 32)
    pk = po.gen_uniform(npb, 0x5EED0601, 2, -100, 3200)
    pp = po.gen_uniform(npb, 0x5EED0601, 3, -(1 << 31), 1 << 32)
    cnt, s, info = join_count_sum(ctx, torch_cuda, bk, bp, pk, pp, load_factor=lf)
    assert (cnt, s) == po.Chain(bk, bp).probe_agg(pk, pp)
    assert info.has_duplicates == 1


@pytest.mark.parametrize("lf", [0.4, 0.5])
def test_region_build_duplicates_large(ctx, torch_cuda, lf):
    """2^18 build rows (the shared-memory region build, 2^16 rows and up)
    with many duplicate keys: the region build's duplicate pass and every
    duplicate's match, against the oracle."""
    nb, npb = 1 << 18, 1 << 20
    bk = po.gen_uniform(nb, 0x5EED0611, 0, 0, 1 << 17)  # about 2 copies per key
    bp = po.gen_uniform(nb, 0x5EED0611, 1, -(1 << 31), 1 << 32)
    pk = po.gen_uniform(npb, 0x5EED0611, 2, -1000, (1 << 17) + 2000)
    pp = po.gen_uniform(npb, 0x5EED0611, 3, -(1 << 31), 1 << 32)
    cnt, s, info = join_count_sum(ctx, torch_cuda, bk, bp, pk, pp, load_factor=lf)
    assert (cnt, s) == po.Chain(bk, bp).probe_agg(pk, pp)
    assert info.has_duplicates == 1 and info.rows == nb


def test_reserved_key_int32_min(ctx, torch_cuda):
    """INT32_MIN is the table's empty marker; such rows still join exactly."""
    mn = -(1 << 31)
    bk = np.array([mn, 5, mn, 7, 5, mn, 2147483647], np.int32)
    bp = np.array([1, 2, 3, 4, 5, 6, 7], np.int32)
    pk = np.array([mn, 5, 7, 8, mn, 2147483647, 0], np.int32)
    pp = np.array([10, 20, 30, 40, 50, 60, 70], np.int32)
    cnt, s, info = join_count_sum(ctx, torch_cuda, bk, bp, pk, pp)
    assert (cnt, s) == po.Chain(bk, bp).probe_agg(pk, pp)
    assert info.reserved_key_rows == 3


@pytest.mark.parametrize("nb,npb", [(0, 100), (100, 0), (1, 1), (129, 4097)])
def test_empty_and_tiny(ctx, torch_cuda, nb, npb):
    bk = po.gen_uniform(nb, 0x5EED0602, 0, 0, 50)
    bp = po.gen_uniform(nb, 0x5EED0602, 1, 0, 1 << 20)
    pk = po.gen_uniform(npb, 0x5EED0602, 2, 0, 60)
    pp = po.gen_uniform(npb, 0x5EED0602, 3, 0, 1 << 20)
    cnt, s, _ = join_count_sum(ctx, torch_cuda, bk, bp, pk, pp)
    assert (cnt, s) == po.Chain(bk, bp).probe_agg(pk, pp)


@pytest.mark.parametrize("case", [c for c in GOLDEN["cases"] if c["op"] == "hashjoin"],
                         ids=lambda c: f"b{c['build']['n']}_p{c['probe']['n']}")
def test_golden_count_join_select(ctx, torch_cuda, case):
    """select(key <= 5000) -> build; probe -> COUNT == sum_hashjoin_select_cpu."""
    b, p = case["build"], case["probe"]
    a = po.gen_uniform(b["n"], b["seed"], b["stream"], b["lo"], b["range"])
    q = po.gen_uniform(p["n"], p["seed"], p["stream"], p["lo"], p["range"])
    zeros_a, zeros_q = np.zeros(a.size, np.int32), np.zeros(q.size, np.int32)
    cnt, _, _ = join_count_sum(ctx, torch_cuda, a, zeros_a, q, zeros_q, build_filter=case["build_filter"],
                               expected=max(a.size, 1))
    assert i32(cnt) == case["count_int32"]


@pytest.mark.parametrize("case", [c for c in GOLDEN["cases"] if c["op"] == "selfjoin"], ids=lambda c: f"n{c['input']['n']}")
def test_golden_selfjoin(ctx, torch_cuda, case):
    """select(a <= 5000) joined with itself == sum_selfjoin_select_cpu (sum of hist^2)."""
    s = case["input"]
    a = po.gen_uniform(s["n"], s["seed"], s["stream"], s["lo"], s["range"])
    z = np.zeros(a.size, np.int32)
    # build: select(a <= 5000) -> hash_build; probe: select(a <= 5000) -> hash_probe -> sink is
    # not needed: probe every row and let the build side's filter decide, then subtract nothing:
    # rows a > 5000 never match a build key <= 5000.
    cnt, _, _ = join_count_sum(ctx, torch_cuda, a, z, a, z, build_filter=5000, expected=max(a.size, 1))
    assert i32(cnt) == case["count_int32"]


def test_table_full_is_reported(ctx, torch_cuda):
    bk = np.arange(1000, dtype=np.int32)
    bp = np.zeros(1000, np.int32)
    hb = mgv.Op.hash_build(ctx, 0, 1, 10, 0.5)
    hb.open()
    hb.consume_columns([dev(torch_cuda, bk), dev(torch_cuda, bp)], 1000)
    with pytest.raises(mgv.MgvError) as e:
        hb.close()
    assert e.value.status == mgv.ENOMEM
    hb.destroy()


def test_probe_before_build_closed_is_rejected(ctx):
    hb = mgv.Op.hash_build(ctx, 0, 1, 100)
    agg = mgv.Op.aggregate(ctx, 1, 2)
    pr = mgv.Op.hash_probe(ctx, 0, hb, agg)
    with pytest.raises(mgv.MgvError) as e:
        pr.open()
    assert e.value.status == mgv.ESTATE
    for o in (pr, agg, hb):
        o.destroy()


def test_duplicate_emit_multiset(ctx, torch_cuda):
    torch = torch_cuda
    nb, npb = 3000, 5000
    bk = po.gen_uniform(nb, 0x5EED0603, 0, 0, 500)
    bp = po.gen_uniform(nb, 0x5EED0603, 1, 0, 1 << 20)
    pk = po.gen_uniform(npb, 0x5EED0603, 2, 0, 600)
    pp = po.gen_uniform(npb, 0x5EED0603, 3, 0, 1 << 20)
    hb = mgv.Op.hash_build(ctx, 0, 1, nb)
    hb.open(); hb.consume_columns([dev(torch, bk), dev(torch, bp)], nb); hb.close()
    pool = mgv.Pool(ctx, 64, 1 << 14, 3)
    sink = mgv.Op.sink(ctx, pool)
    pe = mgv.Op.hash_probe(ctx, 0, hb, sink)
    pe.open(); pe.consume_columns([dev(torch, pk), dev(torch, pp)], npb); pe.close()
    rows = sink.result()
    out = [torch.empty(max(rows, 1), dtype=torch.int32, device="cuda") for _ in range(3)]
    for c in range(3):
        sink.sink_read(c, out[c].data_ptr(), rows)
    got = np.stack([out[0].cpu().numpy()[:rows], out[2].cpu().numpy()[:rows], out[1].cpu().numpy()[:rows]], 1)
    got = got[np.lexsort((got[:, 2], got[:, 1], got[:, 0]))]
    assert np.array_equal(got, po.Chain(bk, bp).probe_emit(pk, pp))
    for o in (pe, sink, hb):
        o.destroy()
    pool.destroy()


@pytest.mark.parametrize("tuned", PROBE_VARIANTS[2:], indirect=True, ids=lambda v: "_".join(f"{k[6:]}{x}" for k, x in v.items()))
def test_staged_probe_is_repeatable(ctx, torch_cuda, tuned):
    """Many probe passes over one table: every pass exact (catches races in
    the shared-memory stage ring and the continuation queue)."""
    torch = torch_cuda
    nb, npb = 1 << 20, 1 << 22
    bk, bp, pk, pp, hits = config2_inputs(nb, npb)
    bhead, hb, probe, agg = mgv.create_count_join_1G_pipeline(ctx, nb)
    bhead.open(); bhead.consume_columns([dev(torch, bk), dev(torch, bp)], nb); bhead.close()
    d = [dev(torch, pk), dev(torch, pp)]
    want = po.Chain(bk, bp).probe_agg(pk, pp)
    for _ in range(8):
        probe.open(); probe.consume_columns(d, npb); probe.close()
        assert agg.result() == want
    for o in (probe, agg, hb):
        o.destroy()


@pytest.mark.parametrize("lf,build_filter", [(0.5, None), (0.95, None), (0.75, 50000)])
def test_shared_memory_build(ctx, torch_cuda, lf, build_filter):
    """Builds of 2^16 rows or more go through the shared-memory region build.
    Duplicate keys, 20000 copies of one key (a run that crosses region ends,
    so rows are finished by the global overflow insert), INT32_MIN rows, a
    build-side filter and two consume calls into the same table."""
    mn = -(1 << 31)
    nb, npb = 300000, 400000
    bk = po.gen_uniform(nb, 0x5EED0603, 0, 0, 60000)
    bk[:20000] = 7
    bk[20000:20010] = mn
    bp = po.gen_uniform(nb, 0x5EED0603, 1, -(1 << 31), 1 << 32)
    pk = po.gen_uniform(npb, 0x5EED0603, 2, -100, 60100)
    pk[:500] = 7
    pk[500:505] = mn
    pp = po.gen_uniform(npb, 0x5EED0603, 3, -(1 << 31), 1 << 32)
    bhead, hb, probe, agg = mgv.create_count_join_1G_pipeline(ctx, nb, lf, build_filter)
    bhead.open()
    half = nb // 2
    bhead.consume_columns([dev(torch_cuda, bk[:half]), dev(torch_cuda, bp[:half])], half)
    bhead.consume_columns([dev(torch_cuda, bk[half:]), dev(torch_cuda, bp[half:])], nb - half)
    bhead.close()
    info = hb.result()
    probe.open()
    probe.consume_columns([dev(torch_cuda, pk), dev(torch_cuda, pp)], npb)
    probe.close()
    keep = np.ones(nb, bool) if build_filter is None else bk <= build_filter
    assert agg.result() == po.Chain(bk[keep], bp[keep]).probe_agg(pk, pp)
    assert info.rows == int(keep.sum()) and info.reserved_key_rows == 10 and info.has_duplicates == 1
    for o in (probe, agg, bhead, hb):
        o.destroy()


@pytest.mark.parametrize("lf", [0.5, 0.95])
@pytest.mark.parametrize("seed", range(4))
def test_shared_memory_build_one_duplicate_pair(ctx, torch_cuda, lf, seed):
    """Unique keys except for one pair.  The region build claims slots by
    per-bucket fill counters and finds duplicates in a pass afterwards, over
    each bucket and the full buckets after it; at load factor 0.95 many runs
    span several buckets, so the two copies often sit in different buckets.
    A pair the pass missed would mark the table unique, and the probe would
    stop at the first of the two matches."""
    nb, npb = 1 << 18, 1 << 19
    bk = po.gen_perm(nb, 0x5EED0700 + seed)
    rng = np.random.default_rng(0x5EED0710 + seed)
    i, j = rng.choice(nb, 2, replace=False)
    bk[j] = bk[i]
    bp = po.gen_uniform(nb, 0x5EED0720 + seed, 1, 0, 1 << 20)
    pk = po.gen_uniform(npb, 0x5EED0730 + seed, 0, 0, nb)
    pk[:64] = bk[i]
    pp = po.gen_uniform(npb, 0x5EED0730 + seed, 1, 0, 1 << 20)
    cnt, s, info = join_count_sum(ctx, torch_cuda, bk, bp, pk, pp, load_factor=lf)
    assert info.has_duplicates == 1 and info.rows == nb
    assert (cnt, s) == po.Chain(bk, bp).probe_agg(pk, pp)


def test_shared_memory_build_unique_full_table(ctx, torch_cuda):
    """Unique keys at load factor 0.95: long runs of full buckets, no false
    duplicate."""
    bk, bp, pk, pp, hits = config2_inputs(1 << 18, 1 << 19, seed=0x5EED0740)
    cnt, s, info = join_count_sum(ctx, torch_cuda, bk, bp, pk, pp, load_factor=0.95)
    assert info.has_duplicates == 0 and info.rows == 1 << 18
    assert cnt == hits and (cnt, s) == po.Chain(bk, bp).probe_agg(pk, pp)


def test_shared_memory_build_unique_keys(ctx, torch_cuda):
    """A region-built table of unique keys is reported duplicate-free (so the
    probe stops at the first match) and joins exactly."""
    bk, bp, pk, pp, hits = config2_inputs(1 << 20, 1 << 21)
    cnt, s, info = join_count_sum(ctx, torch_cuda, bk, bp, pk, pp)
    assert info.has_duplicates == 0 and info.rows == 1 << 20
    assert cnt == hits and (cnt, s) == po.Chain(bk, bp).probe_agg(pk, pp)


MN, MX = -(1 << 31), (1 << 31) - 1


@pytest.mark.parametrize("tuned", [PROBE_VARIANTS[0], PROBE_VARIANTS[1], PROBE_VARIANTS[4], PROBE_VARIANTS[6]],
                         indirect=True, ids=lambda v: "_".join(f"{k[6:]}{x}" for k, x in v.items()))
@pytest.mark.parametrize("case", ["spread", "extremes", "only_reserved", "narrow", "negative"])
def test_probe_keys_around_the_build_range(ctx, torch_cuda, tuned, case):
    """Probe keys at, just inside and just outside both ends of the build
    keys' range, INT32_MIN (the side list) and INT32_MAX, and a build of
    reserved keys only, all against the oracle."""
    rng = np.random.default_rng(sum(map(ord, case)))
    if case == "spread":
        bk = rng.integers(-1000, 1000, 40000).astype(np.int32)
    elif case == "extremes":
        bk = rng.integers(-50, 50, 30000).astype(np.int32)
        bk[:4] = [MN, MX, MN + 1, MX - 1]
    elif case == "only_reserved":
        bk = np.full(5000, MN, np.int32)
    elif case == "narrow":
        bk = np.full(70000, 12345, np.int32)
        bk[::3] = 12346
    else:
        bk = rng.integers(-(1 << 30), -(1 << 29), 100000).astype(np.int32)
    lo = int(bk[bk != MN].min()) if (bk != MN).any() else 0
    hi = int(bk[bk != MN].max()) if (bk != MN).any() else 0
    edge = np.array([lo - 1, lo, lo + 1, hi - 1, hi, hi + 1, MN, MX, MN + 1, MX - 1, 0], np.int64)
    edge = np.clip(edge, MN, MX).astype(np.int32)
    pk = np.concatenate([rng.integers(MN, MX, 300000, dtype=np.int64).astype(np.int32),
                         rng.choice(bk, 300000), np.tile(edge, 1000)])
    pk = pk[rng.permutation(pk.size)]
    bp = rng.integers(MN, MX, bk.size, dtype=np.int64).astype(np.int32)
    pp = rng.integers(MN, MX, pk.size, dtype=np.int64).astype(np.int32)
    c, s, _ = join_count_sum(ctx, torch_cuda, bk, bp, pk, pp)
    assert (c, s) == po.Chain(bk, bp).probe_agg(pk, pp)


def test_reopened_build_with_other_keys(ctx, torch_cuda):
    """One build operator reopened three times, each time with keys in another
    range, probed after each build."""
    torch = torch_cuda
    bhead, hb, probe, agg = mgv.create_count_join_1G_pipeline(ctx, 100000)
    pk = np.arange(-10000, 20000, dtype=np.int32)
    pp = np.ones(pk.size, np.int32)
    dpk, dpp = dev(torch, pk), dev(torch, pp)
    for lo in (0, 5000, -9000):
        bk = np.arange(lo, lo + 1000, dtype=np.int32)
        bp = np.full(bk.size, 7, np.int32)
        bhead.open()
        bhead.consume_columns([dev(torch, bk), dev(torch, bp)], bk.size)
        bhead.close()
        probe.open()
        probe.consume_columns([dpk, dpp], pk.size)
        probe.close()
        assert agg.result() == po.Chain(bk, bp).probe_agg(pk, pp) == (1000, 8000)
    for o in (probe, agg, bhead, hb):
        o.destroy()
