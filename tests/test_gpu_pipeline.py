"""select -> hash join -> group-by, the radix partitioner, and the generic
fused chain, on the GPU against the oracle.

The pipeline is the reference's count_join_select plan shape
(src/main9.cu:260-324: split/hash_exchange before the build, select before
the probe) with the exchange reduced to an in-GPU 8-bit radix partition and
the count widened to a per-group int64 SUM/COUNT."""
import os

import numpy as np
import pytest

import mgv
import pyoracle as po
from gpu_util import dev, sorted_rows

pytestmark = pytest.mark.gpu


def config3_inputs(nb, npb, groups=4096, seed=0x5EED0901, key_range=None):
    bk = po.gen_perm(nb, seed)
    pkey = po.gen_uniform(npb, seed, 1, 0, key_range or nb)
    pfil = po.gen_uniform(npb, seed, 2, 0, 1000)
    pgrp = po.gen_zipf(npb, seed, 3, groups)
    pval = po.gen_uniform(npb, seed, 4, 0, 1 << 16)
    return bk, pkey, pfil, pgrp, pval


def run_pipeline(ctx, torch, bk, probe_cols, groups, bound, radix_bits=8):
    part, hb, sel, gb = mgv.create_join_groupby_pipeline(ctx, bk.size, groups, bound, radix_bits)
    part.open(); part.consume_columns([dev(torch, bk)], bk.size); part.close()
    info = hb.result()
    sel.open(); sel.consume_columns([dev(torch, c) for c in probe_cols], probe_cols[0].size); sel.close()
    r = gb.result()
    for o in (sel, gb, hb, part):
        o.destroy()
    return r, info


@pytest.mark.parametrize("radix_bits", [0, 4, 8])
@pytest.mark.parametrize("nb,npb", [(1 << 12, 1 << 16), (1 << 16, 1 << 20), (100003, 3000017)])
def test_select_join_groupby(ctx, torch_cuda, radix_bits, nb, npb):
    bk, pkey, pfil, pgrp, pval = config3_inputs(nb, npb, key_range=nb + nb // 8)  # some keys miss
    got, info = run_pipeline(ctx, torch_cuda, bk, [pkey, pfil, pgrp, pval], 4096, 99, radix_bits)
    want, _, _ = po.run_query(bk, pkey, pfil, pgrp, pval, 99)
    assert got == [(int(w["group"]), int(w["sum"]), int(w["count"])) for w in want]
    assert info.rows == nb


@pytest.mark.parametrize("radix_bits", [1, 2])
def test_partitioned_build_wide_regions(ctx, torch_cuda, radix_bits):
    """Few partitions of a large table: each partition spans over a hundred
    shared-memory regions, so the warp tiles of the partition op's run span
    more regions than a warp sorts and take the per-row cursor path."""
    nb, npb = 1 << 20, 1 << 20
    bk, pkey, pfil, pgrp, pval = config3_inputs(nb, npb, seed=0x5EED0905, key_range=nb + nb // 8)
    got, info = run_pipeline(ctx, torch_cuda, bk, [pkey, pfil, pgrp, pval], 4096, 499, radix_bits)
    want, _, _ = po.run_query(bk, pkey, pfil, pgrp, pval, 499)
    assert got == [(int(w["group"]), int(w["sum"]), int(w["count"])) for w in want]
    assert info.rows == nb and info.has_duplicates == 0


def test_partitioned_build_of_nothing(ctx, torch_cuda):
    """A partition op that stores no rows closes its (empty) build; every
    probe then misses."""
    bk = np.empty(0, dtype=np.int32)
    _, pkey, pfil, pgrp, pval = config3_inputs(1 << 12, 1 << 14, seed=0x5EED0906)
    got, info = run_pipeline(ctx, torch_cuda, bk, [pkey, pfil, pgrp, pval], 4096, 999, 8)
    assert got == [] and info.rows == 0


@pytest.mark.parametrize("lf", [0.5, 0.6])
def test_config3_full_size(ctx, torch_cuda, lf):
    """probe 2^27 rows, build 2^24 keys, 10% selectivity, Zipf(1) over 4096
    groups, at the default load factor (0.5) and the benchmark's (0.6)."""
    torch = torch_cuda
    nb, npb = 1 << 24, 1 << 27
    cols = [torch.empty(npb, dtype=torch.int32, device="cuda") for _ in range(4)]
    bk = torch.empty(nb, dtype=torch.int32, device="cuda")
    seed = 0x5EED0003
    ctx.gen_perm(bk, nb, seed)
    ctx.gen_uniform(cols[0], npb, seed, 1, 0, nb)
    ctx.gen_uniform(cols[1], npb, seed, 2, 0, 1000)
    ctx.gen_zipf(cols[2], npb, seed, 3, 4096)
    ctx.gen_uniform(cols[3], npb, seed, 4, 0, 1 << 16)
    part, hb, sel, gb = mgv.create_join_groupby_pipeline(ctx, nb, 4096, 99, 8, lf)
    part.open(); part.consume_columns([bk], nb); part.close()
    assert hb.result().rows == nb
    sel.open(); sel.consume_columns(cols, npb); sel.close()
    got = gb.result()
    host = [c.cpu().numpy() for c in cols]
    want, tc, ts = po.run_query(bk.cpu().numpy(), *host, 99)
    assert got == [(int(w["group"]), int(w["sum"]), int(w["count"])) for w in want]
    # every probe key is a build key: the count is the number of qualifying rows
    assert sum(c for _, _, c in got) == int((host[1] <= 99).sum())
    for o in (sel, gb, hb, part):
        o.destroy()


def test_partition_histogram_and_rows(ctx, torch_cuda):
    torch = torch_cuda
    n = 200003
    k = po.gen_uniform(n, 0x5EED0902, 0, -(1 << 31), 1 << 32)
    v = po.gen_uniform(n, 0x5EED0902, 1, 0, 1000)
    pool = mgv.Pool(ctx, 16, 1 << 15, 2)
    sink = mgv.Op.sink(ctx, pool)
    part = mgv.Op.partition(ctx, 0, 8, 3, n, sink)
    part.open()
    part.consume_columns([dev(torch, k[:n // 2]), dev(torch, v[:n // 2])], n // 2)   # two runs
    part.consume_columns([dev(torch, k[n // 2:]), dev(torch, v[n // 2:])], n - n // 2)
    part.close()
    hist = part.result()
    want_hist, _, _ = po.partition(k, 8, 3)
    assert hist == [int(x) for x in want_hist]
    rows = sink.result()
    assert rows == n
    out = [torch.empty(rows, dtype=torch.int32, device="cuda") for _ in range(2)]
    for c in range(2):
        sink.sink_read(c, out[c].data_ptr(), rows)
    got = sorted_rows([o.cpu().numpy() for o in out])
    assert np.array_equal(got, sorted_rows([k, v]))
    for o in (part, sink):
        o.destroy()
    pool.destroy()


def test_partition_more_rows_than_max_rows_is_reported(ctx, torch_cuda):
    """The partition's cursors are computed on the device, so a consume past
    max_rows is reported by close (rows past the store are dropped, none is
    written out of it); the operator then works again after reopening."""
    torch = torch_cuda
    n = 50000
    k = po.gen_uniform(n, 0x5EED0903, 0, -(1 << 31), 1 << 32)
    pool = mgv.Pool(ctx, 4, 1 << 15, 1)
    sink = mgv.Op.sink(ctx, pool)
    part = mgv.Op.partition(ctx, 0, 4, 0, n - 1, sink)
    part.open()
    part.consume_columns([dev(torch, k)], n)
    with pytest.raises(mgv.MgvError) as e:
        part.close()
    assert e.value.status == mgv.ENOMEM
    part.open()
    part.consume_columns([dev(torch, k[:n - 1])], n - 1)
    part.close()
    assert sum(part.result()) == n - 1 and sink.result() == n - 1
    for o in (part, sink):
        o.destroy()
    pool.destroy()


def test_select_partition_aggregate(ctx, torch_cuda):
    n = 100000
    f = po.gen_uniform(n, 0x5EED0903, 0, 0, 100)
    k = po.gen_uniform(n, 0x5EED0903, 1, 0, 1 << 20)
    agg = mgv.Op.aggregate(ctx, 1, -1)
    part = mgv.Op.partition(ctx, 1, 4, 0, n, agg)
    sel = mgv.Op.select(ctx, 0, 49, part)
    sel.open(); sel.consume_columns([dev(torch_cuda, f), dev(torch_cuda, k)], n); sel.close()
    assert agg.result() == po.select_agg(f, k, 49)
    # only the device knows how many rows passed the select: close read the totals back
    want_hist, _, _ = po.partition(k[f <= 49], 4, 0)
    assert part.result() == [int(x) for x in want_hist]
    for o in (sel, part, agg):
        o.destroy()


@pytest.mark.parametrize("dup", [False, True])
def test_select_probe_aggregate_and_sink(ctx, torch_cuda, dup):
    """The generic chain with a select before the probe, both terminals."""
    torch = torch_cuda
    nb, npb = 5000, 200003
    bk = po.gen_uniform(nb, 0x5EED0904, 0, 0, 2000) if dup else po.gen_perm(nb, 0x5EED0904)
    bp = po.gen_uniform(nb, 0x5EED0904, 1, -(1 << 20), 1 << 21)
    pk = po.gen_uniform(npb, 0x5EED0904, 2, 0, 6000)
    pf = po.gen_uniform(npb, 0x5EED0904, 3, 0, 100)
    pp = po.gen_uniform(npb, 0x5EED0904, 4, -(1 << 20), 1 << 21)
    hb = mgv.Op.hash_build(ctx, 0, 1, nb)
    hb.open(); hb.consume_columns([dev(torch, bk), dev(torch, bp)], nb); hb.close()
    keep = pf <= 30
    chain = po.Chain(bk, bp)
    # aggregate: COUNT + SUM(bp + pp) over the selected probe rows
    agg = mgv.Op.aggregate(ctx, 3, 2)        # build payload is column 3 (= ncols)
    pr = mgv.Op.hash_probe(ctx, 0, hb, agg)
    sel = mgv.Op.select(ctx, 1, 30, pr)
    d = [dev(torch, pk), dev(torch, pf), dev(torch, pp)]
    sel.open(); sel.consume_columns(d, npb); sel.close()
    assert agg.result() == chain.probe_agg(pk[keep], pp[keep])
    # sink: (key, filter, pp, bp) rows
    pool = mgv.Pool(ctx, 64, 1 << 15, 4)
    sink = mgv.Op.sink(ctx, pool)
    pr2 = mgv.Op.hash_probe(ctx, 0, hb, sink)
    sel2 = mgv.Op.select(ctx, 1, 30, pr2)
    sel2.open(); sel2.consume_columns(d, npb); sel2.close()
    rows = sink.result()
    out = [torch.empty(max(rows, 1), dtype=torch.int32, device="cuda") for _ in range(4)]
    for c in range(4):
        sink.sink_read(c, out[c].data_ptr(), rows)
    o = [x.cpu().numpy()[:rows] for x in out]
    got = sorted_rows([o[0], o[3], o[2]])               # key, bp, pp
    want = chain.probe_emit(pk[keep], pp[keep])
    assert np.array_equal(got, want.astype(np.int64))
    for x in (sel, pr, agg, sel2, pr2, sink, hb):
        x.destroy()
    pool.destroy()


@pytest.mark.parametrize("offset", [1, 2, 3])
def test_chain_unaligned_columns_and_reserved_keys(ctx, torch_cuda, offset):
    """select -> join -> group-by over columns that start at different 4-byte
    offsets, with duplicate build keys and INT32_MIN keys on both sides."""
    torch = torch_cuda
    mn = -(1 << 31)
    nb, npb = 3000, 100003
    bk = po.gen_uniform(nb, 0x5EED0905, 0, 0, 2000)
    bk[:7] = mn
    pk = po.gen_uniform(npb, 0x5EED0905, 1, 0, 2500)
    pk[::997] = mn
    pf = po.gen_uniform(npb, 0x5EED0905, 2, 0, 100)
    pg = po.gen_zipf(npb, 0x5EED0905, 3, 300)
    pv = po.gen_uniform(npb, 0x5EED0905, 4, -(1 << 31), 1 << 32)
    hb = mgv.Op.hash_build(ctx, 0, -1, nb)
    hb.open(); hb.consume_columns([dev(torch, bk)], nb); hb.close()
    gb = mgv.Op.groupby(ctx, 2, 3, 300)
    pr = mgv.Op.hash_probe(ctx, 0, hb, gb)
    sel = mgv.Op.select(ctx, 1, 60, pr)
    # each column starts at its own 4-byte offset inside a larger allocation
    cols = []
    for i, c in enumerate([pk, pf, pg, pv]):
        o = (offset + i) % 4
        big = torch.empty(npb + 8, dtype=torch.int32, device="cuda")
        big[o:o + npb] = torch.from_numpy(c).to("cuda")
        cols.append(big[o:o + npb])
    sel.open(); sel.consume_columns(cols, npb); sel.close()
    want, _, _ = po.run_query(bk, pk, pf, pg, pv, 60)
    assert gb.result() == [(int(w["group"]), int(w["sum"]), int(w["count"])) for w in want]
    for o in (sel, pr, gb, hb):
        o.destroy()
