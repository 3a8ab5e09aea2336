"""Host ingest with overlapped copies (mgv_op_consume_host).

The reference's generator slices a host column into pool buffers and its
consumer copies each buffer to the device, then launches the consume kernel
(src/operators/generators.cu:55-90, src/operators/exchange.cu:196-291).
mgv_op_consume_host does the same through a bounded pool with the copy of
slice k+1 overlapping the consume of slice k.  Results must equal the
oracle's, whatever the slicing: 2^28 host probe rows through three 4 Mi-row
buffers (columns far larger than the pool), pageable and pinned sources,
ragged and empty inputs, and the select -> aggregate chain."""
import os

import numpy as np
import pytest

import mgv
import pyoracle as po
from gpu_util import dev

pytestmark = pytest.mark.gpu

HIT = 3865470566


def build_join(ctx, torch, nb, seed):
    bk = po.gen_perm(nb, seed)
    bp = po.gen_uniform(nb, seed, 1, 0, 1 << 20)
    bhead, hb, probe, agg = mgv.create_count_join_1G_pipeline(ctx, nb, 0.5)
    bhead.open(); bhead.consume_columns([dev(torch, bk), dev(torch, bp)], nb); bhead.close()
    return bk, bp, bhead, hb, probe, agg


def test_join_probe_of_2_28_host_rows(ctx, torch_cuda):
    torch = torch_cuda
    nb, npb = 1 << 20, 1 << 28
    bk, bp, bhead, hb, probe, agg = build_join(ctx, torch, nb, 0x5EED0A01)
    pk, hits = po.gen_probe_keys(npb, 0x5EED0A02, 0x5EED0A01, nb, HIT, nb, (1 << 31) - nb)
    pp = po.gen_uniform(npb, 0x5EED0A02, 2, 0, 1 << 20)
    pool = mgv.Pool(ctx, 3, mgv.DEFAULT_BUFFER_ROWS, 2)  # 96 MiB of buffers for 2 GiB of columns
    probe.open()
    probe.consume_host(pool, [pk, pp], npb)  # pageable numpy columns
    probe.close()
    got = agg.result()
    want = po.Chain(bk, bp).probe_agg_mt(pk, pp, os.cpu_count() or 1)
    assert got == want and got[0] == hits
    s = pool.stats()
    assert s.available + s.host_cached == 3  # every buffer back in the pool
    for o in (probe, agg, bhead, hb):
        o.destroy()
    pool.destroy()


@pytest.mark.parametrize("rows", [0, 1, 4097, (1 << 22) + 5, 3 * (1 << 20) + 17])
def test_ragged_pinned_and_repeated(ctx, torch_cuda, rows):
    """Pinned torch sources, row counts that are not multiples of the buffer
    capacity (1 Mi rows here), two calls into one open chain."""
    torch = torch_cuda
    nb = 1 << 16
    bk, bp, bhead, hb, probe, agg = build_join(ctx, torch, nb, 0x5EED0A11)
    pk, _ = po.gen_probe_keys(rows, 0x5EED0A12, 0x5EED0A11, nb, HIT, nb, (1 << 31) - nb)
    pp = po.gen_uniform(rows, 0x5EED0A12, 2, -(1 << 31), 1 << 32)
    hpk = torch.from_numpy(pk).pin_memory()
    hpp = torch.from_numpy(pp).pin_memory()
    pool = mgv.Pool(ctx, 4, 1 << 20, 2)
    probe.open()
    half = rows // 2
    probe.consume_host(pool, [hpk.data_ptr(), hpp.data_ptr()], half)
    probe.consume_host(pool, [hpk.data_ptr() + 4 * half, hpp.data_ptr() + 4 * half], rows - half)
    probe.close()
    assert agg.result() == po.Chain(bk, bp).probe_agg(pk, pp)
    for o in (probe, agg, bhead, hb):
        o.destroy()
    pool.destroy()


def test_select_aggregate_from_host(ctx, torch_cuda):
    """Config 1's chain (select c0 <= 2^30 - 1 -> COUNT, SUM(c1)) from host
    columns through a one-buffer pool (no overlap: copy, consume, copy...)."""
    n = (1 << 22) + 333
    c0 = po.gen_uniform(n, 0x5EED0A21, 0, 0, 1 << 31)
    c1 = po.gen_uniform(n, 0x5EED0A21, 1, 0, 1 << 20)
    head, agg = mgv.create_sum_select_pipeline(ctx, (1 << 30) - 1, 0, 1)
    pool = mgv.Pool(ctx, 1, 1 << 20, 2)
    head.open()
    head.consume_host(pool, [c0, c1], n)
    head.close()
    assert agg.result() == po.select_agg(c0, c1, (1 << 30) - 1)
    head.destroy(); agg.destroy(); pool.destroy()


def test_bad_arguments(ctx, torch_cuda):
    head, agg = mgv.create_sum_select_pipeline(ctx, 0, 0, 1)
    pool = mgv.Pool(ctx, 2, 1024, 1)
    a = np.zeros(10, np.int32)
    head.open()
    with pytest.raises(mgv.MgvError) as e:
        head.consume_host(pool, [a, a], 10)  # more columns than the pool has
    assert e.value.status == mgv.EINVAL
    head.close()
    with pytest.raises(mgv.MgvError) as e:
        head.consume_host(pool, [a], 10)  # chain closed
    assert e.value.status == mgv.ESTATE
    head.destroy(); agg.destroy(); pool.destroy()
