"""select -> aggregate and select -> sink on the GPU against the oracle.

Mirrors the reference's select checks (src/main.cu:88-131: count, then a
sorted element-wise compare of the unordered select output) and its
sum_select pipeline (create_sum_select_pipeline, src/main9.cu:202-226).
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


def run_select_agg(ctx, cols, n, bound, filter_col=0, sum_col=1, compact=0):
    """compact=1 routes the select through the warp-ballot compaction into
    128-row vectors (mgv_tuning.select_compact) instead of the masked fold."""
    before = ctx.tuning().select_compact
    ctx.set_tuning(select_compact=compact)
    try:
        head, agg = mgv.create_sum_select_pipeline(ctx, bound, filter_col, sum_col)
        head.open()
        head.consume_columns(cols, n)
        head.close()
        r = agg.result()
        head.destroy()
        agg.destroy()
    finally:
        ctx.set_tuning(select_compact=before)
    return r


@pytest.mark.parametrize("compact", [0, 1], ids=["fold", "ballot"])
def test_config1_full_size(ctx, torch_cuda, compact):
    """2^22 rows, c0 uniform [0, 2^31), c1 uniform [0, 2^20), c0 < 2^30."""
    torch = torch_cuda
    n = 1 << 22
    c0 = torch.empty(n, dtype=torch.int32, device="cuda")
    c1 = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx.gen_uniform(c0, n, 0x5EED0001, 0, 0, 1 << 31)
    ctx.gen_uniform(c1, n, 0x5EED0001, 1, 0, 1 << 20)
    got = run_select_agg(ctx, [c0, c1], n, (1 << 30) - 1, compact=compact)
    want = po.select_agg(po.gen_uniform(n, 0x5EED0001, 0, 0, 1 << 31), po.gen_uniform(n, 0x5EED0001, 1, 0, 1 << 20),
                         (1 << 30) - 1)
    assert got == want


@pytest.mark.parametrize("case", [c for c in GOLDEN["cases"] if c["op"] == "select"],
                         ids=lambda c: f"n{c['input']['n']}_b{c['bound']}")
@pytest.mark.parametrize("compact", [0, 1], ids=["fold", "ballot"])
def test_golden_sum_select(ctx, torch_cuda, case, compact):
    """COUNT and SUM of the selected column equal sum_select_cpu's answers."""
    s = case["input"]
    a = po.gen_uniform(s["n"], s["seed"], s["stream"], s["lo"], s["range"])
    d = dev(torch_cuda, a if a.size else np.zeros(1, np.int32))
    cnt, tot = run_select_agg(ctx, [d], s["n"], case["bound"], 0, 0, compact=compact)
    assert cnt == case["count"]
    assert i32(tot) == case["sum_int32"]


@pytest.mark.parametrize("n", [1, 7, 127, 128, 129, 4095, 4097, 100003])
@pytest.mark.parametrize("offset", [0, 1])
@pytest.mark.parametrize("compact", [0, 1], ids=["fold", "ballot"])
def test_ragged_and_unaligned(ctx, torch_cuda, n, offset, compact):
    f = po.gen_uniform(n + 1, 0x5EED0501, 0, -1000, 2000)
    v = po.gen_uniform(n + 1, 0x5EED0501, 1, -(1 << 31), 1 << 32)
    df, dv = dev(torch_cuda, f), dev(torch_cuda, v)
    cols = [df.data_ptr() + 4 * offset, dv.data_ptr() + 4 * offset]
    for bound in (-2000, -1, 0, 999, 2000):
        got = run_select_agg(ctx, cols, n, bound, compact=compact)
        assert got == po.select_agg(f[offset:offset + n], v[offset:offset + n], bound)


def test_select_sink_multiset(ctx, torch_cuda):
    """Unordered select output materialised in pool buffers, several swaps."""
    torch = torch_cuda
    n = 300001
    a = po.gen_uniform(n, 0x5EED0502, 0, 1, 10000)
    b = po.gen_uniform(n, 0x5EED0502, 1, 0, 1 << 20)
    pool = mgv.Pool(ctx, 64, 4096, 2)
    sink = mgv.Op.sink(ctx, pool)
    sel = mgv.Op.select(ctx, 0, 5000, sink)
    sel.open()
    sel.consume_columns([dev(torch, a), dev(torch, b)], n)
    sel.close()
    rows = sink.result()
    keep = a <= 5000
    assert rows == int(keep.sum())
    out0 = torch.empty(rows, dtype=torch.int32, device="cuda")
    out1 = torch.empty(rows, dtype=torch.int32, device="cuda")
    assert sink.sink_read(0, out0.data_ptr(), rows) == rows
    assert sink.sink_read(1, out1.data_ptr(), rows) == rows
    got = np.stack([out0.cpu().numpy(), out1.cpu().numpy()], 1)
    want = np.stack([a[keep], b[keep]], 1)
    got = got[np.lexsort((got[:, 1], got[:, 0]))]
    want = want[np.lexsort((want[:, 1], want[:, 0]))]
    assert np.array_equal(got, want)
    # reopening returns the buffers to the pool
    sel.open()
    sel.close()
    assert sink.result() == 0
    sel.destroy(); sink.destroy(); pool.destroy()


def test_select_sink_overflow_reports_enomem(ctx, torch_cuda):
    pool = mgv.Pool(ctx, 2, 128, 1)
    sink = mgv.Op.sink(ctx, pool, max_buffers=2)
    sel = mgv.Op.select(ctx, 0, 100, sink)
    a = np.zeros(1000, np.int32)
    sel.open()
    sel.consume_columns([dev(torch_cuda, a)], a.size)
    with pytest.raises(mgv.MgvError) as e:
        sel.close()
    assert e.value.status == mgv.ENOMEM
    assert sink.result() == 1000  # rows that were produced
    sel.destroy(); sink.destroy(); pool.destroy()


def test_consume_pool_buffer(ctx, torch_cuda):
    """generator -> pool buffer (H2D overwrite) -> consume, buffer by buffer."""
    pool = mgv.Pool(ctx, 4, 1 << 16, 2)
    head, agg = mgv.create_sum_select_pipeline(ctx, 500, 0, 1)
    n = 200000
    a = po.gen_uniform(n, 0x5EED0503, 0, 0, 1000)
    v = po.gen_uniform(n, 0x5EED0503, 1, -50, 100)
    head.open()
    for lo in range(0, n, 1 << 16):
        m = min(1 << 16, n - lo)
        buf = pool.acquire()
        mgv.buffer_write(buf, 0, a[lo:lo + m].ctypes.data, m)
        mgv.buffer_write(buf, 1, v[lo:lo + m].ctypes.data, m)
        head.consume(buf)
        ctx.sync()
        pool.release(buf)
    head.close()
    assert agg.result() == po.select_agg(a, v, 500)
    head.destroy(); agg.destroy(); pool.destroy()
