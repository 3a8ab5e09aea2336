"""The result delivery channel: one open sink streams a join's full match
multiset to host memory through a pool much smaller than the output
(gpu_to_cpu + buffer swap, src/operators/gpu_to_cpu.cu:41-165), drained
between consume calls; the multiset equals the oracle's."""
import numpy as np
import pytest

import mgv
import pyoracle as po
from gpu_util import dev

pytestmark = pytest.mark.gpu
HIT = 3865470566  # 0.9 * 2^32


def test_sink_drain_delivers_more_rows_than_the_pool_holds(ctx, torch_cuda):
    torch = torch_cuda
    nb, npb, step = 1 << 16, 1 << 20, 1 << 17
    bk = po.gen_perm(nb, 0x5EED0701)
    bp = po.gen_uniform(nb, 0x5EED0701, 1, -(1 << 31), 1 << 32)
    pk, hits = po.gen_probe_keys(npb, 0x5EED0702, 0x5EED0701, nb, HIT, nb, (1 << 31) - nb)
    pp = po.gen_uniform(npb, 0x5EED0702, 2, -(1 << 31), 1 << 32)
    hb = mgv.Op.hash_build(ctx, 0, 1, nb)
    hb.open(); hb.consume_columns([dev(torch, bk), dev(torch, bp)], nb); hb.close()
    pool = mgv.Pool(ctx, 4, 1 << 16, 3)          # 256 Ki rows: a quarter of the output
    sink = mgv.Op.sink(ctx, pool)
    probe = mgv.Op.hash_probe(ctx, 0, hb, sink)
    dk, dp = dev(torch, pk), dev(torch, pp)
    out = [torch.empty(npb, dtype=torch.int32).pin_memory() for _ in range(3)]
    probe.open()
    total = 0
    assert sink.sink_drain() == 0
    for lo in range(0, npb, step):
        probe.consume_columns([dk[lo:lo + step], dp[lo:lo + step]], step)
        waiting = sink.sink_drain()                       # count only
        got = sink.sink_drain([o.data_ptr() + 4 * total for o in out], npb - total)
        assert got == waiting > 0
        total += got
    probe.close()
    assert total == hits > 4 * (1 << 16)
    rows = np.stack([out[0].numpy()[:total], out[2].numpy()[:total], out[1].numpy()[:total]], 1)
    rows = rows[np.lexsort((rows[:, 2], rows[:, 1], rows[:, 0]))]
    assert np.array_equal(rows, po.Chain(bk, bp).probe_emit(pk, pp))
    for o in (probe, sink, hb):
        o.destroy()
    pool.destroy()


def test_sink_drain_rejects_a_small_destination_and_keeps_the_rows(ctx, torch_cuda):
    torch = torch_cuda
    n = 5000
    keys = np.arange(n, dtype=np.int32)
    pool = mgv.Pool(ctx, 2, 1 << 12, 1)
    sink = mgv.Op.sink(ctx, pool)
    sink.open()
    sink.consume_columns([dev(torch, keys)], n)
    small = torch.empty(100, dtype=torch.int32, device="cuda")
    with pytest.raises(mgv.MgvError) as e:
        sink.sink_drain([small], 100)
    assert e.value.status == mgv.EINVAL
    full = torch.empty(n, dtype=torch.int32, device="cuda")
    assert sink.sink_drain([full], n) == n
    assert sink.sink_drain() == 0                 # the copy is complete once the next drain returns
    assert np.array_equal(np.sort(full.cpu().numpy()), keys)
    sink.close()
    assert sink.result() == 0
    sink.destroy()
    pool.destroy()
