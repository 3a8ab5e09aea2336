"""Hash GROUP BY on the GPU against the oracle (no reference counterpart:
the reference aggregates a global SUM only, src/operators/aggregation.cu)."""
import numpy as np
import pytest

import mgv
import pyoracle as po
from gpu_util import dev

pytestmark = pytest.mark.gpu


@pytest.fixture
def smem_slots(ctx, request):
    old = ctx.tuning().groupby_smem_slots
    ctx.set_tuning(groupby_smem_slots=request.param)
    yield request.param
    ctx.set_tuning(groupby_smem_slots=old)


def rows(res):
    return [(g, s, c) for g, s, c in res]


def oracle_rows(groups, values, mult=None):
    r = po.groupby(groups, values, mult)
    return [(int(x["group"]), int(x["sum"]), int(x["count"])) for x in r]


def run_groupby(ctx, torch, cols, n, group_col, value_col, max_groups, sel=None):
    gb = mgv.Op.groupby(ctx, group_col, value_col, max_groups)
    head = mgv.Op.select(ctx, sel[0], sel[1], gb) if sel else gb
    head.open()
    head.consume_columns([dev(torch, c) for c in cols], n)
    head.close()
    r = gb.result()
    head.destroy()
    gb.destroy()
    return r


@pytest.mark.parametrize("smem_slots", [0, 1024, 4096], indirect=True)
@pytest.mark.parametrize("G,n,dist", [(1, 5000, "uniform"), (16, 100003, "zipf"), (4096, 1 << 20, "zipf"),
                                      (65536, 1 << 20, "uniform"), (300000, 1 << 20, "uniform")])
def test_groupby_matches_oracle(ctx, torch_cuda, smem_slots, G, n, dist):
    g = po.gen_zipf(n, 0x5EED0801, 1, G) if dist == "zipf" else po.gen_uniform(n, 0x5EED0801, 1, -G // 2, G)
    v = po.gen_uniform(n, 0x5EED0801, 2, -(1 << 31), 1 << 32)
    got = run_groupby(ctx, torch_cuda, [g, v], n, 0, 1, max(G, 16))
    assert rows(got) == oracle_rows(g, v)


def test_groupby_count_only_and_reserved_group(ctx, torch_cuda):
    mn = -(1 << 31)
    g = np.array([mn, 3, mn, 3, 7, mn], np.int32)
    got = run_groupby(ctx, torch_cuda, [g], g.size, 0, -1, 8)
    assert rows(got) == oracle_rows(g, None)


def test_select_groupby(ctx, torch_cuda):
    n = 300007
    f = po.gen_uniform(n, 0x5EED0802, 0, 0, 1000)
    g = po.gen_zipf(n, 0x5EED0802, 1, 4096)
    v = po.gen_uniform(n, 0x5EED0802, 2, 0, 1 << 16)
    got = run_groupby(ctx, torch_cuda, [f, g, v], n, 1, 2, 4096, sel=(0, 99))
    keep = f <= 99
    assert rows(got) == oracle_rows(g[keep], v[keep])


def test_groupby_table_full_is_reported(ctx, torch_cuda):
    n = 5000
    g = np.arange(n, dtype=np.int32)
    gb = mgv.Op.groupby(ctx, 0, -1, 16)   # 1024-slot table for 5000 groups
    gb.open()
    gb.consume_columns([dev(torch_cuda, g)], n)
    with pytest.raises(mgv.MgvError) as e:
        gb.close()
    assert e.value.status == mgv.ENOMEM
    gb.destroy()
