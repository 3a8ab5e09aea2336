"""The measurement probes of include/mgv_diag.h run and reject bad arguments
(they are not part of the drop-in API; bench.py uses them to measure the
random-read ceilings the hash probe is compared with)."""
import pytest

import mgv

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method,line", [(0, 32), (0, 64), (0, 128), (1, 32), (1, 64), (2, 32)])
def test_gather_methods_run(ctx, method, line):
    ms = ctx.diag_gather(8 << 20, 1 << 20, line_bytes=line, method=method, ctas_per_sm=2, reps=2, inflight=2,
                         lsu_warps=4, tma_warps=1, tma_share=0.25)
    assert 0.0 < ms < 1000.0


def test_random_gather_runs(ctx):
    assert 0.0 < ctx.diag_random_gather(4 << 20, 1 << 20, 2, 2) < 1000.0


@pytest.mark.parametrize("kw", [dict(line_bytes=48), dict(method=3), dict(inflight=0), dict(ctas_per_sm=9),
                                dict(method=1, tma_warps=0), dict(method=2, tma_share=1.5),
                                dict(method=1, line_bytes=128, tma_warps=4, inflight=8)])
def test_gather_rejects_bad_arguments(ctx, kw):
    args = dict(line_bytes=32, method=0, ctas_per_sm=2, reps=1, inflight=2, lsu_warps=4, tma_warps=1, tma_share=0.0)
    args.update(kw)
    with pytest.raises(mgv.MgvError) as e:
        ctx.diag_gather(8 << 20, 1 << 20, **args)
    assert e.value.status == mgv.EINVAL
