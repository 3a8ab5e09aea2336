"""mgv_hash_join_noalloc, the join entry point that allocates nothing.

It exists for callers that cannot allocate device memory (code running
under another framework's allocator or budget, inside a graph capture or a
real-time loop, or handed only pre-allocated buffers).  The test calls it
through the C ABI twice in a row and checks each result against the
allocating pipeline (hash_build -> hash_probe -> aggregate) on the same
inputs; integer results must match exactly.  This file is collected last so
that a run stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

import mgv
import pyoracle as po

pytestmark = pytest.mark.gpu

HIT = 3865470566


def pipeline_result(ctx, torch, bk, bp, pk, pp):
    bhead, hb, probe, agg = mgv.create_count_join_1G_pipeline(ctx, max(bk.numel(), 1))
    bhead.open(); bhead.consume_columns([bk, bp], bk.numel()); bhead.close()
    probe.open(); probe.consume_columns([pk, pp], pk.numel()); probe.close()
    r = agg.result()
    for o in (probe, agg, hb):
        o.destroy()
    return r


def noalloc_result(torch, bk, bp, pk, pp):
    out = torch.full((2,), -7, dtype=torch.int64, device="cuda")
    mgv.hash_join_noalloc(0, bk, bp, bk.numel(), pk, pp, pk.numel(), out)
    return tuple(int(x) for x in out.cpu().tolist())


def test_noalloc_join_matches_pipeline(torch_cuda):
    torch = torch_cuda
    ctx = mgv.Context(0)
    cases = [(1 << 20, 1 << 22, 0x5EED0701), (12345, 700001, 0x5EED0702)]
    for nb, npb, seed in cases:  # two calls in a row, different sizes
        bk = torch.empty(nb, dtype=torch.int32, device="cuda")
        bp = torch.empty(nb, dtype=torch.int32, device="cuda")
        pk = torch.empty(npb, dtype=torch.int32, device="cuda")
        pp = torch.empty(npb, dtype=torch.int32, device="cuda")
        ctx.gen_perm(bk, nb, seed)
        ctx.gen_uniform(bp, nb, seed, 1, 0, 1 << 20)
        hits = ctx.gen_probe_keys(pk, npb, seed + 1, seed, nb, HIT, nb, (1 << 31) - nb)
        ctx.gen_uniform(pp, npb, seed + 1, 2, 0, 1 << 20)
        ctx.sync()
        want = pipeline_result(ctx, torch, bk, bp, pk, pp)
        got = noalloc_result(torch, bk, bp, pk, pp)
        assert got == want
        assert got[0] == hits
    ctx.close()


def test_noalloc_rejects_oversized_build(torch_cuda):
    torch = torch_cuda
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    k = torch.zeros(4, dtype=torch.int32, device="cuda")
    with pytest.raises(mgv.MgvError) as e:
        mgv.hash_join_noalloc(0, k, k, mgv.NOALLOC_MAX_BUILD_ROWS + 1, k, k, 4, out)
    assert e.value.status == mgv.EINVAL
    assert b"MGV_NOALLOC_MAX_BUILD_ROWS" in mgv.load().mgv_last_error_string()
