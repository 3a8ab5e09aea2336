"""mgv_hash_join_noalloc, the join entry point that allocates nothing.

Some callers of this library cannot allocate device memory: code that runs
under another framework's allocator or memory budget (which owns every byte
and forbids cudaMalloc), and plugins or embedded hosts that are handed only
pre-allocated buffers.  For them the join keeps its hash table in a fixed
device array inside the library.  These tests call it through the C ABI,
twice and more in a row, and check each result against the allocating
pipeline (hash_build -> hash_probe -> aggregate) and against the oracle on
the same inputs; integer results must match exactly.  They also check that
a warm call leaves the device's free memory unchanged and that the caller's
current device is the same after the call.

This file is collected last so that a run stopping at the first failure has
run every other test first.
"""
import numpy as np
import pytest

import mgv
import pyoracle as po
from gpu_util import dev

pytestmark = pytest.mark.gpu

HIT = 3865470566  # 0.9 * 2^32


def pipeline_result(ctx, bk, bp, pk, pp, nb, npb):
    """The allocating entry points: hash_build -> hash_probe -> aggregate."""
    bhead, hb, probe, agg = mgv.create_count_join_1G_pipeline(ctx, max(nb, 1))
    bhead.open()
    if nb:
        bhead.consume_columns([bk, bp], nb)
    bhead.close()
    probe.open()
    if npb:
        probe.consume_columns([pk, pp], npb)
    probe.close()
    r = agg.result()
    for o in (probe, agg, bhead, hb):
        o.destroy()
    return r


def noalloc_result(torch, out, bk, bp, nb, pk, pp, npb):
    out.fill_(-7)
    mgv.hash_join_noalloc(0, bk, bp, nb, pk, pp, npb, out)
    return tuple(int(x) for x in out.cpu().tolist())


def test_noalloc_join_matches_pipeline_and_oracle(ctx, torch_cuda):
    """Two calls in a row (different sizes) against the allocating pipeline and
    the oracle, with the generator's known hit count."""
    torch = torch_cuda
    out = torch.empty(2, dtype=torch.int64, device="cuda")
    cases = [(1 << 20, 1 << 22, 0x5EED0701), (12345, 700001, 0x5EED0702)]
    for nb, npb, seed in cases:
        bk = po.gen_perm(nb, seed)
        bp = po.gen_uniform(nb, seed, 1, 0, 1 << 20)
        pk, hits = po.gen_probe_keys(npb, seed + 1, seed, nb, HIT, nb, (1 << 31) - nb)
        pp = po.gen_uniform(npb, seed + 1, 2, 0, 1 << 20)
        d = [dev(torch, a) for a in (bk, bp, pk, pp)]
        want = po.Chain(bk, bp).probe_agg(pk, pp)
        assert pipeline_result(ctx, d[0], d[1], d[2], d[3], nb, npb) == want
        got = noalloc_result(torch, out, d[0], d[1], nb, d[2], d[3], npb)
        assert got == want
        assert got[0] == hits


def test_noalloc_edge_cases_match_oracle(ctx, torch_cuda):
    """Duplicate build keys (the non-unique probe), INT32_MIN keys (the side
    list), NULL payloads, a probe column offset by 4 bytes (the unaligned
    probe kernel) and an empty build side, one call after another."""
    torch = torch_cuda
    mn = -(1 << 31)
    out = torch.empty(2, dtype=torch.int64, device="cuda")
    nb, npb = 50000, 200003
    bk = po.gen_uniform(nb, 0x5EED0711, 0, 0, 20000)
    bk[::97] = mn
    bp = po.gen_uniform(nb, 0x5EED0711, 1, -(1 << 31), 1 << 32)
    pk = po.gen_uniform(npb + 1, 0x5EED0711, 2, -100, 20200)
    pk[::89] = mn
    pp = po.gen_uniform(npb + 1, 0x5EED0711, 3, -(1 << 31), 1 << 32)
    dbk, dbp, dpk, dpp = (dev(torch, a) for a in (bk, bp, pk, pp))
    zero_b = np.zeros(nb, np.int32)
    zero_p = np.zeros(npb + 1, np.int32)

    # duplicates + INT32_MIN, both payloads
    got = noalloc_result(torch, out, dbk, dbp, nb, dpk, dpp, npb)
    assert got == po.Chain(bk, bp).probe_agg(pk[:npb], pp[:npb])
    # NULL payloads on both sides: SUM is 0, COUNT unchanged
    got = noalloc_result(torch, out, dbk, None, nb, dpk, None, npb)
    assert got == po.Chain(bk, zero_b).probe_agg(pk[:npb], zero_p[:npb])
    # probe columns that start 4 bytes past a 16-byte boundary
    got = noalloc_result(torch, out, dbk, dbp, nb, dpk[1:], dpp[1:], npb)
    assert got == po.Chain(bk, bp).probe_agg(pk[1:], pp[1:])
    # empty build side: nothing matches
    got = noalloc_result(torch, out, dbk, dbp, 0, dpk, dpp, npb)
    assert got == (0, 0)
    # and a full join again, after the empty one
    got = noalloc_result(torch, out, dbk, dbp, nb, dpk, dpp, npb)
    assert got == po.Chain(bk, bp).probe_agg(pk[:npb], pp[:npb])


def test_noalloc_allocates_nothing_and_keeps_the_device(ctx, torch_cuda):
    """Free device memory is the same before and after a warm call, and the
    caller's current device is unchanged."""
    torch = torch_cuda
    nb, npb = 1 << 18, 1 << 21
    bk = po.gen_perm(nb, 0x5EED0721)
    bp = po.gen_uniform(nb, 0x5EED0721, 1, 0, 1 << 20)
    pk, _ = po.gen_probe_keys(npb, 0x5EED0722, 0x5EED0721, nb, HIT, nb, (1 << 31) - nb)
    pp = po.gen_uniform(npb, 0x5EED0722, 2, 0, 1 << 20)
    d = [dev(torch, a) for a in (bk, bp, pk, pp)]
    out = torch.empty(2, dtype=torch.int64, device="cuda")
    want = po.Chain(bk, bp).probe_agg(pk, pp)
    assert noalloc_result(torch, out, d[0], d[1], nb, d[2], d[3], npb) == want  # warm
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    mgv.hash_join_noalloc(0, d[0], d[1], nb, d[2], d[3], npb, out)
    torch.cuda.synchronize()
    after = torch.cuda.mem_get_info()[0]
    assert after == before
    assert tuple(int(x) for x in out.cpu().tolist()) == want
    assert torch.cuda.current_device() == 0


def test_noalloc_rejects_oversized_build(torch_cuda):
    torch = torch_cuda
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    k = torch.zeros(4, dtype=torch.int32, device="cuda")
    with pytest.raises(mgv.MgvError) as e:
        mgv.hash_join_noalloc(0, k, k, mgv.NOALLOC_MAX_BUILD_ROWS + 1, k, k, 4, out)
    assert e.value.status == mgv.EINVAL
    assert b"MGV_NOALLOC_MAX_BUILD_ROWS" in mgv.load().mgv_last_error_string()
