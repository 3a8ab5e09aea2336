"""Key-only join tables: a hash_build without a payload column keeps 8 keys
per 32-byte bucket instead of 4 {key, payload} slots (half the table), and
every match carries build payload 0 -- the reference's own build stores keys
only (src/operators/hashjoin.cu:40-60, the payload store commented out).
Every probe kernel, both builders (one CAS per row under 2^16 rows, the
shared-memory region build above), duplicates, INT32_MIN keys, radix
layouts and the sink's emitted payload column are checked against the
oracle's chained-table join with zero payloads."""
import numpy as np
import pytest

import mgv
import pyoracle as po
from gpu_util import dev, sorted_rows

pytestmark = pytest.mark.gpu

PROBE_VARIANTS = [dict(probe_kernel=0), dict(probe_kernel=1), dict(probe_kernel=2), dict(probe_kernel=3)]


@pytest.fixture
def tuned(ctx, request):
    old = ctx.tuning()
    keep = {k: getattr(old, k) for k in ("probe_kernel", "probe_rows_per_thread", "probe_stages", "probe_ctas_per_sm")}
    ctx.set_tuning(**request.param)
    yield request.param
    ctx.set_tuning(**keep)


def ko_join(ctx, torch, bk, pk, pp, lf=0.0, radix_bits=0, offset=0):
    """hash_build(keys only) then hash_probe -> aggregate(COUNT, SUM(probe payload + build payload))."""
    nb, npb = bk.size, pk.size
    hb = mgv.Op.hash_build(ctx, 0, -1, max(nb, 1), lf, radix_bits, 0)
    agg = mgv.Op.aggregate(ctx, 1, 2)
    probe = mgv.Op.hash_probe(ctx, 0, hb, agg)
    hb.open()
    if nb:
        hb.consume_columns([dev(torch, bk)], nb)
    hb.close()
    info = hb.result()
    dpk = dev(torch, np.concatenate([np.zeros(offset, np.int32), pk]))[offset:]
    dpp = dev(torch, np.concatenate([np.zeros(offset, np.int32), pp]))[offset:]
    probe.open()
    if npb:
        probe.consume_columns([dpk, dpp], npb)
    probe.close()
    r = agg.result()
    for o in (probe, agg, hb):
        o.destroy()
    return r, info


@pytest.mark.parametrize("tuned", PROBE_VARIANTS, indirect=True, ids=lambda v: f"k{v['probe_kernel']}")
@pytest.mark.parametrize("nb,npb,dup", [(5000, 100003, False), (1 << 18, 1 << 21, False), (5000, 100003, True),
                                        (1 << 18, 1 << 21, True)])
def test_key_only_probe_aggregate(ctx, torch_cuda, tuned, nb, npb, dup):
    seed = 0x5EED0D01 + nb + dup
    if dup:
        bk = po.gen_uniform(nb, seed, 0, 0, nb // 2)
        bk[::61] = -(1 << 31)
    else:
        bk = po.gen_perm(nb, seed)
    pk = po.gen_uniform(npb, seed, 1, -100, nb + nb // 4)
    pk[::71] = -(1 << 31)
    pp = po.gen_uniform(npb, seed, 2, -(1 << 31), 1 << 32)
    (cnt, s), info = ko_join(ctx, torch_cuda, bk, pk, pp, 0.5)
    assert (cnt, s) == po.Chain(bk, np.zeros(nb, np.int32)).probe_agg(pk, pp)
    assert info.rows == nb
    assert info.has_duplicates == (1 if dup else 0)
    # 8 keys per bucket: half the buckets of the payload table at the same load factor
    assert info.nbuckets == -(-nb // 4)


@pytest.mark.parametrize("lf", [0.25, 0.5, 0.8, 0.95])
def test_key_only_load_factors_and_unaligned(ctx, torch_cuda, lf):
    nb, npb = 70001, 500009
    bk = po.gen_uniform(nb, 0x5EED0D11, 0, 0, 50000)  # duplicates
    pk = po.gen_uniform(npb, 0x5EED0D11, 1, -10, 50020)
    pp = po.gen_uniform(npb, 0x5EED0D11, 2, -1000, 2000)
    want = po.Chain(bk, np.zeros(nb, np.int32)).probe_agg(pk, pp)
    for offset in (0, 1, 3):  # 4-byte offsets take the register-prefetch probe
        (cnt, s), _ = ko_join(ctx, torch_cuda, bk, pk, pp, lf, offset=offset)
        assert (cnt, s) == want


def test_key_only_radix_table_through_chain_and_sink(ctx, torch_cuda):
    """A radix-laid-out key-only table (partition -> build), probed by the
    generic chain into a sink: the emitted build-payload column is 0."""
    torch = torch_cuda
    nb, npb = 1 << 17, 1 << 16
    bk = po.gen_uniform(nb, 0x5EED0D21, 0, 0, 1 << 16)  # duplicates
    pk = po.gen_uniform(npb, 0x5EED0D21, 1, 0, (1 << 16) + 100)
    pp = po.gen_uniform(npb, 0x5EED0D21, 2, -(1 << 31), 1 << 32)
    hb = mgv.Op.hash_build(ctx, 0, -1, nb, 0.5, 4, 0)
    part = mgv.Op.partition(ctx, 0, 4, 0, nb, hb)
    part.open(); part.consume_columns([dev(torch, bk)], nb); part.close()
    pool = mgv.Pool(ctx, 8, 1 << 18, 3)
    sink = mgv.Op.sink(ctx, pool)
    pr = mgv.Op.hash_probe(ctx, 0, hb, sink)
    pr.open(); pr.consume_columns([dev(torch, pk), dev(torch, pp)], npb); pr.close()
    rows = sink.result()
    out = [torch.empty(max(rows, 1), dtype=torch.int32, device="cuda") for _ in range(3)]
    for c in range(3):
        sink.sink_read(c, out[c].data_ptr(), rows)
    got = sorted_rows([out[0][:rows].cpu().numpy(), out[2][:rows].cpu().numpy(), out[1][:rows].cpu().numpy()])
    want = po.Chain(bk, np.zeros(nb, np.int32)).probe_emit(pk, pp)
    assert np.array_equal(got, sorted_rows([want[:, 0], want[:, 1], want[:, 2]]))
    assert (out[2][:rows].cpu().numpy() == 0).all()
    for o in (pr, sink, hb, part):
        o.destroy()
    pool.destroy()
