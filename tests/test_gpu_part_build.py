"""The build of a partition op's run: partition -> hash_build on the table's
radix bits.  When the partition op stored one run and every partition slice
of the table is whole 64 KiB regions, each partition's rows are staged
region-major inside the partition's own range by one CTA
(k_region_part_scatter in csrc/build_regions.cu) and the regions are built
from there; otherwise the rows take the general staged region build.
Key-only and {key, payload} tables, duplicates, INT32_MIN keys (side list,
their staging slots skipped), a load factor that pushes runs past region
ends, and both fall-backs (several runs, slices that are not whole regions)
are checked against the oracle's chained-table join
(src/operators/hashjoin.cu:40-75, 134-182)."""
import numpy as np
import pytest

import mgv
import pyoracle as po
from gpu_util import dev

pytestmark = pytest.mark.gpu

INT32_MIN = -(1 << 31)
PARTITION_LAUNCHES = 3  # per-partition staging, region build, overflow
STAGED_LAUNCHES = 5     # region histogram, scan, sorted scatter, region build, overflow


def part_join(ctx, torch, bk, bp, pk, pp, bits, lf, runs=1):
    """partition(bits) -> hash_build, then hash_probe -> aggregate(COUNT, SUM(probe + build payload)).
    Returns ((count, sum), build info, launches of the partition's close)."""
    nb = bk.size
    hb = mgv.Op.hash_build(ctx, 0, 1 if bp is not None else -1, max(nb, 1), lf, bits, 0)
    part = mgv.Op.partition(ctx, 0, bits, 0, max(nb, 1), hb)
    agg = mgv.Op.aggregate(ctx, 1, 2)
    probe = mgv.Op.hash_probe(ctx, 0, hb, agg)
    cols = [dev(torch, bk)] + ([dev(torch, bp)] if bp is not None else [])
    part.open()
    cuts = np.linspace(0, nb, runs + 1).astype(np.int64)
    for a, b in zip(cuts[:-1], cuts[1:]):
        part.consume_columns([c[int(a):int(b)] for c in cols], int(b - a))
    l0 = ctx.launches
    part.close()
    launches = ctx.launches - l0
    info = hb.result()
    probe.open()
    probe.consume_columns([dev(torch, pk), dev(torch, pp)], pk.size)
    probe.close()
    r = agg.result()
    for o in (probe, agg, part, hb):
        o.destroy()
    return r, info, launches


def inputs(nb, npb, seed, payload, dup):
    if dup:
        bk = po.gen_uniform(nb, seed, 0, 0, max(nb // 3, 1))
        bk[::97] = INT32_MIN
    else:
        bk = po.gen_perm(nb, seed)
    bp = po.gen_uniform(nb, seed, 1, INT32_MIN, 1 << 32) if payload else None
    pk = po.gen_uniform(npb, seed, 2, 0, nb + nb // 8)
    pk[::89] = INT32_MIN
    pp = po.gen_uniform(npb, seed, 3, INT32_MIN, 1 << 32)
    return bk, bp, pk, pp


def oracle(bk, bp, pk, pp):
    return po.Chain(bk, bp if bp is not None else np.zeros(bk.size, np.int32)).probe_agg(pk, pp)


# (build rows, radix bits, load factor, payload, duplicates): partition slices of
# 1 to 8 whole regions (2048 buckets each)
CASES = [
    (1 << 22, 8, 0.5, False, False),        # key-only, 4096 buckets per partition
    (1 << 22, 6, 0.5, False, True),         # key-only, 16384 buckets, duplicates and INT32_MIN keys
    (1 << 22, 8, 0.5, True, False),         # {key, payload}, 8192 buckets
    (1 << 22, 8, 0.25, True, True),         # {key, payload}, 16384 buckets, duplicates
    (3 << 20, 8, 0.75, False, True),        # key-only, 2048 buckets at 0.75: runs leave their region
    (3 << 19, 8, 0.75, True, False),        # {key, payload}, 2048 buckets at 0.75
]


@pytest.mark.parametrize("nb,bits,lf,payload,dup", CASES)
def test_partition_staged_build_matches_oracle(ctx, torch_cuda, nb, bits, lf, payload, dup):
    seed = 0x5EED0E01 + nb + bits + int(lf * 100) + payload * 7 + dup * 13
    bk, bp, pk, pp = inputs(nb, 1 << 21, seed, payload, dup)
    (cnt, s), info, launches = part_join(ctx, torch_cuda, bk, bp, pk, pp, bits, lf)
    assert launches == PARTITION_LAUNCHES
    assert (cnt, s) == oracle(bk, bp, pk, pp)
    assert info.rows == nb
    assert info.has_duplicates == int(len(np.unique(bk)) < nb)
    assert info.reserved_key_rows == int((bk == INT32_MIN).sum())


@pytest.mark.parametrize("payload", [False, True])
def test_several_runs_take_the_staged_build(ctx, torch_cuda, payload):
    """Two consumes store two partition-major runs: a partition's rows are no
    longer one range, so the build goes through the general staged build."""
    nb = 1 << 22
    bk, bp, pk, pp = inputs(nb, 1 << 20, 0x5EED0E31 + payload, payload, True)
    (cnt, s), info, launches = part_join(ctx, torch_cuda, bk, bp, pk, pp, 8, 0.5, runs=2)
    assert launches == STAGED_LAUNCHES
    assert (cnt, s) == oracle(bk, bp, pk, pp) and info.rows == nb and info.has_duplicates == 1


def test_slices_of_part_regions_take_the_staged_build(ctx, torch_cuda):
    """Load factor 0.6: 13654 buckets per partition, not whole regions, so a
    region can hold rows of two partitions."""
    nb = 1 << 24
    bk, bp, pk, pp = inputs(nb, 1 << 20, 0x5EED0E41, False, False)
    (cnt, s), info, launches = part_join(ctx, torch_cuda, bk, bp, pk, pp, 8, 0.6)
    assert launches == STAGED_LAUNCHES
    assert (cnt, s) == oracle(bk, bp, pk, pp) and info.rows == nb and info.has_duplicates == 0


def test_partition_staged_build_twice_on_one_operator(ctx, torch_cuda):
    """open -> consume -> close twice on the same operators: the second build
    starts from a fresh table again (nothing of the first stays)."""
    torch = torch_cuda
    nb = 1 << 21
    hb = mgv.Op.hash_build(ctx, 0, 1, nb, 0.5, 8, 0)
    part = mgv.Op.partition(ctx, 0, 8, 0, nb, hb)
    agg = mgv.Op.aggregate(ctx, 1, 2)
    probe = mgv.Op.hash_probe(ctx, 0, hb, agg)
    for seed in (0x5EED0E51, 0x5EED0E52):
        bk, bp, pk, pp = inputs(nb, 1 << 20, seed, True, seed & 1 == 0)
        part.open(); part.consume_columns([dev(torch, bk), dev(torch, bp)], nb); part.close()
        probe.open(); probe.consume_columns([dev(torch, pk), dev(torch, pp)], pk.size); probe.close()
        assert agg.result() == po.Chain(bk, bp).probe_agg(pk, pp)
        assert hb.result().rows == nb
    for o in (probe, agg, part, hb):
        o.destroy()
