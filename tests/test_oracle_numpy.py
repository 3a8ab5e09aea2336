"""The oracle's functions without a reference counterpart (hash GROUP BY, the
radix partition's histogram and order, the select -> join -> group-by query,
the join's COUNT / SUM with payloads) checked against independent numpy
restatements on seeded inputs (CPU only).  The reference's own functions are
pinned against its compiled CPU code in test_oracle_golden.py; these are the
oracle's extensions, so they get a second, independent statement here.
"""
import numpy as np
import pytest

import pyoracle as po

MN = -(1 << 31)


def np_groupby(groups, values, mult=None):
    """Sorted (group, int64 SUM(value * mult), int64 COUNT(mult)) of every group with a row."""
    g = np.asarray(groups, np.int64)
    v = np.zeros(g.size, np.int64) if values is None else np.asarray(values, np.int64)
    m = np.ones(g.size, np.int64) if mult is None else np.asarray(mult, np.int64)
    keep = m > 0
    g, v, m = g[keep], v[keep], m[keep]
    uniq, inv = np.unique(g, return_inverse=True)
    sums = np.zeros(uniq.size, np.int64)
    cnts = np.zeros(uniq.size, np.int64)
    np.add.at(sums, inv, v * m)
    np.add.at(cnts, inv, m)
    return [(int(a), int(b), int(c)) for a, b, c in zip(uniq, sums, cnts)]


def rows(out):
    return [(int(r["group"]), int(r["sum"]), int(r["count"])) for r in out]


@pytest.mark.parametrize("n,G,seed", [(1, 1, 1), (1000, 16, 2), (20011, 4096, 3), (50000, 300000, 4)])
def test_groupby_vs_numpy(n, G, seed):
    g = po.gen_zipf(n, 0x5EED0A00 + seed, 1, G)
    v = po.gen_uniform(n, 0x5EED0A00 + seed, 2, -(1 << 31), 1 << 32)
    g[: min(n, 3)] = MN  # the reserved group is a group like any other
    assert rows(po.groupby(g, v)) == np_groupby(g, v)
    mult = po.gen_uniform(n, 0x5EED0A00 + seed, 3, 0, 4)
    assert rows(po.groupby(g, v, mult)) == np_groupby(g, v, mult)


@pytest.mark.parametrize("bits,shift", [(1, 0), (4, 3), (8, 0), (12, 20)])
def test_partition_vs_numpy(bits, shift):
    n = 30011
    k = po.gen_uniform(n, 0x5EED0A10, bits, -(1 << 31), 1 << 32)
    p = po.gen_uniform(n, 0x5EED0A10, 40 + bits, 0, 1000)
    hist, ok, op = po.partition(k, bits, shift, p)
    part = (k.view(np.uint32) >> np.uint32(shift)) & np.uint32((1 << bits) - 1)
    assert np.array_equal(hist, np.bincount(part, minlength=1 << bits).astype(np.uint64))
    # partition-major; the oracle keeps input order within a partition (the GPU partition need not)
    order = np.argsort(part, kind="stable")
    assert np.array_equal(ok, k[order]) and np.array_equal(op, p[order])


def np_join(bk, bp, pk, pp):
    """COUNT and SUM(build payload + probe payload) over every (build, probe) pair with equal keys."""
    mult, bsum = {}, {}
    for key, pay in zip(bk.tolist(), bp.tolist()):
        mult[key] = mult.get(key, 0) + 1
        bsum[key] = bsum.get(key, 0) + pay
    cnt = tot = 0
    for key, pay in zip(pk.tolist(), pp.tolist()):
        m = mult.get(key, 0)
        cnt += m
        tot += bsum.get(key, 0) + m * pay
    return cnt, tot


@pytest.mark.parametrize("nb,npb,seed", [(0, 10, 1), (1, 1, 2), (5000, 20000, 3), (3000, 10000, 4)])
def test_join_vs_numpy(nb, npb, seed):
    bk = po.gen_uniform(nb, 0x5EED0A20 + seed, 0, -50, 2000)  # duplicates, negative keys
    bp = po.gen_uniform(nb, 0x5EED0A20 + seed, 1, -(1 << 31), 1 << 32)
    pk = po.gen_uniform(npb, 0x5EED0A20 + seed, 2, -100, 2200)  # some keys miss
    pp = po.gen_uniform(npb, 0x5EED0A20 + seed, 3, -(1 << 31), 1 << 32)
    if nb > 4 and npb > 4:
        bk[:2] = MN
        pk[:3] = MN  # INT32_MIN keys join like any other key
    assert po.Chain(bk, bp).probe_agg(pk, pp) == np_join(bk, bp, pk, pp)


@pytest.mark.parametrize("nb,npb,bound,seed", [(100, 5000, 499, 1), (4096, 30000, 99, 2), (1000, 1000, -1, 3)])
def test_query_vs_numpy(nb, npb, bound, seed):
    bk = po.gen_uniform(nb, 0x5EED0A30 + seed, 0, 0, nb)  # duplicate build keys
    pk = po.gen_uniform(npb, 0x5EED0A30 + seed, 1, 0, nb + nb // 4)
    pf = po.gen_uniform(npb, 0x5EED0A30 + seed, 2, 0, 1000)
    pg = po.gen_zipf(npb, 0x5EED0A30 + seed, 3, 64)
    pv = po.gen_uniform(npb, 0x5EED0A30 + seed, 4, 0, 1 << 16)
    got, tc, ts = po.run_query(bk, pk, pf, pg, pv, bound)
    mult = np.bincount(bk, minlength=nb + nb // 4)[pk] * (pf <= bound)
    want = np_groupby(pg, pv, mult)
    assert rows(got) == want
    assert tc == sum(c for _, _, c in want) and ts == sum(s for _, s, _ in want)
