"""The server's shared scan restated on the CPU and checked against the
oracle's select -> join -> group-by run once per request.

A shared scan serves requests that differ only in their filter bound.  Its m
distinct bounds b[0] < ... < b[m-1] cut the filter values into ranges (range
j: b[j-1] < f <= b[j]); a row selected at the largest bound is tagged with the
first j with b[j] >= f (the kernel's binary search), each matched row adds
(value, 1) to cell (j, group), and block j of the per-range tables becomes the
sum of blocks 0..j (the prefix pass), which is the result of bound b[j].  The
model keeps the device's layout -- one group directory shared by every range,
blocks of [sums | counts | INT32_MIN group's pair] -- and its int64 wrap."""
import numpy as np
import pytest

import pyoracle as po

MN = -(1 << 31)


def cell_range(b, f):
    """The kernel's search: the first j with b[j] >= f (f <= b[-1])."""
    lo, hi = 0, len(b) - 1
    while lo < hi:
        mid = (lo + hi) >> 1
        if b[mid] >= f:
            hi = mid
        else:
            lo = mid + 1
    return lo


def shared_scan(build_keys, pk, pf, pg, pv, bounds):
    """Per request, its groups as [(group, sum, count)] sorted by group."""
    b = sorted(set(bounds))
    m = len(b)
    keys = {}  # the directory: group -> slot (INT32_MIN has the extra slot)
    build = {}
    for k in build_keys.tolist():
        build[k] = build.get(k, 0) + 1
    blocks = [dict() for _ in range(m)]  # per range: directory slot -> (sum, count)
    for f, k, g, v in zip(pf.tolist(), pk.tolist(), pg.tolist(), pv.tolist()):
        if f > b[-1]:
            continue
        j = cell_range(b, f)
        assert b[j] >= f and (j == 0 or b[j - 1] < f)
        matches = build.get(k, 0)
        if not matches:
            continue
        slot = keys.setdefault(g, len(keys))
        s, c = blocks[j].get(slot, (0, 0))
        blocks[j][slot] = ((s + matches * v) % (1 << 64), c + matches)
    # prefix over the ranges, slot by slot
    run = {}
    prefix = []
    for j in range(m):
        for slot, (s, c) in blocks[j].items():
            s0, c0 = run.get(slot, (0, 0))
            run[slot] = ((s0 + s) % (1 << 64), c0 + c)
        prefix.append(dict(run))
    inv = {slot: g for g, slot in keys.items()}
    out = []
    for bound in bounds:
        p = prefix[b.index(bound)]
        rows = []
        for slot, (s, c) in p.items():
            if c:
                rows.append((inv[slot], s - (1 << 64) if s >= 1 << 63 else s, c))
        out.append(sorted(rows))
    return out


def oracle(bk, pk, pf, pg, pv, bound):
    want, _, _ = po.run_query(bk, pk, pf, pg, pv, bound)
    return [(int(w["group"]), int(w["sum"]), int(w["count"])) for w in want]


@pytest.mark.parametrize("seed", range(4))
def test_shared_scan_model_equals_per_request_oracle(seed):
    rng = np.random.default_rng(700 + seed)
    nb, n = 300, 4000
    bk = rng.integers(-400, 400, nb).astype(np.int32)
    if seed % 2:
        bk[::17] = MN  # reserved build keys (the side list) and duplicates
    pk = rng.integers(-500, 500, n).astype(np.int32)
    pk[::23] = MN
    pf = rng.integers(-50, 1050, n).astype(np.int32)
    pf[::31] = MN
    pf[::37] = (1 << 31) - 1
    pg = rng.integers(0, 64, n).astype(np.int32)
    pg[::13] = MN
    pv = rng.integers(MN, (1 << 31) - 1, n, dtype=np.int64).astype(np.int32)
    bounds = [int(x) for x in rng.integers(-60, 1060, 12)] + [MN, (1 << 31) - 1, 500, 500]
    got = shared_scan(bk, pk, pf, pg, pv, bounds)
    for i, bound in enumerate(bounds):
        assert got[i] == oracle(bk, pk, pf, pg, pv, bound), (i, bound)


def test_cell_range_edges():
    b = [MN, -5, 0, 0 + 1, 999, (1 << 31) - 1]
    for f in (MN, MN + 1, -6, -5, -4, 0, 1, 2, 999, 1000, (1 << 31) - 1):
        j = cell_range(b, f)
        assert b[j] >= f and (j == 0 or b[j - 1] < f)
    assert cell_range([7], 7) == 0 and cell_range([7], MN) == 0


def lut_for(b, limit=8192):
    """The server's range lookup table of a scan's sorted distinct bounds:
    entry d = the first j with b[j] >= b[0] + d, when the bounds span at most
    `limit` values; else none."""
    span = b[-1] - b[0] + 1
    if span > limit:
        return []
    out, j = [], 0
    for d in range(span):
        while b[j] < b[0] + d:
            j += 1
        out.append(j)
    return out


def range_of(b, lut, f):
    """The kernel's lookup: the table for f in [b[0], b[0] + len), the search
    otherwise (unsigned 32-bit difference, as on the device)."""
    d = (f - b[0]) & 0xFFFFFFFF
    return lut[d] if d < len(lut) else cell_range(b, f)


@pytest.mark.parametrize("seed", range(6))
def test_range_lookup_table_equals_the_search(seed):
    rng = np.random.default_rng(900 + seed)
    lo = int(rng.choice([MN, -100, 0, (1 << 31) - 9000]))
    width = int(rng.choice([1, 50, 8192, 9000]))
    b = sorted(set(int(x) for x in rng.integers(lo, min(lo + width, (1 << 31) - 1) + 1, 40)))
    lut = lut_for(b)
    assert (len(lut) > 0) == (b[-1] - b[0] + 1 <= 8192)
    fs = [MN, MN + 1, b[0] - 1, b[0], b[-1]] + [int(x) for x in rng.integers(max(MN, b[0] - 20), b[-1] + 1, 500)]
    for f in fs:
        if f < MN or f > b[-1]:
            continue
        assert range_of(b, lut, f) == cell_range(b, f), (b[:4], f)
