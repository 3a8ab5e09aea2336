"""The kernels' integer bookkeeping restated on the CPU with fixed-width
arithmetic (numpy uint32 / uint64 wrap like the device's):

* the shared group table's int64 SUM kept as two 32-bit words (chain.cu): each
  value adds v + 2^31 (in [0, 2^32)) to the low word and a carry to the high
  word; the flush subtracts count * 2^31;
* the sorted scatters (partition.cu, build_regions.cu): a tile counts its rows
  per destination, reserves one range per destination, and stores sorted
  position j at base[d] + j with base[d] = reserved[d] - first_sorted[d]
  (mod 2^32 / 2^64): every row lands once, inside its destination's range.
"""
import numpy as np
import pytest


@pytest.mark.parametrize("seed", range(6))
def test_biased_two_word_sum(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.choice([1, 1000, 1 << 20]))
    v = rng.integers(-(1 << 31), 1 << 31, n, dtype=np.int64)
    v[: min(n, 4)] = [-(1 << 31), (1 << 31) - 1, -(1 << 31), 0][: min(n, 4)]
    x = (v.astype(np.uint64) ^ np.uint64(0x80000000)) & np.uint64(0xFFFFFFFF)  # v + 2^31 as a u32
    lo = np.uint64(0)
    hi = np.uint64(0)
    for chunk in np.array_split(x, max(1, n // 4096)):  # the running 32-bit low word, carries into hi
        for xi in chunk.tolist():
            s = int(lo) + xi
            if s >= 1 << 32:
                hi += np.uint64(1)
            lo = np.uint64(s & 0xFFFFFFFF)
    biased = (int(hi) << 32) | int(lo)
    total = (biased - n * (1 << 31)) % (1 << 64)
    want = int(v.sum()) % (1 << 64)
    assert total == want


@pytest.mark.parametrize("seed", range(20))
def test_sorted_scatter_positions(seed):
    rng = np.random.default_rng(100 + seed)
    ndest = int(rng.integers(1, 65))
    tiles = int(rng.integers(1, 9))
    rows_per_tile = 256
    dest = [rng.integers(0, ndest, rows_per_tile) for _ in range(tiles)]
    counts = np.bincount(np.concatenate(dest), minlength=ndest)
    start = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint32) + np.uint32(rng.integers(0, 1 << 31))
    cursor = start.copy()
    landed = []
    for d in dest:
        cnt = np.bincount(d, minlength=ndest).astype(np.uint32)
        # rank of each row among its destination's rows of the tile (any order)
        rank = np.zeros(d.size, np.uint32)
        seen = np.zeros(ndest, np.uint32)
        for i in rng.permutation(d.size):
            rank[i] = seen[d[i]]
            seen[d[i]] += np.uint32(1)
        reserved = cursor.copy()  # one reservation per destination
        cursor = cursor + cnt
        first = np.concatenate([[0], np.cumsum(cnt)[:-1]]).astype(np.uint32)  # exclusive scan
        with np.errstate(over="ignore"):
            base = reserved - first  # mod 2^32
            pos = first[d] + rank  # the row's sorted position in the tile
            landed.append((d, (base[d] + pos).astype(np.uint32)))
    all_pos = np.concatenate([p for _, p in landed]).astype(np.int64)
    all_dst = np.concatenate([d for d, _ in landed])
    assert np.unique(all_pos).size == all_pos.size  # every row lands once
    lo = start.astype(np.int64)[all_dst]
    assert ((all_pos >= lo) & (all_pos < lo + counts[all_dst])).all()  # inside its destination's range
