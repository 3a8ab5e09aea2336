"""A model of the shared-memory region build (build_regions.cu), run on the
CPU over random inputs and random arrival orders, checking the properties the
kernel relies on:

* a row claims slot fill[b]++ of its bucket and moves to the next bucket when
  the bucket is full; rows whose run leaves the region are inserted later into
  the whole table, each at the first empty slot of its run (the global CAS
  insert);
* every bucket's occupied slots form a prefix (the probe stops at the first
  bucket with an empty slot);
* a probe walk from a key's home bucket finds every copy of the key;
* the duplicate pass -- each bucket against itself and the full buckets after
  it, within the region -- together with the global insert's own check flags
  a table exactly when it holds a duplicate key.
"""
import random

import pytest

EMPTY = None


def build(keys, homes, nbuckets, region):
    fill = [0] * nbuckets
    tab = [[EMPTY] * 4 for _ in range(nbuckets)]
    order = list(range(len(keys)))
    random.shuffle(order)  # rows claim slots in no particular order
    overflow = []
    for r in order:
        b = homes[r]
        end = (b // region + 1) * region  # the region of the home bucket
        while b < min(end, nbuckets):
            q = fill[b]
            fill[b] += 1
            if q < 4:
                tab[b][q] = keys[r]
                break
            b += 1
        else:
            overflow.append(r)
    # the duplicate pass of every region
    dup = False
    for b in range(nbuckets):
        n = min(fill[b], 4)
        ks = tab[b][:n]
        dup |= len(set(ks)) < len(ks)
        if n < 4:
            continue
        end = (b // region + 1) * region
        c = b + 1
        while c < min(end, nbuckets):
            m = min(fill[c], 4)
            dup |= bool(set(ks) & set(tab[c][:m]))
            if m < 4:
                break
            c += 1
    # overflow rows: the global insert walks from the home bucket through the table
    for r in overflow:
        b = homes[r]
        for _ in range(nbuckets):
            row = tab[b]
            if keys[r] in [k for k in row if k is not EMPTY]:
                dup = True
            if EMPTY in row:
                row[row.index(EMPTY)] = keys[r]
                break
            b = (b + 1) % nbuckets
        else:
            raise AssertionError("table full")
    return tab, dup


def probe(tab, key, home, nbuckets):
    found, b = 0, home
    for _ in range(nbuckets):
        row = tab[b]
        found += sum(1 for k in row if k == key)
        if EMPTY in row:
            return found
        b = (b + 1) % nbuckets
    return found


@pytest.mark.parametrize("seed", range(40))
def test_region_build_model(seed):
    rnd = random.Random(seed)
    random.seed(seed)
    region = rnd.choice([4, 8, 16])
    nbuckets = region * rnd.choice([2, 3, 5])
    lf = rnd.choice([0.3, 0.6, 0.9, 0.95])
    n = int(nbuckets * 4 * lf)
    pool = rnd.sample(range(10**6), n)
    keys = pool[:]
    ndup = rnd.choice([0, 0, 1, 3])  # unique tables are the common case
    for _ in range(ndup):
        i, j = rnd.sample(range(n), 2)
        keys[j] = keys[i]
    home_of = {k: rnd.randrange(nbuckets) for k in set(keys)}
    homes = [home_of[k] for k in keys]
    tab, dup = build(keys, homes, nbuckets, region)
    for row in tab:  # occupied slots form a prefix
        filled = [k is not EMPTY for k in row]
        assert filled == sorted(filled, reverse=True)
    for k in set(keys):  # every copy is found from the home bucket
        assert probe(tab, k, home_of[k], nbuckets) == keys.count(k)
    assert dup == (len(set(keys)) < len(keys))
