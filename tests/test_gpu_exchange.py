"""The hash exchange's GPU steps: mgv_partition_columns (the routing of
split / hash_exchange, src/operators/split.cu:49-118, src/main9.cu:104-148)
against the oracle's partition, and the exchange join with its ranks
emulated one after another on this GPU (each "rank" partitions its slice on
the GPU, partition p of every slice is handed to rank p, each rank joins on
the GPU, the partial results are added) against the oracle's one-process
join.  Only one GPU is used: no collective runs and no kernel waits on
another."""
import numpy as np
import pytest

import exchange
import mgv
import pyoracle as po
from gpu_util import dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bits,shift,n", [(1, 0, 1000003), (3, 5, 77777), (8, 0, 1 << 20), (12, 20, 300001),
                                          (2, 0, 1)])
def test_partition_columns_matches_oracle(ctx, torch_cuda, bits, shift, n):
    torch = torch_cuda
    k = po.gen_uniform(n, 0x5EED0C01 + bits, 0, -(1 << 31), 1 << 32)
    k[::53] = -(1 << 31)
    v = po.gen_uniform(n, 0x5EED0C01 + bits, 1, -(1 << 31), 1 << 32)
    dk, dv = dev(torch, k), dev(torch, v)
    out = torch.empty((2, n + 7), dtype=torch.int32, device="cuda")
    counts = ctx.partition_columns([dk, dv], n, 0, bits, shift, out, n + 7)
    hist, _, _ = po.partition(k, bits, shift)
    assert counts == [int(h) for h in hist]
    hk, hv = out[0, :n].cpu().numpy(), out[1, :n].cpu().numpy()
    part = ((k.astype(np.int64) & 0xFFFFFFFF) >> shift) & ((1 << bits) - 1)
    lo = 0
    for p, c in enumerate(counts):  # partition p's rows, as a multiset of (key, payload)
        got = np.sort(hk[lo:lo + c].astype(np.int64) << 32 | (hv[lo:lo + c].astype(np.int64) & 0xFFFFFFFF))
        sel = part == p
        want = np.sort(k[sel].astype(np.int64) << 32 | (v[sel].astype(np.int64) & 0xFFFFFFFF))
        assert np.array_equal(got, want)
        lo += c


def test_exchange_join_one_rank(ctx, torch_cuda):
    torch = torch_cuda
    nb, npb = 1 << 18, 1 << 21
    bk = po.gen_perm(nb, 0x5EED0C11)
    bp = po.gen_uniform(nb, 0x5EED0C11, 1, 0, 1 << 20)
    pk, hits = po.gen_probe_keys(npb, 0x5EED0C12, 0x5EED0C11, nb, 3865470566, nb, (1 << 31) - nb)
    pp = po.gen_uniform(npb, 0x5EED0C12, 2, 0, 1 << 20)
    d = [dev(torch, a) for a in (bk, bp, pk, pp)]
    got = exchange.exchange_join(None, d[:2], d[2:], exchange.gpu_partition(ctx), exchange.gpu_join(ctx), 0, "cuda")
    assert got == po.Chain(bk, bp).probe_agg(pk, pp) and got[0] == hits


@pytest.mark.parametrize("world,shift", [(2, 0), (4, 7), (8, 0)])
def test_exchange_join_emulated_ranks(ctx, torch_cuda, world, shift):
    torch = torch_cuda
    nb, npb = 200003, 1000003
    bk = po.gen_uniform(nb, 0x5EED0C21, 0, -(1 << 20), 1 << 21)
    bk[::101] = -(1 << 31)
    bp = po.gen_uniform(nb, 0x5EED0C21, 1, -(1 << 31), 1 << 32)
    pk = po.gen_uniform(npb, 0x5EED0C21, 2, -(1 << 20), 1 << 21)
    pk[::97] = -(1 << 31)
    pp = po.gen_uniform(npb, 0x5EED0C21, 3, -(1 << 31), 1 << 32)
    bits = exchange.world_bits(world)
    part = exchange.gpu_partition(ctx)
    join = exchange.gpu_join(ctx)

    def slices(a):
        return [dev(torch, s) for s in np.array_split(a, world)]

    # each emulated rank routes its slice: partition p of every rank goes to rank p
    inbox_b = [[[], []] for _ in range(world)]
    inbox_p = [[[], []] for _ in range(world)]
    for r, (sk, sp, qk, qp) in enumerate(zip(slices(bk), slices(bp), slices(pk), slices(pp))):
        for cols, inbox in (([sk, sp], inbox_b), ([qk, qp], inbox_p)):
            parts, counts = part(cols, 0, bits, shift)
            lo = 0
            for p, c in enumerate(counts):
                for j in range(2):
                    inbox[p][j].append(parts[j][lo:lo + c])
                lo += c
    total = (0, 0)
    for p in range(world):
        rb = [torch.cat(x) for x in inbox_b[p]]
        rp = [torch.cat(x) for x in inbox_p[p]]
        owner = ((rb[0].cpu().numpy().astype(np.int64) & 0xFFFFFFFF) >> shift) & (world - 1)
        assert (owner == p).all()
        c, s = join(rb[0], rb[1], rp[0], rp[1])
        total = (total[0] + c, (total[1] + s + (1 << 63)) % (1 << 64) - (1 << 63))
    assert total == po.Chain(bk, bp).probe_agg(pk, pp)
