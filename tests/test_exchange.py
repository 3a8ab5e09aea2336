"""The multi-GPU hash exchange (exchange.py) on CPU processes over gloo.

The reference routes both join sides by key to the GPU that owns it and
merges the per-GPU joins (hash_exchange, src/main9.cu:104-148; split,
src/operators/split.cu:49-151; union_all, src/operators/union_all.cu:35-57).
Here world-size 2 and 4 process groups run the exchange with the oracle's
partition and chained-table join standing in for the GPU kernels: every
routed row lands on the rank that owns its key, and the merged COUNT / SUM
equal the oracle's one-process join of all rows, duplicates and INT32_MIN
keys included.  No GPU is involved."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (os.path.join(ROOT, "multigpu-vector_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs(nb, npb, seed):
    import pyoracle as po

    bk = po.gen_uniform(nb, seed, 0, -(1 << 20), 1 << 21)  # duplicates and negative keys
    bk[::101] = -(1 << 31)
    bp = po.gen_uniform(nb, seed, 1, -(1 << 31), 1 << 32)
    pk = po.gen_uniform(npb, seed, 2, -(1 << 20), 1 << 21)
    pk[::97] = -(1 << 31)
    pp = po.gen_uniform(npb, seed, 3, -(1 << 31), 1 << 32)
    return bk, bp, pk, pp


def _oracle_partition(cols, key_col, bits, shift):
    import torch
    import pyoracle as po

    keys = cols[key_col].numpy()
    order = np.argsort(((keys.astype(np.int64) & 0xFFFFFFFF) >> shift) & ((1 << bits) - 1), kind="stable")
    hist, _, _ = po.partition(keys, bits, shift)
    return [torch.from_numpy(np.ascontiguousarray(c.numpy()[order])) for c in cols], [int(h) for h in hist]


def _oracle_join(bk, bp, pk, pp):
    import pyoracle as po

    return po.Chain(bk.numpy(), bp.numpy()).probe_agg(pk.numpy(), pp.numpy())


def _rank(rank, world, port, seed, shift, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    for p in (os.path.join(ROOT, "multigpu-vector_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import torch

    import exchange
    import replicas

    dist, w, r, _ = replicas.init("gloo", timeout_s=60)
    bk, bp, pk, pp = _inputs(30011, 70001, seed)
    sl = lambda a: torch.from_numpy(np.ascontiguousarray(np.array_split(a, w)[r]))  # this rank's slice
    mine = [sl(a) for a in (bk, bp, pk, pp)]
    # routing: every received row's key belongs to this rank
    got_bk, got_bp = exchange.route(dist, mine[:2], 0, shift, _oracle_partition)
    owner = ((got_bk.numpy().astype(np.int64) & 0xFFFFFFFF) >> shift) & (w - 1)
    routed_ok = bool((owner == r).all())
    res = exchange.exchange_join(dist, mine[:2], mine[2:], _oracle_partition, _oracle_join, shift)
    replicas.finish(dist)
    q.put((r, routed_ok, int(got_bk.numel()), res))


@pytest.mark.parametrize("world,shift", [(2, 0), (4, 3)])
def test_exchange_join_equals_one_process_join(world, shift):
    import pyoracle as po

    seed = 0x5EED0B01 + world
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, seed, shift, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    bk, bp, pk, pp = _inputs(30011, 70001, seed)
    want = po.Chain(bk, bp).probe_agg(pk, pp)
    assert all(routed for _, routed, _, _ in out)
    assert sum(n for _, _, n, _ in out) == bk.size  # every build row landed somewhere, once
    for _, _, _, res in out:
        assert res == want


def test_world_must_be_a_power_of_two():
    import exchange

    assert exchange.world_bits(1) == 0 and exchange.world_bits(8) == 3
    with pytest.raises(ValueError):
        exchange.world_bits(6)
