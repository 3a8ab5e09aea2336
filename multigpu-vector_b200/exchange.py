"""Multi-GPU hash exchange: the reference's hash_exchange join across GPUs.

The reference joins on two GPUs by routing every row of both sides to the
GPU that owns its key (hash_exchange, src/main9.cu:104-148: a split on
hash3(x) = x & 1, src/operators/split.cu:49-151, feeding one join per GPU),
and merges the GPUs' outputs with union_all (src/operators/union_all.cu:35-57).
Here, one process per GPU (torch.distributed, NCCL over NVLink):

  1. route: each rank partitions its rows by (key >> shift) & (world - 1) on
     its GPU (mgv_partition_columns, partition-major), exchanges the
     per-destination row counts, then moves every column with one
     all_to_all_single whose split sizes are those counts, so partition p
     of every rank lands on rank p (the copy goes into this GPU's memory
     first; no kernel reads a peer's memory);
  2. join: each rank builds a hash table on the build rows it received and
     probes it with the probe rows it received (hash_build, then
     hash_probe -> aggregate: COUNT and SUM(build payload + probe payload));
  3. merge: one all_reduce (sum) of the ranks' int64 (COUNT, SUM); two's
     complement addition makes the merged SUM exact.

A key lives on exactly one rank after routing, so every match is found on
exactly one rank and the merged result equals a one-GPU join of all rows.
`world` must be a power of two (the route takes log2(world) key bits).

The routing and join steps are passed in as functions: on GPUs they are the
mgv kernels (gpu_partition / gpu_join); the CPU tests pass the oracle's, so
the exchange itself runs over gloo without a GPU.
"""
from __future__ import annotations


def world_bits(world: int) -> int:
    """log2(world); world must be a power of two."""
    if world < 1 or world & (world - 1):
        raise ValueError(f"hash exchange needs a power-of-two world size, got {world}")
    return world.bit_length() - 1


def route(dist, cols, key_col: int, shift: int, partition, device="cpu"):
    """Rows of `cols` (equal-length int32 tensors) moved to the rank that owns
    their key: partition p = (key >> shift) & (world - 1) goes to rank p.
    Returns this rank's received columns."""
    import torch

    world = dist.get_world_size() if dist is not None else 1
    bits = world_bits(world)
    if world == 1:
        return list(cols)
    parts, counts = partition(cols, key_col, bits, shift)
    send = torch.tensor([int(c) for c in counts], dtype=torch.int64, device=device)
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send)
    send_l = [int(c) for c in counts]
    recv_l = [int(c) for c in recv.tolist()]
    out = []
    for c in range(len(cols)):
        o = torch.empty(sum(recv_l), dtype=torch.int32, device=device)
        dist.all_to_all_single(o, parts[c].contiguous(), output_split_sizes=recv_l, input_split_sizes=send_l)
        out.append(o)
    return out


def merge(dist, count: int, total: int, device="cpu"):
    """Sum of every rank's (COUNT, SUM) as int64 (union_all of the partial aggregates)."""
    import torch

    if dist is None or dist.get_world_size() == 1:
        return int(count), int(total)
    t = torch.tensor([int(count), int(total)], dtype=torch.int64, device=device)
    dist.all_reduce(t)
    return int(t[0].item()), int(t[1].item())


def exchange_join(dist, build_cols, probe_cols, partition, join, shift: int = 0, device="cpu"):
    """The hash-exchange join: (COUNT, SUM(build payload + probe payload)) over
    every rank's rows.  build_cols = [keys, payloads], probe_cols = [keys,
    payloads] of this rank; `partition` and `join` as gpu_partition /
    gpu_join (or the oracle's on CPU)."""
    bk, bp = route(dist, build_cols, 0, shift, partition, device)
    pk, pp = route(dist, probe_cols, 0, shift, partition, device)
    count, total = join(bk, bp, pk, pp)
    return merge(dist, count, total, device)


def gpu_partition(ctx, stream=None):
    """The routing step on this GPU: mgv_partition_columns into one buffer."""
    import torch

    def partition(cols, key_col, bits, shift):
        n = int(cols[0].numel())
        stride = max(n, 1)
        out = torch.empty((len(cols), stride), dtype=torch.int32, device=cols[0].device)
        counts = ctx.partition_columns(cols, n, key_col, bits, shift, out, stride, stream)
        return [out[c, :n] for c in range(len(cols))], counts

    return partition


def gpu_join(ctx, load_factor: float = 0.0, stream=None):
    """The local join on this GPU: hash_build, then hash_probe -> aggregate."""
    import mgv

    def join(bk, bp, pk, pp):
        nb, npb = int(bk.numel()), int(pk.numel())
        bhead, hb, probe, agg = mgv.create_count_join_1G_pipeline(ctx, max(nb, 1), load_factor)
        try:
            bhead.open(stream)
            if nb:
                bhead.consume_columns([bk, bp], nb, stream)
            bhead.close(stream)
            probe.open(stream)
            if npb:
                probe.consume_columns([pk, pp], npb, stream)
            probe.close(stream)
            return agg.result()
        finally:
            for o in (probe, agg, bhead, hb):
                o.destroy()

    return join
