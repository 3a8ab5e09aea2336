"""Seeded mixes of select -> join -> group-by queries (the batched / served
configurations, scaled) generated on the device, plus their oracle answers."""
import numpy as np

import pyoracle as po

HIT = 3865470566  # 0.9 * 2^32


def make_query_columns(ctx, torch, nb, npr, G, seed, dup=False):
    """Build keys (a permutation, or with duplicates) and probe columns
    (key 90% from the build keys, filter U[0,1000), group Zipf(1) over G,
    value U[0,2^20))."""
    dev = lambda n: torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    bk, pk, pf, pg, pv = dev(nb), dev(npr), dev(npr), dev(npr), dev(npr)
    if nb:
        if dup:
            ctx.gen_uniform(bk, nb, seed, 9, 0, max(1, nb // 3))
        else:
            ctx.gen_perm(bk, nb, seed)
    if npr:
        ctx.gen_probe_keys(pk, npr, seed + 1, seed, max(nb, 1), HIT, max(nb, 1), (1 << 31) - max(nb, 1))
        ctx.gen_uniform(pf, npr, seed + 1, 2, 0, 1000)
        ctx.gen_zipf(pg, npr, seed + 1, 3, G)
        ctx.gen_uniform(pv, npr, seed + 1, 4, 0, 1 << 20)
    return bk, pk, pf, pg, pv


def make_mix(ctx, torch, nq, seed, build=(8, 14), probe=(10, 16), groups=(4, 12)):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nq):
        nb = int(2 ** rng.uniform(*build))
        npr = int(2 ** rng.uniform(*probe))
        bound = int(round(rng.uniform(0.01, 0.9) * 1000)) - 1
        G = int(2 ** rng.uniform(*groups))
        cols = make_query_columns(ctx, torch, nb, npr, G, seed * 1000 + i, dup=(i % 7 == 3))
        out.append(dict(nb=nb, npr=npr, bound=bound, G=G, cols=cols))
    return out


def oracle_answer(q):
    bk, pk, pf, pg, pv = [c.cpu().numpy() for c in q["cols"]]
    want, _, _ = po.run_query(bk[:q["nb"]], pk[:q["npr"]], pf[:q["npr"]], pg[:q["npr"]], pv[:q["npr"]], q["bound"])
    return [(int(w["group"]), int(w["sum"]), int(w["count"])) for w in want]
