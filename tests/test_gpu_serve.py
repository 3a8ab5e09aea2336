"""The query server: continuous batching over resident tables.

Each request's result is the same when it runs alone and when it runs in a
mix of concurrent requests, equals the plain server's result, and equals
the oracle; admission waits for memory instead of failing, and a request
that can never fit is rejected."""
import numpy as np
import pytest

import mgv
import pyoracle as po
from querymix import make_query_columns

pytestmark = pytest.mark.gpu


def setup_tables(ctx, torch, server, ntab=3, seed=21):
    tabs = []
    for t in range(ntab):
        nb = [1000, 30000, 200000][t % 3]
        cols = make_query_columns(ctx, torch, nb, 1 << 18, 4096, seed + t)
        tid = server.add_table(cols[0], nb)
        tabs.append((tid, nb, cols))
    return tabs


def requests(tabs, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        tid, nb, cols = tabs[int(rng.integers(len(tabs)))]
        rows = int(2 ** rng.uniform(8, 18))
        bound = int(rng.integers(10, 900))
        out.append((tid, rows, bound, cols))
    return out


def oracle(nb, cols, rows, bound):
    bk, pk, pf, pg, pv = [c.cpu().numpy() for c in cols]
    want, _, _ = po.run_query(bk[:nb], pk[:rows], pf[:rows], pg[:rows], pv[:rows], bound)
    return [(int(w["group"]), int(w["sum"]), int(w["count"])) for w in want]


def submit(server, r):
    tid, rows, bound, cols = r
    return server.submit(tid, cols[1], cols[2], cols[3], cols[4], rows, bound, 4096)


@pytest.mark.parametrize("batch_solo", [False, True])
def test_alone_equals_in_the_mix(ctx, torch_cuda, batch_solo):
    """A request alone on an idle server runs through the single-query
    operator chain (batch_solo False) or as a batch of one (True); either way
    its groups equal those it gets batched with 59 others."""
    s = mgv.Server(ctx, 8 << 30, max_batch=64, max_inflight=2, batch_solo=batch_solo)
    tabs = setup_tables(ctx, torch_cuda, s)
    reqs = requests(tabs, 60, 5)
    alone = []
    for r in reqs:  # one at a time
        st, rows, _ = s.wait(submit(s, r))
        assert st == mgv.OK
        alone.append(rows)
    tickets = [submit(s, r) for r in reqs]  # all at once: batched together
    mixed = [s.wait(t) for t in tickets]
    for i, (st, rows, lat) in enumerate(mixed):
        assert st == mgv.OK and rows == alone[i], i
        assert lat >= 0
    nbs = {tid: nb for tid, nb, _ in tabs}
    for i in range(0, 60, 7):
        tid, rows_n, bound, cols = reqs[i]
        assert alone[i] == oracle(nbs[tid], cols, rows_n, bound), i
    st = s.stats()
    assert st.completed == 120 and st.batches < 120  # the mix was batched
    assert (st.solo == 0) if batch_solo else (st.solo >= 60)
    s.destroy()


def test_plain_server_and_admission(ctx, torch_cuda):
    plain = mgv.Server(ctx, 8 << 30, plain=True)
    tabs = setup_tables(ctx, torch_cuda, plain)
    reqs = requests(tabs, 20, 6)
    want = []
    for r in reqs:
        st, rows, _ = plain.wait(submit(plain, r))
        assert st == mgv.OK
        want.append(rows)
    table_bytes = plain.stats().resident_table_bytes
    plain.destroy()
    # a budget that fits about two requests at a time: admission queues the rest
    per_req = 4096 * 2 * 20 + 4096 * 24 + 4096  # group table + result region, rounded up
    tight = mgv.Server(ctx, table_bytes + 2 * per_req, max_batch=64, max_inflight=2)
    setup_tables(ctx, torch_cuda, tight)
    tickets = [submit(tight, r) for r in reqs]
    for i, t in enumerate(tickets):
        st, rows, _ = tight.wait(t)
        assert st == mgv.OK and rows == want[i], i
    # a request that can never fit is rejected, not queued forever
    tid, rows_n, bound, cols = reqs[0]
    t = tight.submit(tid, cols[1], cols[2], cols[3], cols[4], rows_n, bound, 1 << 22)
    st, _, _ = tight.wait(t)
    assert st == mgv.ENOMEM
    tight.destroy()
