"""Shared scans in the query server.

Requests of one batch over the same resident table, probe columns and row
count that differ only in their filter bound are answered by one scan: the
columns are read and the table probed once, each matched row is aggregated
into the cell of its filter range, and every request's groups are the prefix
of the ranges up to its bound.  Each request's groups must equal what it
gets alone (a batch of one, no sharing), with scans kept separate, and the
oracle's select -> join -> group-by; integer results match exactly."""
import numpy as np
import pytest

import mgv
import pyoracle as po
from gpu_util import dev
from querymix import make_query_columns

pytestmark = pytest.mark.gpu

MN = -(1 << 31)


def oracle(bk, pk, pf, pg, pv, rows, bound):
    want, _, _ = po.run_query(bk, pk[:rows], pf[:rows], pg[:rows], pv[:rows], bound)
    return [(int(w["group"]), int(w["sum"]), int(w["count"])) for w in want]


def run_all(server, tid, cols, reqs, max_groups):
    """Submits every (rows, bound) at once and returns the groups of each."""
    tickets = [server.submit(tid, cols[0], cols[1], cols[2], cols[3], rows, bound, max_groups)
               for rows, bound in reqs]
    out = []
    for t in tickets:
        st, rows, _ = server.wait(t, timeout_ms=120000)
        assert st == mgv.OK
        out.append(rows)
    return out


def test_shared_scan_equals_alone_separate_and_oracle(ctx, torch_cuda):
    """40 requests on one table and row count, bounds across the filter's
    range (duplicates, nothing selected, everything selected)."""
    torch = torch_cuda
    nb, npr, G = 30000, 1 << 18, 4096
    bk, pk, pf, pg, pv = make_query_columns(ctx, torch, nb, npr, G, 77)
    rng = np.random.default_rng(3)
    bounds = [int(b) for b in rng.integers(0, 1000, 34)] + [-1, -50, 999, 5000, 120, 120]
    reqs = [(npr, b) for b in bounds]
    shared = mgv.Server(ctx, 8 << 30, max_batch=64, max_inflight=2, batch_solo=True)
    tid = shared.add_table(bk, nb)
    got = run_all(shared, tid, (pk, pf, pg, pv), reqs, G)
    st = shared.stats()
    assert st.shared_scans >= 1 and st.scan_queries >= 2
    # alone: one request per batch, so nothing is shared
    alone = []
    for r in reqs:
        alone.append(run_all(shared, tid, (pk, pf, pg, pv), [r], G)[0])
    shared.destroy()
    sep = mgv.Server(ctx, 8 << 30, max_batch=64, max_inflight=2, batch_solo=True, separate_scans=True)
    tid2 = sep.add_table(bk, nb)
    separate = run_all(sep, tid2, (pk, pf, pg, pv), reqs, G)
    assert sep.stats().shared_scans == 0
    sep.destroy()
    hb, hk, hf, hg, hv = (c.cpu().numpy() for c in (bk, pk, pf, pg, pv))
    for i, (rows, b) in enumerate(reqs):
        assert got[i] == alone[i] == separate[i], (i, b)
    for i in range(0, len(reqs), 5):
        assert got[i] == oracle(hb[:nb], hk, hf, hg, hv, npr, reqs[i][1]), i
    for i in range(34, 40):
        assert got[i] == oracle(hb[:nb], hk, hf, hg, hv, npr, reqs[i][1]), i


def test_shared_scan_mixed_with_single_requests(ctx, torch_cuda):
    """One batch holds two shared scans (two row counts on one table), one on
    a second table with duplicate build keys (every copy matches), and
    requests that share with nobody."""
    torch = torch_cuda
    G = 512
    a = make_query_columns(ctx, torch, 5000, 1 << 17, G, 81)
    b = make_query_columns(ctx, torch, 20000, 1 << 16, G, 82, dup=True)
    s = mgv.Server(ctx, 8 << 30, max_batch=128, max_inflight=2, batch_solo=True)
    ta = s.add_table(a[0], 5000)
    tb = s.add_table(b[0], 20000)
    rng = np.random.default_rng(4)
    plan = []
    for _ in range(12):
        plan.append((ta, a, 1 << 17, int(rng.integers(0, 1000))))
    for _ in range(9):
        plan.append((ta, a, 100003, int(rng.integers(0, 1000))))
    for _ in range(10):
        plan.append((tb, b, 1 << 16, int(rng.integers(0, 1000))))
    for rows in (777, 4096, 65000):
        plan.append((tb, b, rows, int(rng.integers(0, 1000))))
    order = rng.permutation(len(plan))
    tickets = [s.submit(plan[i][0], *plan[i][1][1:], plan[i][2], plan[i][3], G) for i in order]
    got = {}
    for i, t in zip(order, tickets):
        st, rows, _ = s.wait(t, timeout_ms=120000)
        assert st == mgv.OK
        got[int(i)] = rows
    assert s.stats().shared_scans >= 3
    s.destroy()
    host = {id(a): [c.cpu().numpy() for c in a], id(b): [c.cpu().numpy() for c in b]}
    nbs = {id(a): 5000, id(b): 20000}
    for i, (_, cols, rows, bound) in enumerate(plan):
        h = host[id(cols)]
        assert got[i] == oracle(h[0][:nbs[id(cols)]], h[1], h[2], h[3], h[4], rows, bound), i


def test_shared_scan_reserved_values_and_many_groups(ctx, torch_cuda):
    """INT32_MIN build and probe keys (the side list), INT32_MIN and extreme
    group ids, negative values, filters at both ends of int32, and more
    distinct groups than a CTA's shared cells hold (the global cells)."""
    torch = torch_cuda
    nb, npr = 3000, 200000
    rng = np.random.default_rng(9)
    bk = rng.integers(-5000, 5000, nb).astype(np.int32)
    bk[::50] = MN
    pk = rng.integers(-6000, 6000, npr).astype(np.int32)
    pk[::37] = MN
    pf = rng.integers(MN, (1 << 31) - 1, npr, dtype=np.int64).astype(np.int32)
    pf[::11] = MN
    pf[::13] = (1 << 31) - 1
    pg = rng.integers(0, 50000, npr).astype(np.int32)
    pg[::7] = MN
    pg[::29] = (1 << 31) - 1
    pv = rng.integers(MN, (1 << 31) - 1, npr, dtype=np.int64).astype(np.int32)
    d = [dev(torch, x) for x in (bk, pk, pf, pg, pv)]
    s = mgv.Server(ctx, 8 << 30, max_batch=64, max_inflight=1, batch_solo=True)
    tid = s.add_table(d[0], nb)
    bounds = [MN, -1, 0, 1 << 30, (1 << 31) - 2, (1 << 31) - 1, -(1 << 30), 12345]
    got = run_all(s, tid, d[1:], [(npr, b) for b in bounds], 65536)
    assert s.stats().shared_scans >= 1
    s.destroy()
    for i, b in enumerate(bounds):
        assert got[i] == oracle(bk, pk, pf, pg, pv, npr, b), (i, b)
