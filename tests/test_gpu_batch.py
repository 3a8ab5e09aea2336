"""Batched select -> join -> group-by queries: the batch, the plain
one-query-at-a-time pipeline and the oracle agree exactly on every query."""
import pytest

import mgv
from querymix import make_mix, make_query_columns, oracle_answer

pytestmark = pytest.mark.gpu


def descs(mgv, mix):
    return [mgv.query_desc(q["cols"][0], q["nb"], *q["cols"][1:], q["npr"], q["bound"], q["G"]) for q in mix]


@pytest.mark.parametrize("use_graph,item_order", [(0, 0), (1, 0), (1, 1)])
def test_batch_matches_plain_and_oracle(ctx, torch_cuda, use_graph, item_order):
    mix = make_mix(ctx, torch_cuda, 48, 11)
    cfg = mgv.BatchConfig(0.5, 4096, 8192, 0, use_graph, item_order)
    b = mgv.Batch(ctx, descs(mgv, mix), cfg)
    b.run()
    b.run()  # second run: graph replay when use_graph
    b.run_plain()
    for i, q in enumerate(mix):
        got = b.result(i)
        assert got == b.result(i, plain=True), i
        assert got == oracle_answer(q), i
    st = b.stats()
    assert st.queries == 48 and st.graph == use_graph
    b.destroy()


def test_batch_edge_queries(ctx, torch_cuda):
    torch = torch_cuda
    qs = [make_query_columns(ctx, torch, nb, npr, G, 77 + i) for i, (nb, npr, G) in
          enumerate([(0, 1000, 16), (1000, 0, 16), (1, 1, 1), (5000, 70001, 65536), (129, 4097, 3)])]
    mix = [dict(nb=nb, npr=npr, bound=b, G=G, cols=c) for (nb, npr, G, b), c in
           zip([(0, 1000, 16, 999), (1000, 0, 16, 500), (1, 1, 1, 999), (5000, 70001, 65536, 300), (129, 4097, 3, 0)],
               qs)]
    b = mgv.Batch(ctx, descs(mgv, mix))
    b.run()
    for i, q in enumerate(mix):
        assert b.result(i) == oracle_answer(q), i
    b.destroy()


def test_autotune_picks_a_config(ctx, torch_cuda):
    mix = make_mix(ctx, torch_cuda, 16, 12)
    cfg = mgv.batch_autotune(ctx, descs(mgv, mix))
    assert 0.3 < cfg.load_factor < 0.7 and cfg.probe_item_rows in (8192, 32768, 131072)
    b = mgv.Batch(ctx, descs(mgv, mix))  # uses the tuned configuration
    b.run()
    for i, q in enumerate(mix):
        assert b.result(i) == oracle_answer(q), i
    b.destroy()


@pytest.mark.parametrize("item_order", [0, 1])
def test_batch_ctas_switch_queries(ctx, torch_cuda, item_order):
    """Hundreds of small queries: every CTA runs several queries in turn,
    flushing one query's shared group table and loading the next query's
    descriptor between them."""
    mix = make_mix(ctx, torch_cuda, 600, 13, build=(6, 12), probe=(8, 13), groups=(2, 10))
    cfg = mgv.BatchConfig(0.5, 4096, 8192, 1, 1, item_order)
    b = mgv.Batch(ctx, descs(mgv, mix), cfg)
    assert b.stats().probe_items > 2 * 148
    for _ in range(3):
        b.run()
    b.run_plain()
    for i, q in enumerate(mix):
        got = b.result(i)
        assert got == b.result(i, plain=True), i
        if i % 5 == 0:
            assert got == oracle_answer(q), i
    b.destroy()
