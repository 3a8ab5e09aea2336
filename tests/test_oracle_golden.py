"""The CPU oracle against the reference's own CPU functions.

tests/golden/reference_outputs.json holds answers of the reference's
stable_select_cpu, sum_select_cpu, sum_selfjoin_select_cpu,
sum_hashjoin_select_cpu and h_hashMurmur (src/main8.cu:49-103,
src/main9.cu:48-69) on seeded inputs; the oracle must reproduce every one
(int32 sums compared as the low 32 bits of the oracle's int64).  When the
reference library oracle/_ref/libmgvref.so is present it is also run live.
"""
import json
import os

import numpy as np
import pytest

import pyoracle as po

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_outputs.json")
DOC = json.load(open(GOLDEN))


def i32(x: int) -> int:
    return ((x + (1 << 31)) % (1 << 32)) - (1 << 31)


def col(spec):
    if spec["kind"] == "uniform":
        return po.gen_uniform(spec["n"], spec["seed"], spec["stream"], spec["lo"], spec["range"])
    return po.gen_perm(spec["n"], spec["seed"])


def poly_hash(a):
    i = np.arange(1, a.size + 1, dtype=np.uint64)
    return int(np.sum(i * a.astype(np.uint32).astype(np.uint64), dtype=np.uint64))


def test_generator_pins():
    p = DOC["generator_pins"]
    assert po.gen_uniform(8, 0x5EED0001, 0, 0, 1 << 31).tolist() == p["uniform"]
    assert po.gen_perm(16, 0x5EED0002).tolist() == p["perm16"]
    keys, _ = po.gen_probe_keys(8, 0x5EED0003, 0x5EED0002, 1 << 22, 3865470566, 1 << 22, (1 << 31) - (1 << 22))
    assert keys.tolist() == p["probe"]
    assert po.gen_zipf(8, 0x5EED0004, 5, 4096).tolist() == p["zipf"]


CASES = DOC["cases"]


@pytest.mark.parametrize("case", [c for c in CASES if c["op"] == "select"],
                         ids=lambda c: f"n{c['input']['n']}_b{c['bound']}")
def test_select_vs_reference(case):
    a = col(case["input"])
    rows = po.select_rows(a, case["bound"])
    assert rows.size == case["count"]
    assert poly_hash(rows) == case["checksum"]  # stable order, as stable_select_cpu
    cnt, s = po.select_agg(a, None, case["bound"])
    assert cnt == case["count"]
    assert i32(s) == case["sum_int32"]


@pytest.mark.parametrize("case", [c for c in CASES if c["op"] == "selfjoin"], ids=lambda c: f"n{c['input']['n']}")
def test_selfjoin_vs_reference(case):
    a = col(case["input"])
    sel = po.select_rows(a, 5000)
    # join of the selection with itself through the chained table
    ch = po.Chain(sel, None)
    cnt, _ = ch.probe_agg(sel, None, False, False)
    assert i32(cnt) == case["count_int32"]


@pytest.mark.parametrize("case", [c for c in CASES if c["op"] == "hashjoin"],
                         ids=lambda c: f"b{c['build']['n']}_p{c['probe']['n']}")
def test_hashjoin_vs_reference(case):
    a, p = col(case["build"]), col(case["probe"])
    ch = po.Chain(a, None, filter_bound=case["build_filter"])
    cnt, _ = ch.probe_agg(p, None, False, False)
    assert i32(cnt) == case["count_int32"]


def test_murmur_vs_reference():
    c = [c for c in CASES if c["op"] == "murmur_masked"][0]
    mask = (1 << c["log_htsize"]) - 1
    assert [po.hash_murmur(x) & mask for x in c["x"]] == c["h"]


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_live_reference_matches_oracle():
    R = po.ref()
    rng_spec = {"kind": "uniform", "n": 30011, "seed": 0x5EED0999, "stream": 9, "lo": 1, "range": 10000}
    a = col(rng_spec)
    p = col(dict(rng_spec, seed=0x5EED0998, n=20011))
    for thres in (0, 1, 77, 5000, 9999, 10000):
        out = np.empty(a.size, np.int32)
        k = int(R.mgvref_stable_select(a.ctypes.data, out.ctypes.data, a.size, thres))
        assert np.array_equal(out[:k], po.select_rows(a, thres))
        assert int(R.mgvref_sum_select(a.ctypes.data, a.size, thres)) == i32(po.select_agg(a, None, thres)[1])
    ch = po.Chain(a, None, filter_bound=5000)
    assert int(R.mgvref_sum_hashjoin_select(a.ctypes.data, a.size, p.ctypes.data, p.size)) == \
        i32(ch.probe_agg(p, None, False, False)[0])
