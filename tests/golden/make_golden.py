"""Generate tests/golden/reference_outputs.json from the reference's own CPU code.

Run here, where the reference checkout exists:

    make -C oracle && python tests/golden/make_golden.py

Inputs come from the seeded generator (mgv_gen.h via the oracle library);
the outputs come from the reference's CPU functions compiled from its
sources by oracle/build_ref.sh (stable_select_cpu, sum_select_cpu,
sum_selfjoin_select_cpu, sum_hashjoin_select_cpu, h_hashMurmur:
src/main8.cu:49-103, src/main9.cu:48-69).  The fixture stores generator
parameters and the reference's answers, never reference source.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as po  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_outputs.json")


def col(spec):
    """Materialise a column from its generator spec."""
    kind = spec["kind"]
    if kind == "uniform":
        return po.gen_uniform(spec["n"], spec["seed"], spec["stream"], spec["lo"], spec["range"])
    if kind == "perm":
        return po.gen_perm(spec["n"], spec["seed"])
    raise ValueError(kind)


def poly_hash(a: np.ndarray) -> int:
    """Order-sensitive 64-bit checksum: sum of (i+1) * (a[i] mod 2^32)."""
    i = np.arange(1, a.size + 1, dtype=np.uint64)
    return int(np.sum(i * a.astype(np.uint32).astype(np.uint64), dtype=np.uint64))


def main():
    R = po.ref()
    cases = []
    # reference driver distribution: e1() % 10000 + 1  (src/main9.cu:560-561)
    small = lambda n, seed, stream: {"kind": "uniform", "n": n, "seed": seed, "stream": stream, "lo": 1, "range": 10000}

    # select: stable_select_cpu count + order-sensitive checksum, sum_select_cpu
    for n, thres, spec in [
        (0, 5000, small(0, 0x5EED0101, 0)),
        (1, 5000, small(1, 0x5EED0102, 0)),
        (127, 5000, small(127, 0x5EED0103, 0)),
        (129, 5000, small(129, 0x5EED0104, 0)),
        (100000, 5000, small(100000, 0x5EED0105, 0)),
        (100000, 0, small(100000, 0x5EED0106, 0)),
        (100000, 10000, small(100000, 0x5EED0107, 0)),
        (4099, 1, small(4099, 0x5EED0108, 0)),
        # config-1 style: uniform [0, 2^31), predicate col < 2^30
        (1 << 20, (1 << 30) - 1, {"kind": "uniform", "n": 1 << 20, "seed": 0x5EED0001, "stream": 0, "lo": 0, "range": 1 << 31}),
        # negative values: uniform over the whole int32 range
        (50000, -7, {"kind": "uniform", "n": 50000, "seed": 0x5EED0109, "stream": 3, "lo": -(1 << 31), "range": 1 << 32}),
    ]:
        a = col(spec)
        sel = np.empty(max(1, n), np.int32)
        k = int(R.mgvref_stable_select(a.ctypes.data, sel.ctypes.data, n, thres))
        cases.append({
            "op": "select", "input": spec, "bound": thres,
            "count": k, "checksum": poly_hash(sel[:k]),
            "sum_int32": int(R.mgvref_sum_select(a.ctypes.data, n, thres)),
        })

    # self join: sum over v of hist[v]^2 for rows <= 5000 (src/main8.cu:64-70)
    for n, seed in [(0, 0x5EED0201), (1000, 0x5EED0202), (50000, 0x5EED0203), (200000, 0x5EED0204)]:
        spec = small(n, seed, 1)
        a = col(spec)
        cases.append({"op": "selfjoin", "input": spec,
                      "count_int32": int(R.mgvref_sum_selfjoin_select(a.ctypes.data, n))})

    # hash join count: build rows <= 5000 of a, probe with p (src/main8.cu:84-103)
    for n, m, seed in [(0, 100, 0x5EED0301), (100, 0, 0x5EED0302), (1, 1, 0x5EED0303),
                       (60000, 70000, 0x5EED0304), (300000, 100000, 0x5EED0305), (129, 4097, 0x5EED0306)]:
        bspec = small(n, seed, 2)
        pspec = small(m, seed, 3)
        a, p = col(bspec), col(pspec)
        cases.append({"op": "hashjoin", "build": bspec, "probe": pspec, "build_filter": 5000,
                      "count_int32": int(R.mgvref_sum_hashjoin_select(a.ctypes.data, n, p.ctypes.data, m))})

    # h_hashMurmur masked to 2^20 buckets (src/main8.cu:75-82)
    xs = [0, 1, 2, 3, 5000, 10000, 65535, 1 << 20, (1 << 31) - 1, 1 << 31, 0xFFFFFFFF, 0x12345678, 0xDEADBEEF]
    cases.append({"op": "murmur_masked", "log_htsize": int(R.mgvref_log_htsize()), "x": xs,
                  "h": [int(R.mgvref_hash_murmur_masked(x)) for x in xs]})

    # generator pins (the fixtures above depend on these streams)
    pins = {
        "uniform": po.gen_uniform(8, 0x5EED0001, 0, 0, 1 << 31).tolist(),
        "perm16": po.gen_perm(16, 0x5EED0002).tolist(),
        "probe": po.gen_probe_keys(8, 0x5EED0003, 0x5EED0002, 1 << 22, 3865470566, 1 << 22, (1 << 31) - (1 << 22))[0].tolist(),
        "zipf": po.gen_zipf(8, 0x5EED0004, 5, 4096).tolist(),
    }
    doc = {"source": "reference CPU functions src/main8.cu:49-103, src/main9.cu:48-69 via oracle/build_ref.sh",
           "generator_pins": pins, "cases": cases}
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=1)
    print(f"wrote {OUT}: {len(cases)} cases")


if __name__ == "__main__":
    main()
