"""ctypes wrapper of the CPU oracle (liboracle.so) and of the reference's own
CPU loops (oracle/_ref/libmgvref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker / timed CPU baseline.  The
product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_int32, c_int64, c_size_t, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmgvref.so")

_lib = None
_ref = None


class ChainTable(ctypes.Structure):
    _fields_ = [("head", c_void_p), ("next", c_void_p), ("keys", c_void_p), ("pay", c_void_p),
                ("n", c_uint64), ("log_size", c_uint32)]


class GroupRow(ctypes.Structure):
    _fields_ = [("group", c_int32), ("pad", c_int32), ("sum", c_int64), ("count", c_int64)]


GROUP_DTYPE = np.dtype([("group", "<i4"), ("pad", "<i4"), ("sum", "<i8"), ("count", "<i8")])


class Query(ctypes.Structure):
    _fields_ = [("build_keys", c_void_p), ("build_rows", c_uint64), ("probe_key", c_void_p),
                ("probe_filter", c_void_p), ("probe_group", c_void_p), ("probe_value", c_void_p),
                ("probe_rows", c_uint64), ("filter_bound", c_int32)]


def build() -> None:
    """Compile liboracle.so (and oracle/_ref when the reference is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        P = c_void_p
        sig = {
            "or_gen_uniform": (None, [P, c_uint64, c_uint64, c_uint32, c_int64, c_uint64]),
            "or_gen_perm": (None, [P, c_uint64, c_uint64]),
            "or_gen_probe_keys": (c_uint64, [P, c_uint64, c_uint64, c_uint64, c_uint64, c_uint32, c_int64, c_uint64]),
            "or_zipf_cdf": (None, [P, c_uint32, c_double]),
            "or_gen_zipf": (None, [P, c_uint64, c_uint64, c_uint32, P, c_uint32]),
            "or_hash_murmur": (c_uint32, [c_uint32]),
            "or_select_rows": (c_size_t, [P, c_size_t, c_int32, P]),
            "or_select_agg": (None, [P, P, c_size_t, c_int32, POINTER(c_int64), POINTER(c_int64)]),
            "or_select_agg_mt": (None, [P, P, c_size_t, c_int32, c_int, POINTER(c_int64), POINTER(c_int64)]),
            "or_chain_build": (c_int, [POINTER(ChainTable), P, P, c_uint64, c_int, c_int32]),
            "or_chain_free": (None, [POINTER(ChainTable)]),
            "or_chain_probe_agg": (None, [POINTER(ChainTable), P, P, c_uint64, c_int, c_int,
                                          POINTER(c_int64), POINTER(c_int64)]),
            "or_chain_probe_agg_mt": (None, [POINTER(ChainTable), P, P, c_uint64, c_int,
                                             POINTER(c_int64), POINTER(c_int64)]),
            "or_chain_probe_emit": (c_uint64, [POINTER(ChainTable), P, P, c_uint64, P, c_uint64]),
            "or_chain_matches": (c_uint64, [POINTER(ChainTable), c_int32]),
            "or_partition": (None, [P, c_uint64, c_uint32, c_uint32, P, P, P, P]),
            "or_groupby": (c_uint64, [P, P, P, c_uint64, P, c_uint64]),
            "or_run_query": (c_uint64, [POINTER(Query), P, c_uint64, POINTER(c_int64), POINTER(c_int64)]),
            "or_run_query_mt": (c_uint64, [POINTER(Query), P, c_uint64, POINTER(c_int64), POINTER(c_int64), c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref() -> ctypes.CDLL:
    """The reference's own CPU functions (src/main8.cu:49-103, src/main9.cu:48-69)."""
    global _ref
    if _ref is None:
        R = ctypes.CDLL(REF_SO)
        P = c_void_p
        R.mgvref_stable_select.restype = c_uint64
        R.mgvref_stable_select.argtypes = [P, P, c_size_t, c_int32]
        R.mgvref_sum_select.restype = c_int32
        R.mgvref_sum_select.argtypes = [P, c_size_t, c_int32]
        R.mgvref_sum_selfjoin_select.restype = c_int32
        R.mgvref_sum_selfjoin_select.argtypes = [P, c_int]
        R.mgvref_sum_hashjoin_select.restype = c_int32
        R.mgvref_sum_hashjoin_select.argtypes = [P, c_int, P, c_int]
        R.mgvref_hash_murmur_masked.restype = c_uint32
        R.mgvref_hash_murmur_masked.argtypes = [c_uint32]
        R.mgvref_log_htsize.restype = c_int
        _ref = R
    return _ref


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


# ---- generators ---------------------------------------------------------

def gen_uniform(n, seed, stream, lo, rng) -> np.ndarray:
    out = np.empty(n, np.int32)
    lib().or_gen_uniform(_p(out), n, seed, stream, lo, rng)
    return out


def gen_perm(n, seed) -> np.ndarray:
    out = np.empty(n, np.int32)
    lib().or_gen_perm(_p(out), n, seed)
    return out


def gen_probe_keys(n, seed, build_seed, nbuild, hit_num, miss_lo, miss_range):
    out = np.empty(n, np.int32)
    hits = lib().or_gen_probe_keys(_p(out), n, seed, build_seed, nbuild, hit_num, miss_lo, miss_range)
    return out, int(hits)


def zipf_cdf(groups, s=1.0) -> np.ndarray:
    cdf = np.empty(groups, np.uint64)
    lib().or_zipf_cdf(_p(cdf), groups, s)
    return cdf


def gen_zipf(n, seed, stream, groups, s=1.0) -> np.ndarray:
    cdf = zipf_cdf(groups, s)
    out = np.empty(n, np.int32)
    lib().or_gen_zipf(_p(out), n, seed, stream, _p(cdf), groups)
    return out


# ---- operators ----------------------------------------------------------

def hash_murmur(x: int) -> int:
    return int(lib().or_hash_murmur(x & 0xFFFFFFFF))


def select_rows(a: np.ndarray, bound: int) -> np.ndarray:
    a = np.ascontiguousarray(a, np.int32)
    out = np.empty(max(1, a.size), np.int32)
    k = lib().or_select_rows(_p(a), a.size, bound, _p(out))
    return out[:k].copy()


def select_agg(f: np.ndarray, v: np.ndarray | None, bound: int):
    f = np.ascontiguousarray(f, np.int32)
    v = None if v is None else np.ascontiguousarray(v, np.int32)
    c, s = c_int64(), c_int64()
    lib().or_select_agg(_p(f), None if v is None else _p(v), f.size, bound, ctypes.byref(c), ctypes.byref(s))
    return c.value, s.value


def select_agg_mt(f: np.ndarray, v: np.ndarray | None, bound: int, threads: int):
    """select_agg split over `threads` host threads."""
    f = np.ascontiguousarray(f, np.int32)
    v = None if v is None else np.ascontiguousarray(v, np.int32)
    c, s = c_int64(), c_int64()
    lib().or_select_agg_mt(_p(f), None if v is None else _p(v), f.size, bound, threads, ctypes.byref(c),
                           ctypes.byref(s))
    return c.value, s.value


class Chain:
    """The reference's chained table (src/main8.cu:84-103), with payloads."""

    def __init__(self, keys: np.ndarray, pay: np.ndarray | None, filter_bound: int | None = None):
        self.keys = np.ascontiguousarray(keys, np.int32)
        self.pay = None if pay is None else np.ascontiguousarray(pay, np.int32)
        self.t = ChainTable()
        rc = lib().or_chain_build(ctypes.byref(self.t), _p(self.keys), None if self.pay is None else _p(self.pay),
                                  self.keys.size, 0 if filter_bound is None else 1,
                                  0 if filter_bound is None else filter_bound)
        if rc != 0:
            raise MemoryError("oracle chain build")

    def probe_agg(self, pk, pp=None, add_build=True, add_probe=True):
        pk = np.ascontiguousarray(pk, np.int32)
        pp = None if pp is None else np.ascontiguousarray(pp, np.int32)
        c, s = c_int64(), c_int64()
        lib().or_chain_probe_agg(ctypes.byref(self.t), _p(pk), None if pp is None else _p(pp), pk.size,
                                 int(add_build), int(add_probe), ctypes.byref(c), ctypes.byref(s))
        return c.value, s.value

    def probe_agg_mt(self, pk, pp, threads):
        c, s = c_int64(), c_int64()
        lib().or_chain_probe_agg_mt(ctypes.byref(self.t), _p(pk), None if pp is None else _p(pp), pk.size,
                                    threads, ctypes.byref(c), ctypes.byref(s))
        return c.value, s.value

    def probe_emit(self, pk, pp=None) -> np.ndarray:
        """Sorted (key, build payload, probe payload) match multiset."""
        pk = np.ascontiguousarray(pk, np.int32)
        pp = None if pp is None else np.ascontiguousarray(pp, np.int32)
        n = lib().or_chain_probe_emit(ctypes.byref(self.t), _p(pk), None if pp is None else _p(pp), pk.size,
                                      None, 0)
        out = np.empty((max(1, n), 3), np.int32)
        lib().or_chain_probe_emit(ctypes.byref(self.t), _p(pk), None if pp is None else _p(pp), pk.size,
                                  _p(out), n)
        out = out[:n]
        return out[np.lexsort((out[:, 2], out[:, 1], out[:, 0]))]

    def matches(self, key: int) -> int:
        return int(lib().or_chain_matches(ctypes.byref(self.t), key))

    def __del__(self):
        try:
            lib().or_chain_free(ctypes.byref(self.t))
        except Exception:
            pass


def partition(keys: np.ndarray, bits: int, shift: int, pay: np.ndarray | None = None):
    keys = np.ascontiguousarray(keys, np.int32)
    hist = np.zeros(1 << bits, np.uint64)
    ok = np.empty(max(1, keys.size), np.int32)
    op = None
    if pay is not None:
        pay = np.ascontiguousarray(pay, np.int32)
        op = np.empty(max(1, keys.size), np.int32)
    lib().or_partition(_p(keys), keys.size, bits, shift, _p(hist), _p(ok), None if pay is None else _p(pay),
                       None if op is None else _p(op))
    return hist, ok[:keys.size], (None if op is None else op[:keys.size])


def groupby(groups, values, mult=None) -> np.ndarray:
    groups = np.ascontiguousarray(groups, np.int32)
    values = None if values is None else np.ascontiguousarray(values, np.int32)
    mult = None if mult is None else np.ascontiguousarray(mult, np.int32)
    n = lib().or_groupby(_p(groups), None if values is None else _p(values), None if mult is None else _p(mult),
                         groups.size, None, 0)
    out = np.zeros(max(1, n), GROUP_DTYPE)
    lib().or_groupby(_p(groups), None if values is None else _p(values), None if mult is None else _p(mult),
                     groups.size, _p(out), n)
    return out[:n]


def run_query(build_keys, probe_key, probe_filter, probe_group, probe_value, bound, threads=1):
    """select(filter <= bound) -> join(build keys) -> group-by(group): SUM(value), COUNT
    (the select + probe phase on `threads` host threads)."""
    arrs = [np.ascontiguousarray(a, np.int32) for a in (build_keys, probe_key, probe_filter, probe_group, probe_value)]
    q = Query(_p(arrs[0]), arrs[0].size, _p(arrs[1]), _p(arrs[2]), _p(arrs[3]), _p(arrs[4]), arrs[1].size, bound)
    tc, ts = c_int64(), c_int64()
    cap = 1 << 17  # more groups than any workload here has; rerun with the exact count otherwise
    out = np.zeros(cap, GROUP_DTYPE)
    n = lib().or_run_query_mt(ctypes.byref(q), _p(out), cap, ctypes.byref(tc), ctypes.byref(ts), threads)
    if n > cap:
        out = np.zeros(n, GROUP_DTYPE)
        lib().or_run_query_mt(ctypes.byref(q), _p(out), n, ctypes.byref(tc), ctypes.byref(ts), threads)
    return out[:n], tc.value, ts.value
