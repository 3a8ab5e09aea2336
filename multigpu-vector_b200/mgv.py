"""ctypes binding of libmgv (include/mgv.h) and the reference-style plans.

The library is the product: every operator runs as a CUDA kernel for
sm_100a inside libmgv.so.  This module only binds the C ABI and builds the
operator chains the reference's drivers build (``create_sum_select_pipeline``
and ``create_count_join_1G_pipeline`` in src/main9.cu:202-367), so that callers
and tests read like the reference's own plans.  There is no CPU fallback:
importing this module without the built library raises.
"""
from __future__ import annotations

import ctypes
import os
import re
from ctypes import POINTER, byref, c_char, c_double, c_float, c_int, c_int32, c_int64, c_size_t
from ctypes import c_uint32, c_uint64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmgv.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
HEADER = os.path.join(INCLUDE, "mgv.h")
# Every public header: the operator API (mgv.h) and the diagnostics (mgv_diag.h).
HEADERS = [os.path.join(INCLUDE, f) for f in ("mgv.h", "mgv_diag.h")]

MAX_COLS = 8
# Rows per pool buffer by default (DEFAULT_BUFF_CAP, src/common.cuh:8-10).
DEFAULT_BUFFER_ROWS = 4 * 1024 * 1024

# mgv_status
OK, EINVAL, ENOMEM, ETIMEDOUT, ECUDA, EDEVICE, ESTATE, EDRAINED, EUNSUPPORTED = range(9)
STATUS_NAMES = {
    OK: "MGV_OK", EINVAL: "MGV_EINVAL", ENOMEM: "MGV_ENOMEM", ETIMEDOUT: "MGV_ETIMEDOUT",
    ECUDA: "MGV_ECUDA", EDEVICE: "MGV_EDEVICE", ESTATE: "MGV_ESTATE", EDRAINED: "MGV_EDRAINED",
    EUNSUPPORTED: "MGV_EUNSUPPORTED",
}


class MgvError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {detail}")
        self.status = status


class Buffer(ctypes.Structure):
    _fields_ = [("cols", c_void_p * MAX_COLS), ("ncols", c_uint32), ("rows", c_uint32),
                ("capacity", c_uint32), ("id", c_uint32), ("device", c_int32), ("reserved", c_uint32)]


class CtxInfo(ctypes.Structure):
    _fields_ = [("device", c_int32), ("sm_count", c_int32), ("l2_bytes", c_uint64),
                ("hbm_bytes", c_uint64), ("cc_major", c_int32), ("cc_minor", c_int32),
                ("name", c_char * 64)]


class Tuning(ctypes.Structure):
    _fields_ = [("probe_kernel", c_uint32), ("probe_rows_per_thread", c_uint32), ("probe_stages", c_uint32),
                ("probe_ctas_per_sm", c_uint32), ("default_load_factor", c_float),
                ("groupby_smem_slots", c_uint32), ("select_ctas_per_sm", c_uint32), ("select_compact", c_uint32)]


class PoolStats(ctypes.Structure):
    _fields_ = [("nbuffers", c_uint32), ("capacity", c_uint32), ("ncols", c_uint32),
                ("available", c_uint32), ("host_cached", c_uint32), ("producers", c_uint32),
                ("bytes", c_uint64)]


class PoolDevice(ctypes.Structure):
    _fields_ = [("head", c_void_p), ("available", c_void_p), ("producers", c_void_p), ("next", c_void_p),
                ("slab", c_void_p), ("nbuffers", c_uint32), ("capacity", c_uint32), ("ncols", c_uint32),
                ("reserved", c_uint32)]


class SelectDesc(ctypes.Structure):
    _fields_ = [("col", c_uint32), ("bound", c_int32)]


class AggregateDesc(ctypes.Structure):
    _fields_ = [("sum_col_a", c_int32), ("sum_col_b", c_int32)]


class AggResult(ctypes.Structure):
    _fields_ = [("count", c_int64), ("sum", c_int64)]


class HashBuildDesc(ctypes.Structure):
    _fields_ = [("key_col", c_uint32), ("payload_col", c_int32), ("expected_rows", c_uint64),
                ("load_factor", c_float), ("radix_bits", c_uint32), ("radix_shift", c_uint32),
                ("reserved", c_uint32)]


class HashBuildInfo(ctypes.Structure):
    _fields_ = [("rows", c_uint64), ("nbuckets", c_uint64), ("table_bytes", c_uint64),
                ("reserved_key_rows", c_uint64), ("has_duplicates", c_uint32), ("reserved", c_uint32)]


class HashProbeDesc(ctypes.Structure):
    _fields_ = [("key_col", c_uint32), ("reserved", c_uint32), ("build", c_void_p)]


class GroupbyDesc(ctypes.Structure):
    _fields_ = [("group_col", c_uint32), ("value_col", c_int32), ("max_groups", c_uint32), ("reserved", c_uint32)]


class GroupRow(ctypes.Structure):
    _fields_ = [("group", c_int32), ("pad", c_int32), ("sum", c_int64), ("count", c_int64)]


class PartitionDesc(ctypes.Structure):
    _fields_ = [("key_col", c_uint32), ("radix_bits", c_uint32), ("radix_shift", c_uint32), ("reserved", c_uint32),
                ("max_rows", c_uint64)]


class QueryDesc(ctypes.Structure):
    _fields_ = [("build_keys", c_void_p), ("build_payloads", c_void_p), ("build_rows", c_uint64),
                ("probe_key", c_void_p), ("probe_filter", c_void_p), ("probe_group", c_void_p),
                ("probe_value", c_void_p), ("probe_rows", c_uint64), ("filter_bound", c_int32),
                ("max_groups", c_uint32)]


class BatchConfig(ctypes.Structure):
    _fields_ = [("load_factor", c_float), ("build_item_rows", c_uint32), ("probe_item_rows", c_uint32),
                ("probe_ctas_per_sm", c_uint32), ("use_graph", c_uint32), ("item_order", c_uint32),
                ("reserved", c_uint32 * 2)]


class BatchStats(ctypes.Structure):
    _fields_ = [("arena_bytes", c_uint64), ("queries", c_uint32), ("build_items", c_uint32),
                ("probe_items", c_uint32), ("graph", c_uint32), ("last_run_ms", c_double)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("memory_budget", c_uint64), ("max_batch", c_uint32), ("max_inflight", c_uint32),
                ("load_factor", c_float), ("plain", c_uint32), ("batch_solo", c_uint32),
                ("separate_scans", c_uint32)]


class ServerRequest(ctypes.Structure):
    _fields_ = [("table", c_uint32), ("reserved", c_uint32), ("probe_key", c_void_p), ("probe_filter", c_void_p),
                ("probe_group", c_void_p), ("probe_value", c_void_p), ("probe_rows", c_uint64),
                ("filter_bound", c_int32), ("max_groups", c_uint32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", c_uint64), ("completed", c_uint64), ("batches", c_uint64), ("rejected", c_uint64),
                ("p50_ms", c_double), ("p99_ms", c_double), ("mean_ms", c_double), ("max_ms", c_double),
                ("mean_batch", c_double), ("resident_table_bytes", c_uint64), ("peak_bytes", c_uint64),
                ("solo", c_uint64), ("shared_scans", c_uint64), ("scan_queries", c_uint64)]


class DiagGatherDesc(ctypes.Structure):
    _fields_ = [("table_bytes", c_uint64), ("lookups", c_uint64), ("line_bytes", c_uint32), ("method", c_uint32),
                ("ctas_per_sm", c_uint32), ("reps", c_uint32), ("inflight", c_uint32), ("lsu_warps", c_uint32),
                ("tma_warps", c_uint32), ("tma_share", c_float)]


class SinkDesc(ctypes.Structure):
    _fields_ = [("pool", c_void_p), ("max_buffers", c_uint32), ("reserved", c_uint32)]


_lib = None


def header_functions(paths=None) -> list[str]:
    """Names of the functions the public headers (include/*.h) declare."""
    names = set()
    for path in paths or HEADERS:
        text = open(path).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(mgv_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libmgv.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libmgv.so is not built ({path}); run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    st = c_int
    sigs = {
        "mgv_status_string": (ctypes.c_char_p, [c_int]),
        "mgv_last_error_string": (ctypes.c_char_p, []),
        "mgv_ctx_create": (st, [c_int, POINTER(c_void_p)]),
        "mgv_ctx_destroy": (st, [c_void_p]),
        "mgv_ctx_info_get": (st, [c_void_p, POINTER(CtxInfo)]),
        "mgv_ctx_sync": (st, [c_void_p, c_void_p]),
        "mgv_ctx_launches": (c_uint64, [c_void_p]),
        "mgv_ctx_set_tuning": (st, [c_void_p, POINTER(Tuning)]),
        "mgv_ctx_get_tuning": (st, [c_void_p, POINTER(Tuning)]),
        "mgv_pool_create": (st, [c_void_p, c_uint32, c_uint32, c_uint32, POINTER(c_void_p)]),
        "mgv_pool_destroy": (st, [c_void_p]),
        "mgv_buffer_acquire": (st, [c_void_p, c_uint32, POINTER(POINTER(Buffer))]),
        "mgv_buffer_release": (st, [c_void_p, POINTER(Buffer)]),
        "mgv_buffer_write": (st, [POINTER(Buffer), c_uint32, c_void_p, c_uint32, c_void_p]),
        "mgv_buffer_read": (st, [POINTER(Buffer), c_uint32, c_void_p, c_uint32, c_void_p]),
        "mgv_pool_register_producer": (st, [c_void_p]),
        "mgv_pool_unregister_producer": (st, [c_void_p]),
        "mgv_pool_stats_get": (st, [c_void_p, POINTER(PoolStats)]),
        "mgv_op_create_select": (st, [c_void_p, POINTER(SelectDesc), c_void_p, POINTER(c_void_p)]),
        "mgv_op_create_aggregate": (st, [c_void_p, POINTER(AggregateDesc), POINTER(c_void_p)]),
        "mgv_op_create_hash_build": (st, [c_void_p, POINTER(HashBuildDesc), POINTER(c_void_p)]),
        "mgv_op_create_hash_probe": (st, [c_void_p, POINTER(HashProbeDesc), c_void_p, POINTER(c_void_p)]),
        "mgv_op_create_sink": (st, [c_void_p, POINTER(SinkDesc), POINTER(c_void_p)]),
        "mgv_op_create_groupby": (st, [c_void_p, POINTER(GroupbyDesc), POINTER(c_void_p)]),
        "mgv_op_create_partition": (st, [c_void_p, POINTER(PartitionDesc), c_void_p, POINTER(c_void_p)]),
        "mgv_op_destroy": (st, [c_void_p]),
        "mgv_op_open": (st, [c_void_p, c_void_p]),
        "mgv_op_consume": (st, [c_void_p, POINTER(Buffer), c_void_p]),
        "mgv_op_consume_columns": (st, [c_void_p, POINTER(c_void_p), c_uint32, c_uint64, c_void_p]),
        "mgv_op_close": (st, [c_void_p, c_void_p]),
        "mgv_op_result": (st, [c_void_p, c_void_p, c_size_t, POINTER(c_size_t)]),
        "mgv_sink_read": (st, [c_void_p, c_uint32, c_void_p, c_uint64, POINTER(c_uint64)]),
        "mgv_sink_drain": (st, [c_void_p, c_void_p, c_uint32, c_uint64, POINTER(c_uint64), c_void_p]),
        "mgv_gen_uniform": (st, [c_void_p, c_void_p, c_uint64, c_uint64, c_uint32, c_int64, c_uint64, c_void_p]),
        "mgv_gen_perm": (st, [c_void_p, c_void_p, c_uint64, c_uint64, c_void_p]),
        "mgv_gen_probe_keys": (st, [c_void_p, c_void_p, c_uint64, c_uint64, c_uint64, c_uint64, c_uint32,
                                    c_int64, c_uint64, POINTER(c_uint64), c_void_p]),
        "mgv_batch_create": (st, [c_void_p, POINTER(QueryDesc), c_uint32, POINTER(BatchConfig), POINTER(c_void_p)]),
        "mgv_batch_run": (st, [c_void_p, c_void_p]),
        "mgv_batch_run_plain": (st, [c_void_p, c_void_p]),
        "mgv_batch_result": (st, [c_void_p, c_uint32, c_int, c_void_p, c_uint64, POINTER(c_uint64)]),
        "mgv_batch_stats_get": (st, [c_void_p, POINTER(BatchStats)]),
        "mgv_batch_destroy": (st, [c_void_p]),
        "mgv_batch_autotune": (st, [c_void_p, POINTER(QueryDesc), c_uint32, POINTER(BatchConfig)]),
        "mgv_server_create": (st, [c_void_p, POINTER(ServerConfig), POINTER(c_void_p)]),
        "mgv_server_add_table": (st, [c_void_p, c_void_p, c_void_p, c_uint64, POINTER(c_uint32)]),
        "mgv_server_submit": (st, [c_void_p, POINTER(ServerRequest), POINTER(c_uint64)]),
        "mgv_server_wait": (st, [c_void_p, c_uint64, c_uint32, c_void_p, c_uint64, POINTER(c_uint64),
                                 POINTER(c_double)]),
        "mgv_server_stats_get": (st, [c_void_p, POINTER(ServerStats)]),
        "mgv_server_reset_stats": (st, [c_void_p]),
        "mgv_server_destroy": (st, [c_void_p]),
        "mgv_hash_join_noalloc": (st, [c_int, c_void_p, c_void_p, c_uint64, c_void_p, c_void_p, c_uint64,
                                       c_void_p, c_void_p]),
        "mgv_diag_random_gather": (st, [c_void_p, c_uint64, c_uint64, c_uint32, c_uint32, POINTER(c_double)]),
        "mgv_pool_device_get": (st, [c_void_p, POINTER(PoolDevice)]),
        "mgv_partition_columns": (st, [c_void_p, POINTER(c_void_p), c_uint32, c_uint64, c_uint32, c_uint32, c_uint32,
                                       c_void_p, c_uint64, POINTER(c_uint64), c_void_p]),
        "mgv_op_consume_host": (st, [c_void_p, c_void_p, POINTER(c_void_p), c_uint32, c_uint64, c_void_p]),
        "mgv_diag_gather": (st, [c_void_p, POINTER(DiagGatherDesc), POINTER(c_double)]),
        "mgv_gen_zipf": (st, [c_void_p, c_void_p, c_uint64, c_uint64, c_uint32, c_uint32, c_double, c_void_p]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, where: str) -> None:
    if status != OK:
        detail = load().mgv_last_error_string().decode(errors="replace")
        raise MgvError(status, where, detail)


def _call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)


def _stream(stream) -> c_void_p:
    if stream is None:
        return c_void_p(0)
    if isinstance(stream, int):
        return c_void_p(stream)
    return c_void_p(stream.cuda_stream)  # torch.cuda.Stream


def _ptr(x) -> int:
    """Device address of a torch tensor or a raw integer pointer."""
    return x if isinstance(x, int) else x.data_ptr()


class Context:
    """mgv_ctx: one device, one stream, one device error word."""

    def __init__(self, device: int = 0):
        h = c_void_p()
        _call("mgv_ctx_create", device, byref(h))
        self.h = h
        self.device = device

    def info(self) -> CtxInfo:
        i = CtxInfo()
        _call("mgv_ctx_info_get", self.h, byref(i))
        return i

    def sync(self, stream=None) -> None:
        _call("mgv_ctx_sync", self.h, _stream(stream))

    def tuning(self) -> Tuning:
        t = Tuning()
        _call("mgv_ctx_get_tuning", self.h, byref(t))
        return t

    def set_tuning(self, **kw) -> Tuning:
        t = self.tuning()
        for k, v in kw.items():
            setattr(t, k, v)
        _call("mgv_ctx_set_tuning", self.h, byref(t))
        return t

    @property
    def launches(self) -> int:
        return int(load().mgv_ctx_launches(self.h))

    def close(self) -> None:
        if self.h:
            load().mgv_ctx_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def diag_random_gather(self, table_bytes: int, n: int, ctas_per_sm: int = 4, reps: int = 20) -> float:
        """Milliseconds per pass of n random 32-byte bucket reads."""
        ms = c_double()
        _call("mgv_diag_random_gather", self.h, table_bytes, n, ctas_per_sm, reps, byref(ms))
        return ms.value

    def diag_gather(self, table_bytes: int, lookups: int, line_bytes: int = 32, method: int = 0,
                    ctas_per_sm: int = 2, reps: int = 10, inflight: int = 4, lsu_warps: int = 8,
                    tma_warps: int = 1, tma_share: float = 0.0) -> float:
        """Milliseconds per pass of `lookups` random reads of line_bytes each
        (method 0 LSU, 1 TMA gather4, 2 both; include/mgv_diag.h)."""
        d = DiagGatherDesc(table_bytes, lookups, line_bytes, method, ctas_per_sm, reps, inflight, lsu_warps,
                           tma_warps, tma_share)
        ms = c_double()
        _call("mgv_diag_gather", self.h, byref(d), byref(ms))
        return ms.value

    def partition_columns(self, cols, rows: int, key_col: int, radix_bits: int, radix_shift: int, out,
                          out_stride: int, stream=None) -> list[int]:
        """mgv_partition_columns: rows of device columns written partition-major into
        `out` (column c at out + c * out_stride); returns the rows per partition."""
        arr = (c_void_p * max(1, len(cols)))(*[_ptr(c) for c in cols])
        counts = (c_uint64 * (1 << radix_bits))()
        _call("mgv_partition_columns", self.h, arr, len(cols), rows, key_col, radix_bits, radix_shift,
              c_void_p(_ptr(out)), out_stride, counts, _stream(stream))
        return list(counts)

    # seeded columns ---------------------------------------------------
    def gen_uniform(self, dst, n, seed, stream_id, lo, rng, stream=None):
        _call("mgv_gen_uniform", self.h, c_void_p(_ptr(dst)), n, seed, stream_id, lo, rng, _stream(stream))

    def gen_perm(self, dst, n, seed, stream=None):
        _call("mgv_gen_perm", self.h, c_void_p(_ptr(dst)), n, seed, _stream(stream))

    def gen_probe_keys(self, dst, n, seed, build_seed, nbuild, hit_num, miss_lo, miss_range, stream=None) -> int:
        hits = c_uint64()
        _call("mgv_gen_probe_keys", self.h, c_void_p(_ptr(dst)), n, seed, build_seed, nbuild, hit_num,
              miss_lo, miss_range, byref(hits), _stream(stream))
        return hits.value

    def gen_zipf(self, dst, n, seed, stream_id, groups, s=1.0, stream=None):
        _call("mgv_gen_zipf", self.h, c_void_p(_ptr(dst)), n, seed, stream_id, groups, s, _stream(stream))


class Pool:
    """mgv_pool: the device buffer pool (buffer_pool / buffer_manager)."""

    def __init__(self, ctx: Context, nbuffers: int, capacity: int, ncols: int):
        h = c_void_p()
        _call("mgv_pool_create", ctx.h, nbuffers, capacity, ncols, byref(h))
        self.h, self.ctx = h, ctx

    def acquire(self, timeout_us: int = 100000):
        b = POINTER(Buffer)()
        _call("mgv_buffer_acquire", self.h, timeout_us, byref(b))
        return b

    def try_acquire(self, timeout_us: int = 0):
        b = POINTER(Buffer)()
        st = load().mgv_buffer_acquire(self.h, timeout_us, byref(b))
        return st, (b if st == OK else None)

    def release(self, b) -> None:
        _call("mgv_buffer_release", self.h, b)

    def register_producer(self) -> None:
        _call("mgv_pool_register_producer", self.h)

    def unregister_producer(self) -> None:
        _call("mgv_pool_unregister_producer", self.h)

    def device_view(self) -> PoolDevice:
        """mgv_pool_device_get: the view a kernel takes for device-side
        acquire / release (include/mgv_device.cuh)."""
        v = PoolDevice()
        _call("mgv_pool_device_get", self.h, byref(v))
        return v

    def stats(self) -> PoolStats:
        s = PoolStats()
        _call("mgv_pool_stats_get", self.h, byref(s))
        return s

    def destroy(self) -> None:
        if self.h:
            load().mgv_pool_destroy(self.h)
            self.h = None


def buffer_write(b, col: int, src_ptr: int, rows: int, stream=None) -> None:
    _call("mgv_buffer_write", b, col, c_void_p(src_ptr), rows, _stream(stream))


def buffer_read(b, col: int, dst_ptr: int, rows: int, stream=None) -> None:
    _call("mgv_buffer_read", b, col, c_void_p(dst_ptr), rows, _stream(stream))


class Op:
    """mgv_op: one operator of a push chain (d_operator_t)."""

    def __init__(self, ctx: Context, h: c_void_p, kind: str, parent: "Op | None" = None):
        self.ctx, self.h, self.kind, self.parent = ctx, h, kind, parent

    # construction --------------------------------------------------------
    @classmethod
    def select(cls, ctx, col: int, bound: int, parent: "Op") -> "Op":
        h = c_void_p()
        _call("mgv_op_create_select", ctx.h, byref(SelectDesc(col, bound)), parent.h, byref(h))
        return cls(ctx, h, "select", parent)

    @classmethod
    def aggregate(cls, ctx, sum_col_a: int = -1, sum_col_b: int = -1) -> "Op":
        h = c_void_p()
        _call("mgv_op_create_aggregate", ctx.h, byref(AggregateDesc(sum_col_a, sum_col_b)), byref(h))
        return cls(ctx, h, "aggregate")

    @classmethod
    def hash_build(cls, ctx, key_col: int, payload_col: int, expected_rows: int, load_factor: float = 0.0,
                   radix_bits: int = 0, radix_shift: int = 0) -> "Op":
        h = c_void_p()
        d = HashBuildDesc(key_col, payload_col, expected_rows, load_factor, radix_bits, radix_shift, 0)
        _call("mgv_op_create_hash_build", ctx.h, byref(d), byref(h))
        return cls(ctx, h, "hash_build")

    @classmethod
    def hash_probe(cls, ctx, key_col: int, build: "Op", parent: "Op") -> "Op":
        h = c_void_p()
        _call("mgv_op_create_hash_probe", ctx.h, byref(HashProbeDesc(key_col, 0, build.h.value)), parent.h, byref(h))
        op = cls(ctx, h, "hash_probe", parent)
        op.build = build
        return op

    @classmethod
    def groupby(cls, ctx, group_col: int, value_col: int, max_groups: int) -> "Op":
        h = c_void_p()
        _call("mgv_op_create_groupby", ctx.h, byref(GroupbyDesc(group_col, value_col, max_groups, 0)), byref(h))
        return cls(ctx, h, "groupby")

    @classmethod
    def partition(cls, ctx, key_col: int, radix_bits: int, radix_shift: int, max_rows: int, parent: "Op") -> "Op":
        h = c_void_p()
        d = PartitionDesc(key_col, radix_bits, radix_shift, 0, max_rows)
        _call("mgv_op_create_partition", ctx.h, byref(d), parent.h, byref(h))
        op = cls(ctx, h, "partition", parent)
        op.radix_bits = radix_bits
        return op

    @classmethod
    def sink(cls, ctx, pool: Pool, max_buffers: int = 0) -> "Op":
        h = c_void_p()
        _call("mgv_op_create_sink", ctx.h, byref(SinkDesc(pool.h.value, max_buffers, 0)), byref(h))
        op = cls(ctx, h, "sink")
        op.pool = pool
        return op

    # lifecycle -------------------------------------------------------------
    def open(self, stream=None) -> None:
        _call("mgv_op_open", self.h, _stream(stream))

    def consume(self, buf, stream=None) -> None:
        _call("mgv_op_consume", self.h, buf, _stream(stream))

    def consume_columns(self, cols, rows: int, stream=None) -> None:
        arr = (c_void_p * max(1, len(cols)))(*[_ptr(c) for c in cols])
        _call("mgv_op_consume_columns", self.h, arr, len(cols), rows, _stream(stream))

    def consume_host(self, pool: "Pool", host_cols, rows: int, stream=None) -> None:
        """mgv_op_consume_host: rows of host columns (numpy arrays, pinned
        torch tensors or raw host addresses) pushed through the chain in
        slices of the pool's buffers, copies overlapped with the consumes."""
        ptrs = []
        for c in host_cols:
            if isinstance(c, int):
                ptrs.append(c)
            elif hasattr(c, "ctypes"):
                ptrs.append(c.ctypes.data)
            else:
                ptrs.append(c.data_ptr())
        arr = (c_void_p * max(1, len(ptrs)))(*ptrs)
        _call("mgv_op_consume_host", self.h, pool.h, arr, len(ptrs), rows, _stream(stream))

    def close(self, stream=None) -> None:
        _call("mgv_op_close", self.h, _stream(stream))

    def try_close(self, stream=None) -> int:
        return load().mgv_op_close(self.h, _stream(stream))

    def result(self):
        if self.kind == "aggregate":
            r = AggResult()
            _call("mgv_op_result", self.h, byref(r), ctypes.sizeof(r), None)
            return r.count, r.sum
        if self.kind == "hash_build":
            r = HashBuildInfo()
            _call("mgv_op_result", self.h, byref(r), ctypes.sizeof(r), None)
            return r
        if self.kind == "sink":
            r = c_uint64()
            _call("mgv_op_result", self.h, byref(r), ctypes.sizeof(r), None)
            return r.value
        if self.kind == "groupby":
            need = c_size_t()
            _call("mgv_op_result", self.h, None, 0, byref(need))
            n = need.value // ctypes.sizeof(GroupRow)
            arr = (GroupRow * max(1, n))()
            _call("mgv_op_result", self.h, arr, ctypes.sizeof(arr), None)
            return [(r.group, r.sum, r.count) for r in arr[:n]]
        if self.kind == "partition":
            arr = (c_uint64 * (1 << self.radix_bits))()
            _call("mgv_op_result", self.h, arr, ctypes.sizeof(arr), None)
            return list(arr)
        raise MgvError(EINVAL, "result", f"{self.kind} has no result")

    def sink_read(self, col: int, dst_ptr: int, max_rows: int) -> int:
        n = c_uint64()
        _call("mgv_sink_read", self.h, col, c_void_p(dst_ptr), max_rows, byref(n))
        return n.value

    def sink_drain(self, dsts=None, cap_rows: int = 0, stream=None) -> int:
        """mgv_sink_drain: move the rows gathered so far to dsts (one address or
        tensor per column) and return the pool buffers; dsts None = only count."""
        n = c_uint64()
        if dsts is None:
            _call("mgv_sink_drain", self.h, None, 0, 0, byref(n), _stream(stream))
        else:
            arr = (c_void_p * len(dsts))(*[_ptr(d) for d in dsts])
            _call("mgv_sink_drain", self.h, arr, len(dsts), cap_rows, byref(n), _stream(stream))
        return n.value

    def destroy(self) -> None:
        if self.h:
            load().mgv_op_destroy(self.h)
            self.h = None


def query_desc(build_keys, build_rows, probe_key, probe_filter, probe_group, probe_value, probe_rows,
               filter_bound, max_groups, build_payloads=None) -> QueryDesc:
    p = lambda x: None if x is None else _ptr(x)
    return QueryDesc(p(build_keys), p(build_payloads), build_rows, p(probe_key), p(probe_filter), p(probe_group),
                     p(probe_value), probe_rows, filter_bound, max_groups)


class Batch:
    """mgv_batch: many select -> join -> group-by queries run together."""

    def __init__(self, ctx: Context, queries, config: BatchConfig | None = None, keep=None):
        self.ctx = ctx
        self.keep = keep  # device tensors the descriptors point into
        arr = (QueryDesc * max(1, len(queries)))(*queries)
        self.nq = len(queries)
        h = c_void_p()
        _call("mgv_batch_create", ctx.h, arr, self.nq, byref(config) if config is not None else None, byref(h))
        self.h = h

    def run(self, stream=None) -> None:
        _call("mgv_batch_run", self.h, _stream(stream))

    def run_plain(self, stream=None) -> None:
        _call("mgv_batch_run_plain", self.h, _stream(stream))

    def result(self, q: int, plain: bool = False):
        n = c_uint64()
        _call("mgv_batch_result", self.h, q, int(plain), None, 0, byref(n))
        arr = (GroupRow * max(1, n.value))()
        _call("mgv_batch_result", self.h, q, int(plain), arr, n.value, byref(n))
        return [(r.group, r.sum, r.count) for r in arr[:n.value]]

    def stats(self) -> BatchStats:
        st = BatchStats()
        _call("mgv_batch_stats_get", self.h, byref(st))
        return st

    def destroy(self) -> None:
        if self.h:
            load().mgv_batch_destroy(self.h)
            self.h = None


def batch_autotune(ctx: Context, queries) -> BatchConfig:
    arr = (QueryDesc * max(1, len(queries)))(*queries)
    cfg = BatchConfig()
    _call("mgv_batch_autotune", ctx.h, arr, len(queries), byref(cfg))
    return cfg


class Server:
    """mgv_server: continuous batching over resident build tables."""

    def __init__(self, ctx: Context, memory_budget: int, max_batch: int = 0, max_inflight: int = 0,
                 load_factor: float = 0.0, plain: bool = False, batch_solo: bool = False,
                 separate_scans: bool = False):
        h = c_void_p()
        cfg = ServerConfig(memory_budget, max_batch, max_inflight, load_factor, int(plain), int(batch_solo),
                           int(separate_scans))
        _call("mgv_server_create", ctx.h, byref(cfg), byref(h))
        self.h, self.ctx = h, ctx

    def add_table(self, keys, rows: int, payloads=None) -> int:
        t = c_uint32()
        _call("mgv_server_add_table", self.h, c_void_p(_ptr(keys)),
              None if payloads is None else c_void_p(_ptr(payloads)), rows, byref(t))
        return t.value

    def submit(self, table: int, key, filt, group, value, rows: int, bound: int, max_groups: int) -> int:
        r = ServerRequest(table, 0, _ptr(key), _ptr(filt), _ptr(group), _ptr(value), rows, bound, max_groups)
        t = c_uint64()
        _call("mgv_server_submit", self.h, byref(r), byref(t))
        return t.value

    def try_submit(self, *args) -> tuple[int, int]:
        table, key, filt, group, value, rows, bound, max_groups = args
        r = ServerRequest(table, 0, _ptr(key), _ptr(filt), _ptr(group), _ptr(value), rows, bound, max_groups)
        t = c_uint64()
        st = load().mgv_server_submit(self.h, byref(r), byref(t))
        return st, t.value

    def wait(self, ticket: int, timeout_ms: int = 60000, max_rows: int = 1 << 20):
        """(status, rows sorted by group, latency_ms); the server returns groups unordered."""
        arr = (GroupRow * max_rows)()
        n = c_uint64()
        lat = c_double()
        st = load().mgv_server_wait(self.h, ticket, timeout_ms, arr, max_rows, byref(n), byref(lat))
        return st, sorted((r.group, r.sum, r.count) for r in arr[:min(n.value, max_rows)]), lat.value

    def stats(self) -> ServerStats:
        st = ServerStats()
        _call("mgv_server_stats_get", self.h, byref(st))
        return st

    def reset_stats(self) -> None:
        _call("mgv_server_reset_stats", self.h)

    def destroy(self) -> None:
        if self.h:
            load().mgv_server_destroy(self.h)
            self.h = None


NOALLOC_MAX_BUILD_ROWS = 1 << 20


def hash_join_noalloc(device: int, build_keys, build_pay, build_rows: int, probe_keys, probe_pay, probe_rows: int,
                      d_result, stream=None) -> None:
    """mgv_hash_join_noalloc: COUNT + SUM(bp + pp) into d_result[0..1] (device int64),
    using the library's fixed scratch table instead of allocating one."""
    p = lambda x: c_void_p(0 if x is None else _ptr(x))
    _call("mgv_hash_join_noalloc", device, p(build_keys), p(build_pay), build_rows, p(probe_keys), p(probe_pay),
          probe_rows, p(d_result), _stream(stream))


# ---- reference-style plans (src/main9.cu:202-367) ---------------------------

def create_sum_select_pipeline(ctx: Context, bound: int, filter_col: int = 0, sum_col: int = 0):
    """select(cols[filter_col] <= bound) -> aggregate(COUNT, SUM(cols[sum_col])).

    create_sum_select_pipeline (src/main9.cu:202-226) with the aggregate
    widened to COUNT + int64 SUM.  Returns (head, aggregate)."""
    agg = Op.aggregate(ctx, sum_col, -1)
    sel = Op.select(ctx, filter_col, bound, agg)
    return sel, agg


def create_join_groupby_pipeline(ctx: Context, build_rows: int, probe_max_groups: int, filter_bound: int,
                                 radix_bits: int = 8, load_factor: float = 0.0):
    """select -> hash join -> group-by with a radix-partitioned build.

    Build side columns: (key,); partitioned on `radix_bits` key bits (the
    reference's split / hash_exchange, src/main9.cu:104-148, reduced to one
    GPU) into a radix-laid-out table.  Probe side columns: (key, filter,
    group, value): select(filter <= filter_bound) -> hash_probe(key) ->
    group-by(group): int64 SUM(value), COUNT.  Returns
    (build_head, build, probe_head, groupby)."""
    hb = Op.hash_build(ctx, 0, -1, build_rows, load_factor, radix_bits, 0)
    part = Op.partition(ctx, 0, radix_bits, 0, max(build_rows, 1), hb) if radix_bits else hb
    gb = Op.groupby(ctx, 2, 3, probe_max_groups)
    probe = Op.hash_probe(ctx, 0, hb, gb)
    sel = Op.select(ctx, 1, filter_bound, probe)
    return part, hb, sel, gb


def create_count_join_1G_pipeline(ctx: Context, build_rows: int, load_factor: float = 0.0,
                                  build_filter_bound: int | None = None):
    """Hash join on one GPU (create_count_join_1G_pipeline, src/main9.cu:326-367).

    Build side columns: (key, payload); probe side columns: (key, payload).
    Returns (build_head, build, probe_head, aggregate) where the aggregate
    yields COUNT(matches) and SUM(build payload + probe payload).  With
    build_filter_bound the build side is select(key <= bound) -> build,
    as the reference's CPU join filters its build rows (src/main8.cu:87)."""
    hb = Op.hash_build(ctx, 0, 1, build_rows, load_factor)
    bhead = Op.select(ctx, 0, build_filter_bound, hb) if build_filter_bound is not None else hb
    agg = Op.aggregate(ctx, 1, 2)  # probe payload (col 1) + build payload (appended col 2)
    probe = Op.hash_probe(ctx, 0, hb, agg)
    return bhead, hb, probe, agg
