// capi.cu -- the extern "C" boundary (include/mgv.h): contexts, pools,
// buffers and the operator graph with open / consume / close.
//
// The operator graph mirrors d_operator_t (src/operators/operator.cuh:42-86,
// src/operators/operator.cu:114-159): operators hold a parent pointer, open()
// opens parents first, close() closes them after the operator's own flush.
// Unlike the reference, a consume() call does not dispatch per 128-row
// vector through a variant: the chain below the consuming operator is
// matched to one fused kernel (kernels.cu) and launched once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "device_common.cuh"
#include "mgv_internal.h"

using namespace mgv;

namespace mgv {

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

mgv_status fail(mgv_status s, const std::string& msg) {
    set_last_error(msg);
    return s;
}

mgv_status cuda_fail(cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    set_last_error(m);
    if (e == cudaErrorMemoryAllocation) return MGV_ENOMEM;
    return MGV_ECUDA;
}

}  // namespace mgv

static cudaStream_t pick_stream(Context* ctx, void* stream) {
    return stream ? (cudaStream_t)stream : ctx->stream;
}

// Maps a device error word to a status (and clears it on the device).
static mgv_status report_device_error(Context* ctx, const uint32_t* h, cudaStream_t s) {
    if (h[0] == 0) return MGV_OK;
    MGV_CUDA_TRY(cudaMemsetAsync(ctx->d_err, 0, 2 * sizeof(uint32_t), s));
    MGV_CUDA_TRY(cudaStreamSynchronize(s));
    char msg[128];
    std::snprintf(msg, sizeof(msg), "device error word %u (site %u)", h[0], h[1]);
    if (h[0] == MGV_ENOMEM) return fail(MGV_ENOMEM, std::string(msg) + ": table, pool or output full");
    if (h[0] == MGV_ETIMEDOUT) return fail(MGV_ETIMEDOUT, std::string(msg) + ": bounded wait ran out");
    return fail(MGV_EDEVICE, msg);
}

// Waits for `s`, then reports and clears the context's device error word.
static mgv_status check_device(Context* ctx, cudaStream_t s) {
    uint32_t w[2];
    {
        std::lock_guard<std::mutex> lk(ctx->mu);  // h_stage is shared by the context
        uint32_t* h = reinterpret_cast<uint32_t*>(ctx->h_stage);
        MGV_CUDA_TRY(cudaMemcpyAsync(h, ctx->d_err, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        MGV_CUDA_TRY(cudaStreamSynchronize(s));
        w[0] = h[0];
        w[1] = h[1];
    }
    return report_device_error(ctx, w, s);
}

static mgv_status consume_cols(Op* head, const int32_t* const* cols, uint32_t ncols, uint64_t n, cudaStream_t s);

namespace mgv {

// Group rows in ascending group order: an LSD radix sort on the biased key,
// three passes of 11 bits, a pass skipped when every key has the same digit
// (small group ids use one or two passes).  A comparison sort of 4096 rows
// took about 180 us on the host, longer than the query's own close.
void sort_group_rows(std::vector<mgv_group_row>& v) {
    const size_t n = v.size();
    if (n < 64) {
        std::sort(v.begin(), v.end(), [](const mgv_group_row& x, const mgv_group_row& y) { return x.group < y.group; });
        return;
    }
    auto digit = [](const mgv_group_row& r, int pass) { return (((uint32_t)r.group ^ 0x80000000u) >> (11 * pass)) & 2047u; };
    static thread_local std::vector<uint32_t> cnt;  // the three digit histograms, from one read
    cnt.assign(3 * 2048, 0u);
    for (size_t i = 0; i < n; ++i)
        for (int pass = 0; pass < 3; ++pass) ++cnt[2048 * pass + digit(v[i], pass)];
    std::unique_ptr<mgv_group_row[]> tmp(new mgv_group_row[n]);
    mgv_group_row* src = v.data();
    mgv_group_row* dst = tmp.get();
    for (int pass = 0; pass < 3; ++pass) {
        uint32_t* c = cnt.data() + 2048 * pass;
        if (c[digit(src[0], pass)] == n) continue;  // every key has this digit: the order stands
        uint32_t sum = 0;
        for (int d = 0; d < 2048; ++d) {
            const uint32_t x = c[d];
            c[d] = sum;
            sum += x;
        }
        for (size_t i = 0; i < n; ++i) dst[c[digit(src[i], pass)]++] = src[i];
        std::swap(src, dst);
    }
    if (src != v.data()) std::copy(src, src + n, v.data());
}

}  // namespace mgv

// A terminal group-by's close: its groups are packed on the device and come
// back with the error word in one copy to pinned memory and one
// synchronisation.  They are ordered by group when first read.
// Group rows read back together with the count at a group-by's close; a
// larger result costs one more copy (most results are smaller).
constexpr uint32_t kGroupRowsFirstCopy = 4096;

static mgv_status close_groupby(Op* o, cudaStream_t s) {
    Context* ctx = o->ctx;
    unsigned char* h = o->gb_land;
    MGV_CUDA_TRY(cudaMemsetAsync(o->gb_dev_count, 0, sizeof(uint32_t), s));
    MGV_CUDA_TRY(launch_group_pack(o->gtab, o->gb_dev_rows, o->gb_dev_count, s, ctx));
    MGV_CUDA_TRY(cudaMemcpyAsync(h, ctx->d_err, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    MGV_CUDA_TRY(cudaMemcpyAsync(h + 8, o->gb_dev_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    // the first rows come with the count; a larger result follows after it
    const uint32_t first = std::min<uint32_t>(o->gb_land_rows, kGroupRowsFirstCopy);
    MGV_CUDA_TRY(cudaMemcpyAsync(h + 16, o->gb_dev_rows, sizeof(mgv_group_row) * (size_t)first,
                                 cudaMemcpyDeviceToHost, s));
    MGV_CUDA_TRY(cudaStreamSynchronize(s));
    const uint32_t w[2] = {reinterpret_cast<uint32_t*>(h)[0], reinterpret_cast<uint32_t*>(h)[1]};
    mgv_status st = report_device_error(ctx, w, s);
    if (st != MGV_OK) return st;
    uint32_t n = 0;
    std::memcpy(&n, h + 8, sizeof(n));
    const mgv_group_row* rows = reinterpret_cast<const mgv_group_row*>(h + 16);
    o->gb_rows.assign(rows, rows + std::min(n, first));
    if (n > first) {  // the rest, through the landing zone while it holds them
        o->gb_rows.resize(n);
        const uint32_t land_more = std::min(n, o->gb_land_rows) - first;
        if (land_more) {
            MGV_CUDA_TRY(cudaMemcpyAsync(h + 16, o->gb_dev_rows + first, sizeof(mgv_group_row) * (size_t)land_more,
                                         cudaMemcpyDeviceToHost, s));
            MGV_CUDA_TRY(cudaStreamSynchronize(s));
            std::memcpy(o->gb_rows.data() + first, h + 16, sizeof(mgv_group_row) * (size_t)land_more);
        }
        if (n > o->gb_land_rows)
            MGV_CUDA_TRY(cudaMemcpy(o->gb_rows.data() + o->gb_land_rows, o->gb_dev_rows + o->gb_land_rows,
                                    sizeof(mgv_group_row) * (size_t)(n - o->gb_land_rows), cudaMemcpyDeviceToHost));
    }
    o->gb_sorted = false;  // ordered by group when first read (mgv_op_result)
    return MGV_OK;
}

// Waits for a sink's copy in flight and returns its buffers to the pool.
static mgv_status sink_finish_drain(Op* o) {
    if (!o->drain_done) return MGV_OK;
    MGV_CUDA_TRY(cudaEventSynchronize(o->drain_done));
    if (!o->drain_ids.empty()) {
        Pool* p = o->sink_pool;
        std::lock_guard<std::mutex> lk(p->mu);
        MGV_CUDA_TRY(pool_push_batch(p, o->drain_ids.data(), (uint32_t)o->drain_ids.size()));
        o->drain_ids.clear();
    }
    return MGV_OK;
}

extern "C" {

const char* mgv_status_string(mgv_status s) {
    switch (s) {
        case MGV_OK: return "ok";
        case MGV_EINVAL: return "invalid argument";
        case MGV_ENOMEM: return "out of memory / capacity";
        case MGV_ETIMEDOUT: return "timed out";
        case MGV_ECUDA: return "CUDA error";
        case MGV_EDEVICE: return "device error";
        case MGV_ESTATE: return "invalid state";
        case MGV_EDRAINED: return "pool drained";
        case MGV_EUNSUPPORTED: return "unsupported operator chain";
    }
    return "unknown status";
}

const char* mgv_last_error_string(void) { return g_last_error.c_str(); }

// ---- context ---------------------------------------------------------------

mgv_status mgv_ctx_create(int device, mgv_ctx** out) {
    if (!out) return fail(MGV_EINVAL, "out is NULL");
    *out = nullptr;
    int n = 0;
    MGV_CUDA_TRY(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(MGV_EINVAL, "no such device");
    MGV_CUDA_TRY(cudaSetDevice(device));
    mgv_ctx* c = new (std::nothrow) mgv_ctx();
    if (!c) return fail(MGV_ENOMEM, "host allocation");
    c->device = device;
    cudaError_t e = cudaGetDeviceProperties(&c->prop, device);
    // A blocking stream: work on it is ordered with the legacy default
    // stream, so callers that use the default stream need no extra sync.
    if (e == cudaSuccess) e = cudaStreamCreate(&c->stream);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_err, 2 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, 2 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMallocHost(&c->h_stage, 8 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        if (c->h_stage) cudaFreeHost(c->h_stage);
        if (c->d_err) cudaFree(c->d_err);
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return cuda_fail(e, "mgv_ctx_create");
    }
    *out = c;
    return MGV_OK;
}

mgv_status mgv_ctx_destroy(mgv_ctx* ctx) {
    if (!ctx) return MGV_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_err);
    cudaFreeHost(ctx->h_stage);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MGV_OK;
}

mgv_status mgv_ctx_info_get(mgv_ctx* ctx, mgv_ctx_info* out) {
    if (!ctx || !out) return fail(MGV_EINVAL, "NULL argument");
    std::memset(out, 0, sizeof(*out));
    out->device = ctx->device;
    out->sm_count = ctx->prop.multiProcessorCount;
    out->l2_bytes = (uint64_t)ctx->prop.l2CacheSize;
    out->hbm_bytes = (uint64_t)ctx->prop.totalGlobalMem;
    out->cc_major = ctx->prop.major;
    out->cc_minor = ctx->prop.minor;
    const size_t len = strnlen(ctx->prop.name, sizeof(out->name) - 1);  // truncated to the field
    std::memcpy(out->name, ctx->prop.name, len);
    out->name[len] = '\0';
    return MGV_OK;
}

mgv_status mgv_ctx_sync(mgv_ctx* ctx, void* stream) {
    if (!ctx) return fail(MGV_EINVAL, "ctx is NULL");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    return check_device(ctx, pick_stream(ctx, stream));
}

uint64_t mgv_ctx_launches(mgv_ctx* ctx) { return ctx ? ctx->launches.load() : 0; }

mgv_status mgv_ctx_set_tuning(mgv_ctx* ctx, const mgv_tuning* t) {
    if (!ctx || !t) return fail(MGV_EINVAL, "NULL argument");
    if (t->probe_kernel > 3) return fail(MGV_EINVAL, "probe_kernel must be 0, 1, 2 or 3");
    if (t->probe_rows_per_thread != 4 && t->probe_rows_per_thread != 8)
        return fail(MGV_EINVAL, "probe_rows_per_thread must be 4 or 8");
    if (t->probe_stages != 2 && t->probe_stages != 4 && t->probe_stages != 6)
        return fail(MGV_EINVAL, "probe_stages must be 2, 4 or 6");
    if (t->probe_ctas_per_sm > 32) return fail(MGV_EINVAL, "probe_ctas_per_sm out of range");
    if (!(t->default_load_factor > 0.0f && t->default_load_factor <= 0.95f))
        return fail(MGV_EINVAL, "default_load_factor must be in (0, 0.95]");
    const uint32_t gs = t->groupby_smem_slots;
    if (gs != 0 && (gs < 64 || gs > kMaxSmemGroups || (gs & (gs - 1)) != 0))
        return fail(MGV_EINVAL, "groupby_smem_slots must be 0 or a power of two in [64, 8192]");
    if (t->select_ctas_per_sm > 8) return fail(MGV_EINVAL, "select_ctas_per_sm must be 0..8");
    if (t->select_compact > 1) return fail(MGV_EINVAL, "select_compact must be 0 or 1");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->tuning = *t;
    return MGV_OK;
}

mgv_status mgv_ctx_get_tuning(mgv_ctx* ctx, mgv_tuning* t) {
    if (!ctx || !t) return fail(MGV_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    *t = ctx->tuning;
    return MGV_OK;
}

// ---- pool ------------------------------------------------------------------

mgv_status mgv_pool_create(mgv_ctx* ctx, uint32_t nbuffers, uint32_t capacity, uint32_t ncols,
                           mgv_pool** out) {
    if (!ctx || !out) return fail(MGV_EINVAL, "NULL argument");
    *out = nullptr;
    if (nbuffers == 0 || nbuffers >= kNil - 1) return fail(MGV_EINVAL, "nbuffers out of range");
    if (capacity == 0 || capacity % 128 != 0)
        return fail(MGV_EINVAL, "capacity must be a positive multiple of 128 rows");
    if (ncols == 0 || ncols > MGV_MAX_COLS) return fail(MGV_EINVAL, "ncols out of range");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    mgv_pool* p = new (std::nothrow) mgv_pool();
    if (!p) return fail(MGV_ENOMEM, "host allocation");
    p->ctx = ctx;
    p->nbuffers = nbuffers;
    p->capacity = capacity;
    p->ncols = ncols;
    const size_t slab_bytes = (size_t)nbuffers * ncols * capacity * sizeof(int32_t);
    cudaError_t e = cudaMalloc(&p->slab, slab_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&p->dev, sizeof(PoolDev) + sizeof(uint32_t) * nbuffers);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_ids, sizeof(uint32_t) * (nbuffers + 2));
    if (e == cudaSuccess) e = cudaMallocHost(&p->h_ids, sizeof(uint32_t) * (nbuffers + 2));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = pool_init_device(p);
    if (e != cudaSuccess) {
        if (p->slab) cudaFree(p->slab);
        if (p->dev) cudaFree(p->dev);
        if (p->d_ids) cudaFree(p->d_ids);
        if (p->h_ids) cudaFreeHost(p->h_ids);
        if (p->stream) cudaStreamDestroy(p->stream);
        delete p;
        return cuda_fail(e, "mgv_pool_create");
    }
    p->bufs.resize(nbuffers);
    p->held.assign(nbuffers, 0);
    for (uint32_t i = 0; i < nbuffers; ++i) {
        mgv_buffer& b = p->bufs[i];
        std::memset(&b, 0, sizeof(b));
        for (uint32_t c = 0; c < ncols; ++c) b.cols[c] = p->slab + ((size_t)i * ncols + c) * capacity;
        b.ncols = ncols;
        b.capacity = capacity;
        b.id = i;
        b.device = ctx->device;
    }
    *out = p;
    return MGV_OK;
}

mgv_status mgv_pool_destroy(mgv_pool* p) {
    if (!p) return MGV_OK;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->stream);
    cudaFree(p->slab);
    cudaFree(p->dev);
    cudaFree(p->d_ids);
    cudaFreeHost(p->h_ids);
    cudaStreamDestroy(p->stream);
    delete p;
    return MGV_OK;
}

mgv_status mgv_buffer_acquire(mgv_pool* p, uint32_t timeout_us, mgv_buffer** out) {
    if (!p || !out) return fail(MGV_EINVAL, "NULL argument");
    *out = nullptr;
    std::lock_guard<std::mutex> lk(p->mu);
    MGV_CUDA_TRY(cudaSetDevice(p->ctx->device));
    if (p->host_cache.empty()) {
        uint32_t got = 0;
        mgv_status st = MGV_OK;
        MGV_CUDA_TRY(pool_pop_batch(p, std::min<uint32_t>(8u, p->nbuffers), timeout_us, &got, &st));
        for (uint32_t i = 0; i < got; ++i) p->host_cache.push_back(p->h_ids[i]);
        if (got == 0) {
            if (st == MGV_EDRAINED) return fail(MGV_EDRAINED, "pool empty and no producer registered");
            return fail(MGV_ETIMEDOUT, "no buffer came back before the timeout");
        }
    }
    uint32_t id = p->host_cache.back();
    p->host_cache.pop_back();
    p->held[id] = 1;
    p->bufs[id].rows = 0;
    *out = &p->bufs[id];
    return MGV_OK;
}

mgv_status mgv_buffer_release(mgv_pool* p, mgv_buffer* b) {
    if (!p || !b) return fail(MGV_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(p->mu);
    if (b->id >= p->nbuffers || &p->bufs[b->id] != b) return fail(MGV_EINVAL, "buffer not from this pool");
    if (!p->held[b->id]) return fail(MGV_ESTATE, "buffer is not held");
    p->held[b->id] = 0;
    b->rows = 0;
    p->host_cache.push_back(b->id);
    if (p->host_cache.size() > 16) {
        MGV_CUDA_TRY(cudaSetDevice(p->ctx->device));
        const uint32_t n = 8;
        std::vector<uint32_t> ids(p->host_cache.end() - n, p->host_cache.end());
        p->host_cache.resize(p->host_cache.size() - n);
        MGV_CUDA_TRY(pool_push_batch(p, ids.data(), n));
    }
    return MGV_OK;
}

mgv_status mgv_buffer_write(mgv_buffer* b, uint32_t col, const void* src, uint32_t rows, void* stream) {
    if (!b || !src) return fail(MGV_EINVAL, "NULL argument");
    if (col >= b->ncols) return fail(MGV_EINVAL, "column out of range");
    if (rows > b->capacity) return fail(MGV_EINVAL, "rows exceed buffer capacity");
    MGV_CUDA_TRY(cudaSetDevice(b->device));
    if (rows) {
        if (stream)
            MGV_CUDA_TRY(cudaMemcpyAsync(b->cols[col], src, sizeof(int32_t) * rows, cudaMemcpyDefault,
                                         (cudaStream_t)stream));
        else  // blocking, as overwrite(blocking = true)
            MGV_CUDA_TRY(cudaMemcpy(b->cols[col], src, sizeof(int32_t) * rows, cudaMemcpyDefault));
    }
    b->rows = rows;
    return MGV_OK;
}

mgv_status mgv_buffer_read(const mgv_buffer* b, uint32_t col, void* dst, uint32_t rows, void* stream) {
    if (!b || !dst) return fail(MGV_EINVAL, "NULL argument");
    if (col >= b->ncols) return fail(MGV_EINVAL, "column out of range");
    if (rows > b->rows) return fail(MGV_EINVAL, "rows exceed the buffer's row count");
    MGV_CUDA_TRY(cudaSetDevice(b->device));
    if (rows) {
        if (stream) {
            MGV_CUDA_TRY(cudaMemcpyAsync(dst, b->cols[col], sizeof(int32_t) * rows, cudaMemcpyDefault,
                                         (cudaStream_t)stream));
            MGV_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
        } else {
            MGV_CUDA_TRY(cudaMemcpy(dst, b->cols[col], sizeof(int32_t) * rows, cudaMemcpyDefault));
        }
    }
    return MGV_OK;
}

mgv_status mgv_pool_register_producer(mgv_pool* p) {
    if (!p) return fail(MGV_EINVAL, "pool is NULL");
    std::lock_guard<std::mutex> lk(p->mu);
    MGV_CUDA_TRY(cudaSetDevice(p->ctx->device));
    MGV_CUDA_TRY(pool_add_producers(p, 1));
    p->producers++;
    return MGV_OK;
}

mgv_status mgv_pool_unregister_producer(mgv_pool* p) {
    if (!p) return fail(MGV_EINVAL, "pool is NULL");
    std::lock_guard<std::mutex> lk(p->mu);
    if (p->producers == 0) return fail(MGV_ESTATE, "no producer registered");
    MGV_CUDA_TRY(cudaSetDevice(p->ctx->device));
    MGV_CUDA_TRY(pool_add_producers(p, -1));
    p->producers--;
    return MGV_OK;
}

mgv_status mgv_pool_stats_get(mgv_pool* p, mgv_pool_stats* out) {
    if (!p || !out) return fail(MGV_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(p->mu);
    MGV_CUDA_TRY(cudaSetDevice(p->ctx->device));
    uint32_t avail = 0, prod = 0;
    MGV_CUDA_TRY(pool_read_counters(p, &avail, &prod));
    out->nbuffers = p->nbuffers;
    out->capacity = p->capacity;
    out->ncols = p->ncols;
    out->available = avail;
    out->host_cached = (uint32_t)p->host_cache.size();
    out->producers = prod;
    out->bytes = (uint64_t)p->nbuffers * p->ncols * p->capacity * sizeof(int32_t);
    return MGV_OK;
}

mgv_status mgv_pool_device_get(mgv_pool* p, mgv_pool_device* out) {
    if (!p || !out) return fail(MGV_EINVAL, "NULL argument");
    std::memset(out, 0, sizeof(*out));
    out->head = &p->dev->head;
    out->available = &p->dev->available;
    out->producers = &p->dev->producers;
    out->next = p->dev->next;
    out->slab = p->slab;
    out->nbuffers = p->nbuffers;
    out->capacity = p->capacity;
    out->ncols = p->ncols;
    return MGV_OK;
}

// ---- operators -------------------------------------------------------------

static mgv_op* new_op(Context* ctx, OpKind k) {
    mgv_op* o = new (std::nothrow) mgv_op();
    if (!o) return nullptr;
    o->kind = k;
    o->ctx = ctx;
    return o;
}

static mgv_status dev_alloc(Op* o, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "device allocation");
    o->allocs.push_back(*p);
    return MGV_OK;
}

mgv_status mgv_op_create_select(mgv_ctx* ctx, const mgv_select_desc* d, mgv_op* parent, mgv_op** out) {
    if (!ctx || !d || !out) return fail(MGV_EINVAL, "NULL argument");
    if (!parent) return fail(MGV_EINVAL, "select needs a parent");
    if (d->col >= MGV_MAX_COLS) return fail(MGV_EINVAL, "select column out of range");
    mgv_op* o = new_op(ctx, OpKind::Select);
    if (!o) return fail(MGV_ENOMEM, "host allocation");
    o->sel = *d;
    o->parent = parent;
    *out = o;
    return MGV_OK;
}

mgv_status mgv_op_create_aggregate(mgv_ctx* ctx, const mgv_aggregate_desc* d, mgv_op** out) {
    if (!ctx || !d || !out) return fail(MGV_EINVAL, "NULL argument");
    if (d->sum_col_a < -1 || d->sum_col_a > MGV_MAX_COLS || d->sum_col_b < -1 || d->sum_col_b > MGV_MAX_COLS)
        return fail(MGV_EINVAL, "sum column out of range");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    mgv_op* o = new_op(ctx, OpKind::Aggregate);
    if (!o) return fail(MGV_ENOMEM, "host allocation");
    o->agg = *d;
    mgv_status st = dev_alloc(o, (void**)&o->d_acc, 2 * sizeof(unsigned long long));
    if (st != MGV_OK) { delete o; return st; }
    cudaError_t e = cudaMallocHost(&o->h_res, 4 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        for (void* p : o->allocs) cudaFree(p);
        delete o;
        return cuda_fail(e, "mgv_op_create_aggregate");
    }
    *out = o;
    return MGV_OK;
}

mgv_status mgv_op_create_hash_build(mgv_ctx* ctx, const mgv_hash_build_desc* d, mgv_op** out) {
    if (!ctx || !d || !out) return fail(MGV_EINVAL, "NULL argument");
    if (d->key_col >= MGV_MAX_COLS || d->payload_col < -1 || d->payload_col >= MGV_MAX_COLS)
        return fail(MGV_EINVAL, "column out of range");
    float lf = d->load_factor == 0.0f ? ctx->tuning.default_load_factor : d->load_factor;
    if (!(lf > 0.0f && lf <= 0.95f)) return fail(MGV_EINVAL, "load_factor must be in (0, 0.95]");
    if (d->radix_bits > 12 || d->radix_shift > 31) return fail(MGV_EINVAL, "radix_bits <= 12, radix_shift <= 31");
    const uint64_t rows = d->expected_rows ? d->expected_rows : 1;
    const uint32_t parts = 1u << d->radix_bits;
    // a build side without payloads keeps keys only: 8 slots per 32-byte bucket
    const bool key_only = d->payload_col < 0;
    // buckets per region: the expected rows of one region at the load factor
    const double bpp = std::ceil((double)rows / parts / ((key_only ? 8.0 : 4.0) * lf));
    if (bpp * parts >= 4294967295.0) return fail(MGV_EINVAL, "expected_rows too large");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    mgv_op* o = new_op(ctx, OpKind::HashBuild);
    if (!o) return fail(MGV_ENOMEM, "host allocation");
    o->hb = *d;
    o->hb.load_factor = lf;
    TableView& t = o->table;
    t.bpp = (uint32_t)std::max(1.0, bpp);
    t.radix_shift = d->radix_shift;
    t.radix_mask = parts - 1;
    t.nbuckets = t.bpp * parts;
    t.key_only = key_only ? 1u : 0u;
    t.side_cap = rows;
    o->table_bytes = (size_t)t.nbuckets * 32;
    mgv_status st = dev_alloc(o, (void**)&t.slots, o->table_bytes);
    if (st == MGV_OK) st = dev_alloc(o, (void**)&t.meta, 4 * sizeof(unsigned long long));
    if (st == MGV_OK) st = dev_alloc(o, (void**)&t.side_pay, sizeof(int32_t) * t.side_cap);
    if (st == MGV_OK && cudaMallocHost(&o->h_res, 5 * sizeof(unsigned long long)) != cudaSuccess)
        st = fail(MGV_ENOMEM, "pinned host allocation");
    if (st != MGV_OK) {
        for (void* p : o->allocs) cudaFree(p);
        delete o;
        return st;
    }
    *out = o;
    return MGV_OK;
}

mgv_status mgv_op_create_hash_probe(mgv_ctx* ctx, const mgv_hash_probe_desc* d, mgv_op* parent,
                                    mgv_op** out) {
    if (!ctx || !d || !out) return fail(MGV_EINVAL, "NULL argument");
    if (!parent) return fail(MGV_EINVAL, "hash_probe needs a parent");
    if (!d->build || d->build->kind != OpKind::HashBuild) return fail(MGV_EINVAL, "build must be a hash_build operator");
    if (d->key_col >= MGV_MAX_COLS) return fail(MGV_EINVAL, "key column out of range");
    mgv_op* o = new_op(ctx, OpKind::HashProbe);
    if (!o) return fail(MGV_ENOMEM, "host allocation");
    o->hp = *d;
    o->parent = parent;
    *out = o;
    return MGV_OK;
}

mgv_status mgv_op_create_groupby(mgv_ctx* ctx, const mgv_groupby_desc* d, mgv_op** out) {
    if (!ctx || !d || !out) return fail(MGV_EINVAL, "NULL argument");
    if (d->group_col > MGV_MAX_COLS || d->value_col < -1 || d->value_col > MGV_MAX_COLS)
        return fail(MGV_EINVAL, "column out of range");
    if (d->max_groups == 0 || d->max_groups > (1u << 30)) return fail(MGV_EINVAL, "max_groups out of range");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    mgv_op* o = new_op(ctx, OpKind::Groupby);
    if (!o) return fail(MGV_ENOMEM, "host allocation");
    o->gb = *d;
    uint32_t cap = 1024;
    while (cap < 2u * d->max_groups) cap <<= 1;
    GroupTableView& g = o->gtab;
    g.cap = cap;
    mgv_status st = dev_alloc(o, (void**)&g.keys, sizeof(int32_t) * cap);
    if (st == MGV_OK) st = dev_alloc(o, (void**)&g.sums, sizeof(unsigned long long) * cap);
    if (st == MGV_OK) st = dev_alloc(o, (void**)&g.counts, sizeof(unsigned long long) * cap);
    if (st == MGV_OK) st = dev_alloc(o, (void**)&g.special, 2 * sizeof(unsigned long long));
    if (st == MGV_OK) st = dev_alloc(o, (void**)&o->gb_dev_rows, sizeof(mgv_group_row) * ((size_t)cap + 1));
    if (st == MGV_OK) st = dev_alloc(o, (void**)&o->gb_dev_count, sizeof(uint32_t));
    // pinned landing zone: results of up to 64 Ki groups come back with one synchronisation
    o->gb_land_rows = std::min<uint32_t>(cap + 1, 1u << 16);
    if (st == MGV_OK &&
        cudaMallocHost(&o->gb_land, 16 + sizeof(mgv_group_row) * (size_t)o->gb_land_rows) != cudaSuccess)
        st = fail(MGV_ENOMEM, "pinned host allocation");
    if (st != MGV_OK) {
        for (void* p : o->allocs) cudaFree(p);
        delete o;
        return st;
    }
    *out = o;
    return MGV_OK;
}

mgv_status mgv_op_create_partition(mgv_ctx* ctx, const mgv_partition_desc* d, mgv_op* parent, mgv_op** out) {
    if (!ctx || !d || !out) return fail(MGV_EINVAL, "NULL argument");
    if (!parent) return fail(MGV_EINVAL, "partition needs a parent");
    if (d->key_col >= MGV_MAX_COLS) return fail(MGV_EINVAL, "key column out of range");
    if (d->radix_bits < 1 || d->radix_bits > 12 || d->radix_shift > 31)
        return fail(MGV_EINVAL, "radix_bits must be in [1, 12], radix_shift <= 31");
    if (d->max_rows == 0) return fail(MGV_EINVAL, "max_rows must be > 0");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    mgv_op* o = new_op(ctx, OpKind::Partition);
    if (!o) return fail(MGV_ENOMEM, "host allocation");
    o->pt = *d;
    o->parent = parent;
    mgv_status st = dev_alloc(o, (void**)&o->pt_dev, sizeof(unsigned long long) << d->radix_bits);
    if (st == MGV_OK) st = dev_alloc(o, (void**)&o->pt_acc, sizeof(unsigned long long) * ((1ull << d->radix_bits) + 1));
    if (st == MGV_OK &&
        cudaMallocHost(&o->h_res, sizeof(unsigned long long) * ((1ull << d->radix_bits) + 2)) != cudaSuccess)
        st = fail(MGV_ENOMEM, "pinned host allocation");
    if (st != MGV_OK) {
        for (void* p : o->allocs) cudaFree(p);
        delete o;
        return st;
    }
    *out = o;
    return MGV_OK;
}

mgv_status mgv_op_create_sink(mgv_ctx* ctx, const mgv_sink_desc* d, mgv_op** out) {
    if (!ctx || !d || !out) return fail(MGV_EINVAL, "NULL argument");
    if (!d->pool) return fail(MGV_EINVAL, "sink needs a pool");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    mgv_op* o = new_op(ctx, OpKind::Sink);
    if (!o) return fail(MGV_ENOMEM, "host allocation");
    o->sk = *d;
    o->sink_pool = d->pool;
    uint32_t maxc = d->max_buffers ? std::min(d->max_buffers, d->pool->nbuffers) : d->pool->nbuffers;
    SinkView& s = o->sink;
    s.slab = d->pool->slab;
    s.max_chunks = maxc;
    s.capacity = d->pool->capacity;
    s.ncols = d->pool->ncols;
    s.pool_ncols = d->pool->ncols;
    s.pool = d->pool->dev;
    mgv_status st = dev_alloc(o, (void**)&s.cursor, sizeof(unsigned long long));
    if (st == MGV_OK) st = dev_alloc(o, (void**)&s.chain, sizeof(uint32_t) * maxc);
    if (st != MGV_OK) {
        for (void* p : o->allocs) cudaFree(p);
        delete o;
        return st;
    }
    *out = o;
    return MGV_OK;
}

static mgv_status sink_return_buffers(Op* o) {
    if (o->sink_chain.empty()) return MGV_OK;
    Pool* p = o->sink_pool;
    std::lock_guard<std::mutex> lk(p->mu);
    MGV_CUDA_TRY(pool_push_batch(p, o->sink_chain.data(), (uint32_t)o->sink_chain.size()));
    o->sink_chain.clear();
    return MGV_OK;
}

mgv_status mgv_op_destroy(mgv_op* o) {
    if (!o) return MGV_OK;
    cudaSetDevice(o->ctx->device);
    cudaStreamSynchronize(o->ctx->stream);
    if (o->kind == OpKind::Sink) {
        sink_finish_drain(o);
        sink_return_buffers(o);
        if (o->drain_done) cudaEventDestroy(o->drain_done);
        if (o->drain_stream) cudaStreamDestroy(o->drain_stream);
    }
    if (o->in_stream) {
        cudaStreamSynchronize(o->in_stream);
        cudaStreamDestroy(o->in_stream);
    }
    for (cudaEvent_t ev : o->in_copied)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : o->in_consumed)
        if (ev) cudaEventDestroy(ev);
    if (o->h_res) cudaFreeHost(o->h_res);
    if (o->rb_scratch) cudaFree(o->rb_scratch);
    if (o->gb_land) cudaFreeHost(o->gb_land);
    for (void* p : o->allocs) cudaFree(p);
    delete o;
    return MGV_OK;
}

// Resets one operator's device state (at_open).
static mgv_status op_reset(Op* o, cudaStream_t s) {
    switch (o->kind) {
        case OpKind::Aggregate:
            MGV_CUDA_TRY(cudaMemsetAsync(o->d_acc, 0, 2 * sizeof(unsigned long long), s));
            o->agg_result = mgv_agg_result{0, 0};
            break;
        case OpKind::HashBuild:
            // The table is cleared lazily: a first shared-memory build writes
            // every bucket itself; otherwise the first consume (or close) fills it.
            MGV_CUDA_TRY(cudaMemsetAsync(o->table.meta, 0, 4 * sizeof(unsigned long long), s));
            o->hb_fresh = true;
            o->unique = false;
            break;
        case OpKind::Sink: {
            mgv_status st = sink_return_buffers(o);
            if (st != MGV_OK) return st;
            MGV_CUDA_TRY(cudaMemsetAsync(o->sink.cursor, 0, sizeof(unsigned long long), s));
            MGV_CUDA_TRY(cudaMemsetAsync(o->sink.chain, 0xff, sizeof(uint32_t) * o->sink.max_chunks, s));
            o->sink_rows = 0;
            break;
        }
        case OpKind::HashProbe:
            if (o->hp.build->state != OpState::Closed)
                return fail(MGV_ESTATE, "hash_probe opened before its build side was closed");
            break;
        case OpKind::Groupby:
            MGV_CUDA_TRY(launch_fill_i32(o->gtab.keys, o->gtab.cap, kEmptyKey, s, o->ctx));
            MGV_CUDA_TRY(cudaMemsetAsync(o->gtab.sums, 0, sizeof(unsigned long long) * o->gtab.cap, s));
            MGV_CUDA_TRY(cudaMemsetAsync(o->gtab.counts, 0, sizeof(unsigned long long) * o->gtab.cap, s));
            MGV_CUDA_TRY(cudaMemsetAsync(o->gtab.special, 0, 2 * sizeof(unsigned long long), s));
            o->gb_rows.clear();
            break;
        case OpKind::Partition:
            o->pt_fill = 0;
            o->pt_runs = 0;
            o->pt_offered = 0;
            o->pt_filtered = false;
            o->pt_hist_valid = true;
            o->pt_hist.assign((size_t)1 << o->pt.radix_bits, 0);
            MGV_CUDA_TRY(cudaMemsetAsync(o->pt_acc, 0, sizeof(unsigned long long) * (o->pt_hist.size() + 1), s));
            break;
        default: break;
    }
    return MGV_OK;
}

mgv_status mgv_op_open(mgv_op* o, void* stream) {
    if (!o) return fail(MGV_EINVAL, "op is NULL");
    if (o->state == OpState::Open) return fail(MGV_ESTATE, "operator already open");
    MGV_CUDA_TRY(cudaSetDevice(o->ctx->device));
    cudaStream_t s = pick_stream(o->ctx, stream);
    if (o->parent) {  // before_open: parents first
        mgv_status st = mgv_op_open(static_cast<mgv_op*>(o->parent), stream);
        if (st != MGV_OK) return st;
    }
    mgv_status st = op_reset(o, s);
    if (st != MGV_OK) return st;
    o->state = OpState::Open;
    return MGV_OK;
}

// A closed build's counters (meta[0..3] of the table) into its info.
static void hash_build_info(Op* o, const unsigned long long* m) {
    mgv_hash_build_info& i = o->hb_info;
    i.rows = m[2] + m[0];
    i.nbuckets = o->table.nbuckets;
    i.table_bytes = o->table_bytes;
    i.reserved_key_rows = m[0];
    i.has_duplicates = (m[3] != 0 || m[0] > 1) ? 1u : 0u;
    o->unique = m[3] == 0;
}

// Reads back a terminal operator's result after its stream completed.
static mgv_status op_finish(Op* o, cudaStream_t s) {
    switch (o->kind) {
        case OpKind::Aggregate: {
            unsigned long long h[2];
            MGV_CUDA_TRY(cudaMemcpyAsync(h, o->d_acc, sizeof(h), cudaMemcpyDeviceToHost, s));
            MGV_CUDA_TRY(cudaStreamSynchronize(s));
            o->agg_result.count = (int64_t)h[0];
            o->agg_result.sum = (int64_t)h[1];
            break;
        }

        case OpKind::Groupby: break;  // read back by close_groupby()
        case OpKind::Sink: {
            unsigned long long rows = 0;
            MGV_CUDA_TRY(cudaMemcpyAsync(&rows, o->sink.cursor, sizeof(rows), cudaMemcpyDeviceToHost, s));
            std::vector<uint32_t> chain(o->sink.max_chunks);
            MGV_CUDA_TRY(cudaMemcpyAsync(chain.data(), o->sink.chain, sizeof(uint32_t) * chain.size(),
                                         cudaMemcpyDeviceToHost, s));
            MGV_CUDA_TRY(cudaStreamSynchronize(s));
            o->sink_rows = rows;
            o->sink_chain.clear();
            for (uint32_t id : chain)
                if (id < o->sink_pool->nbuffers) o->sink_chain.push_back(id);
            break;
        }
        default: break;
    }
    return MGV_OK;
}

mgv_status mgv_op_close(mgv_op* o, void* stream) {
    if (!o) return fail(MGV_EINVAL, "op is NULL");
    if (o->state != OpState::Open) return fail(MGV_ESTATE, "operator is not open");
    MGV_CUDA_TRY(cudaSetDevice(o->ctx->device));
    cudaStream_t s = pick_stream(o->ctx, stream);
    o->state = OpState::Closed;
    mgv_status st = MGV_OK;
    if (o->kind == OpKind::Sink) {  // a drain's copies in flight complete before close returns
        st = sink_finish_drain(o);
        if (st != MGV_OK) return st;
    }
    if (o->kind == OpKind::HashBuild && o->hb_fresh) {  // nothing was built: clear the table now
        MGV_CUDA_TRY(launch_fill_u64(o->table.slots, 4ull * o->table.nbuckets, kEmptySlot, s, o->ctx));
        o->hb_fresh = false;
    }
    if (!o->parent) {  // terminal: wait, check the device error word, read results
        if (o->kind == OpKind::Aggregate) {
            // one pinned landing zone, one synchronisation
            unsigned long long* h = o->h_res;
            MGV_CUDA_TRY(cudaMemcpyAsync(h, o->ctx->d_err, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            MGV_CUDA_TRY(cudaMemcpyAsync(h + 2, o->d_acc, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
            MGV_CUDA_TRY(cudaStreamSynchronize(s));
            const uint32_t w[2] = {reinterpret_cast<uint32_t*>(h)[0], reinterpret_cast<uint32_t*>(h)[1]};
            o->agg_result.count = (int64_t)h[2];
            o->agg_result.sum = (int64_t)h[3];
            return report_device_error(o->ctx, w, s);
        }
        if (o->kind == OpKind::Groupby) return close_groupby(o, s);
        if (o->kind == OpKind::HashBuild) {  // the error word and the table's counters: one copy, one wait
            unsigned long long* h = o->h_res;
            MGV_CUDA_TRY(cudaMemcpyAsync(h, o->ctx->d_err, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            MGV_CUDA_TRY(cudaMemcpyAsync(h + 1, o->table.meta, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                         s));
            MGV_CUDA_TRY(cudaStreamSynchronize(s));
            const uint32_t w[2] = {reinterpret_cast<uint32_t*>(h)[0], reinterpret_cast<uint32_t*>(h)[1]};
            st = report_device_error(o->ctx, w, s);
            if (st == MGV_OK) hash_build_info(o, h + 1);
            return st;
        }
        st = check_device(o->ctx, s);
        mgv_status st2 = op_finish(o, s);
        if (st == MGV_OK) st = st2;
        return st;
    }
    if (o->kind == OpKind::Partition) {
        // the device's totals (and any overflow of max_rows), then the stored
        // rows -- every consume's run partition-major -- go to the parent chain;
        // a hash build on the same radix bits scatters them by sorted warp tiles
        o->pt_close_stream = s;
        if (!o->pt_filtered && o->pt_offered <= o->pt.max_rows) {
            // every consumed row was stored: the replay needs nothing from the device, so
            // the totals are read only if asked for (mgv_op_result) and a device error is
            // reported by the parent's close, which waits for the stream
            o->pt_fill = o->pt_offered;
            o->pt_hist_valid = false;
        } else {
            unsigned long long* h = o->h_res;  // [error word, rows stored, rows per partition]: one copy, one wait
            MGV_CUDA_TRY(cudaMemcpyAsync(h, o->ctx->d_err, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            MGV_CUDA_TRY(cudaMemcpyAsync(h + 1, o->pt_acc, sizeof(unsigned long long) * (o->pt_hist.size() + 1),
                                         cudaMemcpyDeviceToHost, s));
            MGV_CUDA_TRY(cudaStreamSynchronize(s));
            const uint32_t w[2] = {reinterpret_cast<uint32_t*>(h)[0], reinterpret_cast<uint32_t*>(h)[1]};
            st = report_device_error(o->ctx, w, s);
            if (st == MGV_OK) {
                o->pt_fill = h[1];
                for (size_t p = 0; p < o->pt_hist.size(); ++p) o->pt_hist[p] = h[2 + p];
            }
        }
        if (st == MGV_OK && o->pt_fill) {
            Op* hb = o->parent;
            hb->hb_partitioned = hb->kind == OpKind::HashBuild && hb->hb.key_col == o->pt.key_col &&
                                 hb->table.radix_mask == (1u << o->pt.radix_bits) - 1u &&
                                 hb->table.radix_shift == o->pt.radix_shift;
            // one run: the partition ends left by its scatter locate each partition's rows
            hb->hb_part_ends = hb->hb_partitioned && o->pt_runs == 1 ? o->pt_dev : nullptr;
            const int32_t* cols[MGV_MAX_COLS];
            for (uint32_t c = 0; c < o->pt_ncols; ++c) cols[c] = o->pt_store + c * o->pt.max_rows;
            st = consume_cols(o->parent, cols, o->pt_ncols, o->pt_fill, s);
            hb->hb_partitioned = false;
            hb->hb_part_ends = nullptr;
        }
    }
    mgv_status st2 = mgv_op_close(static_cast<mgv_op*>(o->parent), stream);  // after_close
    return st != MGV_OK ? st : st2;
}

mgv_status mgv_op_result(mgv_op* o, void* out, size_t bytes, size_t* needed) {
    if (!o) return fail(MGV_EINVAL, "op is NULL");
    if (o->state != OpState::Closed) return fail(MGV_ESTATE, "operator is not closed");
    const void* src = nullptr;
    size_t n = 0;
    switch (o->kind) {
        case OpKind::Aggregate: src = &o->agg_result; n = sizeof(o->agg_result); break;
        case OpKind::HashBuild: src = &o->hb_info; n = sizeof(o->hb_info); break;
        case OpKind::Sink: src = &o->sink_rows; n = sizeof(o->sink_rows); break;
        case OpKind::Groupby:
            if (!o->gb_sorted) {
                sort_group_rows(o->gb_rows);
                o->gb_sorted = true;
            }
            src = o->gb_rows.data();
            n = o->gb_rows.size() * sizeof(mgv_group_row);
            break;
        case OpKind::Partition:
            if (!o->pt_hist_valid) {  // the rows per partition, read once after the close's stream
                MGV_CUDA_TRY(cudaSetDevice(o->ctx->device));
                unsigned long long* h = o->h_res;
                MGV_CUDA_TRY(cudaMemcpyAsync(h, o->pt_acc, sizeof(unsigned long long) * (o->pt_hist.size() + 1),
                                             cudaMemcpyDeviceToHost, o->pt_close_stream));
                MGV_CUDA_TRY(cudaStreamSynchronize(o->pt_close_stream));
                for (size_t p = 0; p < o->pt_hist.size(); ++p) o->pt_hist[p] = h[1 + p];
                o->pt_hist_valid = true;
            }
            src = o->pt_hist.data();
            n = o->pt_hist.size() * sizeof(uint64_t);
            break;
        default: return fail(MGV_EINVAL, "operator has no result");
    }
    if (needed) *needed = n;
    if (!out) return MGV_OK;
    if (bytes < n) return fail(MGV_EINVAL, "result buffer too small");
    std::memcpy(out, src, n);
    return MGV_OK;
}

mgv_status mgv_sink_read(mgv_op* o, uint32_t col, int32_t* dst, uint64_t max_rows, uint64_t* rows) {
    if (!o || !dst) return fail(MGV_EINVAL, "NULL argument");
    if (o->kind != OpKind::Sink) return fail(MGV_EINVAL, "not a sink");
    if (o->state != OpState::Closed) return fail(MGV_ESTATE, "sink is not closed");
    if (col >= o->sink.ncols) return fail(MGV_EINVAL, "column out of range");
    MGV_CUDA_TRY(cudaSetDevice(o->ctx->device));
    const uint64_t cap = o->sink.capacity;
    uint64_t total = std::min<uint64_t>(o->sink_rows, (uint64_t)o->sink_chain.size() * cap);
    total = std::min(total, max_rows);
    uint64_t done = 0;
    for (size_t c = 0; c < o->sink_chain.size() && done < total; ++c) {
        const uint64_t n = std::min<uint64_t>(cap, total - done);
        const int32_t* src = o->sink.slab + ((size_t)o->sink_chain[c] * o->sink.pool_ncols + col) * cap;
        MGV_CUDA_TRY(cudaMemcpyAsync(dst + done, src, n * sizeof(int32_t), cudaMemcpyDefault, o->ctx->stream));
        done += n;
    }
    MGV_CUDA_TRY(cudaStreamSynchronize(o->ctx->stream));
    if (rows) *rows = done;
    return MGV_OK;
}

mgv_status mgv_sink_drain(mgv_op* o, int32_t* const* dst_cols, uint32_t ncols, uint64_t cap_rows, uint64_t* rows,
                          void* stream) {
    if (!o || !rows) return fail(MGV_EINVAL, "NULL argument");
    if (o->kind != OpKind::Sink) return fail(MGV_EINVAL, "not a sink");
    if (o->state != OpState::Open) return fail(MGV_ESTATE, "sink is not open");
    if (dst_cols && (ncols == 0 || ncols > o->sink.pool_ncols)) return fail(MGV_EINVAL, "column count out of range");
    MGV_CUDA_TRY(cudaSetDevice(o->ctx->device));
    cudaStream_t s = pick_stream(o->ctx, stream);
    // the previous drain's copies complete first: its buffers go back to the pool
    mgv_status st = sink_finish_drain(o);
    if (st != MGV_OK) return st;
    st = check_device(o->ctx, s);  // waits for the consumes; a pool that ran dry is reported here
    if (st != MGV_OK) return st;
    unsigned long long gathered = 0;
    std::vector<uint32_t> chain(o->sink.max_chunks);
    MGV_CUDA_TRY(cudaMemcpyAsync(&gathered, o->sink.cursor, sizeof(gathered), cudaMemcpyDeviceToHost, s));
    MGV_CUDA_TRY(cudaMemcpyAsync(chain.data(), o->sink.chain, sizeof(uint32_t) * chain.size(), cudaMemcpyDeviceToHost,
                                 s));
    MGV_CUDA_TRY(cudaStreamSynchronize(s));
    const uint64_t cap = o->sink.capacity;
    const uint64_t chunks = (gathered + cap - 1) / cap;
    std::vector<uint32_t> ids;
    for (uint64_t c = 0; c < chunks && c < chain.size(); ++c) {
        if (chain[c] >= o->sink_pool->nbuffers) return fail(MGV_EDEVICE, "sink chunk without a buffer");
        ids.push_back(chain[c]);
    }
    *rows = gathered;
    if (!dst_cols) return MGV_OK;
    if (gathered > cap_rows) return fail(MGV_EINVAL, "more rows wait than the destination holds");
    if (!o->drain_stream) {
        MGV_CUDA_TRY(cudaStreamCreateWithFlags(&o->drain_stream, cudaStreamNonBlocking));
        MGV_CUDA_TRY(cudaEventCreateWithFlags(&o->drain_done, cudaEventDisableTiming));
    }
    // The copies run on the sink's own stream, so the next consume on `s`
    // overlaps them; its buffers stay out of the pool until they are done.
    MGV_CUDA_TRY(cudaEventRecord(o->drain_done, s));
    MGV_CUDA_TRY(cudaStreamWaitEvent(o->drain_stream, o->drain_done, 0));
    for (uint32_t col = 0; col < ncols; ++col) {
        uint64_t done = 0;
        for (size_t c = 0; c < ids.size(); ++c) {
            const uint64_t n = std::min<uint64_t>(cap, gathered - done);
            const int32_t* src = o->sink.slab + ((size_t)ids[c] * o->sink.pool_ncols + col) * cap;
            MGV_CUDA_TRY(cudaMemcpyAsync(dst_cols[col] + done, src, n * sizeof(int32_t), cudaMemcpyDefault,
                                         o->drain_stream));
            done += n;
        }
    }
    MGV_CUDA_TRY(cudaEventRecord(o->drain_done, o->drain_stream));
    o->drain_ids = ids;
    // the sink starts over
    MGV_CUDA_TRY(cudaMemsetAsync(o->sink.cursor, 0, sizeof(unsigned long long), s));
    MGV_CUDA_TRY(cudaMemsetAsync(o->sink.chain, 0xff, sizeof(uint32_t) * o->sink.max_chunks, s));
    return MGV_OK;
}

// ---- consume: match the chain to a fused kernel ---------------------------

static bool all_open(Op* o) {
    for (; o; o = o->parent)
        if (o->state != OpState::Open) return false;
    return true;
}

}  // extern "C"

// Partition consume: histogram, cursors and scatter into the op's store, all
// on the device (the totals are read back once, at close).
static mgv_status consume_partition(Op* part, Op* sel, const int32_t* const* cols, uint32_t ncols, uint64_t n,
                                    cudaStream_t s) {
    Context* ctx = part->ctx;
    const uint32_t P = 1u << part->pt.radix_bits;
    if (part->pt_store == nullptr) {
        part->pt_ncols = ncols;
        mgv_status st = dev_alloc(part, (void**)&part->pt_store, sizeof(int32_t) * ncols * part->pt.max_rows);
        if (st != MGV_OK) return st;
    }
    if (ncols != part->pt_ncols) return fail(MGV_EINVAL, "partition: every consume must carry the same columns");
    if (n == 0) return MGV_OK;
    part->pt_offered += n;
    part->pt_runs++;
    if (sel) part->pt_filtered = true;
    MGV_CUDA_TRY(cudaMemsetAsync(part->pt_dev, 0, sizeof(unsigned long long) * P, s));
    MGV_CUDA_TRY(launch_partition_hist(cols, n, sel != nullptr, sel ? sel->sel.col : 0, sel ? sel->sel.bound : 0,
                                       part->pt.key_col, part->pt.radix_shift, part->pt.radix_bits, part->pt_dev, s,
                                       ctx));
    MGV_CUDA_TRY(launch_partition_cursors(part->pt_dev, part->pt.radix_bits, part->pt_acc, part->pt.max_rows, s, ctx));
    MGV_CUDA_TRY(launch_partition_scatter(cols, ncols, n, sel != nullptr, sel ? sel->sel.col : 0,
                                          sel ? sel->sel.bound : 0, part->pt.key_col, part->pt.radix_shift,
                                          part->pt.radix_bits, part->pt_dev, part->pt_store, part->pt.max_rows, s,
                                          ctx));
    return MGV_OK;
}

static mgv_status consume_cols(Op* head, const int32_t* const* cols, uint32_t ncols, uint64_t n, cudaStream_t s) {
    Context* ctx = head->ctx;
    Op* sel = nullptr;
    Op* probe = nullptr;
    Op* o = head;
    if (o->kind == OpKind::Select) { sel = o; o = o->parent; }
    if (o && o->kind == OpKind::HashProbe) { probe = o; o = o->parent; }
    Op* term = o;
    if (!term || (term->parent && term->kind != OpKind::Partition))
        return fail(MGV_EUNSUPPORTED, "chain must be [select] [hash_probe] terminal");
    auto col_ok = [&](int32_t c) { return c >= 0 && (uint32_t)c < ncols; };
    // a column of the chain's rows: an input column, or the build payload (ncols)
    auto ref_ok = [&](int32_t c) { return c == -1 || col_ok(c) || (probe && (uint32_t)c == ncols); };
    if (sel && !col_ok((int32_t)sel->sel.col)) return fail(MGV_EINVAL, "select column not in input");
    if (probe && !col_ok((int32_t)probe->hp.key_col)) return fail(MGV_EINVAL, "probe key column not in input");

    ChainArgs a{};
    for (uint32_t c = 0; c < ncols; ++c) a.cols[c] = cols[c];
    a.ncols = ncols;
    a.n = n;
    a.has_sel = sel != nullptr;
    if (sel) { a.sel_col = sel->sel.col; a.sel_bound = sel->sel.bound; }
    a.has_probe = probe != nullptr;
    if (probe) {
        a.probe_col = probe->hp.key_col;
        a.table = probe->hp.build->table;
        a.unique = probe->hp.build->unique;
    }

    switch (term->kind) {
        case OpKind::Aggregate: {
            const int32_t ca = term->agg.sum_col_a, cb = term->agg.sum_col_b;
            if (!ref_ok(ca) || !ref_ok(cb)) return fail(MGV_EINVAL, "aggregate column not in input");
            if (n == 0) return MGV_OK;
            // select -> aggregate: the masked fold, unless the context asks
            // for the warp-ballot compaction of the chain kernel
            if (!probe && !(sel && ctx->tuning.select_compact)) {
                MGV_CUDA_TRY(launch_select_agg(sel ? cols[sel->sel.col] : nullptr, sel ? sel->sel.bound : 0,
                                               sel != nullptr, ca >= 0 ? cols[ca] : nullptr,
                                               cb >= 0 ? cols[cb] : nullptr, n, term->d_acc, s, ctx));
                return MGV_OK;
            }
            // probe -> aggregate without a select: the warp-specialised probe
            // (sums the build payload and at most one probe column)
            if (!sel && !(ca >= 0 && cb >= 0 && ca != (int32_t)ncols && cb != (int32_t)ncols)) {
                uint32_t mode = 0;
                const int32_t* pays = nullptr;
                for (int32_t c : {ca, cb}) {
                    if (c == -1) continue;
                    if ((uint32_t)c == ncols) mode |= 1u;
                    else { pays = cols[c]; mode |= 2u; }
                }
                Op* hb = probe->hp.build;
                MGV_CUDA_TRY(launch_probe_agg(cols[probe->hp.key_col], pays, n, hb->table, hb->unique, mode,
                                              term->d_acc, s, ctx));
                return MGV_OK;
            }
            a.term = kTermAgg;
            a.ref[0] = ca;
            a.ref[1] = cb;
            a.nref = 2;
            a.acc = term->d_acc;
            MGV_CUDA_TRY(launch_chain(a, s, ctx));
            return MGV_OK;
        }
        case OpKind::Groupby: {
            const int32_t g = (int32_t)term->gb.group_col, v = term->gb.value_col;
            if (!ref_ok(g) || g == -1 || !ref_ok(v)) return fail(MGV_EINVAL, "group-by column not in input");
            if (n == 0) return MGV_OK;
            a.term = kTermGroupby;
            a.ref[0] = g;
            a.ref[1] = v;
            a.nref = 2;
            a.gt = term->gtab;
            a.smem_groups = ctx->tuning.groupby_smem_slots;
            MGV_CUDA_TRY(launch_chain(a, s, ctx));
            return MGV_OK;
        }
        case OpKind::Sink: {
            if (n == 0) return MGV_OK;
            const uint32_t out_cols = std::min(ncols + (probe ? 1u : 0u), term->sink.pool_ncols);
            a.term = kTermSink;
            a.nref = out_cols;
            for (uint32_t c = 0; c < out_cols; ++c) a.ref[c] = (int32_t)c;
            a.sink = term->sink;
            a.sink.ncols = out_cols;
            MGV_CUDA_TRY(launch_chain(a, s, ctx));
            return MGV_OK;
        }
        case OpKind::HashBuild: {
            if (probe) return fail(MGV_EUNSUPPORTED, "hash_probe cannot feed hash_build");
            const int32_t kc = (int32_t)term->hb.key_col, pc = term->hb.payload_col;
            if (!col_ok(kc) || (pc != -1 && !col_ok(pc))) return fail(MGV_EINVAL, "build column not in input");
            if (n == 0) return MGV_OK;
            const int32_t* pays = pc >= 0 ? cols[pc] : nullptr;
            const int32_t* filt = sel ? cols[sel->sel.col] : nullptr;
            const int32_t bound = sel ? sel->sel.bound : 0;
            const uint32_t regions = table_regions(term->table);
            const bool fresh = term->hb_fresh;
            term->hb_fresh = false;
            if (n < kRegionBuildMinRows || n >= (1ull << 31) || regions > kMaxRegionsPerJob) {
                if (fresh)
                    MGV_CUDA_TRY(launch_fill_u64(term->table.slots, 4ull * term->table.nbuckets, kEmptySlot, s, ctx));
                MGV_CUDA_TRY(launch_build(cols[kc], pays, filt, bound, sel != nullptr, n, term->table, s, ctx));
                return MGV_OK;
            }
            // shared-memory build; its scratch is kept by the operator and grown on demand
            const size_t need = region_scratch_bytes(regions, n);
            if (term->rb_bytes < need) {
                if (term->rb_scratch) {
                    MGV_CUDA_TRY(cudaStreamSynchronize(s));
                    MGV_CUDA_TRY(cudaFree(term->rb_scratch));
                    term->rb_scratch = nullptr;
                    term->rb_bytes = 0;
                }
                MGV_CUDA_TRY(cudaMalloc(&term->rb_scratch, need));
                term->rb_bytes = need;
            }
            const RegionJob job{term->table, cols[kc], pays, filt, bound, 0, regions, 0};
            if (fresh && term->hb_part_ends && !sel && region_build_partitioned_fits(term->table)) {
                MGV_CUDA_TRY(launch_build_regions_partitioned(job, term->hb_part_ends, n,
                                                              carve_region_scratch(term->rb_scratch, regions, n), s,
                                                              ctx));
                return MGV_OK;
            }
            // items: two per SM, each worth zeroing and flushing its region histogram
            const uint64_t rows_per_item =
                std::max<uint64_t>({8ull * regions, 4096, n / (2ull * ctx->prop.multiProcessorCount) + 1});
            MGV_CUDA_TRY(launch_build_regions(nullptr, job, 1, nullptr, 0, n, rows_per_item, regions, regions,
                                              carve_region_scratch(term->rb_scratch, regions, n), fresh,
                                              term->hb_partitioned && !sel, s, ctx));
            return MGV_OK;
        }
        case OpKind::Partition: {
            if (probe) return fail(MGV_EUNSUPPORTED, "hash_probe cannot feed a partition");
            if (!col_ok((int32_t)term->pt.key_col)) return fail(MGV_EINVAL, "partition key column not in input");
            return consume_partition(term, sel, cols, ncols, n, s);
        }
        default: return fail(MGV_EUNSUPPORTED, "no kernel for this chain");
    }
}

extern "C" {

mgv_status mgv_op_consume_columns(mgv_op* o, const int32_t* const* cols, uint32_t ncols, uint64_t rows,
                                  void* stream) {
    if (!o || (!cols && ncols)) return fail(MGV_EINVAL, "NULL argument");
    if (ncols > MGV_MAX_COLS) return fail(MGV_EINVAL, "too many columns");
    if (!all_open(o)) return fail(MGV_ESTATE, "chain is not open");
    MGV_CUDA_TRY(cudaSetDevice(o->ctx->device));
    return consume_cols(o, cols, ncols, rows, pick_stream(o->ctx, stream));
}

mgv_status mgv_op_consume(mgv_op* o, const mgv_buffer* b, void* stream) {
    if (!o || !b) return fail(MGV_EINVAL, "NULL argument");
    if (b->rows > b->capacity) return fail(MGV_EINVAL, "buffer rows exceed capacity");
    return mgv_op_consume_columns(o, b->cols, b->ncols, b->rows, stream);
}

mgv_status mgv_partition_columns(mgv_ctx* ctx, const int32_t* const* cols, uint32_t ncols, uint64_t rows,
                                 uint32_t key_col, uint32_t radix_bits, uint32_t radix_shift, int32_t* out,
                                 uint64_t out_stride, uint64_t* counts, void* stream) {
    if (!ctx || !counts || (!cols && ncols) || (rows && !out)) return fail(MGV_EINVAL, "NULL argument");
    if (ncols == 0 || ncols > MGV_MAX_COLS || key_col >= ncols) return fail(MGV_EINVAL, "column out of range");
    if (radix_bits < 1 || radix_bits > 12 || radix_shift > 31) return fail(MGV_EINVAL, "radix bits out of range");
    if (out_stride < rows) return fail(MGV_EINVAL, "out_stride is smaller than rows");
    for (uint32_t c = 0; c < ncols; ++c)
        if (rows && !cols[c]) return fail(MGV_EINVAL, "column is NULL");
    const uint32_t P = 1u << radix_bits;
    std::memset(counts, 0, sizeof(uint64_t) * P);
    if (rows == 0) return MGV_OK;
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t s = pick_stream(ctx, stream);
    // scratch: [histogram -> cursors (P) | rows stored, rows per partition (1 + P)]
    unsigned long long* d = nullptr;
    MGV_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d), sizeof(unsigned long long) * (2 * P + 1), s));
    std::vector<unsigned long long> h(1 + P);
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof(unsigned long long) * (2 * P + 1), s);
    if (e == cudaSuccess)
        e = launch_partition_hist(cols, rows, false, 0, 0, key_col, radix_shift, radix_bits, d, s, ctx);
    if (e == cudaSuccess) e = launch_partition_cursors(d, radix_bits, d + P, out_stride, s, ctx);
    if (e == cudaSuccess)
        e = launch_partition_scatter(cols, ncols, rows, false, 0, 0, key_col, radix_shift, radix_bits, d, out,
                                     out_stride, s, ctx);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h.data(), d + P, sizeof(unsigned long long) * (1 + P), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d, s);
    if (e != cudaSuccess) return cuda_fail(e, "mgv_partition_columns");
    const mgv_status st = check_device(ctx, s);
    if (st != MGV_OK) return st;
    for (uint32_t p = 0; p < P; ++p) counts[p] = h[1 + p];
    return MGV_OK;
}

// Host ingest: slices of the host columns go through `depth` pool buffers;
// the copy stream fills buffer k % depth once its previous slice has been
// consumed, and the consume of slice k waits for its copy only.
mgv_status mgv_op_consume_host(mgv_op* o, mgv_pool* pool, const int32_t* const* host_cols, uint32_t ncols,
                               uint64_t rows, void* stream) {
    constexpr uint32_t kDepth = 3;
    if (!o || !pool || (!host_cols && ncols)) return fail(MGV_EINVAL, "NULL argument");
    if (ncols == 0 || ncols > MGV_MAX_COLS || ncols > pool->ncols)
        return fail(MGV_EINVAL, "column count must be 1..the pool's columns");
    if (pool->ctx->device != o->ctx->device) return fail(MGV_EINVAL, "pool and operator on different devices");
    if (!all_open(o)) return fail(MGV_ESTATE, "chain is not open");
    if (rows == 0) return MGV_OK;
    for (uint32_t c = 0; c < ncols; ++c)
        if (!host_cols[c]) return fail(MGV_EINVAL, "host column is NULL");
    MGV_CUDA_TRY(cudaSetDevice(o->ctx->device));
    cudaStream_t s = pick_stream(o->ctx, stream);
    if (!o->in_stream) {
        MGV_CUDA_TRY(cudaStreamCreateWithFlags(&o->in_stream, cudaStreamNonBlocking));
        o->in_copied.assign(kDepth, nullptr);
        o->in_consumed.assign(kDepth, nullptr);
        for (uint32_t i = 0; i < kDepth; ++i) {
            MGV_CUDA_TRY(cudaEventCreateWithFlags(&o->in_copied[i], cudaEventDisableTiming));
            MGV_CUDA_TRY(cudaEventCreateWithFlags(&o->in_consumed[i], cudaEventDisableTiming));
        }
    }
    const uint64_t cap = pool->capacity;
    const uint64_t slices = (rows + cap - 1) / cap;
    std::vector<mgv_buffer*> bufs;
    for (uint32_t i = 0; i < kDepth && i < slices; ++i) {
        mgv_buffer* b = nullptr;
        const mgv_status st = mgv_buffer_acquire(pool, bufs.empty() ? 1000000u : 0u, &b);
        if (st != MGV_OK) {
            if (bufs.empty()) return st;
            break;  // fewer buffers in flight
        }
        bufs.push_back(b);
    }
    const uint32_t depth = (uint32_t)bufs.size();
    mgv_status st = MGV_OK;
    // the copy stream starts after what `s` already holds (earlier consumes
    // may still read buffers that this call reuses)
    cudaError_t e = cudaEventRecord(o->in_consumed[0], s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(o->in_stream, o->in_consumed[0], 0);
    uint64_t k = 0;
    for (; k < slices && e == cudaSuccess && st == MGV_OK; ++k) {
        const uint32_t j = (uint32_t)(k % depth);
        mgv_buffer* b = bufs[j];
        const uint64_t lo = k * cap;
        const uint32_t m = (uint32_t)std::min<uint64_t>(cap, rows - lo);
        if (k >= depth) e = cudaStreamWaitEvent(o->in_stream, o->in_consumed[j], 0);
        for (uint32_t c = 0; c < ncols && e == cudaSuccess; ++c)
            e = cudaMemcpyAsync(b->cols[c], host_cols[c] + lo, sizeof(int32_t) * m, cudaMemcpyHostToDevice,
                                o->in_stream);
        if (e == cudaSuccess) e = cudaEventRecord(o->in_copied[j], o->in_stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, o->in_copied[j], 0);
        if (e != cudaSuccess) break;
        b->rows = m;
        st = consume_cols(o, b->cols, ncols, m, s);
        if (st == MGV_OK) e = cudaEventRecord(o->in_consumed[j], s);
    }
    // every slice consumed (or the failure reached) before the buffers go back
    const cudaError_t w = cudaStreamSynchronize(s);
    const cudaError_t w2 = cudaStreamSynchronize(o->in_stream);
    for (mgv_buffer* b : bufs) mgv_buffer_release(pool, b);
    if (st != MGV_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "mgv_op_consume_host");
    if (w != cudaSuccess) return cuda_fail(w, "mgv_op_consume_host: stream");
    if (w2 != cudaSuccess) return cuda_fail(w2, "mgv_op_consume_host: copy stream");
    return MGV_OK;
}

}  // extern "C"
