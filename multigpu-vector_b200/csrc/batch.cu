// batch.cu -- host side of batched query execution (kernels in chain.cu).
//
// A batch of select -> hash join -> group-by queries is planned once:
//   * one device arena holds every query's join table, metadata, side list,
//     group table, packed output region, and the descriptors and work-item
//     lists the kernels read;
//   * a run clears the group tables (one fill and memsets over contiguous
//     regions), builds every join table through shared memory (one set of
//     region-build launches for all queries, which also writes the empty
//     parts of the tables), launches one persistent probe kernel over
//     (query, rows) items in query order, packs the groups, and copies the
//     packed regions and their counts to pinned host memory;
//   * with use_graph the run is captured once and replayed as a CUDA graph,
//     so a run costs one graph launch and one synchronisation.
// The plain baseline runs the same queries one at a time through the
// operator API (hash_build, then select -> hash_probe -> groupby).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "device_common.cuh"
#include "mgv_internal.h"

using namespace mgv;

struct mgv_batch {
    mgv_ctx* ctx = nullptr;
    std::vector<mgv_query_desc> q;
    mgv_batch_config cfg{};
    // arena
    unsigned char* arena = nullptr;
    size_t arena_bytes = 0;
    // regions (device pointers into the arena)
    unsigned long long* tables = nullptr;
    uint64_t table_words = 0;  // u64 slots of all tables
    unsigned long long* metas = nullptr;
    int32_t* group_keys = nullptr;
    uint64_t group_slots = 0;
    unsigned char* group_zero = nullptr;  // sums, counts and specials (zeroed per run)
    size_t group_zero_bytes = 0;
    uint32_t* out_counts = nullptr;
    ChainDev* d_qs = nullptr;
    RegionJob* d_jobs = nullptr;  // one shared-memory build job per query
    RegionScratch rsc{};
    uint32_t total_regions = 0, max_job_regions = 0;
    uint32_t key_only = 0;  // every query's build side has no payloads: 8-key buckets
    BatchOut* d_outs = nullptr;
    BatchItem* d_build_items = nullptr;
    BatchItem* d_probe_items = nullptr;
    BatchItem* d_compact_items = nullptr;
    uint32_t n_build = 0, n_probe = 0, n_compact = 0;
    std::vector<uint64_t> out_offset;  // first packed row of each query
    // host landing zone: the packing kernel writes each query's rows straight into
    // it (pinned, mapped), so only the groups found cross to the host, not every
    // query's max_groups rows
    mgv_group_row* h_rows = nullptr;
    mgv_group_row* h_rows_dev = nullptr;  // the same memory as the device addresses it
    uint32_t* h_counts = nullptr;
    uint32_t* h_err = nullptr;
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaStream_t graph_stream = nullptr;
    bool warmed = false;
    double last_ms = 0.0;
    // plain baseline
    struct PlainQuery {
        mgv_op *hb = nullptr, *gb = nullptr, *probe = nullptr, *sel = nullptr;
        std::vector<mgv_group_row> rows;
    };
    std::vector<PlainQuery> plain;
};

namespace {

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

uint32_t group_cap(uint32_t max_groups) {
    uint32_t cap = 64;
    while (cap < 2u * max_groups) cap <<= 1;
    return cap;
}

void free_batch_device(mgv_batch* b) {
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->graph_stream) cudaStreamDestroy(b->graph_stream);
    if (b->arena) cudaFree(b->arena);
    if (b->h_rows) cudaFreeHost(b->h_rows);
    b->graph_exec = nullptr;
    b->graph = nullptr;
    b->graph_stream = nullptr;
    b->arena = nullptr;
    b->h_rows = nullptr;
}

// The body of one run, on stream s (also what the graph captures).
mgv_status enqueue_run(mgv_batch* b, cudaStream_t s) {
    Context* ctx = b->ctx;
    MGV_CUDA_TRY(cudaMemsetAsync(ctx->d_err, 0, 2 * sizeof(uint32_t), s));
    MGV_CUDA_TRY(cudaMemsetAsync(b->metas, 0, 4 * sizeof(unsigned long long) * b->q.size(), s));
    MGV_CUDA_TRY(launch_fill_i32(b->group_keys, b->group_slots, kEmptyKey, s, ctx));
    MGV_CUDA_TRY(cudaMemsetAsync(b->group_zero, 0, b->group_zero_bytes, s));
    MGV_CUDA_TRY(cudaMemsetAsync(b->out_counts, 0, sizeof(uint32_t) * b->q.size(), s));
    // every region of every table is written by the build (no clearing pass)
    RegionJob layout{};  // the jobs themselves are on the device; this carries their slot layout
    layout.t.key_only = b->key_only;
    MGV_CUDA_TRY(launch_build_regions(b->d_jobs, layout, (uint32_t)b->q.size(), b->d_build_items, b->n_build, 0, 0,
                                      b->total_regions, b->max_job_regions, b->rsc, true, false, s, ctx));
    MGV_CUDA_TRY(launch_batch(b->d_qs, b->d_outs, b->d_probe_items, b->n_probe, b->d_compact_items, b->n_compact,
                              (int)b->cfg.probe_ctas_per_sm, b->cfg.item_order, s, ctx));
    MGV_CUDA_TRY(cudaMemcpyAsync(b->h_counts, b->out_counts, sizeof(uint32_t) * b->q.size(), cudaMemcpyDeviceToHost, s));
    MGV_CUDA_TRY(cudaMemcpyAsync(b->h_err, ctx->d_err, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    return MGV_OK;
}

mgv_status check_run(mgv_batch* b) {
    if (b->h_err[0] == 0) return MGV_OK;
    const uint32_t code = b->h_err[0];
    cudaMemset(b->ctx->d_err, 0, 2 * sizeof(uint32_t));
    if (code == MGV_ENOMEM) return fail(MGV_ENOMEM, "batch: a table or result region is full (site " +
                                                        std::to_string(b->h_err[1]) + ")");
    if (code == MGV_ETIMEDOUT) return fail(MGV_ETIMEDOUT, "batch: a bounded wait ran out");
    return fail(MGV_EDEVICE, "batch: device error " + std::to_string(code));
}

void sort_rows(std::vector<mgv_group_row>& v) { sort_group_rows(v); }

}  // namespace

extern "C" {

mgv_status mgv_batch_create(mgv_ctx* ctx, const mgv_query_desc* qs, uint32_t nq, const mgv_batch_config* config,
                            mgv_batch** out) {
    if (!ctx || (!qs && nq) || !out) return fail(MGV_EINVAL, "NULL argument");
    *out = nullptr;
    mgv_batch_config cfg{};
    if (config) cfg = *config;
    else if (ctx->has_batch_tuned) cfg = ctx->batch_tuned;
    else cfg.use_graph = 1;
    if (cfg.load_factor == 0.0f) cfg.load_factor = ctx->tuning.default_load_factor;
    if (!(cfg.load_factor > 0.0f && cfg.load_factor <= 0.95f)) return fail(MGV_EINVAL, "load_factor out of range");
    if (cfg.build_item_rows == 0) cfg.build_item_rows = 65536;
    if (cfg.probe_item_rows == 0) cfg.probe_item_rows = 32768;
    if (cfg.probe_item_rows % 128) return fail(MGV_EINVAL, "probe_item_rows must be a multiple of 128");
    if (cfg.item_order > 1) return fail(MGV_EINVAL, "item_order must be 0 or 1");
    for (uint32_t i = 0; i < nq; ++i) {
        const mgv_query_desc& d = qs[i];
        if ((d.build_rows && !d.build_keys) ||
            (d.probe_rows && (!d.probe_key || !d.probe_filter || !d.probe_group || !d.probe_value)))
            return fail(MGV_EINVAL, "query " + std::to_string(i) + ": NULL column");
        if (d.max_groups == 0 || d.max_groups > (1u << 28)) return fail(MGV_EINVAL, "max_groups out of range");
    }
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    mgv_batch* b = new (std::nothrow) mgv_batch();
    if (!b) return fail(MGV_ENOMEM, "host allocation");
    b->ctx = ctx;
    b->q.assign(qs, qs + nq);
    b->cfg = cfg;

    // ---- plan the arena ----
    std::vector<uint32_t> nbk(nq), gcap(nq);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align256(off + bytes); return o; };
    std::vector<size_t> t_off(nq), side_off(nq), gk_off(nq), gs_off(nq), gc_off(nq), sp_off(nq);
    const size_t tables_begin = off;
    // one slot layout for the whole batch (one region-build launch builds every table)
    b->key_only = 1;
    for (uint32_t i = 0; i < nq; ++i)
        if (qs[i].build_payloads) b->key_only = 0;
    const double spb = b->key_only ? 8.0 : 4.0;  // slots per 32-byte bucket
    for (uint32_t i = 0; i < nq; ++i) {
        nbk[i] = (uint32_t)std::max(1.0, std::ceil((double)std::max<uint64_t>(qs[i].build_rows, 1) / (spb * cfg.load_factor)));
        t_off[i] = off;
        off += (size_t)nbk[i] * 32;  // tables packed back to back: one fill clears all
    }
    const size_t tables_end = off;
    off = align256(off);
    const size_t metas_off = take(4 * sizeof(unsigned long long) * std::max(nq, 1u));
    for (uint32_t i = 0; i < nq; ++i) side_off[i] = take(sizeof(int32_t) * std::max<uint64_t>(qs[i].build_rows, 1));
    const size_t gkeys_begin = off;
    uint64_t gslots = 0;
    for (uint32_t i = 0; i < nq; ++i) {
        gcap[i] = group_cap(qs[i].max_groups);
        gk_off[i] = off;
        off += sizeof(int32_t) * gcap[i];
        gslots += gcap[i];
    }
    off = align256(off);
    const size_t gzero_begin = off;
    for (uint32_t i = 0; i < nq; ++i) {
        gs_off[i] = off; off += 8ull * gcap[i];
        gc_off[i] = off; off += 8ull * gcap[i];
        sp_off[i] = off; off += 16;
    }
    const size_t gzero_end = off;
    off = align256(off);
    const size_t counts_off = take(sizeof(uint32_t) * std::max(nq, 1u));
    b->out_offset.resize(nq);
    uint64_t out_total = 0;
    for (uint32_t i = 0; i < nq; ++i) { b->out_offset[i] = out_total; out_total += qs[i].max_groups; }
    const size_t qs_off = take(sizeof(ChainDev) * std::max(nq, 1u));
    const size_t jobs_off = take(sizeof(RegionJob) * std::max(nq, 1u));
    std::vector<uint32_t> region0(nq);
    uint32_t total_regions = 0, max_job_regions = 1;
    uint64_t build_total = 0;
    for (uint32_t i = 0; i < nq; ++i) {
        const uint32_t r = (nbk[i] + kRegionBuckets - 1) / kRegionBuckets;
        if (r > kMaxRegionsPerJob) {
            delete b;
            return fail(MGV_EUNSUPPORTED, "query " + std::to_string(i) + ": build side too large for a batch");
        }
        region0[i] = total_regions;
        total_regions += r;
        max_job_regions = std::max(max_job_regions, r);
        build_total += qs[i].build_rows;
    }
    if (build_total >= (1ull << 31)) {
        delete b;
        return fail(MGV_EUNSUPPORTED, "a batch holds fewer than 2^31 build rows");
    }
    const size_t rsc_off = take(region_scratch_bytes(total_regions, build_total));
    const size_t outs_off = take(sizeof(BatchOut) * std::max(nq, 1u));
    // work items
    std::vector<BatchItem> bi, pi, ci;
    for (uint32_t i = 0; i < nq; ++i) {
        for (uint64_t lo = 0; lo < qs[i].build_rows; lo += cfg.build_item_rows)
            bi.push_back(BatchItem{i, 0, lo, std::min<uint64_t>(qs[i].build_rows, lo + cfg.build_item_rows)});
        for (uint64_t lo = 0; lo < qs[i].probe_rows; lo += cfg.probe_item_rows)
            pi.push_back(BatchItem{i, 0, lo, std::min<uint64_t>(qs[i].probe_rows, lo + cfg.probe_item_rows)});
        for (uint64_t lo = 0; lo <= gcap[i]; lo += 65536)
            ci.push_back(BatchItem{i, 0, lo, std::min<uint64_t>((uint64_t)gcap[i] + 1, lo + 65536)});
    }
    const size_t bi_off = take(sizeof(BatchItem) * std::max<size_t>(bi.size(), 1));
    const size_t pi_off = take(sizeof(BatchItem) * std::max<size_t>(pi.size(), 1));
    const size_t ci_off = take(sizeof(BatchItem) * std::max<size_t>(ci.size(), 1));
    b->arena_bytes = off;

    cudaError_t e = cudaMalloc(&b->arena, b->arena_bytes);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_rows, sizeof(mgv_group_row) * std::max<uint64_t>(out_total, 1) +
                                                            sizeof(uint32_t) * (nq + 4));
    if (e != cudaSuccess) {
        free_batch_device(b);
        delete b;
        return cuda_fail(e, "mgv_batch_create");
    }
    e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&b->h_rows_dev), b->h_rows, 0);
    if (e != cudaSuccess) {
        free_batch_device(b);
        delete b;
        return cuda_fail(e, "mgv_batch_create: mapped landing zone");
    }
    b->h_counts = reinterpret_cast<uint32_t*>(b->h_rows + std::max<uint64_t>(out_total, 1));
    b->h_err = b->h_counts + nq;
    unsigned char* A = b->arena;
    b->tables = reinterpret_cast<unsigned long long*>(A + tables_begin);
    b->table_words = (tables_end - tables_begin) / 8;
    b->metas = reinterpret_cast<unsigned long long*>(A + metas_off);
    b->group_keys = reinterpret_cast<int32_t*>(A + gkeys_begin);
    b->group_slots = gslots;
    b->group_zero = A + gzero_begin;
    b->group_zero_bytes = gzero_end - gzero_begin;
    b->out_counts = reinterpret_cast<uint32_t*>(A + counts_off);
    b->d_qs = reinterpret_cast<ChainDev*>(A + qs_off);
    b->d_jobs = reinterpret_cast<RegionJob*>(A + jobs_off);
    b->rsc = carve_region_scratch(A + rsc_off, total_regions, build_total);
    b->total_regions = total_regions;
    b->max_job_regions = max_job_regions;
    b->d_outs = reinterpret_cast<BatchOut*>(A + outs_off);
    b->d_build_items = reinterpret_cast<BatchItem*>(A + bi_off);
    b->d_probe_items = reinterpret_cast<BatchItem*>(A + pi_off);
    b->d_compact_items = reinterpret_cast<BatchItem*>(A + ci_off);
    b->n_build = (uint32_t)bi.size();
    b->n_probe = (uint32_t)pi.size();
    b->n_compact = (uint32_t)ci.size();

    // ---- descriptors ----
    std::vector<ChainDev> hq(nq);
    std::vector<RegionJob> hj(nq);
    std::vector<BatchOut> ho(nq);
    for (uint32_t i = 0; i < nq; ++i) {
        TableView t{};
        t.slots = reinterpret_cast<unsigned long long*>(A + t_off[i]);
        t.nbuckets = nbk[i];
        t.bpp = nbk[i];
        t.key_only = b->key_only;
        t.meta = b->metas + 4ull * i;
        t.side_pay = reinterpret_cast<int32_t*>(A + side_off[i]);
        t.side_cap = std::max<uint64_t>(qs[i].build_rows, 1);
        GroupTableView g{};
        g.keys = reinterpret_cast<int32_t*>(A + gk_off[i]);
        g.sums = reinterpret_cast<unsigned long long*>(A + gs_off[i]);
        g.counts = reinterpret_cast<unsigned long long*>(A + gc_off[i]);
        g.special = reinterpret_cast<unsigned long long*>(A + sp_off[i]);
        g.cap = gcap[i];
        ChainDev& c = hq[i];
        c = ChainDev{};
        c.cols[0] = qs[i].probe_key;
        c.cols[1] = qs[i].probe_filter;
        c.cols[2] = qs[i].probe_group;
        c.cols[3] = qs[i].probe_value;
        c.n = qs[i].probe_rows;
        c.ncols = 4;
        c.nslots = 3;  // key, group, value
        c.slot_src[0] = 0;
        c.slot_src[1] = 2;
        c.slot_src[2] = 3;
        c.sel_col = 1;
        c.sel_bound = qs[i].filter_bound;
        c.probe_slot = 0;
        c.table = t;
        c.ref[0] = 1;  // group
        c.ref[1] = 2;  // value
        c.nref = 2;
        c.gt = g;
        c.smem_groups = std::min(gcap[i], kMaxSmemGroups);
        hj[i] = RegionJob{t, qs[i].build_keys, qs[i].build_payloads, nullptr, 0, region0[i],
                          (nbk[i] + kRegionBuckets - 1) / kRegionBuckets, 0};
        ho[i] = BatchOut{g, b->h_rows_dev + b->out_offset[i], b->out_counts + i, qs[i].max_groups, 0};
    }
    e = cudaMemcpy(b->d_qs, hq.data(), sizeof(ChainDev) * nq, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_jobs, hj.data(), sizeof(RegionJob) * nq, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_outs, ho.data(), sizeof(BatchOut) * nq, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !bi.empty())
        e = cudaMemcpy(b->d_build_items, bi.data(), sizeof(BatchItem) * bi.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !pi.empty())
        e = cudaMemcpy(b->d_probe_items, pi.data(), sizeof(BatchItem) * pi.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !ci.empty())
        e = cudaMemcpy(b->d_compact_items, ci.data(), sizeof(BatchItem) * ci.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        free_batch_device(b);
        delete b;
        return cuda_fail(e, "mgv_batch_create");
    }
    *out = b;
    return MGV_OK;
}

mgv_status mgv_batch_run(mgv_batch* b, void* stream) {
    if (!b) return fail(MGV_EINVAL, "batch is NULL");
    Context* ctx = b->ctx;
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    const auto t0 = std::chrono::steady_clock::now();
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    if (!b->cfg.use_graph || !b->warmed) {
        // the first run goes straight to the stream (it also sets kernel
        // attributes that must not be set during a capture)
        mgv_status st = enqueue_run(b, s);
        if (st != MGV_OK) return st;
        MGV_CUDA_TRY(cudaStreamSynchronize(s));
        b->warmed = true;
    } else {
        if (!b->graph_exec) {
            MGV_CUDA_TRY(cudaStreamCreateWithFlags(&b->graph_stream, cudaStreamNonBlocking));
            MGV_CUDA_TRY(cudaStreamBeginCapture(b->graph_stream, cudaStreamCaptureModeThreadLocal));
            mgv_status st = enqueue_run(b, b->graph_stream);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(b->graph_stream, &g);
            if (st != MGV_OK) { if (g) cudaGraphDestroy(g); return st; }
            MGV_CUDA_TRY(e);
            b->graph = g;
            MGV_CUDA_TRY(cudaGraphInstantiate(&b->graph_exec, b->graph, 0));
        }
        MGV_CUDA_TRY(cudaGraphLaunch(b->graph_exec, s));
        MGV_CUDA_TRY(cudaStreamSynchronize(s));
    }
    b->last_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return check_run(b);
}

mgv_status mgv_batch_run_plain(mgv_batch* b, void* stream) {
    if (!b) return fail(MGV_EINVAL, "batch is NULL");
    mgv_ctx* ctx = b->ctx;
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    const uint32_t nq = (uint32_t)b->q.size();
    if (b->plain.empty()) {  // operators are created once, outside the timed runs
        b->plain.resize(nq);
        for (uint32_t i = 0; i < nq; ++i) {
            const mgv_query_desc& d = b->q[i];
            auto& p = b->plain[i];
            mgv_hash_build_desc hd{0, d.build_payloads ? 1 : -1, std::max<uint64_t>(d.build_rows, 1),
                                   b->cfg.load_factor, 0, 0, 0};
            mgv_groupby_desc gd{2, 3, d.max_groups, 0};
            mgv_status st = mgv_op_create_hash_build(ctx, &hd, &p.hb);
            if (st == MGV_OK) st = mgv_op_create_groupby(ctx, &gd, &p.gb);
            mgv_hash_probe_desc pd{0, 0, p.hb};
            if (st == MGV_OK) st = mgv_op_create_hash_probe(ctx, &pd, p.gb, &p.probe);
            mgv_select_desc sd{1, d.filter_bound};
            if (st == MGV_OK) st = mgv_op_create_select(ctx, &sd, p.probe, &p.sel);
            if (st != MGV_OK) return st;
        }
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (uint32_t i = 0; i < nq; ++i) {
        const mgv_query_desc& d = b->q[i];
        auto& p = b->plain[i];
        const int32_t* bcols[2] = {d.build_keys, d.build_payloads};
        mgv_status st = mgv_op_open(p.hb, stream);
        if (st == MGV_OK) st = mgv_op_consume_columns(p.hb, bcols, d.build_payloads ? 2 : 1, d.build_rows, stream);
        if (st == MGV_OK) st = mgv_op_close(p.hb, stream);
        const int32_t* pcols[4] = {d.probe_key, d.probe_filter, d.probe_group, d.probe_value};
        if (st == MGV_OK) st = mgv_op_open(p.sel, stream);
        if (st == MGV_OK) st = mgv_op_consume_columns(p.sel, pcols, 4, d.probe_rows, stream);
        if (st == MGV_OK) st = mgv_op_close(p.sel, stream);
        if (st != MGV_OK) return st;
    }
    b->last_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    // kept as closed (unordered); ordered when read, as the batch's own rows
    for (uint32_t i = 0; i < nq; ++i) b->plain[i].rows = static_cast<Op*>(b->plain[i].gb)->gb_rows;
    return MGV_OK;
}

mgv_status mgv_batch_result(mgv_batch* b, uint32_t q, int plain, mgv_group_row* out, uint64_t cap, uint64_t* rows) {
    if (!b) return fail(MGV_EINVAL, "batch is NULL");
    if (q >= b->q.size()) return fail(MGV_EINVAL, "no such query");
    std::vector<mgv_group_row> v;
    if (plain) {
        if (b->plain.empty()) return fail(MGV_ESTATE, "the plain pipeline has not run");
        v = b->plain[q].rows;
        sort_rows(v);
    } else {
        if (!b->warmed) return fail(MGV_ESTATE, "the batch has not run");
        const uint32_t n = std::min<uint32_t>(b->h_counts[q], b->q[q].max_groups);
        v.assign(b->h_rows + b->out_offset[q], b->h_rows + b->out_offset[q] + n);
        sort_rows(v);
    }
    if (rows) *rows = v.size();
    if (out) std::memcpy(out, v.data(), sizeof(mgv_group_row) * std::min<uint64_t>(cap, v.size()));
    return MGV_OK;
}

mgv_status mgv_batch_stats_get(mgv_batch* b, mgv_batch_stats* out) {
    if (!b || !out) return fail(MGV_EINVAL, "NULL argument");
    out->arena_bytes = b->arena_bytes;
    out->queries = (uint32_t)b->q.size();
    out->build_items = b->n_build;
    out->probe_items = b->n_probe;
    out->graph = b->graph_exec ? 1u : 0u;
    out->last_run_ms = b->last_ms;
    return MGV_OK;
}

mgv_status mgv_batch_destroy(mgv_batch* b) {
    if (!b) return MGV_OK;
    cudaSetDevice(b->ctx->device);
    cudaDeviceSynchronize();
    for (auto& p : b->plain) {
        mgv_op_destroy(p.sel);
        mgv_op_destroy(p.probe);
        mgv_op_destroy(p.gb);
        mgv_op_destroy(p.hb);
    }
    free_batch_device(b);
    delete b;
    return MGV_OK;
}

mgv_status mgv_batch_autotune(mgv_ctx* ctx, const mgv_query_desc* qs, uint32_t nq, mgv_batch_config* out) {
    if (!ctx || (!qs && nq) || !out) return fail(MGV_EINVAL, "NULL argument");
    const float lfs[] = {0.4f, 0.5f, 0.6f, 0.7f, 0.8f};  // key-only tables (8 slots per bucket) take the higher ones
    const uint32_t items[] = {8192, 32768, 131072};
    const uint32_t orders[] = {0, 1};
    double best = 1e30;
    mgv_batch_config best_cfg{};
    for (float lf : lfs)
        for (uint32_t it : items)
            for (uint32_t order : orders) {
                mgv_batch_config cfg{};
                cfg.load_factor = lf;
                cfg.build_item_rows = 65536;
                cfg.probe_item_rows = it;
                cfg.probe_ctas_per_sm = 0;
                cfg.use_graph = 1;
                cfg.item_order = order;
                mgv_batch* b = nullptr;
                mgv_status st = mgv_batch_create(ctx, qs, nq, &cfg, &b);
                if (st != MGV_OK) return st;
                double t = 1e30;
                for (int r = 0; r < 3 && st == MGV_OK; ++r) {  // warm-up, capture, replay
                    st = mgv_batch_run(b, nullptr);
                    if (r > 0) t = std::min(t, b->last_ms);
                }
                mgv_batch_destroy(b);
                if (st != MGV_OK) return st;
                if (t < best) {
                    best = t;
                    best_cfg = cfg;
                }
            }
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->batch_tuned = best_cfg;
    ctx->has_batch_tuned = true;
    *out = best_cfg;
    return MGV_OK;
}

}  // extern "C"
