// serve.cu -- a query server with continuous batching.
//
// Build tables are registered once and stay resident.  Clients submit
// select -> join -> group-by requests against them at any time; a scheduler
// thread admits pending requests in arrival order while the device memory
// budget allows (group table + packed result region per request), launches
// them as one batch (one persistent probe kernel over (query, rows) items,
// then the result packing and one copy to pinned host memory) on a free
// stream, and keeps up to max_inflight batches on the GPU at once, so
// requests that arrive while others run are admitted as soon as a stream
// and memory free up and their work overlaps on the device.  Completion is
// observed through CUDA events; latency runs from submit to the moment the
// scheduler sees the batch's results on the host.  The results stay in the
// batch's pinned landing zone until each waiter copies its own rows out, so
// the scheduler thread copies nothing and is free to launch the next batch.
//
// Requests of a batch over the same table, probe columns and row count that
// differ only in their filter bound share one scan (k_batch_cells): the
// columns are read and the table probed once, each matched row adds to the
// cell of its filter range and group, and one prefix pass over the ranges
// gives every request its own groups (exact: integer sums).
//
// With plain = 1 the server instead runs requests one at a time through the
// operator API (select -> hash_probe -> groupby on the resident table): the
// per-query baseline under the same arrival trace.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "device_common.cuh"
#include "mgv_internal.h"

using namespace mgv;
using Clock = std::chrono::steady_clock;

namespace {

// A pinned host buffer that one batch's results are copied into.  Its rows
// stay there until every request of the batch has been waited for (the
// waiter copies its own rows out), then the buffer serves another batch.
struct Landing {
    mgv_group_row* rows = nullptr;  // pinned: cap rows, then the per-request counts
    uint32_t* counts = nullptr;
    size_t cap = 0;                 // rows
    uint32_t ncounts = 0;
    int refs = 0;                   // requests whose rows are here and not yet waited for (lock held)
    bool attached = false;          // a slot is filling it
};

struct Request {
    uint64_t ticket = 0;
    mgv_server_request r{};
    mgv_op* table = nullptr;  // the resident build table, resolved at submit
    Clock::time_point t_submit;
    double latency_ms = 0.0;
    mgv_status status = MGV_OK;
    bool done = false;
    std::vector<mgv_group_row> rows;  // plain mode
    Landing* land = nullptr;          // batched mode: the rows are land->rows[off, off + n)
    uint64_t off = 0;
    uint32_t n = 0;
    size_t bytes = 0;  // admission charge
};

struct Inflight {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<std::shared_ptr<Request>> reqs;
    void* dmem = nullptr;    // the slot's device region, kept and grown on demand
    size_t dmem_cap = 0;
    unsigned char* hdesc = nullptr;  // pinned staging of the batch's descriptors: one copy per launch
    size_t hdesc_cap = 0;
    size_t charge = 0;
    Landing* land = nullptr;          // where this batch's results land
    std::vector<uint64_t> offs;
    bool busy = false;
};

uint32_t group_cap(uint32_t max_groups) {
    uint32_t cap = 64;
    while (cap < 2u * max_groups) cap <<= 1;
    return cap;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t request_bytes(const mgv_server_request& r) {
    const uint64_t cap = group_cap(r.max_groups);
    return align256(cap * 20 + 16) + align256((size_t)r.max_groups * sizeof(mgv_group_row)) + 512;
}

}  // namespace

struct mgv_server {
    mgv_ctx* ctx = nullptr;
    mgv_server_config cfg{};
    std::vector<mgv_op*> tables;  // resident hash_build operators
    size_t table_bytes = 0;
    std::mutex mu;
    std::condition_variable cv;       // scheduler wake-up
    std::condition_variable done_cv;  // request completion
    std::deque<std::shared_ptr<Request>> pending;
    std::map<uint64_t, std::shared_ptr<Request>> by_ticket;
    uint64_t next_ticket = 1;
    bool stop = false;
    size_t used = 0, peak = 0;
    std::vector<Inflight> slots;
    std::thread th;
    // stats
    std::vector<double> latencies;
    uint64_t submitted = 0, completed = 0, batches = 0, rejected = 0, batched_queries = 0, solo = 0;
    std::atomic<uint64_t> shared_scans{0}, scan_queries{0};  // scans launched, requests they answered
    // plain mode: group-by operators (device tables) reused per max_groups
    std::map<uint32_t, mgv_op*> plain_gb;
    std::vector<std::unique_ptr<Landing>> landings;  // pinned result buffers (lock held)
};

namespace {

void complete(mgv_server* S, const std::shared_ptr<Request>& q, mgv_status st) {
    q->status = st;
    q->latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - q->t_submit).count();
    q->done = true;
    S->latencies.push_back(q->latency_ms);
    S->completed++;
}

constexpr uint64_t kMinLandingRows = 1u << 18;  // 6 MiB of group rows
// Pending requests an idle server still answers one at a time (oldest first)
// through the single-query chain; a longer queue is batched.
constexpr size_t kSoloBacklog = 4;

// A free landing zone of at least `rows` rows and `ncounts` counts (scheduler
// thread, lock not held; the list is read and changed under the lock, a new
// zone is pinned outside it).
mgv_status acquire_landing(mgv_server* S, uint64_t rows, uint32_t ncounts, Landing*& out) {
    {
        std::lock_guard<std::mutex> lk(S->mu);
        Landing* best = nullptr;
        for (auto& L : S->landings)
            if (!L->attached && L->refs == 0 && L->cap >= rows && L->ncounts >= ncounts && (!best || L->cap < best->cap))
                best = L.get();
        if (best) {
            best->attached = true;
            out = best;
            return MGV_OK;
        }
    }
    // pinning is slow (milliseconds for tens of MB): zones get headroom, so a
    // later, larger batch finds one to reuse instead of pinning another
    auto L = std::make_unique<Landing>();
    L->cap = std::max<uint64_t>(rows + rows / 2, kMinLandingRows);
    L->ncounts = std::max<uint32_t>(ncounts, S->cfg.max_batch);
    void* p = nullptr;
    MGV_CUDA_TRY(cudaMallocHost(&p, sizeof(mgv_group_row) * L->cap + 4ull * L->ncounts));
    L->rows = static_cast<mgv_group_row*>(p);
    L->counts = reinterpret_cast<uint32_t*>(L->rows + L->cap);
    L->attached = true;
    out = L.get();
    std::lock_guard<std::mutex> lk(S->mu);
    S->landings.push_back(std::move(L));
    return MGV_OK;
}

// Launch one batch of admitted requests on slot `sl` (scheduler thread, lock
// not held: it reads only the slot and its requests' immutable parameters).
// Requests that can share one scan: the same resident table, probe columns,
// row count and group-table size, differing at most in their filter bound.
struct ScanKey {
    const void* table;
    const int32_t *key, *filter, *group, *value;
    uint64_t rows;
    uint32_t cap;
    bool operator<(const ScanKey& o) const {
        return std::tie(table, key, filter, group, value, rows, cap) <
               std::tie(o.table, o.key, o.filter, o.group, o.value, o.rows, o.cap);
    }
};

// A shared scan of a batch: its requests, its distinct bounds (ascending) and
// each request's range (the index of its bound).
struct Scan {
    std::vector<uint32_t> reqs;
    std::vector<int32_t> bounds;
    std::vector<uint32_t> rank;  // per entry of reqs
    std::vector<uint16_t> lut;   // range of filter value bounds[0] + i, when the bounds span <= kCellLut values
    uint32_t cap = 0;
    size_t dir_off = 0, vals_off = 0, bounds_off = 0, lut_off = 0;
};

// Launch one batch of admitted requests on slot `sl` (scheduler thread, lock
// not held: it reads only the slot and its requests' immutable parameters).
// Requests that can share a scan (ScanKey) and number at least two run as
// one shared scan unless the server was made with separate_scans; the rest
// run as queries of the batch probe kernel.
mgv_status launch(mgv_server* S, Inflight& sl) {
    Context* ctx = S->ctx;
    const uint32_t nq = (uint32_t)sl.reqs.size();
    std::vector<uint32_t> caps(nq);
    for (uint32_t i = 0; i < nq; ++i) caps[i] = group_cap(sl.reqs[i]->r.max_groups);
    // ---- shared scans --------------------------------------------------------
    std::vector<Scan> scans;
    std::vector<int32_t> scan_of(nq, -1);
    if (!S->cfg.separate_scans) {
        std::map<ScanKey, std::vector<uint32_t>> by_key;
        for (uint32_t i = 0; i < nq; ++i) {
            const mgv_server_request& r = sl.reqs[i]->r;
            by_key[ScanKey{sl.reqs[i]->table, r.probe_key, r.probe_filter, r.probe_group, r.probe_value,
                           r.probe_rows, caps[i]}].push_back(i);
        }
        for (auto& kv : by_key) {
            const std::vector<uint32_t>& v = kv.second;
            for (size_t c0 = 0; c0 < v.size(); c0 += kMaxCellRanges) {  // at most kMaxCellRanges bounds a scan
                const size_t c1 = std::min(v.size(), c0 + (size_t)kMaxCellRanges);
                if (c1 - c0 < 2) continue;
                Scan sc;
                sc.reqs.assign(v.begin() + c0, v.begin() + c1);
                sc.cap = kv.first.cap;
                for (uint32_t i : sc.reqs) sc.bounds.push_back(sl.reqs[i]->r.filter_bound);
                std::sort(sc.bounds.begin(), sc.bounds.end());
                sc.bounds.erase(std::unique(sc.bounds.begin(), sc.bounds.end()), sc.bounds.end());
                for (uint32_t i : sc.reqs)
                    sc.rank.push_back((uint32_t)(std::lower_bound(sc.bounds.begin(), sc.bounds.end(),
                                                                  sl.reqs[i]->r.filter_bound) -
                                                 sc.bounds.begin()));
                const int64_t span = (int64_t)sc.bounds.back() - sc.bounds.front() + 1;
                if (span <= (int64_t)kCellLut) {
                    sc.lut.resize((size_t)span);
                    uint16_t j = 0;
                    for (int64_t d = 0; d < span; ++d) {  // the first j with bounds[j] >= bounds[0] + d
                        while ((int64_t)sc.bounds[j] < (int64_t)sc.bounds.front() + d) ++j;
                        sc.lut[(size_t)d] = j;
                    }
                }
                for (uint32_t i : sc.reqs) scan_of[i] = (int32_t)scans.size();
                scans.push_back(std::move(sc));
            }
        }
    }
    // device layout: [group keys, scan directories | zeroed: sums counts specials, scan cells |
    //                 counts | rows | qs | outs | items | compact items | scans | scan items | bounds]
    size_t off = 0;
    std::vector<size_t> gk(nq), gs(nq), gc(nq), sp(nq);
    uint64_t slots = 0, rows = 0;
    for (uint32_t i = 0; i < nq; ++i) {
        if (scan_of[i] >= 0) continue;
        gk[i] = off;
        off += 4ull * caps[i];
        slots += caps[i];
    }
    for (Scan& sc : scans) {
        sc.dir_off = off;
        off += 4ull * sc.cap;
        slots += sc.cap;
    }
    off = align256(off);
    const size_t zero_begin = off;
    for (uint32_t i = 0; i < nq; ++i) {
        if (scan_of[i] >= 0) continue;
        gs[i] = off; off += 8ull * caps[i];
        gc[i] = off; off += 8ull * caps[i];
        sp[i] = off; off += 16;
    }
    for (Scan& sc : scans) {
        sc.vals_off = off;
        off += 8ull * cell_block_words(sc.cap) * sc.bounds.size();
    }
    const size_t zero_end = off;
    off = align256(off);
    const size_t counts_off = off;
    off = align256(off + 4ull * nq);
    sl.offs.resize(nq);
    for (uint32_t i = 0; i < nq; ++i) { sl.offs[i] = rows; rows += sl.reqs[i]->r.max_groups; }
    const size_t rows_off = off;
    off = align256(off + sizeof(mgv_group_row) * std::max<uint64_t>(rows, 1));
    std::vector<BatchItem> pi, ci, si;
    const uint64_t item_rows = 32768;  // < 2^kCellRowBits, as a shared scan's items must be
    for (uint32_t i = 0; i < nq; ++i) {
        if (scan_of[i] < 0)
            for (uint64_t lo = 0; lo < sl.reqs[i]->r.probe_rows; lo += item_rows)
                pi.push_back(BatchItem{i, 0, lo, std::min<uint64_t>(sl.reqs[i]->r.probe_rows, lo + item_rows)});
        for (uint64_t lo = 0; lo <= caps[i]; lo += 65536)
            ci.push_back(BatchItem{i, 0, lo, std::min<uint64_t>((uint64_t)caps[i] + 1, lo + 65536)});
    }
    for (uint32_t g = 0; g < (uint32_t)scans.size(); ++g) {
        const uint64_t n = sl.reqs[scans[g].reqs[0]]->r.probe_rows;
        for (uint64_t lo = 0; lo < n; lo += item_rows) si.push_back(BatchItem{g, 0, lo, std::min(n, lo + item_rows)});
    }
    const size_t qs_off = off;
    off = align256(off + sizeof(ChainDev) * nq);
    const size_t outs_off = off;
    off = align256(off + sizeof(BatchOut) * nq);
    const size_t pi_off = off;
    off = align256(off + sizeof(BatchItem) * std::max<size_t>(pi.size(), 1));
    const size_t ci_off = off;
    off = align256(off + sizeof(BatchItem) * std::max<size_t>(ci.size(), 1));
    const size_t scans_off = off;
    off = align256(off + sizeof(ChainDev) * std::max<size_t>(scans.size(), 1));
    const size_t si_off = off;
    off = align256(off + sizeof(BatchItem) * std::max<size_t>(si.size(), 1));
    for (Scan& sc : scans) {
        sc.bounds_off = off;
        off += 4ull * sc.bounds.size();
        sc.lut_off = off;
        off += 2ull * sc.lut.size();
        off = (off + 3) & ~(size_t)3;
    }
    off = align256(off);

    // Each slot keeps its region and only grows it (the slot's previous batch
    // has completed): no allocator runs per batch, so slots never wait on
    // each other's frees.
    if (off > sl.dmem_cap) {
        if (sl.dmem) MGV_CUDA_TRY(cudaFree(sl.dmem));
        sl.dmem = nullptr;
        sl.dmem_cap = 0;
        const size_t cap = off + off / 4;
        MGV_CUDA_TRY(cudaMalloc(&sl.dmem, cap));
        sl.dmem_cap = cap;
    }
    unsigned char* A = static_cast<unsigned char*>(sl.dmem);
    // a pinned landing zone for the results (rows + counts)
    mgv_status lst = acquire_landing(S, std::max<uint64_t>(rows, 1), nq, sl.land);
    if (lst != MGV_OK) return lst;
    // the descriptors of a single request or of a scan (the scan's bound is its largest)
    auto chain_of = [&](const mgv_server_request& r, const Request& q) {
        ChainDev c{};
        c.cols[0] = r.probe_key;
        c.cols[1] = r.probe_filter;
        c.cols[2] = r.probe_group;
        c.cols[3] = r.probe_value;
        c.n = r.probe_rows;
        c.ncols = 4;
        c.nslots = 3;
        c.slot_src[0] = 0;
        c.slot_src[1] = 2;
        c.slot_src[2] = 3;
        c.sel_col = 1;
        c.sel_bound = r.filter_bound;
        c.probe_slot = 0;
        c.table = q.table->table;
        c.ref[0] = 1;
        c.ref[1] = 2;
        c.nref = 2;
        return c;
    };
    std::vector<ChainDev> hq(nq), hs(scans.size());
    std::vector<BatchOut> ho(nq);
    for (uint32_t g = 0; g < (uint32_t)scans.size(); ++g) {
        const Scan& sc = scans[g];
        const Request& q0 = *sl.reqs[sc.reqs[0]];
        hs[g] = chain_of(q0.r, q0);
        hs[g].sel_bound = sc.bounds.back();
        hs[g].cells = CellsView{reinterpret_cast<const int32_t*>(A + sc.bounds_off), (uint32_t)sc.bounds.size(),
                                sc.cap, reinterpret_cast<int32_t*>(A + sc.dir_off),
                                reinterpret_cast<unsigned long long*>(A + sc.vals_off),
                                reinterpret_cast<const uint16_t*>(A + sc.lut_off), (uint32_t)sc.lut.size(),
                                sc.bounds.front()};
    }
    std::vector<uint32_t> rank_of(nq, 0);
    for (const Scan& sc : scans)
        for (size_t k = 0; k < sc.reqs.size(); ++k) rank_of[sc.reqs[k]] = sc.rank[k];
    for (uint32_t i = 0; i < nq; ++i) {
        const mgv_server_request& r = sl.reqs[i]->r;
        GroupTableView g{};
        if (scan_of[i] >= 0) {
            g = cells_range(hs[scan_of[i]].cells, rank_of[i]);  // the prefix of its ranges
        } else {
            g.keys = reinterpret_cast<int32_t*>(A + gk[i]);
            g.sums = reinterpret_cast<unsigned long long*>(A + gs[i]);
            g.counts = reinterpret_cast<unsigned long long*>(A + gc[i]);
            g.special = reinterpret_cast<unsigned long long*>(A + sp[i]);
            g.cap = caps[i];
            ChainDev& c = hq[i];
            c = chain_of(r, *sl.reqs[i]);
            c.gt = g;
            c.smem_groups = std::min(caps[i], kMaxSmemGroups);
        }
        ho[i] = BatchOut{g, reinterpret_cast<mgv_group_row*>(A + rows_off) + sl.offs[i],
                         reinterpret_cast<uint32_t*>(A + counts_off) + i, r.max_groups, 0};
    }
    cudaStream_t s = sl.stream;
    // The descriptors [qs | outs | probe items | compact items | scans | scan
    // items | bounds] are laid out on the device as in the slot's pinned
    // staging area and go over in one copy.  The staging stays untouched
    // until the slot's batch has completed (a busy slot is never launched on).
    const size_t desc_bytes = off - qs_off;
    if (desc_bytes > sl.hdesc_cap) {
        if (sl.hdesc) MGV_CUDA_TRY(cudaFreeHost(sl.hdesc));
        sl.hdesc = nullptr;
        sl.hdesc_cap = 0;
        const size_t cap = desc_bytes + desc_bytes / 2 + 4096;
        MGV_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&sl.hdesc), cap));
        sl.hdesc_cap = cap;
    }
    std::memcpy(sl.hdesc + (qs_off - qs_off), hq.data(), sizeof(ChainDev) * nq);
    std::memcpy(sl.hdesc + (outs_off - qs_off), ho.data(), sizeof(BatchOut) * nq);
    if (!pi.empty()) std::memcpy(sl.hdesc + (pi_off - qs_off), pi.data(), sizeof(BatchItem) * pi.size());
    std::memcpy(sl.hdesc + (ci_off - qs_off), ci.data(), sizeof(BatchItem) * ci.size());
    if (!hs.empty()) std::memcpy(sl.hdesc + (scans_off - qs_off), hs.data(), sizeof(ChainDev) * hs.size());
    if (!si.empty()) std::memcpy(sl.hdesc + (si_off - qs_off), si.data(), sizeof(BatchItem) * si.size());
    for (const Scan& sc : scans)
        std::memcpy(sl.hdesc + (sc.bounds_off - qs_off), sc.bounds.data(), 4 * sc.bounds.size());
    for (const Scan& sc : scans)
        if (!sc.lut.empty()) std::memcpy(sl.hdesc + (sc.lut_off - qs_off), sc.lut.data(), 2 * sc.lut.size());
    MGV_CUDA_TRY(cudaMemcpyAsync(A + qs_off, sl.hdesc, desc_bytes, cudaMemcpyHostToDevice, s));
    MGV_CUDA_TRY(launch_fill_i32(reinterpret_cast<int32_t*>(A), slots, kEmptyKey, s, ctx));
    MGV_CUDA_TRY(cudaMemsetAsync(A + zero_begin, 0, zero_end - zero_begin, s));
    MGV_CUDA_TRY(cudaMemsetAsync(A + counts_off, 0, 4ull * nq, s));
    MGV_CUDA_TRY(launch_batch(reinterpret_cast<ChainDev*>(A + qs_off), reinterpret_cast<BatchOut*>(A + outs_off),
                              reinterpret_cast<BatchItem*>(A + pi_off), (uint32_t)pi.size(), nullptr, 0u, 0, 0u,
                              s, ctx));
    if (!scans.empty()) {
        MGV_CUDA_TRY(launch_cells(reinterpret_cast<ChainDev*>(A + scans_off), reinterpret_cast<BatchItem*>(A + si_off),
                                  (uint32_t)si.size(), s, ctx));
        for (const ChainDev& h : hs) MGV_CUDA_TRY(launch_cells_prefix(h.cells, s, ctx));
    }
    MGV_CUDA_TRY(launch_batch(nullptr, reinterpret_cast<BatchOut*>(A + outs_off), nullptr, 0u,
                              reinterpret_cast<BatchItem*>(A + ci_off), (uint32_t)ci.size(), 0, 0u, s, ctx));
    MGV_CUDA_TRY(cudaMemcpyAsync(sl.land->counts, A + counts_off, 4ull * nq, cudaMemcpyDeviceToHost, s));
    MGV_CUDA_TRY(cudaMemcpyAsync(sl.land->rows, A + rows_off, sizeof(mgv_group_row) * std::max<uint64_t>(rows, 1),
                                 cudaMemcpyDeviceToHost, s));
    MGV_CUDA_TRY(cudaEventRecord(sl.done, s));
    sl.busy = true;
    S->shared_scans += scans.size();
    for (const Scan& sc : scans) S->scan_queries += sc.reqs.size();
    return MGV_OK;
}

// Hands a finished batch's results to its requests (lock held): each
// request points at its rows in the batch's landing zone, which stays out of
// use until every request has been waited for; the slot takes a new one.
void finish(mgv_server* S, Inflight& sl) {
    Landing* L = sl.land;
    L->attached = false;
    L->refs = (int)sl.reqs.size();
    for (size_t i = 0; i < sl.reqs.size(); ++i) {
        auto& q = sl.reqs[i];
        q->land = L;
        q->off = sl.offs[i];
        q->n = std::min<uint32_t>(L->counts[i], q->r.max_groups);
        complete(S, q, L->counts[i] > q->r.max_groups ? MGV_ENOMEM : MGV_OK);
        S->used -= q->bytes;
    }
    sl.land = nullptr;
    sl.reqs.clear();
    sl.busy = false;
}

// A batch that the GPU reported an error for (lock held): its requests fail
// with MGV_ECUDA, its landing zone and memory charge are released.
void fail_slot(mgv_server* S, Inflight& sl, cudaError_t e) {
    (void)cuda_fail(e, "mgv_server: batch");
    for (auto& q : sl.reqs) {
        S->used -= q->bytes;
        complete(S, q, MGV_ECUDA);
    }
    if (sl.land) sl.land->attached = false;
    sl.land = nullptr;
    sl.reqs.clear();
    sl.busy = false;
}

// Plain mode: one request through the operator API (lock not held).
// The group-by operator of the single-query chain for max_groups.  One per
// power-of-two class: its table (2 x max_groups, rounded up to a power of two)
// is the same for every max_groups of the class, so nothing is created per
// request once the classes up to 2^16 exist (made with the server).
uint32_t groupby_class(uint32_t max_groups) {
    uint32_t c = 16;
    while (c < max_groups) c <<= 1;
    return c;
}

mgv_status plain_groupby(mgv_server* S, uint32_t max_groups, mgv_op** out) {
    const uint32_t c = groupby_class(max_groups);
    auto it = S->plain_gb.find(c);
    if (it != S->plain_gb.end()) {
        *out = it->second;
        return MGV_OK;
    }
    mgv_groupby_desc gd{2, 3, c, 0};
    mgv_status st = mgv_op_create_groupby(S->ctx, &gd, out);
    if (st == MGV_OK) S->plain_gb[c] = *out;
    return st;
}

mgv_status run_plain(mgv_server* S, Request& q) {
    const mgv_server_request& r = q.r;
    mgv_ctx* ctx = S->ctx;
    mgv_op *gb = nullptr, *probe = nullptr, *sel = nullptr;
    mgv_status st = MGV_OK;
    st = plain_groupby(S, r.max_groups, &gb);
    if (st != MGV_OK) return st;
    mgv_hash_probe_desc pd{0, 0, q.table};
    if (st == MGV_OK) st = mgv_op_create_hash_probe(ctx, &pd, gb, &probe);
    mgv_select_desc sd{1, r.filter_bound};
    if (st == MGV_OK) st = mgv_op_create_select(ctx, &sd, probe, &sel);
    const int32_t* cols[4] = {r.probe_key, r.probe_filter, r.probe_group, r.probe_value};
    if (st == MGV_OK) st = mgv_op_open(sel, nullptr);
    if (st == MGV_OK) st = mgv_op_consume_columns(sel, cols, 4, r.probe_rows, nullptr);
    if (st == MGV_OK) st = mgv_op_close(sel, nullptr);
    if (st == MGV_OK) q.rows = static_cast<Op*>(gb)->gb_rows;  // in no particular order, as the batched server's
    mgv_op_destroy(sel);
    mgv_op_destroy(probe);
    return st;
}

void scheduler(mgv_server* S) {
    cudaSetDevice(S->ctx->device);
    std::unique_lock<std::mutex> lk(S->mu);
    while (true) {
        if (S->cfg.plain) {
            S->cv.wait(lk, [&] { return S->stop || !S->pending.empty(); });
            if (S->stop && S->pending.empty()) break;
            auto q = S->pending.front();
            S->pending.pop_front();
            lk.unlock();
            const mgv_status st = run_plain(S, *q);
            lk.lock();
            complete(S, q, st);
            S->done_cv.notify_all();
            continue;
        }
        // 1. harvest finished batches; the host copies run outside the lock.  A
        // batch whose stream reports an error (not just "not ready") fails its
        // requests, so no waiter waits for results that will never come.
        bool any_busy = false;
        for (auto& sl : S->slots) {
            if (sl.busy) {
                const cudaError_t q = cudaEventQuery(sl.done);
                if (q == cudaSuccess) {
                    finish(S, sl);
                    S->done_cv.notify_all();
                } else if (q != cudaErrorNotReady) {
                    fail_slot(S, sl, q);
                    S->done_cv.notify_all();
                }
            }
            any_busy |= sl.busy;
        }
        // 2. admit pending requests into a free slot
        Inflight* free_slot = nullptr;
        for (auto& sl : S->slots)
            if (!sl.busy) { free_slot = &sl; break; }
        const size_t budget = S->cfg.memory_budget > S->table_bytes ? S->cfg.memory_budget - S->table_bytes : 0;
        if (!any_busy && !S->cfg.batch_solo && !S->pending.empty() && S->pending.size() <= kSoloBacklog &&
            S->used + S->pending.front()->bytes <= budget) {
            // a short queue on an idle server: the oldest request runs alone
            // through the single-query chain, without batch planning or event
            // polling (admitted and charged like a batch of one); batches form
            // only once a backlog builds up, where running requests together
            // shortens the queue
            auto q = S->pending.front();
            S->pending.pop_front();
            S->used += q->bytes;
            S->peak = std::max(S->peak, S->used + S->table_bytes);
            lk.unlock();
            const mgv_status st = run_plain(S, *q);
            lk.lock();
            S->used -= q->bytes;
            S->batches++;
            S->batched_queries++;
            S->solo++;
            complete(S, q, st);
            S->done_cv.notify_all();
            continue;
        }
        if (free_slot && !S->pending.empty()) {
            while (!S->pending.empty() && free_slot->reqs.size() < S->cfg.max_batch) {
                auto& q = S->pending.front();
                if (q->bytes > budget) {  // can never fit
                    auto r = q;
                    S->pending.pop_front();
                    S->rejected++;
                    complete(S, r, MGV_ENOMEM);
                    S->done_cv.notify_all();
                    continue;
                }
                if (S->used + q->bytes > budget) break;  // wait for memory to free up
                S->used += q->bytes;
                S->peak = std::max(S->peak, S->used + S->table_bytes);
                free_slot->reqs.push_back(q);
                S->pending.pop_front();
            }
            if (!free_slot->reqs.empty()) {
                lk.unlock();  // submitters and waiters go on while the batch is planned and launched
                const mgv_status st = launch(S, *free_slot);
                lk.lock();
                if (st == MGV_OK) {
                    S->batches++;
                    S->batched_queries += free_slot->reqs.size();
                } else {
                    for (auto& q : free_slot->reqs) { S->used -= q->bytes; complete(S, q, st); }
                    free_slot->reqs.clear();
                    free_slot->busy = false;
                    if (free_slot->land) {  // nothing landed: the zone is free again
                        free_slot->land->attached = false;
                        free_slot->land = nullptr;
                    }
                    S->done_cv.notify_all();
                }
                continue;
            }
        }
        if (S->stop && S->pending.empty() && !any_busy) break;
        if (any_busy)
            S->cv.wait_for(lk, std::chrono::microseconds(20));  // poll the GPU
        else
            S->cv.wait(lk, [&] { return S->stop || !S->pending.empty(); });
    }
}

}  // namespace

extern "C" {

mgv_status mgv_server_create(mgv_ctx* ctx, const mgv_server_config* cfg, mgv_server** out) {
    if (!ctx || !cfg || !out) return fail(MGV_EINVAL, "NULL argument");
    *out = nullptr;
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    mgv_server* S = new (std::nothrow) mgv_server();
    if (!S) return fail(MGV_ENOMEM, "host allocation");
    S->ctx = ctx;
    S->cfg = *cfg;
    if (S->cfg.max_batch == 0) S->cfg.max_batch = 256;
    if (S->cfg.max_inflight == 0) S->cfg.max_inflight = 2;
    if (S->cfg.max_inflight > 16) S->cfg.max_inflight = 16;
    if (S->cfg.load_factor == 0.0f) S->cfg.load_factor = ctx->tuning.default_load_factor;
    for (uint32_t c = 16; c <= (1u << 16); c <<= 1) {  // the single-query chain's group-by classes
        mgv_op* gb = nullptr;
        const mgv_status st = plain_groupby(S, c, &gb);
        if (st != MGV_OK) {
            for (auto& kv : S->plain_gb) mgv_op_destroy(kv.second);
            delete S;
            return st;
        }
        // the host rows of the class's largest result, written once now: the
        // first request of a class then finds its pages present instead of
        // faulting them in (a tenth of a millisecond for 65536 groups)
        std::vector<mgv_group_row>& rows = static_cast<Op*>(gb)->gb_rows;
        rows.resize(c);
        rows.clear();
    }
    // landing zones pinned up front (four per in-flight slot, at most eight),
    // so serving rarely pins (slow) while batches are in flight and waiters
    // still hold earlier zones
    for (uint32_t i = 0; i < std::min(4 * S->cfg.max_inflight, 8u); ++i) {
        auto L = std::make_unique<Landing>();
        L->cap = kMinLandingRows;
        L->ncounts = S->cfg.max_batch;
        void* p = nullptr;
        if (cudaMallocHost(&p, sizeof(mgv_group_row) * L->cap + 4ull * L->ncounts) != cudaSuccess) {
            for (auto& Z : S->landings) cudaFreeHost(Z->rows);
            for (auto& kv : S->plain_gb) mgv_op_destroy(kv.second);
            delete S;
            return fail(MGV_ENOMEM, "pinned host allocation");
        }
        L->rows = static_cast<mgv_group_row*>(p);
        L->counts = reinterpret_cast<uint32_t*>(L->rows + L->cap);
        S->landings.push_back(std::move(L));
    }
    S->slots.resize(S->cfg.max_inflight);
    for (auto& sl : S->slots) {
        cudaError_t e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(e, "mgv_server_create");
    }
    S->th = std::thread(scheduler, S);
    *out = S;
    return MGV_OK;
}

mgv_status mgv_server_add_table(mgv_server* S, const int32_t* keys, const int32_t* payloads, uint64_t rows,
                                uint32_t* table_id) {
    if (!S || (!keys && rows) || !table_id) return fail(MGV_EINVAL, "NULL argument");
    mgv_hash_build_desc d{0, payloads ? 1 : -1, std::max<uint64_t>(rows, 1), S->cfg.load_factor, 0, 0, 0};
    mgv_op* hb = nullptr;
    mgv_status st = mgv_op_create_hash_build(S->ctx, &d, &hb);
    const int32_t* cols[2] = {keys, payloads};
    if (st == MGV_OK) st = mgv_op_open(hb, nullptr);
    if (st == MGV_OK) st = mgv_op_consume_columns(hb, cols, payloads ? 2 : 1, rows, nullptr);
    if (st == MGV_OK) st = mgv_op_close(hb, nullptr);
    if (st != MGV_OK) {
        if (hb) mgv_op_destroy(hb);
        return st;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    S->tables.push_back(hb);
    S->table_bytes += hb->table_bytes + sizeof(int32_t) * hb->table.side_cap;
    *table_id = (uint32_t)(S->tables.size() - 1);
    return MGV_OK;
}

mgv_status mgv_server_submit(mgv_server* S, const mgv_server_request* r, uint64_t* ticket) {
    if (!S || !r || !ticket) return fail(MGV_EINVAL, "NULL argument");
    if (r->max_groups == 0 || r->max_groups > (1u << 28)) return fail(MGV_EINVAL, "max_groups out of range");
    if (r->probe_rows && (!r->probe_key || !r->probe_filter || !r->probe_group || !r->probe_value))
        return fail(MGV_EINVAL, "NULL probe column");
    auto q = std::make_shared<Request>();
    q->r = *r;
    q->bytes = request_bytes(*r);
    q->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (r->table >= S->tables.size()) return fail(MGV_EINVAL, "no such table");
        if (S->stop) return fail(MGV_ESTATE, "server is stopping");
        q->table = S->tables[r->table];
        q->ticket = S->next_ticket++;
        S->by_ticket[q->ticket] = q;
        S->pending.push_back(q);
        S->submitted++;
    }
    S->cv.notify_all();
    *ticket = q->ticket;
    return MGV_OK;
}

mgv_status mgv_server_wait(mgv_server* S, uint64_t ticket, uint32_t timeout_ms, mgv_group_row* out, uint64_t cap,
                           uint64_t* rows, double* latency_ms) {
    if (!S) return fail(MGV_EINVAL, "server is NULL");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->by_ticket.find(ticket);
    if (it == S->by_ticket.end()) return fail(MGV_EINVAL, "unknown ticket");
    auto q = it->second;
    if (!S->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return q->done; }))
        return fail(MGV_ETIMEDOUT, "request not finished");
    S->by_ticket.erase(it);
    lk.unlock();  // the request is this caller's now: copy its rows outside the lock
    const mgv_group_row* src = q->land ? q->land->rows + q->off : q->rows.data();
    const uint64_t n = q->land ? q->n : q->rows.size();
    if (rows) *rows = n;
    if (latency_ms) *latency_ms = q->latency_ms;
    if (out) std::copy(src, src + std::min<uint64_t>(cap, n), out);
    if (q->land) {  // the landing zone is free again once its last request is waited for
        lk.lock();
        q->land->refs--;
        q->land = nullptr;
    }
    if (q->status != MGV_OK) return fail(q->status, "request failed");
    return MGV_OK;
}

mgv_status mgv_server_stats_get(mgv_server* S, mgv_server_stats* out) {
    if (!S || !out) return fail(MGV_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(S->mu);
    *out = mgv_server_stats{};
    out->submitted = S->submitted;
    out->completed = S->completed;
    out->batches = S->batches;
    out->rejected = S->rejected;
    out->mean_batch = S->batches ? (double)S->batched_queries / S->batches : 0.0;
    out->solo = S->solo;
    out->shared_scans = S->shared_scans.load();
    out->scan_queries = S->scan_queries.load();
    out->resident_table_bytes = S->table_bytes;
    out->peak_bytes = S->peak;
    if (!S->latencies.empty()) {
        std::vector<double> v = S->latencies;
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) { return v[std::min<size_t>(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5))]; };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        out->max_ms = v.back();
        double s = 0;
        for (double x : v) s += x;
        out->mean_ms = s / v.size();
    }
    return MGV_OK;
}

mgv_status mgv_server_reset_stats(mgv_server* S) {
    if (!S) return fail(MGV_EINVAL, "server is NULL");
    std::lock_guard<std::mutex> lk(S->mu);
    S->latencies.clear();
    S->submitted = S->completed = S->batches = S->rejected = S->batched_queries = S->solo = 0;
    S->shared_scans = 0;
    S->scan_queries = 0;
    S->peak = S->used + S->table_bytes;
    return MGV_OK;
}

mgv_status mgv_server_destroy(mgv_server* S) {
    if (!S) return MGV_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv.notify_all();
    if (S->th.joinable()) S->th.join();
    cudaSetDevice(S->ctx->device);
    for (auto& sl : S->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        if (sl.dmem) cudaFree(sl.dmem);
        if (sl.hdesc) cudaFreeHost(sl.hdesc);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    for (auto& kv : S->plain_gb) mgv_op_destroy(kv.second);
    for (mgv_op* t : S->tables) mgv_op_destroy(t);
    for (auto& L : S->landings) cudaFreeHost(L->rows);
    delete S;
    return MGV_OK;
}

}  // extern "C"
