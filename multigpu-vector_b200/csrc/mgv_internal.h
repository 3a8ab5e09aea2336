// mgv_internal.h -- host-side objects behind the C ABI and the kernel
// launchers they call.  Not part of the public interface.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mgv.h"

namespace mgv {

// ---- error reporting ---------------------------------------------------

void set_last_error(const std::string& msg);
mgv_status fail(mgv_status s, const std::string& msg);
mgv_status cuda_fail(cudaError_t e, const char* what);

#define MGV_CUDA_TRY(expr)                                    \
    do {                                                      \
        cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) return ::mgv::cuda_fail(e_, #expr); \
    } while (0)

// ---- device views passed to kernels by value ----------------------------

// Open-addressing join table: nbuckets buckets of 32 bytes (32-byte
// aligned), either 4 slots of 64-bit {key (low word), payload (high word)}
// or, for a build side without payloads (key_only), 8 slots of a 32-bit key
// (every match then has payload 0): half the bytes per key.
struct TableView {
    unsigned long long* slots;
    uint32_t nbuckets;
    // Radix layout: the home bucket of a key lies in the region of its
    // partition ((key >> radix_shift) & radix_mask), bpp buckets per region;
    // radix_mask 0 and bpp == nbuckets for an unpartitioned table.  Runs
    // continue linearly across regions.
    uint32_t radix_shift;
    uint32_t radix_mask;
    uint32_t bpp;
    uint32_t key_only;  // 1: 8 key slots per bucket, no payloads
    uint32_t pad;
    // Rows whose key is the reserved empty marker INT32_MIN:
    // meta[0] = their count, meta[1] = their payload sum, meta[2] = rows
    // inserted into the table, meta[3] = duplicate-key flag.
    unsigned long long* meta;
    int32_t* side_pay;      // payloads of those rows (for emitting matches)
    uint64_t side_cap;
};

// Group-by table in global memory: cap (power of two) slots of {key, sum,
// count}, empty key INT32_MIN; the group INT32_MIN has its own counters.
struct GroupTableView {
    int32_t* keys;
    unsigned long long* sums;
    unsigned long long* counts;
    unsigned long long* special;  // [0] sum, [1] count of group INT32_MIN
    uint32_t cap;
    uint32_t pad;
};

// Output rows appended to a chain of pool buffers.
struct SinkView {
    int32_t* slab;              // pool slab base
    unsigned long long* cursor; // rows reserved so far
    uint32_t* chain;            // buffer id per chunk, 0xffffffff = not yet taken
    uint32_t max_chunks;
    uint32_t capacity;          // rows per buffer
    uint32_t ncols;             // columns written
    uint32_t pool_ncols;
    struct PoolDev* pool;       // device free stack for swap-on-full
};

// Device free stack of a pool (tagged Treiber stack of buffer ids).
struct PoolDev {
    unsigned long long head;    // low 32 bits: top id (0xffffffff = empty), high: tag
    uint32_t available;
    uint32_t producers;
    uint32_t nbuffers;
    uint32_t pad;
    uint32_t next[1];           // nbuffers entries follow
};

constexpr uint32_t kNil = 0xffffffffu;
#ifndef MGV_BUILD_ROWS_PER_THREAD
#define MGV_BUILD_ROWS_PER_THREAD 1
#endif
constexpr int kBuildRows = MGV_BUILD_ROWS_PER_THREAD;  // build rows per thread in flight (1 measured fastest: more in flight contends in L2)
constexpr uint32_t kMaxSmemGroups = 8192;  // largest per-CTA shared group table (slots; 128 KiB)

// ---- host objects --------------------------------------------------------

struct Context;

struct Pool {
    Context* ctx = nullptr;
    uint32_t nbuffers = 0, capacity = 0, ncols = 0;
    int32_t* slab = nullptr;
    PoolDev* dev = nullptr;         // device free stack
    uint32_t* d_ids = nullptr;      // device scratch for host batch ops
    uint32_t* h_ids = nullptr;      // pinned mirror
    cudaStream_t stream = nullptr;  // the pool's own stream (release_streams)
    std::mutex mu;
    std::vector<uint32_t> host_cache;   // ids cached on the host side
    std::vector<mgv_buffer> bufs;       // descriptors, indexed by id
    std::vector<uint8_t> held;          // 1 = handed out to the caller
    uint32_t producers = 0;
};

struct Context {
    int device = 0;
    cudaDeviceProp prop{};
    cudaStream_t stream = nullptr;
    uint32_t* d_err = nullptr;      // device error word [code, detail]
    // pinned landing zone for close(): [0..1] error word, [2..] result words
    unsigned long long* h_stage = nullptr;
    std::atomic<uint64_t> launches{0};
    mgv_tuning tuning{0u, 4u, 4u, 3u, 0.5f, kMaxSmemGroups, 0u, 0u};
    mgv_batch_config batch_tuned{};  // the batch autotuner's last choice
    bool has_batch_tuned = false;
    std::mutex mu;
};

enum class OpKind { Select, Aggregate, HashBuild, HashProbe, Sink, Groupby, Partition };
enum class OpState { Created, Open, Closed };

struct Op {
    OpKind kind;
    Context* ctx = nullptr;
    Op* parent = nullptr;
    OpState state = OpState::Created;
    // select
    mgv_select_desc sel{};
    // aggregate
    mgv_aggregate_desc agg{};
    unsigned long long* d_acc = nullptr;    // [count, sum]
    unsigned long long* h_res = nullptr;    // pinned: the error word and the results read back at close
    mgv_agg_result agg_result{};
    // hash build
    mgv_hash_build_desc hb{};
    TableView table{};
    size_t table_bytes = 0;
    mgv_hash_build_info hb_info{};
    bool unique = false;
    // hash probe
    mgv_hash_probe_desc hp{};
    // sink
    mgv_sink_desc sk{};
    Pool* sink_pool = nullptr;
    SinkView sink{};
    uint64_t sink_rows = 0;
    std::vector<uint32_t> sink_chain;
    // delivery channel (mgv_sink_drain): copies run on their own stream; the
    // buffers of the copy in flight return to the pool when it completes
    cudaStream_t drain_stream = nullptr;
    cudaEvent_t drain_done = nullptr;
    std::vector<uint32_t> drain_ids;
    // group-by
    mgv_groupby_desc gb{};
    GroupTableView gtab{};
    std::vector<mgv_group_row> gb_rows;
    bool gb_sorted = false;  // gb_rows ordered by group (done at the first result read)
    mgv_group_row* gb_dev_rows = nullptr;  // [cap + 1] packed by close()
    uint32_t* gb_dev_count = nullptr;
    unsigned char* gb_land = nullptr;      // pinned: {err[2], count, pad} then kGroupLandRows rows
    uint32_t gb_land_rows = 0;
    // partition
    mgv_partition_desc pt{};
    int32_t* pt_store = nullptr;          // ncols x capacity, partition-major runs
    uint32_t pt_ncols = 0;
    uint64_t pt_fill = 0;                 // rows stored (read back at close)
    uint64_t pt_offered = 0;              // rows consumed since open (host count)
    uint32_t pt_runs = 0;                 // consumes with rows since open (each stores one partition-major run)
    bool pt_filtered = false;             // a select fed a consume: only the device knows pt_fill
    bool pt_hist_valid = true;            // pt_hist read back (else read at mgv_op_result)
    cudaStream_t pt_close_stream = nullptr;
    unsigned long long* pt_dev = nullptr; // [P] histogram / cursors of a consume
    unsigned long long* pt_acc = nullptr; // [1 + P] rows stored, rows per partition
    std::vector<uint64_t> pt_hist;        // rows per partition (read back at close)
    bool hb_fresh = false;  // opened, nothing consumed yet: the table is not cleared yet
    bool hb_partitioned = false;  // the rows being consumed are a partition op's run on the table's radix bits
    const unsigned long long* hb_part_ends = nullptr;  // that run's partition ends (device), when it is the only run
    // host ingest (mgv_op_consume_host): the copy stream and, per buffer in
    // flight, events for "slice copied" and "slice consumed"
    cudaStream_t in_stream = nullptr;
    std::vector<cudaEvent_t> in_copied, in_consumed;
    // shared-memory build scratch (hash_build), grown on demand
    void* rb_scratch = nullptr;
    size_t rb_bytes = 0;
    // device allocations owned by this op
    std::vector<void*> allocs;
};

// ---- kernel launchers (kernels.cu, pool.cu) -----------------------------

struct LaunchCfg {
    int grid;
    int block;
};

int occupancy_grid(const void* kernel, int block, size_t smem, const Context* ctx);

cudaError_t launch_fill_u64(unsigned long long* p, uint64_t n, unsigned long long v, cudaStream_t s,
                            Context* ctx);
cudaError_t launch_select_agg(const int32_t* filt, int32_t bound, bool has_sel, const int32_t* a,
                              const int32_t* b, uint64_t n, unsigned long long* acc, cudaStream_t s,
                              Context* ctx);
cudaError_t launch_build(const int32_t* keys, const int32_t* pays, const int32_t* filt,
                         int32_t bound, bool has_sel, uint64_t n, const TableView& t,
                         cudaStream_t s, Context* ctx);
// sum_mode bit 0: add build payload, bit 1: add probe payload column.
cudaError_t launch_probe_agg_staged(const int32_t* keys, const int32_t* pays, uint64_t n, const TableView& t,
                                    bool unique, uint32_t sum_mode, unsigned long long* acc, cudaStream_t s,
                                    Context* ctx);
cudaError_t launch_probe_agg(const int32_t* keys, const int32_t* pays, uint64_t n,
                             const TableView& t, bool unique, uint32_t sum_mode,
                             unsigned long long* acc, cudaStream_t s, Context* ctx);
// Generic fused chain (chain.cu): [select] -> [probe] -> terminal.
enum TermKind : int { kTermAgg = 0, kTermGroupby = 1, kTermSink = 2, kTermCells = 3 };

// A shared scan: several select -> join -> group-by requests over the same
// probe columns and join table that differ only in their filter bound read
// the columns and probe the table once.  The m distinct bounds, ascending,
// cut the filter values into m ranges (range j: b[j-1] < f <= b[j]); a
// matched row adds its (group, value) to one cell (range of its filter,
// group) only, whatever the number of requests.  A request with bound b[j]
// is then the sum of ranges 0..j, which one prefix pass over the ranges
// computes for every request at once.
//
// Cells live in m group tables that share one key array (the group
// directory, `cap` slots): range j's table is {keys, v + j*(2 cap + 2),
// +cap, +2 cap} over one block of u64 values, so a group has the same slot
// in every range and the prefix is a flat sum over the blocks.
struct CellsView {
    const int32_t* bounds;       // m ascending distinct filter bounds
    uint32_t m;
    uint32_t cap;                // directory slots, power of two
    int32_t* keys;               // the group directory (EMPTY = INT32_MIN)
    unsigned long long* vals;    // m blocks of [sums (cap) | counts (cap) | special sum, count]
    const uint16_t* lut;         // range of filter value lut_base + i, i < lut_len (0: none)
    uint32_t lut_len;
    int32_t lut_base;
};
constexpr uint32_t kCellRowBits = 20;        // ring entries: row offset (low bits) | range (high bits)
constexpr uint32_t kMaxCellRanges = 2048;    // distinct bounds per shared scan (range index < 2^11)
constexpr uint32_t kCellLut = 8192;          // longest range lookup table (filter values b[0]..b[m-1])
__host__ __device__ __forceinline__ size_t cell_block_words(uint32_t cap) { return 2ull * cap + 2; }
__host__ __device__ __forceinline__ GroupTableView cells_range(const CellsView& c, uint32_t j) {
    GroupTableView g;
    g.keys = c.keys;
    g.sums = c.vals + (size_t)j * cell_block_words(c.cap);
    g.counts = g.sums + c.cap;
    g.special = g.sums + 2ull * c.cap;
    g.cap = c.cap;
    g.pad = 0;
    return g;
}

struct ChainArgs {
    const int32_t* cols[MGV_MAX_COLS];
    uint32_t ncols;
    uint64_t n;
    bool has_sel;
    uint32_t sel_col;
    int32_t sel_bound;
    bool has_probe;
    uint32_t probe_col;
    TableView table;
    bool unique;
    int term;
    // terminal column references (input column, ncols = build payload, -1 none):
    //   aggregate: ref[0], ref[1] summed;  group-by: ref[0] group, ref[1] value;
    //   sink: ref[i] = source of output column i
    int32_t ref[MGV_MAX_COLS + 2];
    uint32_t nref;
    unsigned long long* acc;
    GroupTableView gt;
    uint32_t smem_groups;
    SinkView sink;
};
cudaError_t launch_chain(const ChainArgs& a, cudaStream_t s, Context* ctx);

// Device-side parameters of one chain (one query of a batch).
struct ChainDev {
    const int32_t* cols[MGV_MAX_COLS];
    uint64_t n;
    uint32_t ncols;
    uint32_t nslots;                 // carried columns
    int32_t slot_src[MGV_MAX_COLS];  // input column of each carried slot
    uint32_t sel_col;
    int32_t sel_bound;
    int32_t probe_slot;
    uint32_t unique;  // the table has no duplicate keys: a probe stops at its match
    TableView table;
    // terminal column references: carried slot, kBP (build payload) or -1
    int32_t ref[MGV_MAX_COLS + 2];
    uint32_t nref;
    unsigned long long* acc;
    GroupTableView gt;
    uint32_t smem_groups;  // shared group-table slots: power of two <= kMaxSmemGroups, 0 = none
    SinkView sink;
    CellsView cells;       // shared scan (kTermCells): the ranges' cells
};

constexpr int32_t kBP = 100;  // terminal reference to the build payload

// Batched execution (chain.cu kernels, batch.cu host side).
struct BatchItem {  // rows [lo, hi) of query q
    uint32_t q;
    uint32_t pad;
    uint64_t lo, hi;
};
// Shared-memory hash-table build (build_regions.cu).  A table is cut into
// regions of kRegionBuckets buckets; build rows are bucketed by the region of
// their home bucket, then one CTA per region inserts the region's rows into
// a shared-memory copy of the region and writes it back with coalesced
// stores.  A row whose run leaves its region is inserted afterwards into the
// global table.  A "job" is one table's build; a launch can build many.
constexpr uint32_t kRegionBuckets = 2048;      // 64 KiB of table per region
constexpr uint32_t kMaxRegionsPerJob = 16384;  // per-CTA region histogram: 64 KiB
constexpr uint64_t kRegionBuildMinRows = 1u << 16;  // smaller builds: one global CAS per row
struct RegionJob {
    TableView t;
    const int32_t* keys;
    const int32_t* pays;      // nullable
    const int32_t* filt;      // nullable: rows with filt <= bound only
    int32_t bound;
    uint32_t region0;         // first region of this job in the launch
    uint32_t nregions;
    uint32_t pad;
};
struct RegionScratch {
    uint32_t* hist;           // [regions] rows per region
    uint32_t* start;          // [regions + 1] first staging row of each region
    uint32_t* cursor;         // [regions]
    uint32_t* ovf_count;      // [1]
    unsigned long long* staging;  // [rows] {key, payload}, region-major
    unsigned long long* ovf;  // [rows] job << 32 | staging row, left for the global insert
};
// Host: group rows in ascending group order (radix sort).
void sort_group_rows(std::vector<mgv_group_row>& v);
inline uint32_t table_regions(const TableView& t) { return (t.nbuckets + kRegionBuckets - 1) / kRegionBuckets; }
size_t region_scratch_bytes(uint32_t regions, uint64_t rows);
RegionScratch carve_region_scratch(void* base, uint32_t regions, uint64_t rows);
// Items: explicit (job, rows) items, or (items == nullptr) rows [0, n) of
// job0 cut into items of rows_per_item.  fresh: the tables hold nothing yet
// and are not cleared beforehand; every region is written.  partitioned
// (one job, no items): the rows arrive partitioned on the table's radix bits,
// and are scattered by warps that sort their tiles by region.
// A fresh radix-laid-out table built from a partition op's single run on its
// radix bits (ends[p] = one past partition p's last row): per-partition
// staging in the partition's own range, then the region build.  Only when
// every partition slice is whole regions (region_build_partitioned_fits).
bool region_build_partitioned_fits(const TableView& t);
cudaError_t launch_build_regions_partitioned(const RegionJob& job, const unsigned long long* ends, uint64_t n,
                                             const RegionScratch& sc, cudaStream_t s, Context* ctx);
cudaError_t launch_build_regions(const RegionJob* d_jobs, const RegionJob& job0, uint32_t njobs,
                                 const struct BatchItem* items, uint32_t nitems, uint64_t n, uint64_t rows_per_item,
                                 uint32_t total_regions, uint32_t max_job_regions, const RegionScratch& sc,
                                 bool fresh, bool partitioned, cudaStream_t s, Context* ctx);

struct BatchOut {  // packed result region of a query
    GroupTableView gt;
    mgv_group_row* rows;
    uint32_t* count;
    uint32_t capacity;
    uint32_t pad;
};
cudaError_t launch_group_pack(const GroupTableView& gt, mgv_group_row* out, uint32_t* count, cudaStream_t s,
                              Context* ctx);
cudaError_t launch_batch(const ChainDev* d_qs, const BatchOut* d_outs, const BatchItem* probe_items, uint32_t n_probe,
                         const BatchItem* compact_items, uint32_t n_compact, int ctas_per_sm, uint32_t item_order,
                         cudaStream_t s, Context* ctx);
// Shared scans: the persistent probe -> cells kernel over (scan, rows)
// items (rows per item < 2^kCellRowBits), then the prefix over each scan's
// ranges (`scans` are host-side copies of the device descriptors' cells).
cudaError_t launch_cells(const ChainDev* d_scans, const BatchItem* items, uint32_t nitems, cudaStream_t s,
                         Context* ctx);
cudaError_t launch_cells_prefix(const CellsView& c, cudaStream_t s, Context* ctx);

// partition.cu
cudaError_t launch_partition_hist(const int32_t* const* cols, uint64_t n, bool has_sel, uint32_t sel_col,
                                  int32_t sel_bound, uint32_t key_col, uint32_t shift, uint32_t bits,
                                  unsigned long long* hist, cudaStream_t s, Context* ctx);
cudaError_t launch_partition_cursors(unsigned long long* hc, uint32_t bits, unsigned long long* acc, uint64_t max_rows,
                                    cudaStream_t s, Context* ctx);
cudaError_t launch_partition_scatter(const int32_t* const* cols, uint32_t ncols, uint64_t n, bool has_sel,
                                     uint32_t sel_col, int32_t sel_bound, uint32_t key_col, uint32_t shift,
                                     uint32_t bits, unsigned long long* cursors, int32_t* out, uint64_t out_stride,
                                     cudaStream_t s, Context* ctx);
cudaError_t launch_fill_i32(int32_t* p, uint64_t n, int32_t v, cudaStream_t s, Context* ctx);

// pool.cu
cudaError_t pool_init_device(Pool* p);
// Pops up to `want` ids into p->h_ids (sync); returns the count taken or
// reports drained / timeout through *status.
cudaError_t pool_pop_batch(Pool* p, uint32_t want, uint32_t timeout_us, uint32_t* got,
                           mgv_status* status);
cudaError_t pool_push_batch(Pool* p, const uint32_t* ids, uint32_t n);
cudaError_t pool_read_counters(Pool* p, uint32_t* available, uint32_t* producers);
cudaError_t pool_add_producers(Pool* p, int delta);

}  // namespace mgv

struct mgv_ctx : mgv::Context {};
struct mgv_pool : mgv::Pool {};
struct mgv_op : mgv::Op {};
