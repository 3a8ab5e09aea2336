/*
 * mgv.h -- C ABI of the B200 vector-at-a-time operator pipeline.
 *
 * Plain C: opaque handles, plain pointers and sizes, no C++ or torch types.
 * Every call returns an mgv_status; nothing here calls exit() or aborts
 * (the reference's gpu() macro exits on any CUDA error, src/common.cuh:12-23).
 * Device pointers are CUDA device addresses on the context's device;
 * `stream` arguments are cudaStream_t values (NULL = the context's stream).
 *
 * Each entry point names the reference interface it replaces
 * (paths relative to the reference project).
 */
#ifndef MGV_H_
#define MGV_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MGV_MAX_COLS 8
/* Rows per pool buffer by default: DEFAULT_BUFF_CAP, src/common.cuh:8-10. */
#define MGV_DEFAULT_BUFFER_ROWS (4u * 1024u * 1024u)

typedef enum mgv_status {
    MGV_OK = 0,
    MGV_EINVAL = 1,      /* bad argument                                  */
    MGV_ENOMEM = 2,      /* allocation failed / pool, table or output full */
    MGV_ETIMEDOUT = 3,   /* a bounded wait ran out                         */
    MGV_ECUDA = 4,       /* CUDA runtime error (see mgv_last_error_string) */
    MGV_EDEVICE = 5,     /* a kernel reported an error word                */
    MGV_ESTATE = 6,      /* call not valid in the object's current state   */
    MGV_EDRAINED = 7,    /* pool empty and no producer registered          */
    MGV_EUNSUPPORTED = 8 /* operator chain has no kernel                   */
} mgv_status;

typedef struct mgv_ctx mgv_ctx;
typedef struct mgv_pool mgv_pool;
typedef struct mgv_op mgv_op;

/* A vector buffer: up to MGV_MAX_COLS int32 columns of `capacity` rows in
 * device memory, `rows` of them valid.  Replaces buffer<int32_t, 4Mi>
 * (src/buffer.cuh:15-31: cnt, data, device), extended to several columns. */
typedef struct mgv_buffer {
    int32_t *cols[MGV_MAX_COLS];
    uint32_t ncols;
    uint32_t rows;
    uint32_t capacity;
    uint32_t id;
    int32_t device;
    uint32_t reserved;
} mgv_buffer;

/* ---- errors ----------------------------------------------------------- */

const char *mgv_status_string(mgv_status s);
/* Detail of the last failing call on this thread. */
const char *mgv_last_error_string(void);

/* ---- context ---------------------------------------------------------- */

typedef struct mgv_ctx_info {
    int32_t device;
    int32_t sm_count;
    uint64_t l2_bytes;
    uint64_t hbm_bytes;
    int32_t cc_major, cc_minor;
    char name[64];
} mgv_ctx_info;

/* Replaces the per-device set-up of buffer_manager::init
 * (src/buffer_manager.cu:38-61): device selection and a context stream. */
mgv_status mgv_ctx_create(int device, mgv_ctx **out);
mgv_status mgv_ctx_destroy(mgv_ctx *ctx);
mgv_status mgv_ctx_info_get(mgv_ctx *ctx, mgv_ctx_info *out);
/* Waits for `stream`, then reports and clears the device error word. */
mgv_status mgv_ctx_sync(mgv_ctx *ctx, void *stream);
/* Number of mgv kernel launches issued by this context so far. */
uint64_t mgv_ctx_launches(mgv_ctx *ctx);

/* Kernel tuning of a context (the reference fixes its launch shapes per
 * driver, e.g. <<<128, 1024>>> in src/main9.cu:593-594; here they are
 * runtime parameters, set by the caller or by the autotuner). */
typedef struct mgv_tuning {
    uint32_t probe_kernel;          /* 0 auto (= 3), 1 register prefetch, 2 bulk-copy
                                       staged, 3 staged with software-pipelined rounds */
    uint32_t probe_rows_per_thread; /* staged probe: 4 or 8 rows per thread per tile   */
    uint32_t probe_stages;          /* staged probe: 2, 4 or 6 tiles in flight         */
    uint32_t probe_ctas_per_sm;     /* 0 = as many as fit; 3 with 4 rows per thread
                                       selects the 3-CTA register budget               */
    float default_load_factor;      /* hash_build tables whose desc gives 0            */
    uint32_t groupby_smem_slots;    /* largest per-CTA shared group table: 0 (off) or a
                                       power of 2 in [64, 8192]; default 8192        */
    uint32_t select_ctas_per_sm;    /* select -> aggregate kernel: CTAs of 256 threads
                                       per SM, 1..8 (0 = the default, 2)             */
    uint32_t select_compact;        /* select -> aggregate: 0 = masked fold of every row
                                       (the default), 1 = warp-ballot compaction of the
                                       qualifying rows into 128-row vectors that the
                                       aggregate reads (unstable_select::consume_warp,
                                       src/operators/select3.cu:19-85); same results */
} mgv_tuning;

mgv_status mgv_ctx_set_tuning(mgv_ctx *ctx, const mgv_tuning *t);
mgv_status mgv_ctx_get_tuning(mgv_ctx *ctx, mgv_tuning *t);

/* ---- buffer pool (buffer_pool / buffer_manager) ------------------------ */

typedef struct mgv_pool_stats {
    uint32_t nbuffers;
    uint32_t capacity;
    uint32_t ncols;
    uint32_t available;     /* buffers on the device free stack           */
    uint32_t host_cached;   /* buffers held in the host-side cache        */
    uint32_t producers;
    uint64_t bytes;
} mgv_pool_stats;

/* One device slab carved into `nbuffers` buffers of `ncols` x `capacity`
 * int32 (buffer_manager::init's cudaMallocPitch slab,
 * src/buffer_manager.cu:98-134), with a device free stack
 * (src/threadsafe_device_stack.cuh:19-87, src/lockfree_stack.cuh:19-208). */
mgv_status mgv_pool_create(mgv_ctx *ctx, uint32_t nbuffers, uint32_t capacity,
                           uint32_t ncols, mgv_pool **out);
mgv_status mgv_pool_destroy(mgv_pool *pool);
/* Host acquire: buffer_manager::h_get_buffer (src/buffer_manager.cuh:78-94),
 * batching device pops through a host cache, with the bounded wait of
 * buffer_pool::acquire_buffer_blocked_unsafe (src/buffer_pool.cuh:83-96):
 * MGV_EDRAINED when the pool is empty and no producer is registered,
 * MGV_ETIMEDOUT when a producer is registered but nothing came back within
 * timeout_us. */
mgv_status mgv_buffer_acquire(mgv_pool *pool, uint32_t timeout_us, mgv_buffer **out);
/* Host release: buffer_manager::release_buffer (src/buffer_manager.cuh:96-118). */
mgv_status mgv_buffer_release(mgv_pool *pool, mgv_buffer *buf);
/* Copy `rows` int32 from host or device memory into column `col` and set
 * the buffer's row count: buffer_manager::overwrite
 * (src/buffer_manager.cu:214-218) / buffer_inspector::overwrite
 * (src/buffer.cuh:190-196).  Asynchronous on `stream`; with stream NULL
 * the copy has completed when the call returns (blocking = true). */
mgv_status mgv_buffer_write(mgv_buffer *buf, uint32_t col, const void *src, uint32_t rows,
                            void *stream);
/* Copy `rows` of column `col` to host or device memory and wait for it:
 * buffer_inspector::read (src/buffer.cuh:198-202). */
mgv_status mgv_buffer_read(const mgv_buffer *buf, uint32_t col, void *dst, uint32_t rows,
                           void *stream);
/* buffer_pool::register_producer / unregister_producer
 * (src/buffer_pool.cuh:136-165). */
mgv_status mgv_pool_register_producer(mgv_pool *pool);
mgv_status mgv_pool_unregister_producer(mgv_pool *pool);
mgv_status mgv_pool_stats_get(mgv_pool *pool, mgv_pool_stats *out);

/* Device view of a pool for kernels that acquire and release buffers
 * themselves (include/mgv_device.cuh: mgv_dev_buffer_acquire /
 * mgv_dev_buffer_release, the device-side get_buffer / release_buffer of
 * src/buffer_manager.cuh:50-64,96-129).  Every pointer is a device address. */
typedef struct mgv_pool_device {
    unsigned long long *head;  /* free stack head: {top id, tag}              */
    uint32_t *available;       /* buffers on the free stack                   */
    uint32_t *producers;       /* registered producers                        */
    uint32_t *next;            /* [nbuffers] free-stack links                 */
    int32_t *slab;             /* buffer i, column c at slab + (i*ncols + c)*capacity */
    uint32_t nbuffers;
    uint32_t capacity;
    uint32_t ncols;
    uint32_t reserved;
} mgv_pool_device;

/* Fills *out with the pool's device view (buffer_manager's __constant__ pool
 * pointer, src/buffer_manager.cuh:40-48, handed to kernels explicitly). */
mgv_status mgv_pool_device_get(mgv_pool *pool, mgv_pool_device *out);

/* ---- operators -------------------------------------------------------- */
/*
 * Operators form push chains as in the reference (d_operator_t with a
 * parent pointer, src/operators/operator.cuh:42-86): rows pushed into an
 * operator flow to its parent.  A chain from the operator that receives
 * data up to its terminal (aggregate, groupby, hash_build, sink, partition)
 * runs as ONE fused kernel per consume call; there is no per-row dispatch.
 *
 * Column numbering: the rows entering a chain carry the consumed buffer's
 * columns 0..ncols-1; select keeps them all; hash_probe appends the
 * matching build row's payload as column `ncols` (one output row per
 * match).
 */

/* unstable_select with less_eq_than (src/operators/select3.cuh:10-48):
 * keeps rows with cols[col] <= bound (signed compare). */
typedef struct mgv_select_desc {
    uint32_t col;
    int32_t bound;
} mgv_select_desc;

/* aggregation (src/operators/aggregation.cu:5-66), widened: COUNT(*) and
 * int64 SUM(cols[sum_col_a] + cols[sum_col_b]); -1 leaves a term out. */
typedef struct mgv_aggregate_desc {
    int32_t sum_col_a;
    int32_t sum_col_b;
} mgv_aggregate_desc;

typedef struct mgv_agg_result {
    int64_t count;
    int64_t sum;
} mgv_agg_result;

/* hashjoin_builder (src/operators/hashjoin.cu:40-60), as an open-addressing
 * table of 32-byte buckets (4 {key, payload} slots, one L2 sector).
 * expected_rows sizes the table; load_factor in (0, 0.95] (0 = the context's
 * default); payload_col -1 stores payload 0.  radix_bits > 0 lays the table
 * out in 2^radix_bits regions, one per value of (key >> radix_shift) &
 * (2^radix_bits - 1), so that a build fed partition by partition (by a
 * partition operator with the same bits) touches one region at a time. */
typedef struct mgv_hash_build_desc {
    uint32_t key_col;
    int32_t payload_col;
    uint64_t expected_rows;
    float load_factor;
    uint32_t radix_bits;
    uint32_t radix_shift;
    uint32_t reserved;
} mgv_hash_build_desc;

typedef struct mgv_hash_build_info {
    uint64_t rows;            /* rows inserted                               */
    uint64_t nbuckets;
    uint64_t table_bytes;
    uint64_t reserved_key_rows; /* build rows whose key is INT32_MIN         */
    uint32_t has_duplicates;  /* 1 if some key was inserted more than once   */
    uint32_t reserved;
} mgv_hash_build_info;

/* hashjoin probe (src/operators/hashjoin.cu:134-182): each row is matched
 * against every build row with an equal key (duplicates all match). */
typedef struct mgv_hash_probe_desc {
    uint32_t key_col;
    uint32_t reserved;
    mgv_op *build;            /* a closed hash_build operator              */
} mgv_hash_probe_desc;

/* Materialises rows into buffers of `pool` (the pool's ncols columns are
 * filled from the incoming columns 0..ncols-1): the reference's
 * gpu_to_cpu output buffers with swap-on-full
 * (src/operators/gpu_to_cpu.cu:41-105, src/buffer_manager.cuh:147-176). */
typedef struct mgv_sink_desc {
    mgv_pool *pool;
    uint32_t max_buffers;     /* 0 = as many as the pool has               */
    uint32_t reserved;
} mgv_sink_desc;

/* Hash GROUP BY (no reference counterpart; the reference has a global SUM
 * only): int64 SUM(cols[value_col]) and COUNT(*) per distinct
 * cols[group_col] (value_col -1: COUNT only; either may be `ncols`, the
 * build payload appended by a hash_probe).  max_groups sizes the table. */
typedef struct mgv_groupby_desc {
    uint32_t group_col;
    int32_t value_col;
    uint32_t max_groups;
    uint32_t reserved;
} mgv_groupby_desc;

typedef struct mgv_group_row {
    int32_t group;
    int32_t pad;
    int64_t sum;
    int64_t count;
} mgv_group_row;

/* split (src/operators/split.cu:49-118, partition by x & 1), generalised to
 * 2^radix_bits partitions by (cols[key_col] >> radix_shift) & (2^bits - 1):
 * the in-GPU exchange.  Rows are stored partition-major (capacity
 * max_rows; a consume does not wait for the device); close() pushes them
 * into the parent chain and then closes it.  Rows past max_rows are dropped
 * and close() returns MGV_ENOMEM. */
typedef struct mgv_partition_desc {
    uint32_t key_col;
    uint32_t radix_bits;
    uint32_t radix_shift;
    uint32_t reserved;
    uint64_t max_rows;
} mgv_partition_desc;

/* The routing step of split / hash_exchange on its own
 * (src/operators/split.cu:49-118, src/main9.cu:104-148), for callers that
 * move the partitions themselves (the multi-GPU hash exchange sends
 * partition p to rank p): the rows of device columns cols[0..ncols) are
 * written partition-major, by (cols[key_col] >> radix_shift) &
 * (2^radix_bits - 1), into `out` (column c at out + c * out_stride,
 * out_stride >= rows), and counts[p] (host memory, 2^radix_bits entries)
 * receives the rows of partition p.  Rows keep no order within a partition.
 * radix_bits in 1..12.  Waits for `stream`. */
mgv_status mgv_partition_columns(mgv_ctx *ctx, const int32_t *const *cols, uint32_t ncols, uint64_t rows,
                                 uint32_t key_col, uint32_t radix_bits, uint32_t radix_shift, int32_t *out,
                                 uint64_t out_stride, uint64_t *counts, void *stream);

mgv_status mgv_op_create_select(mgv_ctx *ctx, const mgv_select_desc *desc, mgv_op *parent,
                                mgv_op **out);
mgv_status mgv_op_create_groupby(mgv_ctx *ctx, const mgv_groupby_desc *desc, mgv_op **out);
mgv_status mgv_op_create_partition(mgv_ctx *ctx, const mgv_partition_desc *desc, mgv_op *parent,
                                   mgv_op **out);
mgv_status mgv_op_create_aggregate(mgv_ctx *ctx, const mgv_aggregate_desc *desc, mgv_op **out);
mgv_status mgv_op_create_hash_build(mgv_ctx *ctx, const mgv_hash_build_desc *desc, mgv_op **out);
mgv_status mgv_op_create_hash_probe(mgv_ctx *ctx, const mgv_hash_probe_desc *desc,
                                    mgv_op *parent, mgv_op **out);
mgv_status mgv_op_create_sink(mgv_ctx *ctx, const mgv_sink_desc *desc, mgv_op **out);
/* Operators are destroyed explicitly (the reference never frees them,
 * src/operators/operator.cu:161-163); parents are not destroyed. */
mgv_status mgv_op_destroy(mgv_op *op);

/* d_operator_t::open (src/operators/operator.cu:126-135): opens the
 * parents first, then resets this operator's device state. */
mgv_status mgv_op_open(mgv_op *op, void *stream);
/* launch_consume_pipeline over one buffer (src/operators/exchange.cu:160-194):
 * every valid row of `buf` is pushed through the chain in one launch. */
mgv_status mgv_op_consume(mgv_op *op, const mgv_buffer *buf, void *stream);
/* The same over device-resident columns of any length (the reference's
 * generator aliasing a user array into buffers, src/operators/generators.cu:55-90). */
mgv_status mgv_op_consume_columns(mgv_op *op, const int32_t *const *cols, uint32_t ncols,
                                  uint64_t rows, void *stream);
/* Host ingest: the reference's generator slicing a host column into pool
 * buffers, and consumer::consume copying each buffer to the device before
 * its consume kernel (src/operators/generators.cu:55-90,
 * src/operators/exchange.cu:196-291), with the copies overlapped.  `rows`
 * rows of the host columns host_cols[0..ncols) are cut into slices of the
 * pool's buffer capacity (ncols <= the pool's columns; up to 3 buffers of
 * `pool` in flight); slice k+1 is copied host -> device on the operator's
 * own copy stream while slice k is consumed on `stream`, so the copies
 * and the kernels run at the same time.  Pinned host memory copies fastest;
 * pageable memory works.  Returns when every slice has been consumed: the
 * host columns may be reused and the buffers are back in the pool.  Columns
 * larger than device memory stream through a bounded pool this way. */
mgv_status mgv_op_consume_host(mgv_op *op, mgv_pool *pool, const int32_t *const *host_cols, uint32_t ncols,
                               uint64_t rows, void *stream);
/* d_operator_t::close (src/operators/operator.cu:150-159): flushes, closes
 * the parents, waits for the stream and reports device errors. */
mgv_status mgv_op_close(mgv_op *op, void *stream);
/* Result of a closed terminal operator, copied to host memory:
 *   aggregate  -> mgv_agg_result
 *   hash_build -> mgv_hash_build_info
 *   sink       -> uint64_t row count
 *   groupby    -> mgv_group_row[groups], sorted by group
 *   partition  -> uint64_t[2^radix_bits] rows per partition
 * `needed` (may be NULL) receives the size in bytes. */
mgv_status mgv_op_result(mgv_op *op, void *out, size_t bytes, size_t *needed);

/* Rows of a closed sink: copies up to `max_rows` rows of column `col`
 * (in buffer order) into dst (host or device memory). */
mgv_status mgv_sink_read(mgv_op *sink, uint32_t col, int32_t *dst, uint64_t max_rows,
                         uint64_t *rows);

/* Result delivery channel (replaces gpu_to_cpu's catcher thread and the pool
 * buffer swap, src/operators/gpu_to_cpu.cu:41-165, src/buffer_manager.cuh:147-176).
 * Between consume calls of an open sink: waits for `stream`, then starts
 * copying every row gathered so far (column c to dst_cols[c], c < ncols;
 * host or device memory, pinned host memory copies fastest) on the sink's
 * own copy stream and starts the sink over, so the next consume overlaps
 * the copy and one open sink can deliver any number of rows through a
 * bounded pool.  The copy is complete, and its buffers are back in the
 * pool, when the next mgv_sink_drain or mgv_op_close of the sink returns;
 * read the destination only then.  Each consume between drains must fit
 * the pool's free buffers (otherwise the drain reports MGV_ENOMEM).  With
 * dst_cols NULL it only completes the copy in flight and sets *rows to the
 * rows waiting.  If more rows wait than cap_rows, nothing is copied and the
 * call fails with MGV_EINVAL. */
mgv_status mgv_sink_drain(mgv_op *sink, int32_t *const *dst_cols, uint32_t ncols, uint64_t cap_rows,
                          uint64_t *rows, void *stream);

/* ---- seeded synthetic columns ------------------------------------------ */
/*
 * Fill device memory with seeded columns; value i is a pure function of
 * (seed, stream_id, i), identical to the CPU oracle's generator.  No
 * reference counterpart: the reference fills host arrays with unseeded
 * rand() / mt19937 (src/main8.cu:169, src/main9.cu:556-566).
 */
/* Uniform int32 in [lo, lo + range), range in [1, 2^32]. */
mgv_status mgv_gen_uniform(mgv_ctx *ctx, int32_t *dst, uint64_t n, uint64_t seed, uint32_t stream_id,
                           int64_t lo, uint64_t range, void *stream);
/* A seeded permutation of 0..n-1. */
mgv_status mgv_gen_perm(mgv_ctx *ctx, int32_t *dst, uint64_t n, uint64_t seed, void *stream);
/* Join probe keys: with probability hit_num/2^32 a uniformly chosen key of
 * the permutation mgv_gen_perm(build_seed, nbuild), else uniform in
 * [miss_lo, miss_lo + miss_range).  *hits (may be NULL) receives how many
 * rows took the first branch. */
mgv_status mgv_gen_probe_keys(mgv_ctx *ctx, int32_t *dst, uint64_t n, uint64_t seed, uint64_t build_seed,
                              uint64_t nbuild, uint32_t hit_num, int64_t miss_lo, uint64_t miss_range,
                              uint64_t *hits, void *stream);
/* Zipf(s) group ids in [0, groups), 0 the most frequent. */
mgv_status mgv_gen_zipf(mgv_ctx *ctx, int32_t *dst, uint64_t n, uint64_t seed, uint32_t stream_id,
                        uint32_t groups, double s, void *stream);

/* ---- batched queries ---------------------------------------------------- */
/*
 * Many independent select -> hash join -> group-by queries executed
 * together: per-query tables in one device arena, one persistent build
 * launch and one persistent probe launch over (query, rows) work items,
 * results packed into one copy to the host, the whole sequence captured
 * once and replayed as a CUDA graph.  No reference counterpart (the
 * reference runs one pipeline per plan, src/main9.cu:371-631).
 */
typedef struct mgv_query_desc {
    const int32_t *build_keys;      /* device columns                          */
    const int32_t *build_payloads;  /* may be NULL                             */
    uint64_t build_rows;
    const int32_t *probe_key;
    const int32_t *probe_filter;
    const int32_t *probe_group;
    const int32_t *probe_value;
    uint64_t probe_rows;
    int32_t filter_bound;           /* rows with filter <= bound are probed    */
    uint32_t max_groups;            /* upper bound on distinct groups          */
} mgv_query_desc;

typedef struct mgv_batch_config {
    float load_factor;          /* join tables (0 = the context's default)      */
    uint32_t build_item_rows;   /* rows per build work item (0 = 65536)         */
    uint32_t probe_item_rows;   /* rows per probe work item (0 = 32768)         */
    uint32_t probe_ctas_per_sm; /* 0 = as many as fit                           */
    uint32_t use_graph;         /* 1 = capture once, replay as a CUDA graph     */
    uint32_t item_order;        /* 0 = work items dealt round-robin to the CTAs
                                   (all CTAs on neighbouring items, so the
                                   tables in use stay in L2); 1 = one
                                   contiguous run of items per CTA             */
    uint32_t reserved[2];
} mgv_batch_config;

typedef struct mgv_batch mgv_batch;

typedef struct mgv_batch_stats {
    uint64_t arena_bytes;
    uint32_t queries, build_items, probe_items, graph;
    double last_run_ms;         /* host wall clock of the last run (incl. the copy to host) */
} mgv_batch_stats;

/* config NULL: the configuration the context's autotuner chose last, else defaults. */
mgv_status mgv_batch_create(mgv_ctx *ctx, const mgv_query_desc *queries, uint32_t nq,
                            const mgv_batch_config *config, mgv_batch **out);
/* Runs every query; results are on the host when it returns. */
mgv_status mgv_batch_run(mgv_batch *b, void *stream);
/* The same queries one at a time through the plain operator pipeline
 * (partition-free select -> hash_probe -> groupby after a hash_build), the
 * comparison baseline; its results are kept apart from the batch's. */
mgv_status mgv_batch_run_plain(mgv_batch *b, void *stream);
/* Groups of query q sorted by group (plain = 1: of the last plain run). */
mgv_status mgv_batch_result(mgv_batch *b, uint32_t q, int plain, mgv_group_row *out, uint64_t cap,
                            uint64_t *rows);
mgv_status mgv_batch_stats_get(mgv_batch *b, mgv_batch_stats *out);
mgv_status mgv_batch_destroy(mgv_batch *b);
/* Project autotuner: times candidate configurations (load factor, probe
 * item rows, CTAs per SM) on these queries and returns the fastest; the
 * context remembers it for mgv_batch_create(config = NULL). */
mgv_status mgv_batch_autotune(mgv_ctx *ctx, const mgv_query_desc *queries, uint32_t nq, mgv_batch_config *out);

/* ---- serving ------------------------------------------------------------ */
/*
 * A query server with continuous batching over resident build tables (no
 * reference counterpart).  Requests (select -> join -> group-by against a
 * registered table) may be submitted at any time; a scheduler thread
 * admits them in arrival order while `memory_budget` bytes of device memory
 * allow (group table and result region per request, plus the resident
 * tables), launches admitted requests together as one batch on a free
 * stream, and keeps up to `max_inflight` batches on the GPU, so requests
 * arriving while others run are admitted as streams and memory free up.
 * plain = 1 serves requests one at a time through the operator API instead
 * (the per-query baseline).
 */
typedef struct mgv_server_config {
    uint64_t memory_budget;  /* bytes for resident tables + in-flight requests */
    uint32_t max_batch;      /* requests per batch (0 = 256)                  */
    uint32_t max_inflight;   /* batches on the GPU at once (0 = 2, max 16)    */
    float load_factor;       /* resident join tables (0 = context default)    */
    uint32_t plain;          /* 1 = one request at a time, operator API       */
    uint32_t batch_solo;     /* 0: while nothing is in flight and at most four
                              * requests wait, the oldest runs alone through
                              * the operator chain (lower latency); batches
                              * form once a longer queue builds up;
                              * 1: every request is batched                   */
    uint32_t separate_scans; /* 0: requests of one batch over the same table,
                              * probe columns and row count that differ only in
                              * their filter bound share one scan (the columns
                              * read and the table probed once, each matched row
                              * aggregated once per filter range); 1: every
                              * request scans alone                          */
} mgv_server_config;

typedef struct mgv_server_request {
    uint32_t table;          /* from mgv_server_add_table                     */
    uint32_t reserved;
    const int32_t *probe_key, *probe_filter, *probe_group, *probe_value;  /* device */
    uint64_t probe_rows;
    int32_t filter_bound;
    uint32_t max_groups;
} mgv_server_request;

typedef struct mgv_server_stats {
    uint64_t submitted, completed, batches, rejected;
    double p50_ms, p99_ms, mean_ms, max_ms;  /* submit -> result on the host */
    double mean_batch;
    uint64_t resident_table_bytes, peak_bytes;
    uint64_t solo;           /* requests answered alone by the operator chain */
    uint64_t shared_scans;   /* shared scans launched                         */
    uint64_t scan_queries;   /* requests answered by shared scans             */
} mgv_server_stats;

typedef struct mgv_server mgv_server;

mgv_status mgv_server_create(mgv_ctx *ctx, const mgv_server_config *cfg, mgv_server **out);
/* Builds a hash table on (keys, payloads) and keeps it resident. */
mgv_status mgv_server_add_table(mgv_server *s, const int32_t *keys, const int32_t *payloads, uint64_t rows,
                                uint32_t *table_id);
mgv_status mgv_server_submit(mgv_server *s, const mgv_server_request *r, uint64_t *ticket);
/* Waits (bounded by timeout_ms) for a request and copies up to cap of its
 * groups to out, in no particular order (as GROUP BY defines); *rows = the
 * number of groups. */
mgv_status mgv_server_wait(mgv_server *s, uint64_t ticket, uint32_t timeout_ms, mgv_group_row *out,
                           uint64_t cap, uint64_t *rows, double *latency_ms);
mgv_status mgv_server_stats_get(mgv_server *s, mgv_server_stats *out);
mgv_status mgv_server_reset_stats(mgv_server *s);
mgv_status mgv_server_destroy(mgv_server *s);

/* ---- hash join without allocation ------------------------------------- */

/* Largest build side mgv_hash_join_noalloc accepts. */
#define MGV_NOALLOC_MAX_BUILD_ROWS (1u << 20)

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory: code running under another framework's allocator or memory budget
 * (which owns every byte and forbids cudaMalloc), plugins and embedded hosts
 * that are handed only pre-allocated buffers, and processes whose device
 * memory is already spoken for.  Builds a hash table on the build columns and
 * probes it with the probe columns, writing d_result[0] = COUNT(matches) and
 * d_result[1] = SUM(build payload + probe payload) (int64, device memory) --
 * the result of create_count_join_1G_pipeline.  Needs no context and
 * allocates nothing: the table lives in a fixed file-scope device array of
 * MGV_NOALLOC_MAX_BUILD_ROWS rows (about 20 MiB per device, committed by the
 * first call on that device -- or at module load under
 * CUDA_MODULE_LOADING=EAGER -- and held until the process exits); a larger
 * build side is rejected with MGV_EINVAL.  The first call on a device looks
 * up the array's device address and should come before any stream capture.
 * All calls share the array and clear it first: calls that overlap on the
 * GPU race.  Payload pointers may be NULL (payload 0).  Runs with `device`
 * current and restores the caller's current device; waits for `stream`
 * before returning. */
mgv_status mgv_hash_join_noalloc(int device, const int32_t *build_keys, const int32_t *build_payloads,
                                 uint64_t build_rows, const int32_t *probe_keys, const int32_t *probe_payloads,
                                 uint64_t probe_rows, int64_t *d_result, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MGV_H_ */
