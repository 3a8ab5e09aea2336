// kernels.cu -- fused operator kernels for sm_100a.
//
// One kernel per operator chain shape (static dispatch; the reference
// dispatches through a variant visitor for every 128-row vector,
// src/operators/operator.cu:137-148).  Columns are streamed with 256-bit
// loads that skip L1 and are evicted first from L2; hash buckets are read
// as one 32-byte sector each.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_common.cuh"
#include "hash_table.cuh"
#include "mgv_internal.h"

namespace mgv {

constexpr int kBlock = 256;

int occupancy_grid(const void* kernel, int block, size_t smem, const Context* ctx) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    return per_sm * ctx->prop.multiProcessorCount;
}

static inline bool aligned32(const void* p) { return p == nullptr || ((uintptr_t)p & 31u) == 0; }

// ---------------------------------------------------------------------------
// fill
// ---------------------------------------------------------------------------

__global__ void k_fill_u64(unsigned long long* p, uint64_t n, unsigned long long v) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

cudaError_t launch_fill_u64(unsigned long long* p, uint64_t n, unsigned long long v, cudaStream_t s,
                            Context* ctx) {
    if (n == 0) return cudaSuccess;
    uint64_t want = (n + kBlock - 1) / kBlock;
    int grid = (int)(want < (uint64_t)ctx->prop.multiProcessorCount * 8
                         ? want
                         : (uint64_t)ctx->prop.multiProcessorCount * 8);
    k_fill_u64<<<grid, kBlock, 0, s>>>(p, n, v);
    ctx->launches++;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// select -> aggregate  (select3 + aggregation, src/operators/select3.cu:19-85,
// src/operators/aggregation.cu:26-52)
//
// COUNT and int64 SUM(a + b) over rows with f <= bound.  The reference
// compacts qualifying rows into 128-row vectors and re-reads them in the
// aggregation; for an associative aggregate the masked sum is exact and
// needs no compaction, so each thread folds 8 rows per 256-bit load.
// ---------------------------------------------------------------------------

template <bool SEL, bool HASA, bool HASB, bool VEC>
__global__ void __launch_bounds__(kBlock) k_select_agg(const int32_t* __restrict__ f, int32_t bound,
                                                       const int32_t* __restrict__ a,
                                                       const int32_t* __restrict__ b, uint64_t n,
                                                       unsigned long long* acc) {
    unsigned long long cnt = 0, sum = 0;
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    uint64_t done = 0;
    if (VEC) {
        const uint64_t nvec = n / 8;
        for (uint64_t v = (uint64_t)blockIdx.x * kBlock + threadIdx.x; v < nvec; v += stride) {
            int32_t fv[8], av[8], bv[8];
            if (SEL) ld_stream8(f + 8 * v, fv);
            if (HASA) ld_stream8(a + 8 * v, av);
            if (HASB) ld_stream8(b + 8 * v, bv);
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const bool p = !SEL || fv[r] <= bound;
                long long t = 0;
                if (HASA) t += av[r];
                if (HASB) t += bv[r];
                cnt += p;
                sum += p ? (unsigned long long)t : 0ull;
            }
        }
        done = nvec * 8;
    }
    for (uint64_t i = done + (uint64_t)blockIdx.x * kBlock + threadIdx.x; i < n; i += stride) {
        const bool p = !SEL || f[i] <= bound;
        long long t = 0;
        if (HASA) t += a[i];
        if (HASB) t += b[i];
        cnt += p;
        sum += p ? (unsigned long long)t : 0ull;
    }
    block_accumulate2<kBlock>(cnt, sum, acc);
}

template <bool SEL, bool HASA, bool HASB>
static cudaError_t select_agg_v(const int32_t* f, int32_t bound, const int32_t* a, const int32_t* b,
                                uint64_t n, unsigned long long* acc, cudaStream_t s, Context* ctx) {
    const bool vec = aligned32(f) && aligned32(a) && aligned32(b);
    const void* k = vec ? (const void*)k_select_agg<SEL, HASA, HASB, true>
                        : (const void*)k_select_agg<SEL, HASA, HASB, false>;
    int grid = occupancy_grid(k, kBlock, 0, ctx);
    uint64_t need = (n / 8 + kBlock - 1) / kBlock + 1;
    if ((uint64_t)grid > need) grid = (int)need;
    if (vec)
        k_select_agg<SEL, HASA, HASB, true><<<grid, kBlock, 0, s>>>(f, bound, a, b, n, acc);
    else
        k_select_agg<SEL, HASA, HASB, false><<<grid, kBlock, 0, s>>>(f, bound, a, b, n, acc);
    ctx->launches++;
    return cudaGetLastError();
}

cudaError_t launch_select_agg(const int32_t* filt, int32_t bound, bool has_sel, const int32_t* a,
                              const int32_t* b, uint64_t n, unsigned long long* acc, cudaStream_t s,
                              Context* ctx) {
    if (n == 0) return cudaSuccess;
    const int code = (has_sel ? 4 : 0) | (a ? 2 : 0) | (b ? 1 : 0);
    switch (code) {
        case 0: return select_agg_v<false, false, false>(filt, bound, a, b, n, acc, s, ctx);
        case 1: return select_agg_v<false, false, true>(filt, bound, a, b, n, acc, s, ctx);
        case 2: return select_agg_v<false, true, false>(filt, bound, a, b, n, acc, s, ctx);
        case 3: return select_agg_v<false, true, true>(filt, bound, a, b, n, acc, s, ctx);
        case 4: return select_agg_v<true, false, false>(filt, bound, a, b, n, acc, s, ctx);
        case 5: return select_agg_v<true, false, true>(filt, bound, a, b, n, acc, s, ctx);
        case 6: return select_agg_v<true, true, false>(filt, bound, a, b, n, acc, s, ctx);
        default: return select_agg_v<true, true, true>(filt, bound, a, b, n, acc, s, ctx);
    }
}

// ---------------------------------------------------------------------------
// hash build  (hashjoin_builder::consume_warp, src/operators/hashjoin.cu:40-60)
//
// The reference head-inserts into chains with atomicExch on a 2^L bucket
// array plus a separate next[] array (two dependent random accesses per
// probe step).  Here a row is claimed into the first free slot of its
// bucket run with one 64-bit atomicCAS of {key, payload}; slots of a run
// fill in order, so a lookup stops at the first empty slot.  Duplicate keys
// are kept (every one matches, as in the reference) and flagged, so that a
// table without duplicates can be probed with early exit.
// ---------------------------------------------------------------------------

template <bool SEL>
__global__ void __launch_bounds__(kBlock) k_build(const int32_t* __restrict__ keys,
                                                  const int32_t* __restrict__ pays,
                                                  const int32_t* __restrict__ filt, int32_t bound,
                                                  uint64_t n, TableView t, uint32_t* err) {
    bool dup = false;
    uint32_t inserted = 0;
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    for (uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x; i < n; i += stride) {
        if (SEL && !(filt[i] <= bound)) continue;
        bool ok;
        table_insert(t, keys[i], pays ? pays[i] : 0, err, dup, ok);
        inserted += ok;
    }
    unsigned long long tot = warp_sum_u64(inserted);
    const unsigned any_dup = __any_sync(0xffffffffu, dup);
    if (lane_id() == 0) {
        if (tot) atomicAdd(t.meta + 2, tot);
        if (any_dup) atomicOr(t.meta + 3, 1ull);
    }
}

cudaError_t launch_build(const int32_t* keys, const int32_t* pays, const int32_t* filt,
                         int32_t bound, bool has_sel, uint64_t n, const TableView& t,
                         cudaStream_t s, Context* ctx) {
    if (n == 0) return cudaSuccess;
    const void* k = has_sel ? (const void*)k_build<true> : (const void*)k_build<false>;
    int grid = occupancy_grid(k, kBlock, 0, ctx);
    uint64_t need = (n + kBlock - 1) / kBlock;
    if ((uint64_t)grid > need) grid = (int)need;
    if (has_sel)
        k_build<true><<<grid, kBlock, 0, s>>>(keys, pays, filt, bound, n, t, ctx->d_err);
    else
        k_build<false><<<grid, kBlock, 0, s>>>(keys, pays, filt, bound, n, t, ctx->d_err);
    ctx->launches++;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// hash probe -> aggregate  (hashjoin::consume_warp, src/operators/hashjoin.cu:134-182,
// then aggregation)
//
// The reference walks 4 chains per lane with dependent loads.  Here each
// thread takes 8 probe rows from one 256-bit load per column, issues 8
// independent 32-byte bucket loads, and only continues to the next bucket
// when a bucket is full and (for unique tables) the key was not found.
// The next tile's keys are loaded before the current tile's buckets are
// examined, so column streaming and table lookups overlap.
// ---------------------------------------------------------------------------

template <bool UNIQUE, bool VEC>
__global__ void __launch_bounds__(kBlock, 2)
    k_probe_agg(const int32_t* __restrict__ keys, const int32_t* __restrict__ pays, uint64_t n,
                TableView t, uint32_t sum_mode, unsigned long long* acc) {
    constexpr int R = 8;
    constexpr uint64_t kTile = (uint64_t)kBlock * R;
    const uint64_t ntiles = (n + kTile - 1) / kTile;
    const bool add_bp = sum_mode & 1u, add_pp = (sum_mode & 2u) && pays;
    unsigned long long cnt = 0, sum = 0;

    int32_t k[R], p[R];
    uint32_t valid = 0;
    auto load_tile = [&](uint64_t tile, int32_t (&kk)[R], int32_t (&pp)[R], uint32_t& vv) {
        const uint64_t r0 = tile * kTile + (uint64_t)threadIdx.x * R;
        if (VEC && r0 + R <= n) {
            ld_stream8(keys + r0, kk);
            if (add_pp) ld_stream8(pays + r0, pp);
            else {
#pragma unroll
                for (int r = 0; r < R; ++r) pp[r] = 0;
            }
            vv = 0xffu;
        } else {
            vv = 0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const bool in = r0 + r < n;
                kk[r] = in ? keys[r0 + r] : 0;
                pp[r] = (in && add_pp) ? pays[r0 + r] : 0;
                vv |= (uint32_t)in << r;
            }
        }
    };

    uint64_t tile = blockIdx.x;
    if (tile < ntiles) load_tile(tile, k, p, valid);
    while (tile < ntiles) {
        uint32_t w[R][8];
#pragma unroll
        for (int r = 0; r < R; ++r) ld_bucket(t.slots + 4ull * bucket_of(k[r], t.nbuckets), w[r]);

        // Prefetch the next tile while the bucket loads are in flight.
        const uint64_t next = tile + gridDim.x;
        int32_t nk[R], np[R];
        uint32_t nvalid = 0;
        if (next < ntiles) load_tile(next, nk, np, nvalid);

#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (!((valid >> r) & 1u)) continue;
            uint32_t mc;
            long long ms;
            if (k[r] == kEmptyKey) {
                mc = (uint32_t)t.meta[0];
                ms = (long long)t.meta[1];
            } else {
                bool more;
                match_bucket<UNIQUE>(w[r], k[r], mc, ms, more);
                if (more) {
                    const Matches x = probe_rest<UNIQUE>(t.slots, t.nbuckets, k[r], bucket_of(k[r], t.nbuckets));
                    mc += x.count;
                    ms += (long long)x.sum;
                }
            }
            cnt += mc;
            long long add = 0;
            if (add_bp) add += ms;
            if (add_pp) add += (long long)mc * p[r];
            sum += (unsigned long long)add;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            k[r] = nk[r];
            p[r] = np[r];
        }
        valid = nvalid;
        tile = next;
    }
    block_accumulate2<kBlock>(cnt, sum, acc);
}

cudaError_t launch_probe_agg(const int32_t* keys, const int32_t* pays, uint64_t n,
                             const TableView& t, bool unique, uint32_t sum_mode,
                             unsigned long long* acc, cudaStream_t s, Context* ctx) {
    if (n == 0) return cudaSuccess;
    if (ctx->tuning.probe_kernel != 1) {
        cudaError_t e = launch_probe_agg_staged(keys, pays, n, t, unique, sum_mode, acc, s, ctx);
        if (e != cudaErrorNotSupported) return e;
    }
    const bool vec = aligned32(keys) && aligned32(pays);
    const void* k = unique ? (vec ? (const void*)k_probe_agg<true, true> : (const void*)k_probe_agg<true, false>)
                           : (vec ? (const void*)k_probe_agg<false, true> : (const void*)k_probe_agg<false, false>);
    int grid = occupancy_grid(k, kBlock, 0, ctx);
    const uint64_t ntiles = (n + (uint64_t)kBlock * 8 - 1) / ((uint64_t)kBlock * 8);
    if ((uint64_t)grid > ntiles) grid = (int)ntiles;
    if (unique) {
        if (vec) k_probe_agg<true, true><<<grid, kBlock, 0, s>>>(keys, pays, n, t, sum_mode, acc);
        else k_probe_agg<true, false><<<grid, kBlock, 0, s>>>(keys, pays, n, t, sum_mode, acc);
    } else {
        if (vec) k_probe_agg<false, true><<<grid, kBlock, 0, s>>>(keys, pays, n, t, sum_mode, acc);
        else k_probe_agg<false, false><<<grid, kBlock, 0, s>>>(keys, pays, n, t, sum_mode, acc);
    }
    ctx->launches++;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Generic chain: [select] -> [probe] -> sink
//
// Warp-ballot select as in unstable_select::consume_warp
// (src/operators/select3.cu:19-85): each warp takes 128-row windows,
// evaluates the predicate, and compacts the qualifying rows with
// __ballot_sync/__popc into a per-warp shared-memory ring of 256 rows per
// carried column, then pushes full 128-row vectors on (the reference's
// 160-slot ring and consume_warp(x, 128)).  The downstream stage (probe,
// sink) therefore always works on dense vectors.
// ---------------------------------------------------------------------------

struct ChainDev {
    const int32_t* cols[MGV_MAX_COLS];
    uint32_t ncols;
    uint32_t sel_col;
    int32_t sel_bound;
    uint32_t probe_col;
    uint64_t n;
    TableView table;
};

__device__ __forceinline__ uint32_t pool_pop(PoolDev* p, uint32_t tries) {
    for (uint32_t i = 0; i < tries; ++i) {
        unsigned long long h = atomicAdd(&p->head, 0ull);
        uint32_t top = (uint32_t)h;
        if (top == kNil) return kNil;
        uint32_t nxt = *((volatile uint32_t*)&p->next[top]);
        unsigned long long nh = (((h >> 32) + 1ull) << 32) | nxt;
        if (atomicCAS(&p->head, h, nh) == h) {
            atomicSub(&p->available, 1u);
            return top;
        }
    }
    return kNil;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Buffer id for chunk c of a sink; the warp that owns row c*capacity takes
// a buffer from the pool and publishes it, everyone else waits for it with
// a bounded wait (swap-on-full, src/buffer_manager.cuh:147-176).
__device__ uint32_t sink_chunk(const SinkView& s, uint32_t c, bool opener, uint32_t* err) {
    if (opener) {
        uint32_t id = pool_pop(s.pool, 4096);
        if (id == kNil) {
            set_error(err, kDevOverflow, 3);
            id = kNil - 1;  // published "no buffer" marker
        }
        atomicExch(s.chain + c, id);
        return id;
    }
    const unsigned long long t0 = global_ns();
    for (;;) {
        uint32_t id = *((volatile uint32_t*)(s.chain + c));
        if (id != kNil) return id;
        if (global_ns() - t0 > 2000000000ull) {  // 2 s
            set_error(err, kDevTimeout, 4);
            return kNil - 1;
        }
        __nanosleep(64);
    }
}

// Write `cnt` rows per lane, reserved warp-wide; vals(lane_row_index, col).
template <class RowFn>
__device__ __forceinline__ void sink_emit_warp(const SinkView& s, uint32_t my_cnt, RowFn row_val,
                                               uint32_t* err) {
    const uint32_t lane = lane_id();
    uint32_t incl = my_cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) return;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(s.cursor, (unsigned long long)total);
    base = __shfl_sync(0xffffffffu, base, 0);
    const unsigned long long limit = (unsigned long long)s.max_chunks * s.capacity;
    // chunks touched by [base, base + total)
    const unsigned long long first_c = base / s.capacity;
    const unsigned long long last_c = (base + total - 1) / s.capacity;
    // resolve chunk ids (lane j handles chunk first_c + j; at most 32 per call)
    uint32_t my_chunk_id = kNil - 1;
    const unsigned long long c = first_c + lane;
    if (c <= last_c && c < s.max_chunks) {
        const bool opener = c * s.capacity >= base;  // this warp owns the chunk's first row
        my_chunk_id = sink_chunk(s, (uint32_t)c, opener, err);
    }
    if (lane == 0 && (last_c - first_c >= 32 || base + total > limit)) set_error(err, kDevOverflow, 5);
    // Every lane runs the same number of iterations so that the chunk-id
    // shuffle always reads from a converged lane.
    const uint32_t maxc = __reduce_max_sync(0xffffffffu, my_cnt);
    const unsigned long long pos0 = base + incl - my_cnt;
    for (uint32_t i = 0; i < maxc; ++i) {
        const bool act = i < my_cnt;
        const unsigned long long pos = pos0 + i;
        const unsigned long long rel = act ? pos / s.capacity - first_c : 0ull;
        const uint32_t id = __shfl_sync(0xffffffffu, my_chunk_id, (int)(rel & 31ull));
        if (!act || pos >= limit || rel >= 32 || id >= s.pool->nbuffers) continue;
        const uint32_t off = (uint32_t)(pos % s.capacity);
        int32_t* base_ptr = s.slab + (size_t)id * s.pool_ncols * s.capacity;
        for (uint32_t col = 0; col < s.ncols; ++col)
            base_ptr[(size_t)col * s.capacity + off] = row_val(i, col);
    }
}

template <bool SEL, bool PROBE, bool UNIQUE>
__global__ void __launch_bounds__(kBlock) k_chain_sink(ChainDev a, SinkView s, uint32_t* err) {
    // per-warp ring: [ncols][256]
    extern __shared__ int32_t smem[];
    const uint32_t warp = threadIdx.x / kWarp, lane = lane_id();
    int32_t* ring = smem + (size_t)warp * a.ncols * 256;
    uint32_t head = 0, fill = 0;
    const uint64_t nwin = (a.n + 127) / 128;
    const uint64_t gwarp = (uint64_t)blockIdx.x * (kBlock / kWarp) + warp;
    const uint64_t nwarps = (uint64_t)gridDim.x * (kBlock / kWarp);

    // Process `cnt` (<= 128) dense rows starting at ring position `start`.
    auto push_vector = [&](uint32_t start, uint32_t cnt) {
        __syncwarp();
#pragma unroll 1
        for (int j = 0; j < 4; ++j) {
            const uint32_t idx = j * 32 + lane;
            const bool in = idx < cnt;
            const uint32_t rp = (start + idx) & 255u;
            if (!PROBE) {
                sink_emit_warp(s, in ? 1u : 0u,
                               [&](uint32_t, uint32_t col) { return ring[col * 256 + rp]; }, err);
            } else {
                const int32_t key = in ? ring[a.probe_col * 256 + rp] : 0;
                // pass 1: count matches
                uint32_t m = 0;
                if (in) {
                    if (key == kEmptyKey) {
                        m = (uint32_t)a.table.meta[0];
                    } else {
                        uint32_t b = bucket_of(key, a.table.nbuckets);
                        for (uint32_t it = 0; it < a.table.nbuckets; ++it) {
                            uint32_t w[8];
                            ld_bucket(a.table.slots + 4ull * b, w);
                            uint32_t c;
                            long long sdum;
                            bool more;
                            match_bucket<UNIQUE>(w, key, c, sdum, more);
                            m += c;
                            if (!more) break;
                            b = (b + 1 == a.table.nbuckets) ? 0u : b + 1;
                        }
                    }
                }
                // pass 2: emit the i-th match's payload
                const uint32_t side_n = (uint32_t)min((unsigned long long)a.table.meta[0],
                                                      (unsigned long long)a.table.side_cap);
                sink_emit_warp(
                    s, m,
                    [&](uint32_t i, uint32_t col) -> int32_t {
                        if (col < a.ncols) return ring[col * 256 + rp];
                        // build payload of the i-th match
                        if (key == kEmptyKey) return i < side_n ? a.table.side_pay[i] : 0;
                        uint32_t b = bucket_of(key, a.table.nbuckets);
                        uint32_t seen = 0;
                        for (uint32_t it = 0; it < a.table.nbuckets; ++it) {
                            uint32_t w[8];
                            ld_bucket(a.table.slots + 4ull * b, w);
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                if (w[2 * q] == (uint32_t)key) {
                                    if (seen == i) return (int32_t)w[2 * q + 1];
                                    ++seen;
                                }
                            }
                            if (w[6] == (uint32_t)kEmptyKey) break;
                            b = (b + 1 == a.table.nbuckets) ? 0u : b + 1;
                        }
                        return 0;
                    },
                    err);
            }
        }
        __syncwarp();
    };

    for (uint64_t win = gwarp; win < nwin; win += nwarps) {
        const uint64_t r0 = win * 128;
#pragma unroll 1
        for (int j = 0; j < 4; ++j) {
            const uint64_t row = r0 + j * 32 + lane;
            bool pass = row < a.n;
            if (SEL && pass) pass = a.cols[a.sel_col][row] <= a.sel_bound;
            const unsigned m = __ballot_sync(0xffffffffu, pass);
            if (pass) {
                const uint32_t pos = (head + fill + __popc(m & ((1u << lane) - 1u))) & 255u;
                for (uint32_t c = 0; c < a.ncols; ++c) ring[c * 256 + pos] = a.cols[c][row];
            }
            fill += __popc(m);
            if (fill >= 128) {
                push_vector(head, 128);
                head = (head + 128) & 255u;
                fill -= 128;
            }
        }
    }
    if (fill) push_vector(head, fill);
}

cudaError_t launch_chain_sink(const ChainArgs& a, const SinkView& sink, cudaStream_t s,
                              Context* ctx) {
    if (a.n == 0) return cudaSuccess;
    ChainDev d{};
    for (uint32_t c = 0; c < a.ncols; ++c) d.cols[c] = a.cols[c];
    d.ncols = a.ncols;
    d.sel_col = a.sel_col;
    d.sel_bound = a.sel_bound;
    d.probe_col = a.probe_col;
    d.n = a.n;
    d.table = a.table;
    const size_t smem = (size_t)(kBlock / kWarp) * a.ncols * 256 * sizeof(int32_t);
    const void* k;
    if (a.has_probe)
        k = a.has_sel ? (a.unique ? (const void*)k_chain_sink<true, true, true> : (const void*)k_chain_sink<true, true, false>)
                      : (a.unique ? (const void*)k_chain_sink<false, true, true> : (const void*)k_chain_sink<false, true, false>);
    else
        k = a.has_sel ? (const void*)k_chain_sink<true, false, false> : (const void*)k_chain_sink<false, false, false>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int grid = occupancy_grid(k, kBlock, smem, ctx);
    const uint64_t need = ((a.n + 127) / 128 + kBlock / kWarp - 1) / (kBlock / kWarp);
    if ((uint64_t)grid > need) grid = (int)need;
    void* args[] = {(void*)&d, (void*)&sink, (void*)&ctx->d_err};
    cudaError_t e = cudaLaunchKernel(k, dim3(grid), dim3(kBlock), args, smem, s);
    ctx->launches++;
    return e;
}

}  // namespace mgv
