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

constexpr int kSelVecs = 4;  // k_select_agg: 8-row vectors per thread per step

template <bool SEL, bool HASA, bool HASB, bool VEC>
__global__ void __launch_bounds__(kBlock) k_select_agg(const int32_t* __restrict__ f, int32_t bound,
                                                       const int32_t* __restrict__ a,
                                                       const int32_t* __restrict__ b, uint64_t n,
                                                       unsigned long long* acc) {
    unsigned long long cnt = 0, sum = 0;
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    uint64_t done = 0;
    if (VEC) {
        // kSelVecs 8-row vectors per thread per step, every load issued before any is used
        const uint64_t nvec = n / 8;
        for (uint64_t v0 = (uint64_t)blockIdx.x * kBlock + threadIdx.x; v0 < nvec; v0 += stride * kSelVecs) {
            int32_t fv[kSelVecs][8], av[kSelVecs][8], bv[kSelVecs][8];
#pragma unroll
            for (int u = 0; u < kSelVecs; ++u) {
                const uint64_t v = v0 + u * stride;
                if (v >= nvec) continue;
                if (SEL) ld_stream8(f + 8 * v, fv[u]);
                if (HASA) ld_stream8(a + 8 * v, av[u]);
                if (HASB) ld_stream8(b + 8 * v, bv[u]);
            }
#pragma unroll
            for (int u = 0; u < kSelVecs; ++u) {
                if (v0 + u * stride >= nvec) continue;
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    const bool p = !SEL || fv[u][r] <= bound;
                    long long t = 0;
                    if (HASA) t += av[u][r];
                    if (HASB) t += bv[u][r];
                    cnt += p;
                    sum += p ? (unsigned long long)t : 0ull;
                }
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
    // two CTAs per SM by default: enough loads in flight to fill HBM, and few
    // CTAs adding into the one accumulator (same-address atomics serialise in L2)
    const int per_sm = ctx->tuning.select_ctas_per_sm ? (int)ctx->tuning.select_ctas_per_sm : 2;
    int grid = std::min(occupancy_grid(k, kBlock, 0, ctx), per_sm * ctx->prop.multiProcessorCount);
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
    constexpr int R = kBuildRows;
    bool dup = false;
    uint32_t inserted = 0;
    const uint64_t stride = (uint64_t)gridDim.x * kBlock * R;
    for (uint64_t i0 = (uint64_t)blockIdx.x * kBlock * R + threadIdx.x; i0 < n; i0 += stride) {
        int32_t k[R], p[R];
        bool valid[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const uint64_t i = i0 + (uint64_t)j * kBlock;
            valid[j] = i < n && (!SEL || filt[i] <= bound);
            k[j] = valid[j] ? keys[i] : 0;
            p[j] = (valid[j] && pays) ? pays[i] : 0;
        }
        table_insert_rows<R>(t, k, p, valid, err, dup, inserted);
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
    uint64_t need = (n + (uint64_t)kBuildRows * kBlock - 1) / ((uint64_t)kBuildRows * kBlock);
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

template <bool UNIQUE, bool VEC, bool KO>
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
        for (int r = 0; r < R; ++r) ld_bucket(t.slots + 4ull * home_bucket(k[r], t), w[r]);

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
                match_bucket<UNIQUE, KO>(w[r], k[r], mc, ms, more);
                if (more) {
                    const Matches x = probe_rest<UNIQUE, KO>(t.slots, t.nbuckets, k[r], home_bucket(k[r], t));
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

template <bool KO>
static cudaError_t probe_agg_v(const int32_t* keys, const int32_t* pays, uint64_t n, const TableView& t, bool unique,
                               bool vec, uint32_t sum_mode, unsigned long long* acc, cudaStream_t s, Context* ctx);

// sum_mode bit 0 (add the build payload) is dropped for a key-only table:
// its payloads are all 0.
cudaError_t launch_probe_agg(const int32_t* keys, const int32_t* pays, uint64_t n,
                             const TableView& t, bool unique, uint32_t sum_mode,
                             unsigned long long* acc, cudaStream_t s, Context* ctx) {
    if (n == 0) return cudaSuccess;
    if (ctx->tuning.probe_kernel != 1) {
        cudaError_t e = launch_probe_agg_staged(keys, pays, n, t, unique, sum_mode, acc, s, ctx);
        if (e != cudaErrorNotSupported) return e;
    }
    const bool vec = aligned32(keys) && aligned32(pays);
    if (t.key_only) return probe_agg_v<true>(keys, pays, n, t, unique, vec, sum_mode & ~1u, acc, s, ctx);
    return probe_agg_v<false>(keys, pays, n, t, unique, vec, sum_mode, acc, s, ctx);
}

template <bool KO>
static cudaError_t probe_agg_v(const int32_t* keys, const int32_t* pays, uint64_t n, const TableView& t, bool unique,
                               bool vec, uint32_t sum_mode, unsigned long long* acc, cudaStream_t s, Context* ctx) {
    const void* k = unique ? (vec ? (const void*)k_probe_agg<true, true, KO> : (const void*)k_probe_agg<true, false, KO>)
                           : (vec ? (const void*)k_probe_agg<false, true, KO> : (const void*)k_probe_agg<false, false, KO>);
    int grid = occupancy_grid(k, kBlock, 0, ctx);
    const uint64_t ntiles = (n + (uint64_t)kBlock * 8 - 1) / ((uint64_t)kBlock * 8);
    if ((uint64_t)grid > ntiles) grid = (int)ntiles;
    if (unique) {
        if (vec) k_probe_agg<true, true, KO><<<grid, kBlock, 0, s>>>(keys, pays, n, t, sum_mode, acc);
        else k_probe_agg<true, false, KO><<<grid, kBlock, 0, s>>>(keys, pays, n, t, sum_mode, acc);
    } else {
        if (vec) k_probe_agg<false, true, KO><<<grid, kBlock, 0, s>>>(keys, pays, n, t, sum_mode, acc);
        else k_probe_agg<false, false, KO><<<grid, kBlock, 0, s>>>(keys, pays, n, t, sum_mode, acc);
    }
    ctx->launches++;
    return cudaGetLastError();
}

}  // namespace mgv
