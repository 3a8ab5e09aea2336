// build_regions.cu -- hash-table build through shared memory.
//
// Inserting build rows one 64-bit atomicCAS at a time into a table in global
// memory is bound by the L2's atomic throughput (about 20 G inserts/s on
// B200 even with the table in L2, and slower with more rows in flight).  Here
// the table is cut into regions of kRegionBuckets buckets (64 KiB) and built
// region by region in shared memory:
//   1. k_region_hist     rows per region (per-CTA shared histogram per item)
//   2. k_region_scan     exclusive prefix sum -> each region's staging range
//   3. k_region_scatter  every row, packed {key, payload} (the key alone for a
//                        key-only table), to its region's
//                        range (per item: one global reservation per region,
//                        then shared-memory cursors); for input already
//                        partitioned on the table's radix bits,
//                        k_region_scatter_sorted instead: each warp sorts its
//                        256-row tile by region and stores runs
//   4. k_region_build    one CTA per region: the region is loaded into shared
//                        memory (or starts empty), each row claims a slot
//                        with one shared atomicAdd on its bucket's fill
//                        counter (linear probing on a full bucket), a
//                        conflict-free pass finds duplicate keys, and the
//                        region is written back with one bulk copy
//   5. k_region_overflow rows whose run leaves their region (rare) are
//                        inserted into the finished global table
// The table is the same open-addressing table (hash_table.cuh): a row goes to
// the first empty slot of its run from its home bucket, slots fill in order,
// so probes are unchanged.  Rows with the reserved key INT32_MIN go to the
// side list during the scatter.
#include <cuda_runtime.h>

#include <algorithm>

#include "device_common.cuh"
#include "hash_table.cuh"
#include "mgv_internal.h"

namespace mgv {
namespace {

constexpr int kRBlock = 512;      // histogram / scatter CTA
constexpr int kRBuildBlock = 512; // region build CTA
constexpr int kScanBlock = 1024;

// The job of item / region lookups, cached in shared memory by the caller.
__device__ __forceinline__ void load_job(RegionJob& dst, const RegionJob* jobs, const RegionJob& job0, uint32_t j) {
    static_assert(sizeof(RegionJob) % 4 == 0, "RegionJob is copied as 32-bit words");
    const uint32_t* src = jobs ? reinterpret_cast<const uint32_t*>(jobs + j) : reinterpret_cast<const uint32_t*>(&job0);
    for (uint32_t i = threadIdx.x; i < sizeof(RegionJob) / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(&dst)[i] = src[i];
}

__device__ __forceinline__ BatchItem item_at(const BatchItem* items, uint32_t it, uint64_t n, uint64_t rpi) {
    if (items) return items[it];
    BatchItem b;
    b.q = 0;
    b.pad = 0;
    b.lo = (uint64_t)it * rpi;
    b.hi = min(n, b.lo + rpi);
    return b;
}

// Staging rows: {key, payload} as 8 bytes, or the key alone (4 bytes) for a
// key-only table -- half the scatter's stores and the build's loads.
template <bool KO>
__device__ __forceinline__ void stage_put(unsigned long long* staging, uint32_t pos, unsigned long long v) {
    if (KO) reinterpret_cast<uint32_t*>(staging)[pos] = (uint32_t)v;
    else staging[pos] = v;
}

template <bool KO>
__device__ __forceinline__ unsigned long long stage_get(const unsigned long long* staging, uint32_t i) {
    if (KO) return (unsigned long long)reinterpret_cast<const uint32_t*>(staging)[i];
    return staging[i];
}

__device__ __forceinline__ uint32_t region_of(int32_t key, const TableView& t) {
    return home_bucket(key, t) / kRegionBuckets;
}

// Loads of kPrefetch rows per thread are issued before any is used.
constexpr int kPrefetch = 8;

// Adds the item's rows to the shared per-region counters.
__device__ __forceinline__ void count_regions(const RegionJob& sj, const BatchItem& item, uint32_t* sh) {
    for (uint64_t i0 = item.lo + threadIdx.x; i0 < item.hi; i0 += (uint64_t)kRBlock * kPrefetch) {
        int32_t key[kPrefetch];
        bool in[kPrefetch];
#pragma unroll
        for (int u = 0; u < kPrefetch; ++u) {
            const uint64_t i = i0 + (uint64_t)u * kRBlock;
            in[u] = i < item.hi;
            key[u] = in[u] ? __ldg(sj.keys + i) : 0;
            if (in[u] && sj.filt) in[u] = __ldg(sj.filt + i) <= sj.bound;
        }
#pragma unroll
        for (int u = 0; u < kPrefetch; ++u)
            if (in[u] && key[u] != kEmptyKey) atomicAdd(sh + region_of(key[u], sj.t), 1u);
    }
}

__global__ void __launch_bounds__(kRBlock) k_region_hist(const RegionJob* __restrict__ jobs, RegionJob job0,
                                                         const BatchItem* __restrict__ items, uint32_t nitems,
                                                         uint64_t n, uint64_t rpi, uint32_t* __restrict__ hist) {
    extern __shared__ uint32_t sh[];
    __shared__ RegionJob sj;
    int64_t cur = -1;
    for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        const BatchItem item = item_at(items, it, n, rpi);
        __syncthreads();  // the previous item is done with sh and sj
        if ((int64_t)item.q != cur) {
            load_job(sj, jobs, job0, item.q);
            cur = item.q;
            __syncthreads();
        }
        for (uint32_t r = threadIdx.x; r < sj.nregions; r += kRBlock) sh[r] = 0;
        __syncthreads();
        count_regions(sj, item, sh);
        __syncthreads();
        for (uint32_t r = threadIdx.x; r < sj.nregions; r += kRBlock)
            if (sh[r]) atomicAdd(hist + sj.region0 + r, sh[r]);
    }
}

// One CTA: start[i] = sum of hist[0..i), start[regions] = total; cursor = start.
__global__ void __launch_bounds__(kScanBlock) k_region_scan(const uint32_t* __restrict__ hist, uint32_t regions,
                                                            uint32_t* __restrict__ start, uint32_t* __restrict__ cursor) {
    __shared__ uint32_t part[kScanBlock];
    const uint32_t per = (regions + kScanBlock - 1) / kScanBlock;
    const uint32_t lo = min(regions, threadIdx.x * per), hi = min(regions, lo + per);
    uint32_t sum = 0;
    for (uint32_t i = lo; i < hi; ++i) sum += hist[i];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (uint32_t o = 1; o < kScanBlock; o <<= 1) {  // inclusive Hillis-Steele scan of the chunk sums
        const uint32_t add = threadIdx.x >= o ? part[threadIdx.x - o] : 0u;
        __syncthreads();
        part[threadIdx.x] += add;
        __syncthreads();
    }
    uint32_t run = part[threadIdx.x] - sum;
    for (uint32_t i = lo; i < hi; ++i) {
        start[i] = run;
        cursor[i] = run;
        run += hist[i];
    }
    if (threadIdx.x == kScanBlock - 1) start[regions] = part[kScanBlock - 1];
}

template <bool KO>
__global__ void __launch_bounds__(kRBlock) k_region_scatter(const RegionJob* __restrict__ jobs, RegionJob job0,
                                                            const BatchItem* __restrict__ items, uint32_t nitems,
                                                            uint64_t n, uint64_t rpi, uint32_t* __restrict__ cursor,
                                                            unsigned long long* __restrict__ staging, uint32_t* err) {
    extern __shared__ uint32_t sh[];
    __shared__ RegionJob sj;
    int64_t cur = -1;
    for (uint32_t it = blockIdx.x; it < nitems; it += gridDim.x) {
        const BatchItem item = item_at(items, it, n, rpi);
        __syncthreads();
        if ((int64_t)item.q != cur) {
            load_job(sj, jobs, job0, item.q);
            cur = item.q;
            __syncthreads();
        }
        for (uint32_t r = threadIdx.x; r < sj.nregions; r += kRBlock) sh[r] = 0;
        __syncthreads();
        count_regions(sj, item, sh);
        __syncthreads();
        // one reservation per region and item; sh[r] becomes the region's next staging row
        for (uint32_t r = threadIdx.x; r < sj.nregions; r += kRBlock) {
            const uint32_t c = sh[r];
            if (c) sh[r] = atomicAdd(cursor + sj.region0 + r, c);
        }
        __syncthreads();
        for (uint64_t i0 = item.lo + threadIdx.x; i0 < item.hi; i0 += (uint64_t)kRBlock * kPrefetch) {
            int32_t key[kPrefetch], pay[kPrefetch];
            bool in[kPrefetch];
#pragma unroll
            for (int u = 0; u < kPrefetch; ++u) {
                const uint64_t i = i0 + (uint64_t)u * kRBlock;
                in[u] = i < item.hi;
                key[u] = in[u] ? __ldg(sj.keys + i) : 0;
                pay[u] = (in[u] && sj.pays) ? __ldg(sj.pays + i) : 0;
                if (in[u] && sj.filt) in[u] = __ldg(sj.filt + i) <= sj.bound;
            }
#pragma unroll
            for (int u = 0; u < kPrefetch; ++u) {
                if (!in[u]) continue;
                if (key[u] == kEmptyKey) {  // the side list (its duplicates are seen from its count)
                    bool dup, ok;
                    table_insert(sj.t, key[u], pay[u], err, dup, ok);
                    continue;
                }
                const uint32_t pos = atomicAdd(sh + region_of(key[u], sj.t), 1u);
                stage_put<KO>(staging, pos, ((unsigned long long)(uint32_t)pay[u] << 32) | (uint32_t)key[u]);
            }
        }
    }
}

constexpr int kWarpTileRows = 8;                          // rows per lane of a warp tile
constexpr uint32_t kWarpTile = 32u * kWarpTileRows;       // 256 rows
constexpr uint32_t kWarpSpan = 64;                        // widest region span a warp tile sorts

// One warp's sorting space in k_region_scatter_sorted.
struct WarpSort {
    unsigned long long val[kWarpTile];  // the tile's rows in region order
    uint32_t off[kWarpSpan];            // counts, then each region's first sorted position
    uint32_t base[kWarpSpan];           // staging row of sorted position 0 of each region (mod 2^32)
    uint8_t reg[kWarpTile];             // region (minus the tile's lowest) of each sorted position
};

// Rows of input that is already partitioned on the table's radix bits (a
// partition op's run: each partition's rows together, so a warp's tile of 256
// rows falls in the regions of one or two partitions).  Each warp sorts its
// tile by region in its own shared memory -- ranks by shared atomics, one
// global cursor reservation per region -- and stores runs of consecutive
// staging rows, with no block-wide barrier.  A tile whose regions span more
// than kWarpSpan takes one cursor increment per row instead.
template <bool KO>
__global__ void __launch_bounds__(kRBlock, 2) k_region_scatter_sorted(RegionJob job, uint64_t n,
                                                                    uint32_t* __restrict__ cursor,
                                                                    unsigned long long* __restrict__ staging,
                                                                    uint32_t* err) {
    extern __shared__ __align__(16) unsigned char ws_raw[];
    WarpSort& ws = reinterpret_cast<WarpSort*>(ws_raw)[threadIdx.x / 32];
    const uint32_t lane = lane_id();
    const uint64_t ntiles = (n + kWarpTile - 1) / kWarpTile;
    const uint64_t nw = (uint64_t)gridDim.x * (kRBlock / 32);
    for (uint64_t tile = (uint64_t)blockIdx.x * (kRBlock / 32) + threadIdx.x / 32; tile < ntiles; tile += nw) {
        const uint64_t t0 = tile * kWarpTile;
        int32_t key[kWarpTileRows], pay[kWarpTileRows];
        bool in[kWarpTileRows];
#pragma unroll
        for (int u = 0; u < kWarpTileRows; ++u) {
            const uint64_t i = t0 + 32u * u + lane;
            in[u] = i < n;
            key[u] = in[u] ? __ldg(job.keys + i) : 0;
            pay[u] = (in[u] && job.pays) ? __ldg(job.pays + i) : 0;
            if (in[u] && job.filt) in[u] = __ldg(job.filt + i) <= job.bound;
        }
        uint32_t reg[kWarpTileRows];
        uint32_t lo = ~0u, hi = 0;
#pragma unroll
        for (int u = 0; u < kWarpTileRows; ++u) {
            reg[u] = 0;
            if (!in[u]) continue;
            if (key[u] == kEmptyKey) {  // the side list (its duplicates are seen from its count)
                bool dup, ok;
                table_insert(job.t, key[u], pay[u], err, dup, ok);
                in[u] = false;
                continue;
            }
            reg[u] = region_of(key[u], job.t);
            lo = min(lo, reg[u]);
            hi = max(hi, reg[u]);
        }
        lo = __reduce_min_sync(0xffffffffu, lo);
        hi = __reduce_max_sync(0xffffffffu, hi);
        if (lo > hi) continue;  // no row of the tile goes to the table
        if (hi - lo >= kWarpSpan) {
#pragma unroll
            for (int u = 0; u < kWarpTileRows; ++u)
                if (in[u]) {
                    const uint32_t pos = atomicAdd(cursor + job.region0 + reg[u], 1u);
                    stage_put<KO>(staging, pos, ((unsigned long long)(uint32_t)pay[u] << 32) | (uint32_t)key[u]);
                }
            continue;
        }
        const uint32_t span = hi - lo + 1;
        for (uint32_t j = lane; j < span; j += 32) ws.off[j] = 0;
        __syncwarp();
        uint32_t rank[kWarpTileRows];
#pragma unroll
        for (int u = 0; u < kWarpTileRows; ++u) {
            reg[u] -= lo;
            rank[u] = in[u] ? atomicAdd(&ws.off[reg[u]], 1u) : 0u;
        }
        __syncwarp();
        // lane l owns regions l and l + 32: reserve their staging ranges, then
        // an exclusive scan of the counts gives their first sorted positions
        const uint32_t c0 = lane < span ? ws.off[lane] : 0u;
        const uint32_t c1 = lane + 32 < span ? ws.off[lane + 32] : 0u;
        const uint32_t g0 = c0 ? atomicAdd(cursor + job.region0 + lo + lane, c0) : 0u;
        const uint32_t g1 = c1 ? atomicAdd(cursor + job.region0 + lo + lane + 32, c1) : 0u;
        uint32_t x0 = c0, x1 = c1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y0 = __shfl_up_sync(0xffffffffu, x0, o);
            const uint32_t y1 = __shfl_up_sync(0xffffffffu, x1, o);
            if (lane >= (uint32_t)o) {
                x0 += y0;
                x1 += y1;
            }
        }
        const uint32_t tot0 = __shfl_sync(0xffffffffu, x0, 31);
        const uint32_t total = tot0 + __shfl_sync(0xffffffffu, x1, 31);
        const uint32_t e0 = x0 - c0, e1 = tot0 + x1 - c1;
        if (lane < span) {
            ws.off[lane] = e0;
            ws.base[lane] = g0 - e0;
        }
        if (lane + 32 < span) {
            ws.off[lane + 32] = e1;
            ws.base[lane + 32] = g1 - e1;
        }
        __syncwarp();
#pragma unroll
        for (int u = 0; u < kWarpTileRows; ++u)
            if (in[u]) {
                const uint32_t p = ws.off[reg[u]] + rank[u];
                ws.val[p] = ((unsigned long long)(uint32_t)pay[u] << 32) | (uint32_t)key[u];
                ws.reg[p] = (uint8_t)reg[u];
            }
        __syncwarp();
        for (uint32_t j = lane; j < total; j += 32) stage_put<KO>(staging, ws.base[ws.reg[j]] + j, ws.val[j]);
        __syncwarp();  // the warp's buffers are free for its next tile
    }
}

__device__ __forceinline__ uint32_t job_of_region(const RegionJob* jobs, uint32_t njobs, uint32_t g) {
    uint32_t lo = 0, hi = njobs;  // last job whose region0 <= g
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (jobs[mid].region0 <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

// 16-byte shared-memory read.
__device__ __forceinline__ uint4 lds_v4(const void* p) {
    uint4 r;
    asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "r"(smem_u32(p))
                 : "memory");
    return r;
}

// Slots per bucket: 4 {key, payload} slots, or 8 keys in a key-only table.
template <bool KO>
constexpr uint32_t slots_per_bucket() { return KO ? 8u : 4u; }

// The key words of shared bucket b (4, or 8 for a key-only table).
template <bool KO>
__device__ __forceinline__ void bucket_keys(const unsigned long long* tab, uint32_t b,
                                            uint32_t (&k)[slots_per_bucket<KO>()]) {
    const uint32_t* words = reinterpret_cast<const uint32_t*>(tab) + 8 * b;
    const uint4 s01 = lds_v4(words), s23 = lds_v4(words + 4);
    if constexpr (KO) {
        k[0] = s01.x; k[1] = s01.y; k[2] = s01.z; k[3] = s01.w;
        k[4] = s23.x; k[5] = s23.y; k[6] = s23.z; k[7] = s23.w;
    } else {
        k[0] = s01.x;
        k[1] = s01.z;
        k[2] = s23.x;
        k[3] = s23.z;
    }
}

// Inserts one staged row into the shared region.  fill[b] counts the rows
// that asked bucket b for a slot: the first four (eight in a key-only table)
// get slots 0, 1, ... in that order (so slots fill as a prefix, as the global
// insert leaves them), later ones move on to the next bucket.  A bucket that
// has turned a row away stays full, so every row ends in the first bucket of
// its run that had room.
template <bool KO>
__device__ __forceinline__ bool region_insert(unsigned long long* tab, uint32_t* fill, uint32_t nb, uint32_t b,
                                              unsigned long long v) {
    for (; b < nb; ++b) {
        const uint32_t q = atomicAdd(fill + b, 1u);
        if (q < slots_per_bucket<KO>()) {
            if (KO) reinterpret_cast<uint32_t*>(tab)[8 * b + q] = (uint32_t)v;  // the key alone
            else tab[4 * b + q] = v;
            return true;
        }
    }
    return false;  // the run leaves the region
}

// Whether bucket b holds a key that also appears later in its run: in b
// itself, or in the buckets after b up to the first one that is not full.
// Two rows with one key share their home bucket, and every bucket between
// the two is full, so this finds every duplicate pair inside the region.
template <bool KO>
__device__ __forceinline__ bool bucket_has_dup(const unsigned long long* tab, const uint32_t* fill, uint32_t nb,
                                               uint32_t b) {
    constexpr uint32_t S = slots_per_bucket<KO>();
    const uint32_t n = min(fill[b], S);
    if (n < 2) return false;  // no pair in b, and b is not full
    uint32_t k[S];
    bucket_keys<KO>(tab, b, k);
    bool dup = false;
#pragma unroll
    for (int i = 0; i < (int)S; ++i)
#pragma unroll
        for (int j = i + 1; j < (int)S; ++j) dup |= (uint32_t)j < n && k[i] == k[j];
    if (n < S) return dup;
    for (uint32_t c = b + 1; c < nb && !dup; ++c) {
        const uint32_t m = min(fill[c], S);
        uint32_t o[S];
        bucket_keys<KO>(tab, c, o);
#pragma unroll
        for (int i = 0; i < (int)S; ++i)
#pragma unroll
            for (int j = 0; j < (int)S; ++j) dup |= (uint32_t)j < m && k[i] == o[j];
        if (m < S) break;
    }
    return dup;
}

constexpr int kBuildRows = 8;  // staging rows per thread in one load batch (4096 per region)

// The next region of this CTA at or after g (stride gridDim.x); without
// `fresh`, regions that receive no rows are left as they are.
__device__ __forceinline__ uint32_t next_region(uint32_t g, uint32_t regions, const uint32_t* start, uint32_t fresh) {
    for (; g < regions; g += gridDim.x)
        if (fresh || start[g] != start[g + 1]) return g;
    return regions;
}

// Staging rows [s0, s1) of a region, the first kBuildRows * kRBuildBlock of
// them, into registers (rows past s1 read as empty).
template <bool KO>
__device__ __forceinline__ void load_region_rows(const unsigned long long* staging, uint32_t s0, uint32_t s1,
                                                 unsigned long long (&v)[kBuildRows]) {
#pragma unroll
    for (int u = 0; u < kBuildRows; ++u) {
        const uint32_t i = s0 + threadIdx.x + u * kRBuildBlock;
        v[u] = i < s1 ? stage_get<KO>(staging, i) : kEmptySlot;
    }
}

// Regions one at a time per CTA, several CTAs per SM; the next region's
// first rows are loaded into registers before this region's duplicate pass
// and bulk store, so their latency overlaps that work.
template <bool KO>
__global__ void __launch_bounds__(kRBuildBlock, 3) k_region_build(const RegionJob* __restrict__ jobs, RegionJob job0,
                                                                  uint32_t njobs, uint32_t regions,
                                                                  const uint32_t* __restrict__ start,
                                                                  const unsigned long long* __restrict__ staging,
                                                                  unsigned long long* __restrict__ ovf,
                                                                  uint32_t* ovf_count, uint32_t fresh, uint32_t* err) {
    extern __shared__ __align__(128) unsigned long long tab[];  // kRegionBuckets * 4 slots, then the fill counters
    uint32_t* fill = reinterpret_cast<uint32_t*>(tab + 4 * kRegionBuckets);
    __shared__ RegionJob sj;
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    uint32_t phase = 0;
    int64_t cur = -1;
    uint32_t g = next_region(blockIdx.x, regions, start, fresh);
    unsigned long long v[kBuildRows];
    if (g < regions) load_region_rows<KO>(staging, start[g], start[g + 1], v);
    while (g < regions) {
        const uint32_t s0 = start[g], s1 = start[g + 1];
        const uint32_t j = (jobs && njobs > 1) ? job_of_region(jobs, njobs, g) : 0u;
        __syncthreads();  // the previous region's store has read the buffer; sj is free
        if ((int64_t)j != cur) {
            load_job(sj, jobs, job0, j);
            cur = j;
            __syncthreads();
        }
        const uint32_t b0 = (g - sj.region0) * kRegionBuckets;
        const uint32_t nb = min(kRegionBuckets, sj.t.nbuckets - b0);
        unsigned long long* gslots = sj.t.slots + 4ull * b0;
        if (fresh) {
            const uint4 empty = make_uint4(0x80000000u, 0x80000000u, 0x80000000u, 0x80000000u);  // 2 x kEmptySlot
            static_assert(kEmptySlot == 0x8000000080000000ull, "empty slot pattern");
            for (uint32_t w = threadIdx.x; w < 2 * nb; w += kRBuildBlock) reinterpret_cast<uint4*>(tab)[w] = empty;
            for (uint32_t b = threadIdx.x; b < nb; b += kRBuildBlock) fill[b] = 0;
        } else {
            if (threadIdx.x == 0) {  // the region's current contents, one bulk copy
                mbar_expect_tx(&bar, nb * 32);
                bulk_g2s(tab, gslots, nb * 32, &bar);
            }
            if (!mbar_wait_bounded(&bar, phase, 1u << 24)) {
                if (threadIdx.x == 0) {
                    set_error(err, kDevTimeout, 40);
                    bulk_wait_all();
                }
                return;
            }
            phase ^= 1u;
            // slots fill as a prefix: a bucket's count is the index of its first empty slot
            for (uint32_t b = threadIdx.x; b < nb; b += kRBuildBlock) {
                uint32_t k[slots_per_bucket<KO>()];
                bucket_keys<KO>(tab, b, k);
                uint32_t n = 0;
#pragma unroll
                for (int q = 0; q < (int)slots_per_bucket<KO>(); ++q) n += k[q] != (uint32_t)kEmptyKey;
                fill[b] = n;
            }
        }
        __syncthreads();
        uint32_t ins = 0;
        for (uint32_t i0 = s0 + threadIdx.x;; i0 += kRBuildBlock * kBuildRows) {
#pragma unroll
            for (int u = 0; u < kBuildRows; ++u) {
                const uint32_t i = i0 + u * kRBuildBlock;
                // past the region, or a gap slot of a partition's range (the
                // reserved key goes to the side list, never into staging)
                if (i >= s1 || (int32_t)(uint32_t)v[u] == kEmptyKey) continue;
                const uint32_t hb = home_bucket((int32_t)(uint32_t)v[u], sj.t) - b0;
                if (region_insert<KO>(tab, fill, nb, hb, v[u])) ++ins;
                else ovf[atomicAdd(ovf_count, 1u)] = ((unsigned long long)j << 32) | i;  // the run leaves the region
            }
            if (i0 + kRBuildBlock * kBuildRows >= s1) break;
            load_region_rows<KO>(staging, i0 + kRBuildBlock * kBuildRows - threadIdx.x, s1, v);  // a large region
        }
        __syncthreads();
        const uint32_t gn = next_region(g + gridDim.x, regions, start, fresh);
        if (gn < regions) load_region_rows<KO>(staging, start[gn], start[gn + 1], v);  // in flight from here on
        bool dup = false;
        for (uint32_t b = threadIdx.x; b < nb; b += kRBuildBlock) dup |= bucket_has_dup<KO>(tab, fill, nb, b);
        fence_proxy_async_smem();  // the inserts, before the bulk store reads them
        __syncthreads();
        if (threadIdx.x == 0) {
            bulk_s2g(gslots, tab, nb * 32);
            bulk_commit();
            bulk_wait_reads();  // the buffer may be refilled; the write itself completes in the background
        }
        const unsigned long long tot = warp_sum_u64(ins);
        const bool any_dup = __any_sync(0xffffffffu, dup);
        if (lane_id() == 0) {
            if (tot) atomicAdd(sj.t.meta + 2, tot);
            if (any_dup) atomicOr(sj.t.meta + 3, 1ull);
        }
        g = gn;
    }
    if (threadIdx.x == 0) bulk_wait_all();  // every region store is complete before the CTA ends
}

// Rows whose run left their region, into the global table (each entry:
// job << 32 | staging row).
template <bool KO>
__global__ void k_region_overflow(const RegionJob* __restrict__ jobs, RegionJob job0,
                                  const unsigned long long* __restrict__ staging,
                                  const unsigned long long* __restrict__ ovf, const uint32_t* ovf_count, uint32_t* err) {
    const uint32_t cnt = *ovf_count;
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < cnt; x += gridDim.x * blockDim.x) {
        const unsigned long long e = ovf[x];
        const TableView t = jobs ? jobs[e >> 32].t : job0.t;
        const unsigned long long v = stage_get<KO>(staging, (uint32_t)e);
        bool dup = false, ok = false;
        table_insert(t, (int32_t)(uint32_t)v, (int32_t)(uint32_t)(v >> 32), err, dup, ok);
        if (ok) atomicAdd(t.meta + 2, 1ull);
        if (dup) atomicOr(t.meta + 3, 1ull);
    }
}

// ---- staging of a partition op's single run ---------------------------------
//
// A partition op's single run gives each partition's rows as one range
// [ends[p-1], ends[p]), and when the table's partition slices are whole
// regions (bpp a multiple of kRegionBuckets) every region lies in one
// partition.  One CTA per partition then counts its rows per region in
// shared memory, and stages them region-major inside the partition's own
// range -- the regions' starts are the range's start plus a prefix sum, so
// no global histogram, scan or cursor is needed, and the partition's rows
// (just written by the partition op) are read from L2 twice.  Rows with the
// reserved key go to the side list; their slots at the range's end are
// filled with the reserved key, which the region build skips.
constexpr int kPartScatterBlock = 1024;
constexpr int kPartScatterRows = 8;  // loads per thread in flight

template <bool KO>
__global__ void __launch_bounds__(kPartScatterBlock) k_region_part_scatter(RegionJob job,
                                                                           const unsigned long long* __restrict__ ends,
                                                                           uint32_t P, uint32_t rpp,
                                                                           uint32_t* __restrict__ start,
                                                                           unsigned long long* __restrict__ staging,
                                                                           uint32_t* err) {
    extern __shared__ uint32_t cnt[];  // rpp counters, then rpp cursors
    uint32_t* cur = cnt + rpp;
    __shared__ uint32_t side_rows;
    const uint32_t lane = lane_id();
    const uint32_t bpp = job.t.bpp;
    for (uint32_t p = blockIdx.x; p < P; p += gridDim.x) {
        const uint64_t lo = p ? ends[p - 1] : 0ull, hi = ends[p];
        __syncthreads();  // the previous partition is done with the counters
        for (uint32_t r = threadIdx.x; r < rpp; r += kPartScatterBlock) cnt[r] = 0;
        if (threadIdx.x == 0) side_rows = 0;
        __syncthreads();
        // 1. rows per region
        for (uint64_t i0 = lo + threadIdx.x; i0 < hi; i0 += (uint64_t)kPartScatterBlock * kPartScatterRows) {
            int32_t key[kPartScatterRows];
#pragma unroll
            for (int u = 0; u < kPartScatterRows; ++u) {
                const uint64_t i = i0 + (uint64_t)u * kPartScatterBlock;
                key[u] = i < hi ? __ldg(job.keys + i) : kEmptyKey;
            }
#pragma unroll
            for (int u = 0; u < kPartScatterRows; ++u)
                if (key[u] != kEmptyKey) atomicAdd(cnt + __umulhi(murmur32((uint32_t)key[u]), bpp) / kRegionBuckets, 1u);
        }
        __syncthreads();
        // the regions' starts inside the partition's range
        if (threadIdx.x < 32) {
            uint32_t run = 0;
            for (uint32_t r0 = 0; r0 < rpp; r0 += 32) {
                const uint32_t r = r0 + lane;
                const uint32_t c = r < rpp ? cnt[r] : 0u;
                uint32_t x = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= (uint32_t)o) x += y;
                }
                if (r < rpp) {
                    const uint32_t off = (uint32_t)lo + run + x - c;
                    cur[r] = off;
                    start[(uint64_t)p * rpp + r] = off;
                }
                run += __shfl_sync(0xffffffffu, x, 31);
            }
        }
        if (p == P - 1 && threadIdx.x == 0) start[(uint64_t)P * rpp] = (uint32_t)hi;
        __syncthreads();
        // 2. the rows, region-major; a warp's rows of one region take consecutive slots
        for (uint64_t i0 = lo + threadIdx.x;; i0 += (uint64_t)kPartScatterBlock * kPartScatterRows) {
            const uint64_t base = i0 - threadIdx.x;  // uniform across the CTA
            if (base >= hi) break;
            int32_t key[kPartScatterRows], pay[kPartScatterRows];
#pragma unroll
            for (int u = 0; u < kPartScatterRows; ++u) {
                const uint64_t i = i0 + (uint64_t)u * kPartScatterBlock;
                const bool in = i < hi;
                key[u] = in ? __ldg(job.keys + i) : kEmptyKey;
                pay[u] = (!KO && in && job.pays) ? __ldg(job.pays + i) : 0;
                if (in && key[u] == kEmptyKey) {  // the side list (its duplicates are seen from its count)
                    bool d, ok;
                    table_insert(job.t, key[u], pay[u], err, d, ok);
                    atomicAdd(&side_rows, 1u);
                }
            }
#pragma unroll
            for (int u = 0; u < kPartScatterRows; ++u) {
                const bool row = key[u] != kEmptyKey;
                const uint32_t r = row ? __umulhi(murmur32((uint32_t)key[u]), bpp) / kRegionBuckets : 0xffffffffu;
                const uint32_t peers = __match_any_sync(0xffffffffu, r);
                const uint32_t leader = __ffs(peers) - 1;
                uint32_t pos = 0;
                if (row && lane == leader) pos = atomicAdd(cur + r, (uint32_t)__popc(peers));
                pos = __shfl_sync(0xffffffffu, pos, leader) + __popc(peers & ((1u << lane) - 1u));
                if (row) stage_put<KO>(staging, pos, ((unsigned long long)(uint32_t)pay[u] << 32) | (uint32_t)key[u]);
            }
        }
        __syncthreads();
        // the reserved-key rows' slots at the end of the range
        const uint32_t nside = side_rows;
        for (uint32_t k = threadIdx.x; k < nside; k += kPartScatterBlock)
            stage_put<KO>(staging, (uint32_t)(hi - nside) + k, kEmptySlot);
    }
}

}  // namespace

bool region_build_partitioned_fits(const TableView& t) {
    return t.bpp % kRegionBuckets == 0 && t.bpp / kRegionBuckets <= 4096;
}

cudaError_t launch_build_regions_partitioned(const RegionJob& job, const unsigned long long* ends, uint64_t n,
                                             const RegionScratch& sc, cudaStream_t s, Context* ctx) {
    const uint32_t P = job.t.radix_mask + 1;
    const uint32_t rpp = job.t.bpp / kRegionBuckets;
    const uint32_t regions = P * rpp;
    const bool ko = job.t.key_only != 0;
    const size_t psmem = 8ull * rpp;
    const size_t tsmem = (32ull + 4ull) * kRegionBuckets;
    const void* kp = ko ? (const void*)k_region_part_scatter<true> : (const void*)k_region_part_scatter<false>;
    const void* kb = ko ? (const void*)k_region_build<true> : (const void*)k_region_build<false>;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem)) ||
        (e = cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem)))
        return e;
    if ((e = cudaMemsetAsync(sc.ovf_count, 0, 4, s))) return e;
    if (n) {
        const int grid = (int)std::min<uint64_t>(P, (uint64_t)occupancy_grid(kp, kPartScatterBlock, psmem, ctx));
        if (ko)
            k_region_part_scatter<true><<<grid, kPartScatterBlock, psmem, s>>>(job, ends, P, rpp, sc.start, sc.staging,
                                                                                ctx->d_err);
        else
            k_region_part_scatter<false><<<grid, kPartScatterBlock, psmem, s>>>(job, ends, P, rpp, sc.start,
                                                                                 sc.staging, ctx->d_err);
        ctx->launches++;
        if ((e = cudaGetLastError())) return e;
    } else {  // nothing staged: every region is empty
        if ((e = cudaMemsetAsync(sc.start, 0, 4ull * (regions + 1), s))) return e;
    }
    const int grid = (int)std::min<uint64_t>(regions, (uint64_t)occupancy_grid(kb, kRBuildBlock, tsmem, ctx));
    if (ko)
        k_region_build<true><<<grid, kRBuildBlock, tsmem, s>>>(nullptr, job, 1, regions, sc.start, sc.staging, sc.ovf,
                                                               sc.ovf_count, 1u, ctx->d_err);
    else
        k_region_build<false><<<grid, kRBuildBlock, tsmem, s>>>(nullptr, job, 1, regions, sc.start, sc.staging,
                                                                sc.ovf, sc.ovf_count, 1u, ctx->d_err);
    ctx->launches++;
    if ((e = cudaGetLastError())) return e;
    const int sms = ctx->prop.multiProcessorCount;
    if (ko) k_region_overflow<true><<<sms * 2, 256, 0, s>>>(nullptr, job, sc.staging, sc.ovf, sc.ovf_count, ctx->d_err);
    else k_region_overflow<false><<<sms * 2, 256, 0, s>>>(nullptr, job, sc.staging, sc.ovf, sc.ovf_count, ctx->d_err);
    ctx->launches++;
    return cudaGetLastError();
}

size_t region_scratch_bytes(uint32_t regions, uint64_t rows) {
    auto a = [](size_t x) { return (x + 255) & ~(size_t)255; };
    return a(4ull * regions) + a(4ull * (regions + 1)) + a(4ull * regions) + a(4) + a(8ull * rows) + a(8ull * rows);
}

RegionScratch carve_region_scratch(void* base, uint32_t regions, uint64_t rows) {
    auto a = [](size_t x) { return (x + 255) & ~(size_t)255; };
    unsigned char* p = static_cast<unsigned char*>(base);
    RegionScratch s;
    s.hist = reinterpret_cast<uint32_t*>(p);
    p += a(4ull * regions);
    s.start = reinterpret_cast<uint32_t*>(p);
    p += a(4ull * (regions + 1));
    s.cursor = reinterpret_cast<uint32_t*>(p);
    p += a(4ull * regions);
    s.ovf_count = reinterpret_cast<uint32_t*>(p);
    p += a(4);
    s.staging = reinterpret_cast<unsigned long long*>(p);
    p += a(8ull * rows);
    s.ovf = reinterpret_cast<unsigned long long*>(p);
    return s;
}

cudaError_t launch_build_regions(const RegionJob* d_jobs, const RegionJob& job0, uint32_t njobs,
                                 const BatchItem* items, uint32_t nitems, uint64_t n, uint64_t rows_per_item,
                                 uint32_t total_regions, uint32_t max_job_regions, const RegionScratch& sc,
                                 bool fresh, bool partitioned, cudaStream_t s, Context* ctx) {
    if (total_regions == 0) return cudaSuccess;
    if (!items) nitems = (uint32_t)((n + rows_per_item - 1) / rows_per_item);
    const int sms = ctx->prop.multiProcessorCount;
    const size_t hsmem = 4ull * std::max(max_job_regions, 1u);
    const bool sorted = partitioned && !items && njobs == 1;
    const size_t wsmem = sizeof(WarpSort) * (kRBlock / 32);
    const size_t tsmem = (32ull + 4ull) * kRegionBuckets;  // the region, then its fill counters
    // every job of one launch has the same slot layout (all key-only or none); a
    // key-only launch stages 4-byte keys
    const bool ko = job0.t.key_only != 0;
    const void* kscat = ko ? (const void*)k_region_scatter<true> : (const void*)k_region_scatter<false>;
    const void* ksort = ko ? (const void*)k_region_scatter_sorted<true> : (const void*)k_region_scatter_sorted<false>;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_region_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem)) ||
        (e = cudaFuncSetAttribute(kscat, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem)) ||
        (e = cudaFuncSetAttribute(ksort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsmem)) ||
        (e = cudaFuncSetAttribute(k_region_build<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem)) ||
        (e = cudaFuncSetAttribute(k_region_build<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem)))
        return e;
    if ((e = cudaMemsetAsync(sc.hist, 0, 4ull * total_regions, s))) return e;
    if ((e = cudaMemsetAsync(sc.ovf_count, 0, 4, s))) return e;
    if (nitems) {
        const int grid = (int)std::min<uint64_t>(nitems, (uint64_t)occupancy_grid((const void*)k_region_hist, kRBlock,
                                                                                   hsmem, ctx));
        k_region_hist<<<grid, kRBlock, hsmem, s>>>(d_jobs, job0, items, nitems, n, rows_per_item, sc.hist);
        ctx->launches++;
        if ((e = cudaGetLastError())) return e;
    }
    k_region_scan<<<1, kScanBlock, 0, s>>>(sc.hist, total_regions, sc.start, sc.cursor);
    ctx->launches++;
    if ((e = cudaGetLastError())) return e;
    if (sorted && n) {
        const uint64_t tiles = (n + kWarpTile - 1) / kWarpTile;
        const uint64_t ctas = (tiles + kRBlock / 32 - 1) / (kRBlock / 32);
        const int grid = (int)std::min<uint64_t>(ctas, (uint64_t)occupancy_grid(ksort, kRBlock, wsmem, ctx));
        if (ko) k_region_scatter_sorted<true><<<grid, kRBlock, wsmem, s>>>(job0, n, sc.cursor, sc.staging, ctx->d_err);
        else k_region_scatter_sorted<false><<<grid, kRBlock, wsmem, s>>>(job0, n, sc.cursor, sc.staging, ctx->d_err);
        ctx->launches++;
        if ((e = cudaGetLastError())) return e;
    } else if (nitems) {
        const int grid = (int)std::min<uint64_t>(nitems, (uint64_t)occupancy_grid(kscat, kRBlock, hsmem, ctx));
        if (ko)
            k_region_scatter<true><<<grid, kRBlock, hsmem, s>>>(d_jobs, job0, items, nitems, n, rows_per_item,
                                                                sc.cursor, sc.staging, ctx->d_err);
        else
            k_region_scatter<false><<<grid, kRBlock, hsmem, s>>>(d_jobs, job0, items, nitems, n, rows_per_item,
                                                                 sc.cursor, sc.staging, ctx->d_err);
        ctx->launches++;
        if ((e = cudaGetLastError())) return e;
    }
    {
        const void* kb = ko ? (const void*)k_region_build<true> : (const void*)k_region_build<false>;
        const int grid = (int)std::min<uint64_t>(total_regions,
                                                 (uint64_t)occupancy_grid(kb, kRBuildBlock, tsmem, ctx));
        if (ko)
            k_region_build<true><<<grid, kRBuildBlock, tsmem, s>>>(d_jobs, job0, njobs, total_regions, sc.start,
                                                                   sc.staging, sc.ovf, sc.ovf_count, fresh ? 1u : 0u,
                                                                   ctx->d_err);
        else
            k_region_build<false><<<grid, kRBuildBlock, tsmem, s>>>(d_jobs, job0, njobs, total_regions, sc.start,
                                                                    sc.staging, sc.ovf, sc.ovf_count,
                                                                    fresh ? 1u : 0u, ctx->d_err);
        ctx->launches++;
        if ((e = cudaGetLastError())) return e;
    }
    if (ko) k_region_overflow<true><<<sms * 2, 256, 0, s>>>(d_jobs, job0, sc.staging, sc.ovf, sc.ovf_count, ctx->d_err);
    else k_region_overflow<false><<<sms * 2, 256, 0, s>>>(d_jobs, job0, sc.staging, sc.ovf, sc.ovf_count, ctx->d_err);
    ctx->launches++;
    return cudaGetLastError();
}

}  // namespace mgv
