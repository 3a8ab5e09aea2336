// build_regions.cu -- hash-table build through shared memory.
//
// Inserting build rows one 64-bit atomicCAS at a time into a table in global
// memory is bound by the L2's atomic throughput (about 20 G inserts/s on
// B200 even with the table in L2, and slower with more rows in flight).  Here
// the table is cut into regions of kRegionBuckets buckets (64 KiB) and built
// region by region in shared memory:
//   1. k_region_hist     rows per region (per-CTA shared histogram per item)
//   2. k_region_scan     exclusive prefix sum -> each region's staging range
//   3. k_region_scatter  every row, packed {key, payload}, to its region's
//                        range (per item: one global reservation per region,
//                        then shared-memory cursors)
//   4. k_region_build    one CTA per region: the region is loaded into shared
//                        memory (or starts empty), its rows are inserted with
//                        shared-memory CAS and linear probing, and it is
//                        written back with coalesced stores
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
constexpr int kRBuildBlock = 256; // region build CTA
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
                staging[pos] = ((unsigned long long)(uint32_t)pay[u] << 32) | (uint32_t)key[u];
            }
        }
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

// 16-byte shared-memory read, issued where it stands (not cached across CAS).
__device__ __forceinline__ uint4 lds_v4(const void* p) {
    uint4 r;
    asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "r"(smem_u32(p))
                 : "memory");
    return r;
}

// Inserts one staged row into the shared region (linear probing inside it).
// A slot is claimed with a 32-bit CAS on its key word, then its payload word
// is stored: nothing reads payloads before the region is written back.
__device__ __forceinline__ bool region_insert(unsigned long long* tab, uint32_t nb, uint32_t b,
                                              unsigned long long v, bool& dup) {
    const uint32_t key = (uint32_t)v;
    uint32_t* words = reinterpret_cast<uint32_t*>(tab);  // slot q of bucket b: words[8b + 2q] key, +1 payload
    for (; b < nb; ++b) {
        // the whole bucket in two 16-byte reads; a stale empty key only costs a failed CAS
        const uint4 s01 = lds_v4(words + 8 * b);
        const uint4 s23 = lds_v4(words + 8 * b + 4);
        const uint32_t ks[4] = {s01.x, s01.z, s23.x, s23.z};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t c = ks[q];
            if (c == (uint32_t)kEmptyKey) {
                c = atomicCAS(words + 8 * b + 2 * q, (uint32_t)kEmptyKey, key);
                if (c == (uint32_t)kEmptyKey) {
                    words[8 * b + 2 * q + 1] = (uint32_t)(v >> 32);
                    return true;
                }
            }
            if (c == key) dup = true;
        }
    }
    return false;  // the run leaves the region
}

__global__ void __launch_bounds__(kRBuildBlock) k_region_build(const RegionJob* __restrict__ jobs, RegionJob job0,
                                                               uint32_t njobs, uint32_t regions,
                                                               const uint32_t* __restrict__ start,
                                                               const unsigned long long* __restrict__ staging,
                                                               unsigned long long* __restrict__ ovf,
                                                               uint32_t* ovf_count, uint32_t fresh, uint32_t* err) {
    extern __shared__ __align__(128) unsigned long long tab[];  // kRegionBuckets * 4 slots
    __shared__ RegionJob sj;
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    uint32_t phase = 0;
    int64_t cur = -1;
    for (uint32_t g = blockIdx.x; g < regions; g += gridDim.x) {
        const uint32_t s0 = start[g], s1 = start[g + 1];
        if (!fresh && s0 == s1) continue;  // nothing to add, the region stays as it is
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
        }
        __syncthreads();
        uint32_t ins = 0;
        bool dup = false;
        for (uint32_t i0 = s0 + threadIdx.x; i0 < s1; i0 += kRBuildBlock * kPrefetch) {
            unsigned long long v[kPrefetch];
#pragma unroll
            for (int u = 0; u < kPrefetch; ++u) {
                const uint32_t i = i0 + u * kRBuildBlock;
                v[u] = i < s1 ? staging[i] : kEmptySlot;
            }
#pragma unroll
            for (int u = 0; u < kPrefetch; ++u) {
                const uint32_t i = i0 + u * kRBuildBlock;
                if (i >= s1) continue;
                const uint32_t hb = home_bucket((int32_t)(uint32_t)v[u], sj.t) - b0;
                if (region_insert(tab, nb, hb, v[u], dup)) ++ins;
                else ovf[atomicAdd(ovf_count, 1u)] = ((unsigned long long)j << 32) | i;  // the run leaves the region
            }
        }
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
    }
    if (threadIdx.x == 0) bulk_wait_all();  // every region store is complete before the CTA ends
}

// Rows whose run left their region, into the global table (each entry:
// job << 32 | staging row).
__global__ void k_region_overflow(const RegionJob* __restrict__ jobs, RegionJob job0,
                                  const unsigned long long* __restrict__ staging,
                                  const unsigned long long* __restrict__ ovf, const uint32_t* ovf_count, uint32_t* err) {
    const uint32_t cnt = *ovf_count;
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < cnt; x += gridDim.x * blockDim.x) {
        const unsigned long long e = ovf[x];
        const TableView t = jobs ? jobs[e >> 32].t : job0.t;
        const unsigned long long v = staging[(uint32_t)e];
        bool dup = false, ok = false;
        table_insert(t, (int32_t)(uint32_t)v, (int32_t)(uint32_t)(v >> 32), err, dup, ok);
        if (ok) atomicAdd(t.meta + 2, 1ull);
        if (dup) atomicOr(t.meta + 3, 1ull);
    }
}

}  // namespace

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
                                 bool fresh, cudaStream_t s, Context* ctx) {
    if (total_regions == 0) return cudaSuccess;
    if (!items) nitems = (uint32_t)((n + rows_per_item - 1) / rows_per_item);
    const int sms = ctx->prop.multiProcessorCount;
    const size_t hsmem = 4ull * std::max(max_job_regions, 1u);
    const size_t tsmem = 32ull * kRegionBuckets;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_region_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem)) ||
        (e = cudaFuncSetAttribute(k_region_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem)) ||
        (e = cudaFuncSetAttribute(k_region_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem)))
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
    if (nitems) {
        const int grid = (int)std::min<uint64_t>(
            nitems, (uint64_t)occupancy_grid((const void*)k_region_scatter, kRBlock, hsmem, ctx));
        k_region_scatter<<<grid, kRBlock, hsmem, s>>>(d_jobs, job0, items, nitems, n, rows_per_item, sc.cursor,
                                                      sc.staging, ctx->d_err);
        ctx->launches++;
        if ((e = cudaGetLastError())) return e;
    }
    {
        const int grid = (int)std::min<uint64_t>(
            total_regions, (uint64_t)occupancy_grid((const void*)k_region_build, kRBuildBlock, tsmem, ctx));
        k_region_build<<<grid, kRBuildBlock, tsmem, s>>>(d_jobs, job0, njobs, total_regions, sc.start, sc.staging,
                                                         sc.ovf, sc.ovf_count, fresh ? 1u : 0u, ctx->d_err);
        ctx->launches++;
        if ((e = cudaGetLastError())) return e;
    }
    k_region_overflow<<<sms * 2, 256, 0, s>>>(d_jobs, job0, sc.staging, sc.ovf, sc.ovf_count, ctx->d_err);
    ctx->launches++;
    return cudaGetLastError();
}

}  // namespace mgv
