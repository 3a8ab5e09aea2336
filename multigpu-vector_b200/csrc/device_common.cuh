// device_common.cuh -- device-side helpers shared by every mgv kernel.
//
// Replaces the reference's device utilities (src/common.cuh:211-293): lane
// and warp ids, broadcast, warp reductions.  Everything here uses the *_sync
// warp intrinsics; the reference's legacy __shfl/__ballot rely on implicit
// warp synchrony, which independent thread scheduling does not give.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mgv {

constexpr int kWarp = 32;
// Key value reserved as the empty-slot marker of the open-addressing hash
// tables.  Build rows that carry this key are kept in a side list instead.
constexpr int32_t kEmptyKey = INT32_MIN;
constexpr unsigned long long kEmptySlot = 0x8000000080000000ull;

// Device error word layout: [0] = first error code (mgv_status), [1] = detail.
enum DevErr : uint32_t {
    kDevOk = 0,
    kDevTableFull = 2,      // MGV_ENOMEM
    kDevTimeout = 3,        // MGV_ETIMEDOUT
    kDevOverflow = 2,       // output capacity exceeded (MGV_ENOMEM)
};

__device__ __forceinline__ uint32_t lane_id() {
    uint32_t l;
    asm("mov.u32 %0, %%laneid;" : "=r"(l));
    return l;
}

// MurmurHash3 32-bit finaliser; the reference's hashMurmur
// (src/operators/hashjoin.cu:4-11).
__host__ __device__ __forceinline__ uint32_t murmur32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

// Bucket of a key in a table of nbuckets buckets: multiply-shift range
// reduction of the murmur hash, so nbuckets need not be a power of two.
__device__ __forceinline__ uint32_t bucket_of(int32_t key, uint32_t nbuckets) {
    return __umulhi(murmur32((uint32_t)key), nbuckets);
}

__device__ __forceinline__ void set_error(uint32_t* err, uint32_t code, uint32_t detail) {
    if (atomicCAS(err, 0u, code) == 0u) atomicExch(err + 1, detail);
}

// 32 bytes of a streamed column: no L1 allocation and first-out in L2, so
// that streamed input does not push resident hash tables out of L2.
__device__ __forceinline__ void ld_stream8(const int32_t* p, int32_t (&v)[8]) {
    asm volatile(
        "ld.global.nc.L1::no_allocate.L2::evict_first.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
        : "l"(p));
}

// One int32 of a column read once: no L1 allocation and, with an
// evict-first policy (l2_policy_evict_first), first-out in L2, so the
// column's lines do not push a hash table's lines out of L2.
__device__ __forceinline__ int32_t ld_stream1(const int32_t* p, uint64_t policy) {
    int32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(policy));
    return v;
}

// One 32-byte hash bucket (4 slots of {key, payload}), read-only during a
// probe: kept in L2 with evict_last priority, not allocated in L1.
__device__ __forceinline__ void ld_bucket(const unsigned long long* p, uint32_t (&w)[8]) {
    asm volatile(
        "ld.global.nc.L1::no_allocate.L2::evict_last.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
        : "l"(p));
}

// The same bucket read coherently at gpu scope while it is being filled.
__device__ __forceinline__ void ld_bucket_relaxed(const unsigned long long* p, unsigned long long (&s)[4]) {
    asm volatile("ld.relaxed.gpu.global.v4.b64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(s[0]), "=l"(s[1]), "=l"(s[2]), "=l"(s[3])
                 : "l"(p));
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of two u64 values, then one atomicAdd each into acc[0..1].
// Two's-complement addition makes this exact for int64 sums too.
template <int BLOCK>
__device__ __forceinline__ void block_accumulate2(unsigned long long a, unsigned long long b,
                                                  unsigned long long* acc) {
    __shared__ unsigned long long red[2][BLOCK / kWarp];
    a = warp_sum_u64(a);
    b = warp_sum_u64(b);
    const int w = threadIdx.x / kWarp;
    if (lane_id() == 0) { red[0][w] = a; red[1][w] = b; }
    __syncthreads();
    if (threadIdx.x < kWarp) {
        unsigned long long x = threadIdx.x < BLOCK / kWarp ? red[0][threadIdx.x] : 0ull;
        unsigned long long y = threadIdx.x < BLOCK / kWarp ? red[1][threadIdx.x] : 0ull;
        x = warp_sum_u64(x);
        y = warp_sum_u64(y);
        if (threadIdx.x == 0) {
            if (x) atomicAdd(acc + 0, x);
            if (y) atomicAdd(acc + 1, y);
        }
    }
}

// In-place exclusive prefix sum of a[0..n) in shared memory over a CTA of
// BLOCK threads; returns the total.  Every thread of the CTA calls it; a[] is
// complete and the scratch free again when it returns.
template <int BLOCK, typename T = uint32_t>
__device__ __forceinline__ T block_exclusive_scan(T* a, uint32_t n) {
    static_assert(BLOCK % kWarp == 0 && BLOCK / kWarp <= kWarp, "one warp scans the warp totals");
    __shared__ T wsum[BLOCK / kWarp];
    const uint32_t per = (n + BLOCK - 1) / BLOCK;
    const uint32_t lo = threadIdx.x * per;
    const uint32_t lane = lane_id(), warp = threadIdx.x / kWarp;
    T local = 0;
    for (uint32_t i = 0; i < per; ++i)
        if (lo + i < n) local += a[lo + i];
    T x = local;  // inclusive scan over the warp
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == kWarp - 1) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < BLOCK / kWarp ? wsum[lane] : T(0);
#pragma unroll
        for (int o = 1; o < kWarp; o <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        if (lane < BLOCK / kWarp) wsum[lane] = w;
    }
    __syncthreads();
    T base = (warp ? wsum[warp - 1] : T(0)) + x - local;
    for (uint32_t i = 0; i < per; ++i)
        if (lo + i < n) {
            const T c = a[lo + i];
            a[lo + i] = base;
            base += c;
        }
    const T total = wsum[BLOCK / kWarp - 1];
    __syncthreads();
    return total;
}

}  // namespace mgv

namespace mgv {

// ---- mbarrier + bulk async copy (TMA engine, non-tensor form) -------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bulk copy global -> shared, completion counted on `bar` (bytes % 16 == 0,
// both addresses 16-byte aligned).  Never multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// An L2 policy that evicts the lines it touches first: for streamed data
// read once, so it does not push out data kept for reuse (a hash table).
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// bulk_g2s with an L2 cache policy for the source lines.
__device__ __forceinline__ void bulk_g2s_hint(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                              uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
        "%4;" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of `bar`; false if it ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t max_tries) {
    for (uint32_t i = 0; i < max_tries; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Bulk copy shared -> global (bytes % 16 == 0, 16-byte aligned), tracked by
// the issuing thread's bulk async-group.
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// The shared-memory sources of this thread's committed bulk stores have been read.
__device__ __forceinline__ void bulk_wait_reads() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// This thread's committed bulk stores are complete.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Orders this thread's generic-proxy shared-memory writes before later
// async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

}  // namespace mgv
