// probe_staged.cu -- hash probe -> aggregate, warp-specialised.
//
// A random 32-byte bucket read costs one L1TEX request, and an SM retires
// about one such request per clock; the probe is bound by that rate, not by
// HBM.  The kernel therefore spends the SM's request slots on bucket reads
// only:
//
//   * a producer warp streams the probe columns (key, payload) into an
//     S-stage shared-memory ring with cp.async.bulk (TMA engine), one
//     mbarrier pair (full / empty) per stage, so column streaming issues no
//     L1 requests and runs S tiles ahead;
//   * 8 consumer warps take R rows per lane from a landed stage, release the
//     stage, and issue R independent bucket loads;
//   * a probe whose run continues past a full bucket (about 5% at load
//     factor 0.5) is not chased on the spot, which would add a dependent L2
//     round trip to nearly every warp iteration; it is appended to the
//     warp's continuation queue in shared memory, and once 32 are queued
//     each lane takes one and issues its load together with the next
//     round's home-bucket loads.  Before each round the warp drains until
//     the round cannot overflow the queue, so nothing is ever dropped.
//
// Every mbarrier wait is bounded; a wait that runs out sets the context's
// error word and the kernel ends (after a bounded drain of the copies in
// flight), so the host sees MGV_ETIMEDOUT instead of a hung GPU.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "hash_table.cuh"
#include "mgv_internal.h"

namespace mgv {

namespace {

constexpr int kConsumerWarps = 8;
constexpr int kThreads = (kConsumerWarps + 1) * 32;
constexpr uint32_t kWaitTries = 1u << 24;

// continuation queue entries per consumer warp: room for two full rounds
template <int R>
constexpr int queue_len() { return 32 * (R + 1) <= 160 ? 256 : 512; }

struct Acc {
    uint32_t cnt;            // matches of this thread (fits: rows per thread < 2^32)
    unsigned long long sum;  // two's-complement int64
};

// Per-warp continuation queue (ring) in shared memory.  `tail` is a shared
// counter bumped with atomicAdd by the (few) lanes that append; `head` is
// warp-uniform and private to the warp.
struct ContQueue {
    int32_t* key;
    int32_t* pay;
    uint32_t* bucket;
    uint32_t* tail;
    uint32_t head;
};

__device__ __forceinline__ uint32_t next_bucket(uint32_t b, uint32_t nb) { return (b + 1 == nb) ? 0u : b + 1; }

// Home bucket of a key: the radix-laid-out form (RADIX), or the plain
// multiply-shift of the hash for an unpartitioned table (fewer instructions
// per probe on the common path).
template <bool RADIX>
__device__ __forceinline__ uint32_t home(int32_t key, const TableView& t) {
    return RADIX ? home_bucket(key, t) : __umulhi(murmur32((uint32_t)key), t.nbuckets);
}

// Fold one bucket's matches for (key, pay); returns whether the run goes on.
// KO: a key-only bucket of eight keys (build payloads 0, ADD_BP unused).
template <bool UNIQUE, bool ADD_BP, bool ADD_PP, bool KO>
__device__ __forceinline__ bool fold(const uint32_t (&w)[8], int32_t key, int32_t pay, Acc& a) {
    const uint32_t k = (uint32_t)key;
    if (KO) {
        uint32_t c = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) c += w[q] == k;
        const bool full = w[7] != (uint32_t)kEmptyKey;
        if (UNIQUE) c = c != 0;
        a.cnt += c;
        if (ADD_PP) a.sum += (unsigned long long)((long long)c * pay);
        return UNIQUE ? (c == 0 && full) : full;
    }
    const bool m0 = w[0] == k, m1 = w[2] == k, m2 = w[4] == k, m3 = w[6] == k;
    const bool full = w[6] != (uint32_t)kEmptyKey;
    if (UNIQUE) {
        const bool f = m0 | m1 | m2 | m3;
        long long v = 0;
        if (ADD_BP) v += (int32_t)(m0 ? w[1] : m1 ? w[3] : m2 ? w[5] : w[7]);
        if (ADD_PP) v += pay;
        a.cnt += f;
        if (ADD_BP || ADD_PP) a.sum += f ? (unsigned long long)v : 0ull;
        return !f && full;
    }
    const uint32_t mc = (uint32_t)m0 + m1 + m2 + m3;
    a.cnt += mc;
    long long v = 0;
    if (ADD_BP)
        v += (m0 ? (long long)(int32_t)w[1] : 0ll) + (m1 ? (long long)(int32_t)w[3] : 0ll) +
             (m2 ? (long long)(int32_t)w[5] : 0ll) + (m3 ? (long long)(int32_t)w[7] : 0ll);
    if (ADD_PP) v += (long long)mc * pay;
    if (ADD_BP || ADD_PP) a.sum += (unsigned long long)v;
    return full;
}

template <int Q>
__device__ __forceinline__ void enqueue(const ContQueue& q, int32_t key, int32_t pay, uint32_t b) {
    const uint32_t pos = atomicAdd(q.tail, 1u) & (Q - 1);
    q.key[pos] = key;
    q.pay[pos] = pay;
    q.bucket[pos] = b;
}

// Probe rows of the reserved key INT32_MIN against the side list.
template <bool ADD_BP, bool ADD_PP>
__device__ __forceinline__ void fold_reserved(const TableView& t, int32_t pay, Acc& a) {
    const unsigned long long c = t.meta[0];
    a.cnt += (uint32_t)c;
    long long add = 0;
    if (ADD_BP) add += (long long)t.meta[1];
    if (ADD_PP) add += (long long)c * pay;
    a.sum += (unsigned long long)add;
}

// One round for a warp: R rows per lane, row r of lane l at rk[32 r + l] /
// rp[32 r + l] (so each read of the warp is one conflict-free 128-byte
// wavefront; shared or global memory, valid bits in `valid`) plus, when the queue holds a batch
// (or `drain`), one continuation per lane.  The rows are read twice --
// to issue the bucket loads and again to fold the results -- so that no
// key or payload stays in a register across the L2 latency.  Returns a
// value that depends on every row read (for releasing a stage safely).
template <int R, int Q, bool UNIQUE, bool ADD_BP, bool ADD_PP, bool RADIX, bool KO>
__device__ __forceinline__ uint32_t round(const int32_t* rk, const int32_t* rp, uint32_t valid, ContQueue& q,
                                          bool drain, const TableView& t, Acc& a) {
    const uint32_t lane = lane_id();
    __syncwarp();
    const uint32_t avail = *((volatile uint32_t*)q.tail) - q.head;
    int32_t ck = 0, cp = 0;
    uint32_t cb = 0;
    bool has_c = false;
    if (avail >= 32 || (drain && avail > 0)) {
        const uint32_t m = avail < 32 ? avail : 32;
        if (lane < m) {
            const uint32_t idx = (q.head + lane) & (Q - 1);
            ck = q.key[idx];
            cp = q.pay[idx];
            cb = q.bucket[idx];
            has_c = true;
        }
        q.head += m;
    }
    // issue every load of the round before looking at any of them
    uint32_t w[R][8];
#pragma unroll
    for (int r = 0; r < R; ++r)
        if ((valid >> r) & 1u) ld_bucket(t.slots + 4ull * home<RADIX>(rk[32 * r], t), w[r]);
    uint32_t wc[8];
    if (has_c) ld_bucket(t.slots + 4ull * cb, wc);
    __syncwarp();  // every lane has read its queue entry before anyone appends

    uint32_t dep = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        if (!((valid >> r) & 1u)) continue;
        const int32_t key = rk[32 * r];
        const int32_t pay = ADD_PP ? rp[32 * r] : 0;
        dep ^= (uint32_t)key ^ (uint32_t)pay;
        if (key == kEmptyKey) {
            fold_reserved<ADD_BP, ADD_PP>(t, pay, a);
        } else if (fold<UNIQUE, ADD_BP, ADD_PP, KO>(w[r], key, pay, a)) {
            enqueue<Q>(q, key, pay, next_bucket(home<RADIX>(key, t), t.nbuckets));
        }
    }
    if (has_c && fold<UNIQUE, ADD_BP, ADD_PP, KO>(wc, ck, cp, a)) enqueue<Q>(q, ck, cp, next_bucket(cb, t.nbuckets));
    return dep;
}

// Continuation-only rounds until a full round can no longer overflow the
// queue.  They never grow it, and every run ends, so this terminates.
template <int R, int Q, bool UNIQUE, bool ADD_BP, bool ADD_PP, bool RADIX, bool KO>
__device__ __forceinline__ void make_room(ContQueue& q, const TableView& t, Acc& a, uint32_t limit) {
    for (uint32_t guard = 0; guard < (1u << 24); ++guard) {
        __syncwarp();
        if (*((volatile uint32_t*)q.tail) - q.head <= limit) break;
        round<R, Q, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>(nullptr, nullptr, 0u, q, true, t, a);
    }
}

template <int R, int S, int MB, bool UNIQUE, bool ADD_BP, bool ADD_PP, bool RADIX, bool KO = false>
__global__ void __launch_bounds__(kThreads, MB)
    k_probe_agg_ws(const int32_t* __restrict__ keys, const int32_t* __restrict__ pays, uint64_t n, TableView t,
                   unsigned long long* acc, uint32_t* err) {
    constexpr int T = kConsumerWarps * 32 * R;  // rows per tile
    constexpr int Q = queue_len<R>();
    constexpr uint32_t kRoomLimit = (uint32_t)(Q - 32 * (R + 1));
    extern __shared__ __align__(128) unsigned char smem_raw[];
    int32_t* sk = reinterpret_cast<int32_t*>(smem_raw);
    int32_t* sp = sk + S * T;
    int32_t* qbase = sp + (ADD_PP ? S * T : 0);
    uint32_t* tails = reinterpret_cast<uint32_t*>(qbase + 3 * kConsumerWarps * Q);
    uint64_t* full = reinterpret_cast<uint64_t*>(tails + kConsumerWarps);
    uint64_t* empty = full + S;

    const uint64_t nfull = n / T;
    const uint64_t my_tiles = nfull > blockIdx.x ? (nfull - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const uint32_t tile_bytes = (uint32_t)T * sizeof(int32_t);
    const int warp = threadIdx.x / 32;
    const uint32_t lane = lane_id();
    const uint32_t zero = (uint32_t)(n >> 63);  // 0 for every real row count

    if (threadIdx.x < kConsumerWarps) tails[threadIdx.x] = 0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kConsumerWarps);
        }
        fence_barrier_init();
    }
    __syncthreads();

    Acc a{0u, 0ull};
    if (warp == kConsumerWarps) {
        // ---- producer warp: keep S tiles of the probe columns in flight ----
        if (lane == 0) {
            const uint64_t stream_policy = l2_policy_evict_first();  // columns are read once; the table stays
            uint64_t i = 0;
            for (; i < my_tiles; ++i) {
                const int s = (int)(i % S);
                if (i >= (uint64_t)S &&
                    !mbar_wait_bounded(&empty[s], (uint32_t)(((i / S) - 1) & 1), kWaitTries)) {
                    set_error(err, kDevTimeout, 11);
                    break;
                }
                const uint64_t tile = blockIdx.x + i * gridDim.x;
                mbar_expect_tx(&full[s], ADD_PP ? 2 * tile_bytes : tile_bytes);
                bulk_g2s_hint(sk + s * T, keys + tile * T, tile_bytes, &full[s], stream_policy);
                if (ADD_PP) bulk_g2s_hint(sp + s * T, pays + tile * T, tile_bytes, &full[s], stream_policy);
            }
            // let every copy issued land before the CTA can exit
            const uint64_t lo = i > (uint64_t)S ? i - S : 0;
            for (uint64_t j = lo; j < i; ++j) mbar_wait_bounded(&full[j % S], (uint32_t)((j / S) & 1), kWaitTries);
        }
    } else {
        // ---- consumer warps ----
        ContQueue q;
        q.key = qbase + warp * Q;
        q.pay = qbase + (kConsumerWarps + warp) * Q;
        q.bucket = reinterpret_cast<uint32_t*>(qbase + (2 * kConsumerWarps + warp) * Q);
        q.tail = tails + warp;
        q.head = 0;
        const int row0 = warp * 32 * R + (int)lane;
        bool ok = true;
        for (uint64_t i = 0; i < my_tiles; ++i) {
            const int s = (int)(i % S);
            if (!mbar_wait_bounded(&full[s], (uint32_t)((i / S) & 1), kWaitTries)) ok = false;
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) set_error(err, kDevTimeout, 12);
                break;
            }
            make_room<R, Q, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>(q, t, a, kRoomLimit);
            const uint32_t dep = round<R, Q, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>(sk + s * T + row0, sp + s * T + row0,
                                                                     (1u << R) - 1u, q, false, t, a);
            // Release the stage once every lane's reads of it have landed:
            // combine the values read across the warp (the reduction waits
            // for each lane's loads), order the reads before the async-proxy
            // (TMA) refill, and make the arrive's address depend on the
            // combined value through a run-time zero the compiler cannot fold.
            const uint32_t wdep = __reduce_or_sync(0xffffffffu, dep);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            if (lane == 0) {
                const uint32_t addr = smem_u32(&empty[s]) + ((wdep & zero) << 3);
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(addr) : "memory");
            }
        }
        if (ok && blockIdx.x == gridDim.x - 1) {
            // rows of the last partial tile, straight from global memory
            const uint64_t base = nfull * T + (uint64_t)row0;
            uint32_t valid = 0;
#pragma unroll
            for (int r = 0; r < R; ++r) valid |= (uint32_t)(base + 32 * r < n) << r;
            make_room<R, Q, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>(q, t, a, kRoomLimit);
            round<R, Q, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>(keys + base, ADD_PP ? pays + base : nullptr, valid, q, false, t, a);
        }
        // drain the continuation queue
        make_room<R, Q, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>(q, t, a, 0u);
    }
    block_accumulate2<kThreads>((unsigned long long)a.cnt, a.sum, acc);
}

// The same probe with the consumer rounds software-pipelined: a consumer
// warp issues the bucket loads of its next tile row by row as it folds the
// current tile's rows, so the register of row r is refilled right after its
// fold and the warp always has R bucket loads in flight; the current tile's
// stage is released once its folds are done.  Continuations are served by
// continuation-only rounds (one load per lane) whenever the queue holds a
// batch, which also keeps room for a tile's appends.
template <int R, int S, int MB, bool UNIQUE, bool ADD_BP, bool ADD_PP, bool RADIX, bool KO = false>
__global__ void __launch_bounds__(kThreads, MB)
    k_probe_agg_pipe(const int32_t* __restrict__ keys, const int32_t* __restrict__ pays, uint64_t n, TableView t,
                     unsigned long long* acc, uint32_t* err) {
    constexpr int T = kConsumerWarps * 32 * R;  // rows per tile
    constexpr int Q = queue_len<R>();
    constexpr uint32_t kRoomLimit = (uint32_t)(Q - 32 * (R + 1));
    extern __shared__ __align__(128) unsigned char smem_raw[];
    int32_t* sk = reinterpret_cast<int32_t*>(smem_raw);
    int32_t* sp = sk + S * T;
    int32_t* qbase = sp + (ADD_PP ? S * T : 0);
    uint32_t* tails = reinterpret_cast<uint32_t*>(qbase + 3 * kConsumerWarps * Q);
    uint64_t* full = reinterpret_cast<uint64_t*>(tails + kConsumerWarps);
    uint64_t* empty = full + S;

    const uint64_t nfull = n / T;
    const uint64_t my_tiles = nfull > blockIdx.x ? (nfull - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
    const uint32_t tile_bytes = (uint32_t)T * sizeof(int32_t);
    const int warp = threadIdx.x / 32;
    const uint32_t lane = lane_id();
    const uint32_t zero = (uint32_t)(n >> 63);  // 0 for every real row count

    if (threadIdx.x < kConsumerWarps) tails[threadIdx.x] = 0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kConsumerWarps);
        }
        fence_barrier_init();
    }
    __syncthreads();

    Acc a{0u, 0ull};
    if (warp == kConsumerWarps) {
        // ---- producer warp: keep S tiles of the probe columns in flight ----
        if (lane == 0) {
            const uint64_t stream_policy = l2_policy_evict_first();  // columns are read once; the table stays
            uint64_t i = 0;
            for (; i < my_tiles; ++i) {
                const int s = (int)(i % S);
                if (i >= (uint64_t)S &&
                    !mbar_wait_bounded(&empty[s], (uint32_t)(((i / S) - 1) & 1), kWaitTries)) {
                    set_error(err, kDevTimeout, 13);
                    break;
                }
                const uint64_t tile = blockIdx.x + i * gridDim.x;
                mbar_expect_tx(&full[s], ADD_PP ? 2 * tile_bytes : tile_bytes);
                bulk_g2s_hint(sk + s * T, keys + tile * T, tile_bytes, &full[s], stream_policy);
                if (ADD_PP) bulk_g2s_hint(sp + s * T, pays + tile * T, tile_bytes, &full[s], stream_policy);
            }
            const uint64_t lo = i > (uint64_t)S ? i - S : 0;
            for (uint64_t j = lo; j < i; ++j) mbar_wait_bounded(&full[j % S], (uint32_t)((j / S) & 1), kWaitTries);
        }
    } else {
        // ---- consumer warps ----
        ContQueue q;
        q.key = qbase + warp * Q;
        q.pay = qbase + (kConsumerWarps + warp) * Q;
        q.bucket = reinterpret_cast<uint32_t*>(qbase + (2 * kConsumerWarps + warp) * Q);
        q.tail = tails + warp;
        q.head = 0;
        const int row0 = warp * 32 * R + (int)lane;
        bool ok = true;
        uint32_t w[R][8];
        if (my_tiles) {
            if (!mbar_wait_bounded(&full[0], 0u, kWaitTries)) ok = false;
            if (__all_sync(0xffffffffu, ok)) {
                const int32_t* rk = sk + row0;
#pragma unroll
                for (int r = 0; r < R; ++r) ld_bucket(t.slots + 4ull * home<RADIX>(rk[32 * r], t), w[r]);
            } else if (lane == 0) {
                set_error(err, kDevTimeout, 14);
            }
        }
        for (uint64_t i = 0; i < my_tiles && __all_sync(0xffffffffu, ok); ++i) {
            const int s = (int)(i % S);
            const bool next = i + 1 < my_tiles;
            const int s1 = (int)((i + 1) % S);
            if (next && !mbar_wait_bounded(&full[s1], (uint32_t)(((i + 1) / S) & 1), kWaitTries)) ok = false;
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) set_error(err, kDevTimeout, 15);
                break;
            }
            // room for this tile's appends; the rounds use their own registers
            make_room<R, Q, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>(q, t, a, kRoomLimit);
            const int32_t* rk = sk + s * T + row0;
            const int32_t* rp = sp + s * T + row0;
            const int32_t* nk = sk + s1 * T + row0;
            uint32_t dep = 0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int32_t key = rk[32 * r];
                const int32_t pay = ADD_PP ? rp[32 * r] : 0;
                dep ^= (uint32_t)key ^ (uint32_t)pay;
                if (key == kEmptyKey) {
                    fold_reserved<ADD_BP, ADD_PP>(t, pay, a);
                } else if (fold<UNIQUE, ADD_BP, ADD_PP, KO>(w[r], key, pay, a)) {
                    enqueue<Q>(q, key, pay, next_bucket(home<RADIX>(key, t), t.nbuckets));
                }
                if (next) ld_bucket(t.slots + 4ull * home<RADIX>(nk[32 * r], t), w[r]);  // row r of the next tile
            }
            // release the stage as the plain kernel does (see k_probe_agg_ws)
            const uint32_t wdep = __reduce_or_sync(0xffffffffu, dep);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            if (lane == 0) {
                const uint32_t addr = smem_u32(&empty[s]) + ((wdep & zero) << 3);
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(addr) : "memory");
            }
        }
        if (ok && blockIdx.x == gridDim.x - 1) {
            // rows of the last partial tile, straight from global memory
            const uint64_t base = nfull * T + (uint64_t)row0;
            uint32_t valid = 0;
#pragma unroll
            for (int r = 0; r < R; ++r) valid |= (uint32_t)(base + 32 * r < n) << r;
            make_room<R, Q, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>(q, t, a, kRoomLimit);
            round<R, Q, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>(keys + base, ADD_PP ? pays + base : nullptr, valid, q, false,
                                                           t, a);
        }
        // drain the continuation queue
        make_room<R, Q, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>(q, t, a, 0u);
    }
    block_accumulate2<kThreads>((unsigned long long)a.cnt, a.sum, acc);
}

template <int R, int S, int MB, bool UNIQUE, bool ADD_BP, bool ADD_PP, bool RADIX, bool KO = false>
cudaError_t launch_v(const int32_t* keys, const int32_t* pays, uint64_t n, const TableView& t,
                     unsigned long long* acc, int ctas_per_sm, cudaStream_t s, Context* ctx) {
    // probe_kernel 0 (auto) and 3: the software-pipelined consumer rounds
    // (measured faster); 2: the plain rounds
    auto k = ctx->tuning.probe_kernel == 2 ? k_probe_agg_ws<R, S, MB, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>
                                           : k_probe_agg_pipe<R, S, MB, UNIQUE, ADD_BP, ADD_PP, RADIX, KO>;
    constexpr int T = kConsumerWarps * 32 * R;
    const size_t smem = (size_t)(ADD_PP ? 2 : 1) * S * T * sizeof(int32_t) +
                        (size_t)3 * kConsumerWarps * queue_len<R>() * sizeof(int32_t) +
                        kConsumerWarps * sizeof(uint32_t) + 2 * S * sizeof(uint64_t);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    if (ctas_per_sm > 0 && ctas_per_sm < per_sm) per_sm = ctas_per_sm;
    uint64_t grid = (uint64_t)per_sm * ctx->prop.multiProcessorCount;
    const uint64_t nfull = n / T;
    if (grid > nfull) grid = nfull ? nfull : 1;
    k<<<(int)grid, kThreads, smem, s>>>(keys, pays, n, t, acc, ctx->d_err);
    ctx->launches++;
    return cudaGetLastError();
}

template <int R, int S, int MB, bool UNIQUE, bool RADIX>
cudaError_t launch_mode_r(const int32_t* keys, const int32_t* pays, uint64_t n, const TableView& t, uint32_t mode,
                          unsigned long long* acc, int ctas, cudaStream_t s, Context* ctx) {
    switch (mode) {
        case 0: return launch_v<R, S, MB, UNIQUE, false, false, RADIX>(keys, pays, n, t, acc, ctas, s, ctx);
        case 1: return launch_v<R, S, MB, UNIQUE, true, false, RADIX>(keys, pays, n, t, acc, ctas, s, ctx);
        case 2: return launch_v<R, S, MB, UNIQUE, false, true, RADIX>(keys, pays, n, t, acc, ctas, s, ctx);
        default: return launch_v<R, S, MB, UNIQUE, true, true, RADIX>(keys, pays, n, t, acc, ctas, s, ctx);
    }
}

template <int R, int S, int MB, bool UNIQUE>
cudaError_t launch_mode(const int32_t* keys, const int32_t* pays, uint64_t n, const TableView& t, uint32_t mode,
                        unsigned long long* acc, int ctas, cudaStream_t s, Context* ctx) {
    if (t.radix_mask != 0) return launch_mode_r<R, S, MB, UNIQUE, true>(keys, pays, n, t, mode, acc, ctas, s, ctx);
    return launch_mode_r<R, S, MB, UNIQUE, false>(keys, pays, n, t, mode, acc, ctas, s, ctx);
}

}  // namespace

// Returns cudaErrorNotSupported when this kernel does not apply (columns
// not 16-byte aligned); the caller then uses the register-prefetch kernel.
cudaError_t launch_probe_agg_staged(const int32_t* keys, const int32_t* pays, uint64_t n, const TableView& t,
                                    bool unique, uint32_t sum_mode, unsigned long long* acc, cudaStream_t s,
                                    Context* ctx) {
    if (((uintptr_t)keys & 15u) || ((uintptr_t)pays & 15u)) return cudaErrorNotSupported;
    const uint32_t mode = (sum_mode & 1u) | ((sum_mode & 2u) && pays ? 2u : 0u);
    if (t.key_only) {  // eight keys per bucket, payloads 0: the default shape only
        const bool radix = t.radix_mask != 0, pp = (mode & 2u) != 0;
        const int ctas = (int)ctx->tuning.probe_ctas_per_sm;
#define MGV_KO(U, P, X) return launch_v<4, 4, 3, U, false, P, X, true>(keys, pays, n, t, acc, ctas, s, ctx)
        if (unique) {
            if (pp) { if (radix) MGV_KO(true, true, true); MGV_KO(true, true, false); }
            if (radix) MGV_KO(true, false, true);
            MGV_KO(true, false, false);
        }
        if (pp) { if (radix) MGV_KO(false, true, true); MGV_KO(false, true, false); }
        if (radix) MGV_KO(false, false, true);
        MGV_KO(false, false, false);
#undef MGV_KO
    }
    const mgv_tuning& tu = ctx->tuning;
    const int ctas = (int)tu.probe_ctas_per_sm;
    const int st = tu.probe_stages <= 2 ? 2 : tu.probe_stages <= 4 ? 4 : 6;
    // Register budgets: R = 4 at 2, 3 or 4 CTAs per SM (3 and 4 when
    // probe_ctas_per_sm asks for them), R = 8 at 1 (at 2 it spills).
#define MGV_WS(RR, SS, MBB)                                                                        \
    return unique ? launch_mode<RR, SS, MBB, true>(keys, pays, n, t, mode, acc, ctas, s, ctx)     \
                  : launch_mode<RR, SS, MBB, false>(keys, pays, n, t, mode, acc, ctas, s, ctx)
    if (tu.probe_rows_per_thread == 8) {
        switch (st) {
            case 2: MGV_WS(8, 2, 1);
            case 4: MGV_WS(8, 4, 1);
            default: MGV_WS(8, 6, 1);
        }
    }
    if (ctas == 3) {
        switch (st) {
            case 2: MGV_WS(4, 2, 3);
            case 4: MGV_WS(4, 4, 3);
            default: MGV_WS(4, 6, 3);
        }
    }
    if (ctas == 4) {
        switch (st) {
            case 2: MGV_WS(4, 2, 4);
            default: MGV_WS(4, 4, 4);
        }
    }
    switch (st) {
        case 2: MGV_WS(4, 2, 2);
        case 4: MGV_WS(4, 4, 2);
        default: MGV_WS(4, 6, 2);
    }
#undef MGV_WS
}

}  // namespace mgv
