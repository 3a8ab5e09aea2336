// diag.cu -- roofline diagnostics: the rates at which the GPU serves random
// reads of hash buckets, the operation every hash probe is built on
// (include/mgv_diag.h; not part of the drop-in operator API).
//
// mgv_diag_random_gather: each thread hashes R streamed keys, issues R
// independent 32-byte loads at the hashed bucket of a table, and folds the
// words it read.
//
// mgv_diag_gather: the same question by line width (32 / 64 / 128 bytes per
// lookup) and by path: LSU loads, where line_bytes / 32 lanes read one
// aligned block together (one cache line per lookup, whatever its width),
// or the TMA engine's tile::gather4 (four table rows per instruction into
// shared memory, bypassing the LSU request path), or both at once.  The
// lookups hash the row index, so no column is streamed: the figure is the
// bare lookup rate.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "../../include/mgv_diag.h"
#include "device_common.cuh"
#include "mgv_internal.h"

namespace mgv {
namespace {

constexpr uint32_t kDiagWaitTries = 1u << 24;

__global__ void k_diag_fill(uint32_t* p, uint64_t n, uint32_t salt) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = murmur32((uint32_t)i ^ salt) ^ (uint32_t)(i * 2654435761u);
}

template <int R>
__global__ void __launch_bounds__(256) k_diag_gather(const uint32_t* __restrict__ keys, uint64_t n,
                                                     const unsigned long long* __restrict__ table, uint32_t nb,
                                                     uint32_t* sink) {
    const uint64_t T = 256ull * R;
    uint32_t acc = 0;
    for (uint64_t t = blockIdx.x; t * T < n; t += gridDim.x) {
        const uint64_t r0 = t * T + threadIdx.x * (uint64_t)R;
        uint32_t k[R];
#pragma unroll
        for (int r = 0; r < R; ++r) k[r] = (r0 + r < n) ? __ldg(keys + r0 + r) : 0u;
        uint32_t w[R][8];
#pragma unroll
        for (int r = 0; r < R; ++r) ld_bucket(table + 4ull * __umulhi(murmur32(k[r]), nb), w[r]);
#pragma unroll
        for (int r = 0; r < R; ++r) acc ^= w[r][0] ^ w[r][3] ^ w[r][6] ^ w[r][7] ^ (w[r][2] == k[r]);
    }
    if (acc == 0x9E3779B9u) sink[0] = acc;  // keeps the loads alive
}

// Line of lookup j in a table of nlines lines.
__device__ __forceinline__ uint32_t diag_line(uint64_t j, uint32_t nlines) {
    return __umulhi(murmur32((uint32_t)j ^ 0x2545F491u) ^ (uint32_t)(j >> 32), nlines);
}

// One tile::gather4 of four table rows into shared memory, completion counted
// on `bar`.  The tensor map covers this GPU's own table; no multicast.
__device__ __forceinline__ void tma_gather4(void* dst, const CUtensorMap* map, int32_t r0, int32_t r1, int32_t r2,
                                            int32_t r3, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(smem_u32(bar))
        : "memory");
}

// LB bytes per lookup; R lookups in flight per lane group (LSU warps); D
// gather4 instructions in flight per lane (TMA warps).
template <int LB, int R>
__global__ void k_diag_lines(const __grid_constant__ CUtensorMap map, const unsigned char* __restrict__ table,
                             uint32_t nlines, uint64_t n_lsu, uint64_t n_tma, uint32_t lsu_warps, uint32_t tma_warps,
                             uint32_t D, uint32_t* sink, uint32_t* err) {
    constexpr int LPL = LB / 32;  // lanes per line
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t warp = threadIdx.x / 32, lane = lane_id();
    uint32_t acc = 0;
    if (warp < lsu_warps) {
        const uint64_t groups = (uint64_t)gridDim.x * lsu_warps * (32 / LPL);
        const uint64_t g = ((uint64_t)blockIdx.x * lsu_warps + warp) * (32 / LPL) + lane / LPL;
        const uint32_t sub = lane % LPL;
        for (uint64_t base = g * R; base < n_lsu; base += groups * R) {
            uint32_t w[R][8];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint64_t j = base + r;
                if (j < n_lsu)
                    ld_bucket(reinterpret_cast<const unsigned long long*>(table + (uint64_t)diag_line(j, nlines) * LB +
                                                                          32 * sub),
                              w[r]);
            }
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (base + r < n_lsu) acc ^= w[r][0] ^ w[r][5] ^ w[r][7];
        }
    } else if (warp < lsu_warps + tma_warps) {
        // every lane issues its own gathers: D slots of 4 rows, one mbarrier each
        const uint32_t t = (warp - lsu_warps) * 32 + lane;
        unsigned char* slots = smem + (size_t)t * D * 4 * LB;
        uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)tma_warps * 32 * D * 4 * LB) + (size_t)t * D;
        for (uint32_t d = 0; d < D; ++d) mbar_init(&bars[d], 1);
        fence_barrier_init();
        const uint64_t issuers = (uint64_t)gridDim.x * tma_warps * 32;
        const uint64_t quads = n_tma / 4;
        uint64_t it = 0;
        bool ok = true;
        for (uint64_t q = (uint64_t)blockIdx.x * tma_warps * 32 + t; q < quads && ok; q += issuers, ++it) {
            const uint32_t d = (uint32_t)(it % D);
            if (it >= D) {
                if (!mbar_wait_bounded(&bars[d], (uint32_t)((it / D - 1) & 1), kDiagWaitTries)) {
                    set_error(err, kDevTimeout, 21);
                    ok = false;
                    break;
                }
                const uint32_t* v = reinterpret_cast<const uint32_t*>(slots + (size_t)d * 4 * LB);
                acc ^= v[0] ^ v[LB / 4] ^ v[LB / 2] ^ v[3 * LB / 4];
                fence_proxy_async_smem();
            }
            mbar_expect_tx(&bars[d], 4 * LB);
            const uint64_t j = 4 * q + n_lsu;
            tma_gather4(slots + (size_t)d * 4 * LB, &map, (int32_t)diag_line(j, nlines),
                        (int32_t)diag_line(j + 1, nlines), (int32_t)diag_line(j + 2, nlines),
                        (int32_t)diag_line(j + 3, nlines), &bars[d]);
        }
        // drain what is in flight
        const uint64_t lo = it > D ? it - D : 0;
        for (uint64_t k = lo; k < it; ++k) {
            const uint32_t d = (uint32_t)(k % D);
            if (mbar_wait_bounded(&bars[d], (uint32_t)((k / D) & 1), kDiagWaitTries)) {
                const uint32_t* v = reinterpret_cast<const uint32_t*>(slots + (size_t)d * 4 * LB);
                acc ^= v[0];
            } else {
                set_error(err, kDevTimeout, 22);
            }
        }
    }
    if (acc == 0x9E3779B9u) sink[0] = acc;  // keeps the loads alive
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

mgv_status encode_rows_map(CUtensorMap* map, void* base, uint32_t nlines, uint32_t line_bytes) {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
            return fail(MGV_ECUDA, "cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    const cuuint64_t dims[2] = {line_bytes / 4u, nlines};
    const cuuint64_t strides[1] = {line_bytes};
    const cuuint32_t box[2] = {line_bytes / 4u, 1u};  // one row high (tile::gather4)
    const cuuint32_t estr[2] = {1u, 1u};
    const CUtensorMapL2promotion prom = line_bytes >= 128 ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B
                                        : line_bytes >= 64 ? CU_TENSOR_MAP_L2_PROMOTION_L2_64B
                                                           : CU_TENSOR_MAP_L2_PROMOTION_NONE;
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, base, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, prom,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(MGV_ECUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return MGV_OK;
}

template <int LB>
cudaError_t launch_lines(const CUtensorMap& map, const unsigned char* table, uint32_t nlines, uint64_t n_lsu,
                         uint64_t n_tma, uint32_t lsu_warps, uint32_t tma_warps, uint32_t inflight, int grid,
                         size_t smem, uint32_t* sink, uint32_t* err, cudaStream_t s) {
    const int threads = (int)(lsu_warps + tma_warps) * 32;
#define MGV_DIAG_R(RR)                                                                                       \
    do {                                                                                                     \
        auto k = k_diag_lines<LB, RR>;                                                                       \
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);     \
        if (e != cudaSuccess) return e;                                                                      \
        k<<<grid, threads, smem, s>>>(map, table, nlines, n_lsu, n_tma, lsu_warps, tma_warps, inflight, sink, \
                                      err);                                                                  \
        return cudaGetLastError();                                                                           \
    } while (0)
    if (inflight <= 2) MGV_DIAG_R(2);
    if (inflight <= 4) MGV_DIAG_R(4);
    MGV_DIAG_R(8);
#undef MGV_DIAG_R
}

}  // namespace
}  // namespace mgv

using namespace mgv;

extern "C" mgv_status mgv_diag_random_gather(mgv_ctx* ctx, uint64_t table_bytes, uint64_t n, uint32_t ctas_per_sm,
                                             uint32_t reps, double* ms_per_pass) {
    if (!ctx || !ms_per_pass) return fail(MGV_EINVAL, "NULL argument");
    if (table_bytes < 32 || table_bytes > (1ull << 36) || n == 0 || reps == 0 || ctas_per_sm == 0 || ctas_per_sm > 8)
        return fail(MGV_EINVAL, "argument out of range");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const uint32_t nb = (uint32_t)(table_bytes / 32);
    uint32_t *keys = nullptr, *sink = nullptr;
    unsigned long long* table = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    mgv_status st = MGV_OK;
    cudaError_t e = cudaMallocAsync(&keys, n * 4, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&table, (size_t)nb * 32, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&sink, 4, s);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) {
        const int sms = ctx->prop.multiProcessorCount;
        k_diag_fill<<<sms * 8, 256, 0, s>>>(keys, n, 1u);
        k_diag_fill<<<sms * 8, 256, 0, s>>>(reinterpret_cast<uint32_t*>(table), (uint64_t)nb * 8, 2u);
        const int grid = sms * (int)ctas_per_sm;
        k_diag_gather<4><<<grid, 256, 0, s>>>(keys, n, table, nb, sink);  // warm-up
        cudaEventRecord(e0, s);
        for (uint32_t i = 0; i < reps; ++i) k_diag_gather<4><<<grid, 256, 0, s>>>(keys, n, table, nb, sink);
        cudaEventRecord(e1, s);
        ctx->launches += 3 + reps;
        e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        *ms_per_pass = (double)ms / reps;
    }
    if (e != cudaSuccess) st = cuda_fail(e, "mgv_diag_random_gather");
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (keys) cudaFreeAsync(keys, s);
    if (table) cudaFreeAsync(table, s);
    if (sink) cudaFreeAsync(sink, s);
    cudaStreamSynchronize(s);
    return st;
}

extern "C" mgv_status mgv_diag_gather(mgv_ctx* ctx, const mgv_diag_gather_desc* d, double* ms_per_pass) {
    if (!ctx || !d || !ms_per_pass) return fail(MGV_EINVAL, "NULL argument");
    const uint32_t lb = d->line_bytes;
    if (lb != 32 && lb != 64 && lb != 128) return fail(MGV_EINVAL, "line_bytes must be 32, 64 or 128");
    if (d->table_bytes < 4096 || d->table_bytes > (1ull << 36) || d->table_bytes / lb > 0x7fffffffull)
        return fail(MGV_EINVAL, "table_bytes out of range");
    if (d->lookups == 0 || d->reps == 0 || d->ctas_per_sm == 0 || d->ctas_per_sm > 8 || d->method > 2 ||
        d->inflight == 0 || d->inflight > 8)
        return fail(MGV_EINVAL, "argument out of range");
    const uint32_t lsu_warps = d->method == 1 ? 0u : d->lsu_warps;
    const uint32_t tma_warps = d->method == 0 ? 0u : d->tma_warps;
    if (lsu_warps + tma_warps == 0 || lsu_warps + tma_warps > 32 || (d->method == 0 && !lsu_warps) ||
        (d->method >= 1 && !tma_warps))
        return fail(MGV_EINVAL, "warp counts out of range");
    const float share = d->method == 0 ? 0.f : d->method == 1 ? 1.f : d->tma_share;
    if (!(share >= 0.f && share <= 1.f)) return fail(MGV_EINVAL, "tma_share out of range");
    const uint64_t n_tma = ((uint64_t)((double)d->lookups * share)) & ~3ull;
    const uint64_t n_lsu = d->lookups - n_tma;
    const size_t smem = tma_warps ? (size_t)tma_warps * 32 * d->inflight * (4 * lb + 8) : 0;
    if (smem > 200 * 1024) return fail(MGV_EINVAL, "TMA slots exceed shared memory");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const uint32_t nlines = (uint32_t)(d->table_bytes / lb);
    unsigned char* table = nullptr;
    uint32_t* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CUtensorMap map;
    memset(&map, 0, sizeof(map));
    cudaError_t e = cudaMallocAsync(&table, (size_t)nlines * lb, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&sink, 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_err, 0, 8, s);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    mgv_status st = MGV_OK;
    if (e == cudaSuccess && tma_warps) st = encode_rows_map(&map, table, nlines, lb);
    if (e == cudaSuccess && st == MGV_OK) {
        const int sms = ctx->prop.multiProcessorCount;
        k_diag_fill<<<sms * 8, 256, 0, s>>>(reinterpret_cast<uint32_t*>(table), (uint64_t)nlines * lb / 4, 2u);
        const int grid = sms * (int)d->ctas_per_sm;
        auto run = [&]() -> cudaError_t {
            switch (lb) {
                case 32: return launch_lines<32>(map, table, nlines, n_lsu, n_tma, lsu_warps, tma_warps, d->inflight,
                                                 grid, smem, sink, ctx->d_err, s);
                case 64: return launch_lines<64>(map, table, nlines, n_lsu, n_tma, lsu_warps, tma_warps, d->inflight,
                                                 grid, smem, sink, ctx->d_err, s);
                default: return launch_lines<128>(map, table, nlines, n_lsu, n_tma, lsu_warps, tma_warps,
                                                  d->inflight, grid, smem, sink, ctx->d_err, s);
            }
        };
        e = run();  // warm-up
        if (e == cudaSuccess) e = cudaEventRecord(e0, s);
        for (uint32_t i = 0; i < d->reps && e == cudaSuccess; ++i) e = run();
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        ctx->launches += 2 + d->reps;
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        *ms_per_pass = (double)ms / d->reps;
        uint32_t err[2] = {0, 0};
        if (e == cudaSuccess) e = cudaMemcpy(err, ctx->d_err, sizeof(err), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && err[0]) st = fail(MGV_ETIMEDOUT, "a gather wait ran out");
    }
    if (e != cudaSuccess) st = cuda_fail(e, "mgv_diag_gather");
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (table) cudaFreeAsync(table, s);
    if (sink) cudaFreeAsync(sink, s);
    cudaStreamSynchronize(s);
    return st;
}
