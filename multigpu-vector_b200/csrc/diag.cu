// diag.cu -- roofline diagnostic: the rate at which the GPU serves random
// 32-byte bucket reads, the operation every hash probe is built on.
//
// Each thread hashes R streamed keys, issues R independent 32-byte loads at
// the hashed bucket of a table of `table_bytes`, and folds the words it
// read.  The result is the random-sector ceiling that bounds any hash
// probe, whatever its bookkeeping; the probe kernel is measured against it.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "mgv_internal.h"

namespace mgv {
namespace {

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
