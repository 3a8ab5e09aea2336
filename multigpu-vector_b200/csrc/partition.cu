// partition.cu -- the exchange reduced to an in-GPU radix partitioner.
//
// The reference's split (src/operators/split.cu:49-118) routes each row to
// one of its parents by hash3(x) = x & 1, ballot-compacting per destination
// into 160-row staging areas in global memory.  Here a [select] -> partition
// consume makes two passes over its input:
//   1. k_part_hist: per-CTA shared histograms of (key >> shift) & mask,
//      merged with one global atomic per partition and CTA;
//   2. k_part_cursors (one CTA): the partitions' ranges in the store,
//      fill + exclusive prefix sum of the histogram, and the running totals
//      (rows stored, rows per partition), all on the device;
//   3. k_part_scatter: tiles of 4096 rows get a local rank per row from a
//      shared-memory histogram, reserve one contiguous range per partition
//      from the global cursors,
//      and are counting-sorted by partition in shared memory, column by
//      column; consecutive threads then store consecutive rows of a
//      partition's range, so a warp's store touches a few lines instead of
//      one line per row (random 4-byte stores are bound by the memory
//      pipeline's request rate, not by bytes).
// No step waits for the host.  The result is partition-major storage that
// close() replays into the parent chain, so a radix-laid-out hash table is
// built one region at a time.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "mgv_internal.h"

namespace mgv {
namespace {

constexpr int kPartBlock = 256;
constexpr int kPartRows = 16;  // rows per thread per tile: one reservation per partition per 4096 rows
constexpr int kHistRows = 8;   // histogram: key loads per thread in flight

template <bool SEL>
__global__ void __launch_bounds__(kPartBlock)
    k_part_hist(const int32_t* __restrict__ keys, const int32_t* __restrict__ filt, int32_t bound, uint64_t n,
                uint32_t shift, uint32_t mask, unsigned long long* hist) {
    extern __shared__ uint32_t sh[];
    for (uint32_t p = threadIdx.x; p <= mask; p += kPartBlock) sh[p] = 0;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * kPartBlock;
    for (uint64_t i0 = (uint64_t)blockIdx.x * kPartBlock + threadIdx.x; i0 < n; i0 += stride * kHistRows) {
        int32_t k[kHistRows];
        bool in[kHistRows];
#pragma unroll
        for (int u = 0; u < kHistRows; ++u) {
            const uint64_t i = i0 + u * stride;
            in[u] = i < n;
            k[u] = in[u] ? __ldg(keys + i) : 0;
            if (SEL && in[u]) in[u] = __ldg(filt + i) <= bound;
        }
#pragma unroll
        for (int u = 0; u < kHistRows; ++u)
            if (in[u]) atomicAdd(&sh[((uint32_t)k[u] >> shift) & mask], 1u);
    }
    __syncthreads();
    for (uint32_t p = threadIdx.x; p <= mask; p += kPartBlock)
        if (sh[p]) atomicAdd(hist + p, (unsigned long long)sh[p]);
}

struct ScatterCols {
    const int32_t* cols[MGV_MAX_COLS];
};

constexpr int kCursorBlock = 1024;

// acc[0] = rows stored so far, acc[1 + p] = rows of partition p so far.  The
// consume's histogram in hc[] becomes its cursors: acc[0] + the exclusive
// prefix sum.  Rows past max_rows are an error; the scatter drops them.
__global__ void __launch_bounds__(kCursorBlock) k_part_cursors(unsigned long long* hc, uint32_t P,
                                                               unsigned long long* acc, uint64_t max_rows,
                                                               uint32_t* err) {
    for (uint32_t p = threadIdx.x; p < P; p += kCursorBlock) acc[1 + p] += hc[p];
    const unsigned long long fill = acc[0];
    const unsigned long long total = block_exclusive_scan<kCursorBlock, unsigned long long>(hc, P);
    for (uint32_t p = threadIdx.x; p < P; p += kCursorBlock) hc[p] += fill;
    if (threadIdx.x == 0) {
        acc[0] = fill + total;
        if (fill + total > max_rows) set_error(err, kDevOverflow, 60);
    }
}

constexpr uint32_t kPartTile = (uint32_t)kPartBlock * kPartRows;

// Shared memory of k_part_scatter for 2^bits partitions.
__host__ __device__ constexpr size_t part_scatter_smem(uint32_t P) {
    return 8ull * P + 4ull * P + 2ull * kPartTile + 4ull * kPartTile;
}

template <bool SEL>
__global__ void __launch_bounds__(kPartBlock, 2)
    k_part_scatter(ScatterCols in, uint32_t ncols, uint32_t key_col, const int32_t* __restrict__ filt, int32_t bound,
                   uint64_t n, uint32_t shift, uint32_t mask, unsigned long long* cursors, int32_t* out,
                   uint64_t out_stride) {
    // [P] u64: global row of local position 0 of each partition (base - local offset, mod 2^64),
    // [P] u32: counts, then local offsets, [T] u16: partition of each sorted position, [T] i32: one column
    extern __shared__ unsigned long long shb[];
    const uint32_t P = mask + 1;
    uint32_t* cnt = reinterpret_cast<uint32_t*>(shb + P);
    uint16_t* spart = reinterpret_cast<uint16_t*>(cnt + P);
    int32_t* sval = reinterpret_cast<int32_t*>(spart + kPartTile);
    const uint64_t ntiles = (n + kPartTile - 1) / kPartTile;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        for (uint32_t p = threadIdx.x; p < P; p += kPartBlock) cnt[p] = 0;
        __syncthreads();
        int32_t key[kPartRows];
        uint32_t part[kPartRows], pos[kPartRows];
        bool keep[kPartRows];
        // every load of the tile first, then the ranks
#pragma unroll
        for (int r = 0; r < kPartRows; ++r) {
            const uint64_t i = tile * kPartTile + (uint64_t)r * kPartBlock + threadIdx.x;
            keep[r] = i < n;
            key[r] = keep[r] ? __ldg(in.cols[key_col] + i) : 0;
            if (SEL && keep[r]) keep[r] = __ldg(filt + i) <= bound;
        }
#pragma unroll
        for (int r = 0; r < kPartRows; ++r) {
            part[r] = ((uint32_t)key[r] >> shift) & mask;
            pos[r] = keep[r] ? atomicAdd(&cnt[part[r]], 1u) : 0u;
        }
        __syncthreads();
        for (uint32_t p = threadIdx.x; p < P; p += kPartBlock)
            shb[p] = cnt[p] ? atomicAdd(cursors + p, (unsigned long long)cnt[p]) : 0ull;
        const uint32_t total = block_exclusive_scan<kPartBlock>(cnt, P);  // cnt[p] = the partition's first sorted position
        for (uint32_t p = threadIdx.x; p < P; p += kPartBlock) shb[p] -= cnt[p];
#pragma unroll
        for (int r = 0; r < kPartRows; ++r)
            if (keep[r]) {
                pos[r] += cnt[part[r]];
                spart[pos[r]] = (uint16_t)part[r];
            }
        // column by column: the tile's loads, its sorted copy in shared memory, then runs of stores
        for (uint32_t c = 0; c < ncols; ++c) {
            int32_t v[kPartRows];
#pragma unroll
            for (int r = 0; r < kPartRows; ++r) {
                const uint64_t i = tile * kPartTile + (uint64_t)r * kPartBlock + threadIdx.x;
                v[r] = c == key_col ? key[r] : (keep[r] ? __ldg(in.cols[c] + i) : 0);
            }
#pragma unroll
            for (int r = 0; r < kPartRows; ++r)
                if (keep[r]) sval[pos[r]] = v[r];
            __syncthreads();  // also publishes spart and shb for the first column
            int32_t* dst = out + (uint64_t)c * out_stride;
            for (uint32_t j = threadIdx.x; j < total; j += kPartBlock) {
                const uint64_t row = shb[spart[j]] + j;
                if (row < out_stride) dst[row] = sval[j];  // past max_rows: dropped, the error is set
            }
            __syncthreads();  // sval is free for the next column
        }
    }
}

}  // namespace

cudaError_t launch_partition_hist(const int32_t* const* cols, uint64_t n, bool has_sel, uint32_t sel_col,
                                  int32_t sel_bound, uint32_t key_col, uint32_t shift, uint32_t bits,
                                  unsigned long long* hist, cudaStream_t s, Context* ctx) {
    if (n == 0) return cudaSuccess;
    const uint32_t mask = (1u << bits) - 1u;
    const size_t smem = sizeof(uint32_t) * (mask + 1);
    const void* k = has_sel ? (const void*)k_part_hist<true> : (const void*)k_part_hist<false>;
    int grid = occupancy_grid(k, kPartBlock, smem, ctx);
    const uint64_t need = (n + kPartBlock - 1) / kPartBlock;
    if ((uint64_t)grid > need) grid = (int)need;
    if (has_sel)
        k_part_hist<true><<<grid, kPartBlock, smem, s>>>(cols[key_col], cols[sel_col], sel_bound, n, shift, mask, hist);
    else
        k_part_hist<false><<<grid, kPartBlock, smem, s>>>(cols[key_col], nullptr, 0, n, shift, mask, hist);
    ctx->launches++;
    return cudaGetLastError();
}

cudaError_t launch_partition_cursors(unsigned long long* hc, uint32_t bits, unsigned long long* acc, uint64_t max_rows,
                                    cudaStream_t s, Context* ctx) {
    k_part_cursors<<<1, kCursorBlock, 0, s>>>(hc, 1u << bits, acc, max_rows, ctx->d_err);
    ctx->launches++;
    return cudaGetLastError();
}

cudaError_t launch_partition_scatter(const int32_t* const* cols, uint32_t ncols, uint64_t n, bool has_sel,
                                     uint32_t sel_col, int32_t sel_bound, uint32_t key_col, uint32_t shift,
                                     uint32_t bits, unsigned long long* cursors, int32_t* out, uint64_t out_stride,
                                     cudaStream_t s, Context* ctx) {
    if (n == 0) return cudaSuccess;
    const uint32_t mask = (1u << bits) - 1u;
    ScatterCols in{};
    for (uint32_t c = 0; c < ncols; ++c) in.cols[c] = cols[c];
    const size_t smem = part_scatter_smem(mask + 1);
    const void* k = has_sel ? (const void*)k_part_scatter<true> : (const void*)k_part_scatter<false>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int grid = occupancy_grid(k, kPartBlock, smem, ctx);
    const uint64_t need = (n + kPartTile - 1) / kPartTile;
    if ((uint64_t)grid > need) grid = (int)need;
    const int32_t* filt = has_sel ? cols[sel_col] : nullptr;
    if (has_sel)
        k_part_scatter<true><<<grid, kPartBlock, smem, s>>>(in, ncols, key_col, filt, sel_bound, n, shift, mask,
                                                            cursors, out, out_stride);
    else
        k_part_scatter<false><<<grid, kPartBlock, smem, s>>>(in, ncols, key_col, filt, sel_bound, n, shift, mask,
                                                             cursors, out, out_stride);
    ctx->launches++;
    return cudaGetLastError();
}

// ---- int32 fill (group table keys) ------------------------------------------

__global__ void k_fill_i32(int32_t* p, uint64_t n, int32_t v) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

cudaError_t launch_fill_i32(int32_t* p, uint64_t n, int32_t v, cudaStream_t s, Context* ctx) {
    if (n == 0) return cudaSuccess;
    const uint64_t want = (n + 255) / 256;
    const uint64_t cap = (uint64_t)ctx->prop.multiProcessorCount * 8;
    k_fill_i32<<<(int)(want < cap ? want : cap), 256, 0, s>>>(p, n, v);
    ctx->launches++;
    return cudaGetLastError();
}

}  // namespace mgv
