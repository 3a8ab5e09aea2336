// gen.cu -- seeded synthetic columns generated directly in device memory.
//
// The same counter-based streams as mgv_gen.h on the host, so a column made
// here equals the one the CPU oracle makes row for row.  (The reference
// fills host arrays with unseeded rand()/mt19937, src/main8.cu:169,
// src/main9.cu:556-566, and copies them to the device buffer by buffer.)
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "mgv_gen.h"
#include "mgv_internal.h"

namespace mgv {

enum GenKind : int { kUniform = 0, kPerm = 1, kProbe = 2, kZipf = 3 };

struct GenArgs {
    int kind;
    uint32_t stream;
    uint64_t seed, build_seed, nbuild, range, miss_range, n;
    int64_t lo, miss_lo;
    uint32_t hit_num, groups;
    const uint64_t* cdf;
    unsigned long long* hits;
};

__global__ void k_gen(int32_t* __restrict__ dst, GenArgs a) {
    unsigned long long hits = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        int32_t v;
        switch (a.kind) {
            case kUniform: v = mgv_gen_uniform(a.seed, a.stream, i, a.lo, a.range); break;
            case kPerm: v = (int32_t)mgv_gen_perm(a.seed, a.n, i); break;
            case kProbe: {
                int h = 0;
                v = mgv_gen_probe_key(a.seed, a.build_seed, a.nbuild, a.hit_num, a.miss_lo, a.miss_range, i, &h);
                hits += (unsigned long long)h;
                break;
            }
            default: v = mgv_gen_zipf(a.seed, a.stream, i, a.cdf, a.groups); break;
        }
        dst[i] = v;
    }
    if (a.hits) {
        for (int o = 16; o > 0; o >>= 1) hits += __shfl_xor_sync(0xffffffffu, hits, o);
        if ((threadIdx.x & 31) == 0 && hits) atomicAdd(a.hits, hits);
    }
}

static mgv_status run_gen(Context* ctx, int32_t* dst, GenArgs a, cudaStream_t s) {
    if (a.n == 0) return MGV_OK;
    const int block = 256;
    uint64_t want = (a.n + block - 1) / block;
    uint64_t cap = (uint64_t)ctx->prop.multiProcessorCount * 16;
    k_gen<<<(int)(want < cap ? want : cap), block, 0, s>>>(dst, a);
    ctx->launches++;
    MGV_CUDA_TRY(cudaGetLastError());
    return MGV_OK;
}

// Same table as the oracle's or_zipf_cdf: cdf[g] = floor(2^32 H(g+1)/H(G)).
void zipf_cdf(std::vector<uint64_t>& cdf, uint32_t G, double s) {
    cdf.assign(G, 0);
    double total = 0.0;
    for (uint32_t g = 1; g <= G; ++g) total += (s == 1.0) ? 1.0 / (double)g : 1.0 / std::pow((double)g, s);
    double acc = 0.0;
    for (uint32_t g = 1; g <= G; ++g) {
        acc += (s == 1.0) ? 1.0 / (double)g : 1.0 / std::pow((double)g, s);
        double v = acc / total * 4294967296.0;
        cdf[g - 1] = (v >= 4294967296.0) ? 4294967296ull : (uint64_t)v;
    }
    cdf[G - 1] = 4294967296ull;
}

}  // namespace mgv

using namespace mgv;

static cudaStream_t gen_stream(mgv_ctx* ctx, void* stream) {
    return stream ? (cudaStream_t)stream : ctx->stream;
}

extern "C" {

mgv_status mgv_gen_uniform(mgv_ctx* ctx, int32_t* dst, uint64_t n, uint64_t seed, uint32_t stream_id,
                           int64_t lo, uint64_t range, void* stream) {
    if (!ctx || (!dst && n)) return fail(MGV_EINVAL, "NULL argument");
    if (range == 0 || range > (1ull << 32)) return fail(MGV_EINVAL, "range must be in [1, 2^32]");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    GenArgs a{};
    a.kind = kUniform;
    a.seed = seed;
    a.stream = stream_id;
    a.lo = lo;
    a.range = range;
    a.n = n;
    return run_gen(ctx, dst, a, gen_stream(ctx, stream));
}

mgv_status mgv_gen_perm(mgv_ctx* ctx, int32_t* dst, uint64_t n, uint64_t seed, void* stream) {
    if (!ctx || (!dst && n)) return fail(MGV_EINVAL, "NULL argument");
    if (n > (1ull << 31)) return fail(MGV_EINVAL, "n must be <= 2^31");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    GenArgs a{};
    a.kind = kPerm;
    a.seed = seed;
    a.n = n;
    return run_gen(ctx, dst, a, gen_stream(ctx, stream));
}

mgv_status mgv_gen_probe_keys(mgv_ctx* ctx, int32_t* dst, uint64_t n, uint64_t seed, uint64_t build_seed,
                              uint64_t nbuild, uint32_t hit_num, int64_t miss_lo, uint64_t miss_range,
                              uint64_t* hits, void* stream) {
    if (!ctx || (!dst && n)) return fail(MGV_EINVAL, "NULL argument");
    if (nbuild == 0 || nbuild > (1ull << 31) || miss_range == 0 || miss_range > (1ull << 32))
        return fail(MGV_EINVAL, "nbuild or miss_range out of range");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t s = gen_stream(ctx, stream);
    unsigned long long* d_hits = nullptr;
    if (hits) {
        MGV_CUDA_TRY(cudaMallocAsync(&d_hits, sizeof(unsigned long long), s));
        MGV_CUDA_TRY(cudaMemsetAsync(d_hits, 0, sizeof(unsigned long long), s));
    }
    GenArgs a{};
    a.kind = kProbe;
    a.seed = seed;
    a.build_seed = build_seed;
    a.nbuild = nbuild;
    a.hit_num = hit_num;
    a.miss_lo = miss_lo;
    a.miss_range = miss_range;
    a.n = n;
    a.hits = d_hits;
    mgv_status st = run_gen(ctx, dst, a, s);
    if (hits) {
        unsigned long long h = 0;
        if (st == MGV_OK) {
            MGV_CUDA_TRY(cudaMemcpyAsync(&h, d_hits, sizeof(h), cudaMemcpyDeviceToHost, s));
            MGV_CUDA_TRY(cudaStreamSynchronize(s));
        }
        cudaFreeAsync(d_hits, s);
        *hits = h;
    }
    return st;
}

mgv_status mgv_gen_zipf(mgv_ctx* ctx, int32_t* dst, uint64_t n, uint64_t seed, uint32_t stream_id,
                        uint32_t groups, double s_exp, void* stream) {
    if (!ctx || (!dst && n)) return fail(MGV_EINVAL, "NULL argument");
    if (groups == 0) return fail(MGV_EINVAL, "groups must be >= 1");
    MGV_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t s = gen_stream(ctx, stream);
    std::vector<uint64_t> cdf;
    zipf_cdf(cdf, groups, s_exp);
    uint64_t* d_cdf = nullptr;
    MGV_CUDA_TRY(cudaMallocAsync(&d_cdf, sizeof(uint64_t) * groups, s));
    MGV_CUDA_TRY(cudaMemcpyAsync(d_cdf, cdf.data(), sizeof(uint64_t) * groups, cudaMemcpyHostToDevice, s));
    GenArgs a{};
    a.kind = kZipf;
    a.seed = seed;
    a.stream = stream_id;
    a.groups = groups;
    a.cdf = d_cdf;
    a.n = n;
    mgv_status st = run_gen(ctx, dst, a, s);
    MGV_CUDA_TRY(cudaStreamSynchronize(s));  // cdf is pageable host memory
    cudaFreeAsync(d_cdf, s);
    return st;
}

}  // extern "C"
