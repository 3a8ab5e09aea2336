// noalloc.cu -- a hash join that allocates nothing.
//
// Some callers cannot allocate device memory: code that runs inside another
// framework's memory budget or allocator (which owns every byte and forbids
// cudaMalloc), plugins and embedded hosts that are only handed
// pre-allocated buffers, and processes whose device memory is already spoken
// for.  They cannot create a context or a hash_build operator, because both
// allocate.  mgv_hash_join_noalloc gives them the join of
// create_count_join_1G_pipeline -- build, then probe, then COUNT(matches) and
// SUM(build payload + probe payload) -- with its hash table in a file-scope
// device array instead of allocated memory.
//
// The array is fixed at MGV_NOALLOC_MAX_BUILD_ROWS build rows (a 16 MiB
// table at load factor 0.5 plus a 4 MiB side list for INT32_MIN keys).  With
// lazy module loading (the CUDA default) a device commits it when the first
// call on that device looks up its address, or when the module loads under
// CUDA_MODULE_LOADING=EAGER; it is then held until the process exits.  Host
// code cannot use the array's name as a device address, so each device's
// address is looked up once with cudaGetSymbolAddress (with that device
// current) by the first call on that device.  All calls share the array and
// each call clears it, so calls that overlap on the GPU (other threads,
// other streams) race and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "device_common.cuh"
#include "mgv_internal.h"

namespace mgv {
namespace {

constexpr uint64_t kMaxBuildRows = MGV_NOALLOC_MAX_BUILD_ROWS;
constexpr uint32_t kBuckets = (uint32_t)((kMaxBuildRows + 1) / 2);  // rows / (4 slots * 0.5)
constexpr size_t kTableBytes = (size_t)kBuckets * 32;
constexpr size_t kSideBytes = kMaxBuildRows * sizeof(int32_t);
constexpr size_t kMetaBytes = 4 * sizeof(unsigned long long);
constexpr size_t kErrBytes = 64;  // error word, padded
constexpr size_t kScratchBytes = kTableBytes + kSideBytes + kMetaBytes + kErrBytes;

// The scratch memory of the join: [table | side list | meta | error word].
static __device__ __align__(256) unsigned char g_join_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;

struct DeviceSlot {
    bool ready = false;
    unsigned char* scratch = nullptr;  // device address of g_join_scratch
    Context ctx;                       // host-side launch state; its d_err points into scratch
};

std::mutex g_mu;
DeviceSlot g_slots[kMaxDevices];

// Per-device set-up, with `device` current: the array's device address and
// the launch parameters.  Allocates nothing.
mgv_status setup(int device, DeviceSlot*& out) {
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceSlot& s = g_slots[device];
    if (!s.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_join_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_join_scratch)");
        e = cudaGetDeviceProperties(&s.ctx.prop, device);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
        s.scratch = static_cast<unsigned char*>(p);
        s.ctx.device = device;
        s.ctx.d_err = reinterpret_cast<uint32_t*>(s.scratch + kTableBytes + kSideBytes + kMetaBytes);
        s.ready = true;
    }
    out = &s;
    return MGV_OK;
}

mgv_status join_on_device(int device, const int32_t* build_keys, const int32_t* build_payloads, uint64_t build_rows,
                          const int32_t* probe_keys, const int32_t* probe_payloads, uint64_t probe_rows,
                          int64_t* d_result, void* stream);

}  // namespace
}  // namespace mgv

using namespace mgv;

extern "C" mgv_status mgv_hash_join_noalloc(int device, const int32_t* build_keys, const int32_t* build_payloads,
                                            uint64_t build_rows, const int32_t* probe_keys,
                                            const int32_t* probe_payloads, uint64_t probe_rows, int64_t* d_result,
                                            void* stream) {
    if (!d_result) return fail(MGV_EINVAL, "d_result is NULL");
    if (build_rows && !build_keys) return fail(MGV_EINVAL, "build_keys is NULL");
    if (probe_rows && !probe_keys) return fail(MGV_EINVAL, "probe_keys is NULL");
    if (build_rows > kMaxBuildRows)
        return fail(MGV_EINVAL, "build_rows exceeds MGV_NOALLOC_MAX_BUILD_ROWS (" +
                                    std::to_string(kMaxBuildRows) + "); use the hash_build operator");
    int ndev = 0;
    MGV_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev || device >= kMaxDevices) return fail(MGV_EINVAL, "no such device");
    // The join runs with `device` current; the caller's current device is
    // restored on every return path.
    int caller_device = 0;
    MGV_CUDA_TRY(cudaGetDevice(&caller_device));
    if (caller_device == device) return join_on_device(device, build_keys, build_payloads, build_rows, probe_keys,
                                                       probe_payloads, probe_rows, d_result, stream);
    MGV_CUDA_TRY(cudaSetDevice(device));
    const mgv_status st = join_on_device(device, build_keys, build_payloads, build_rows, probe_keys, probe_payloads,
                                         probe_rows, d_result, stream);
    const cudaError_t back = cudaSetDevice(caller_device);
    if (st == MGV_OK && back != cudaSuccess) return cuda_fail(back, "cudaSetDevice(caller's device)");
    return st;
}

namespace mgv {
namespace {

// The join itself, with `device` current.
mgv_status join_on_device(int device, const int32_t* build_keys, const int32_t* build_payloads, uint64_t build_rows,
                          const int32_t* probe_keys, const int32_t* probe_payloads, uint64_t probe_rows,
                          int64_t* d_result, void* stream) {
    DeviceSlot* slot = nullptr;
    mgv_status st = setup(device, slot);
    if (st != MGV_OK) return st;
    Context* ctx = &slot->ctx;
    cudaStream_t s = (cudaStream_t)stream;

    TableView t{};
    t.slots = reinterpret_cast<unsigned long long*>(slot->scratch);
    t.nbuckets = kBuckets;
    t.bpp = kBuckets;
    t.radix_mask = 0;
    t.radix_shift = 0;
    t.side_pay = reinterpret_cast<int32_t*>(slot->scratch + kTableBytes);
    t.side_cap = kMaxBuildRows;
    t.meta = reinterpret_cast<unsigned long long*>(slot->scratch + kTableBytes + kSideBytes);

    // Clear what must start at zero: the table (empty slots), the metadata,
    // the error word and the caller's result.
    MGV_CUDA_TRY(launch_fill_u64(t.slots, 4ull * kBuckets, kEmptySlot, s, ctx));
    MGV_CUDA_TRY(cudaMemsetAsync(t.meta, 0, kMetaBytes, s));
    MGV_CUDA_TRY(cudaMemsetAsync(ctx->d_err, 0, 2 * sizeof(uint32_t), s));
    MGV_CUDA_TRY(cudaMemsetAsync(d_result, 0, 2 * sizeof(int64_t), s));
    MGV_CUDA_TRY(launch_build(build_keys, build_payloads, nullptr, 0, false, build_rows, t, s, ctx));

    // The probe kernel is chosen by whether the build side had duplicate keys.
    unsigned long long meta[4];
    MGV_CUDA_TRY(cudaMemcpyAsync(meta, t.meta, sizeof(meta), cudaMemcpyDeviceToHost, s));
    MGV_CUDA_TRY(cudaStreamSynchronize(s));
    const bool unique = meta[3] == 0;
    const uint32_t mode = 1u | (probe_payloads ? 2u : 0u);
    MGV_CUDA_TRY(launch_probe_agg(probe_keys, probe_payloads, probe_rows, t, unique, mode,
                                  reinterpret_cast<unsigned long long*>(d_result), s, ctx));

    uint32_t err[2] = {0, 0};
    MGV_CUDA_TRY(cudaMemcpyAsync(err, ctx->d_err, sizeof(err), cudaMemcpyDeviceToHost, s));
    MGV_CUDA_TRY(cudaStreamSynchronize(s));
    if (err[0] != 0) {
        if (err[0] == MGV_ENOMEM) return fail(MGV_ENOMEM, "join scratch table full");
        if (err[0] == MGV_ETIMEDOUT) return fail(MGV_ETIMEDOUT, "a bounded wait ran out");
        return fail(MGV_EDEVICE, "device error word " + std::to_string(err[0]));
    }
    return MGV_OK;
}

}  // namespace
}  // namespace mgv
