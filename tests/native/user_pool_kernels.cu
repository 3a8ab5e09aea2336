// user_pool_kernels.cu -- a "user" library for the device-side pool tests:
// kernels written only against the public headers (include/mgv.h and
// include/mgv_device.cuh) that acquire, fill and release pool buffers
// themselves, as a caller's own kernels would.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mgv_device.cuh"

// Thread t (< n) acquires a buffer, fills `rows` rows of column 0 with
// tag * 2^20 + row, and records the id and the status; it does not release.
__global__ void k_user_fill(mgv_pool_device p, uint32_t n, uint32_t rows, int32_t tag,
                            unsigned long long timeout_ns, uint32_t* ids, uint32_t* status) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    uint32_t id = MGV_DEV_NIL;
    const mgv_status s = mgv_dev_buffer_acquire(&p, timeout_ns, &id);
    status[t] = (uint32_t)s;
    ids[t] = s == MGV_OK ? id : MGV_DEV_NIL;
    if (s != MGV_OK) return;
    int32_t* c0 = mgv_dev_buffer_col(&p, id, 0);
    for (uint32_t r = 0; r < rows && r < p.capacity; ++r) c0[r] = (tag + (int32_t)t) * (1 << 20) + (int32_t)r;
}

__global__ void k_user_release(mgv_pool_device p, const uint32_t* ids, uint32_t n, uint32_t* status) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    status[t] = (uint32_t)mgv_dev_buffer_release(&p, ids[t]);
}

// Every thread acquires and releases `iters` times; owner[id] records the
// holder (CAS from NIL), so two holders of one buffer are counted in
// counters[1]; counters[0] counts successful acquisitions, counters[2]
// failed ones (timed out or drained), counters[3] failed releases.
__global__ void k_user_churn(mgv_pool_device p, uint32_t iters, unsigned long long timeout_ns, uint32_t* owner,
                             unsigned long long* counters) {
    const uint32_t me = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t i = 0; i < iters; ++i) {
        uint32_t id;
        if (mgv_dev_buffer_acquire(&p, timeout_ns, &id) != MGV_OK) {
            atomicAdd(&counters[2], 1ull);
            continue;
        }
        if (atomicCAS(&owner[id], MGV_DEV_NIL, me) != MGV_DEV_NIL) atomicAdd(&counters[1], 1ull);
        int32_t* c0 = mgv_dev_buffer_col(&p, id, 0);
        c0[me % p.capacity] = (int32_t)me;
        atomicExch(&owner[id], MGV_DEV_NIL);
        __threadfence();
        if (mgv_dev_buffer_release(&p, id) != MGV_OK) atomicAdd(&counters[3], 1ull);
        atomicAdd(&counters[0], 1ull);
    }
}

extern "C" int user_fill(const mgv_pool_device* p, uint32_t n, uint32_t rows, int32_t tag,
                         unsigned long long timeout_ns, uint32_t* d_ids, uint32_t* d_status) {
    k_user_fill<<<(n + 127) / 128, 128>>>(*p, n, rows, tag, timeout_ns, d_ids, d_status);
    return (int)cudaDeviceSynchronize();
}

extern "C" int user_release(const mgv_pool_device* p, const uint32_t* d_ids, uint32_t n, uint32_t* d_status) {
    k_user_release<<<(n + 127) / 128, 128>>>(*p, d_ids, n, d_status);
    return (int)cudaDeviceSynchronize();
}

extern "C" int user_churn(const mgv_pool_device* p, uint32_t threads, uint32_t iters, unsigned long long timeout_ns,
                          uint32_t* d_owner, unsigned long long* d_counters) {
    k_user_churn<<<(threads + 127) / 128, 128>>>(*p, iters, timeout_ns, d_owner, d_counters);
    return (int)cudaDeviceSynchronize();
}

extern "C" int user_read(void* host_dst, const void* dev_src, size_t bytes) {
    return (int)cudaMemcpy(host_dst, dev_src, bytes, cudaMemcpyDeviceToHost);
}
