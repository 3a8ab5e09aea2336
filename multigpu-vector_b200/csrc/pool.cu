// pool.cu -- device buffer pool: one slab of fixed-size multi-column
// buffers and a tagged lock-free stack of free buffer ids in device memory.
//
// Mirrors buffer_pool / buffer_manager (src/buffer_pool.cuh:35-170,
// src/buffer_manager.cuh:40-181, src/buffer_manager.cu:38-134): the device
// stack is the one authority on free buffers; the host takes and returns
// buffers in batches through single-thread kernels on the pool's own stream
// (get_buffer_host / release_buffer_host, src/buffer_manager.cu:16-26) and
// keeps a small host cache.  Every device-side wait is bounded: a stack
// operation gives up after a fixed number of CAS attempts and a blocked
// acquire gives up at a deadline on %globaltimer, returning a status
// instead of spinning forever (the reference's stacks spin without limit,
// src/lockfree_stack.cuh:122, src/threadsafe_device_stack.cuh:48).
#include <cuda_runtime.h>

#include "../../include/mgv_device.cuh"
#include "device_common.cuh"
#include "mgv_internal.h"

namespace mgv {

// The device view of a pool, the form the public device header's stack
// operations take (one implementation for the library and for user kernels).
__device__ __forceinline__ mgv_pool_device pool_view(PoolDev* p) {
    mgv_pool_device v;
    v.head = &p->head;
    v.available = &p->available;
    v.producers = &p->producers;
    v.next = p->next;
    v.slab = nullptr;
    v.nbuffers = p->nbuffers;
    v.capacity = 0;
    v.ncols = 0;
    v.reserved = 0;
    return v;
}

__global__ void k_pool_init(PoolDev* p, uint32_t n) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    p->nbuffers = n;
    p->producers = 0;
    p->available = n;
    // ids pushed so that id 0 is on top
    for (uint32_t i = 0; i < n; ++i) p->next[i] = (i + 1 < n) ? i + 1 : kNil;
    p->head = n ? 0ull : (unsigned long long)kNil;
}

// Pops up to `want` ids.  status: 0 ok (got == want), 1 timed out,
// 2 drained (empty and no producer).  acquire_buffer_blocked_unsafe,
// src/buffer_pool.cuh:83-96.
__global__ void k_pool_pop_batch(PoolDev* p, uint32_t want, uint64_t timeout_ns, uint32_t* out,
                                 uint32_t* got_status) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint32_t got = 0, status = 0;
    const mgv_pool_device v = pool_view(p);
    const unsigned long long t0 = mgv_dev_now_ns();
    while (got < want) {
        uint32_t id;
        if (mgv_dev_stack_pop(&v, &id)) {
            out[got++] = id;
            continue;
        }
        if (got > 0) break;  // partial batch is fine
        if (*((volatile uint32_t*)&p->producers) == 0 && *((volatile uint32_t*)&p->available) == 0) {
            status = 2;
            break;
        }
        if (mgv_dev_now_ns() - t0 >= timeout_ns) {
            status = 1;
            break;
        }
        __nanosleep(1000);
    }
    got_status[0] = got;
    got_status[1] = status;
}

__global__ void k_pool_push_batch(PoolDev* p, const uint32_t* ids, uint32_t n, uint32_t* err) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const mgv_pool_device v = pool_view(p);
    for (uint32_t i = 0; i < n; ++i)
        if (!mgv_dev_stack_push(&v, ids[i])) set_error(err, kDevTimeout, 7);
}

__global__ void k_pool_producers(PoolDev* p, int delta) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    if (delta > 0) atomicAdd(&p->producers, (uint32_t)delta);
    else if (p->producers >= (uint32_t)(-delta)) atomicSub(&p->producers, (uint32_t)(-delta));
}

cudaError_t pool_init_device(Pool* p) {
    k_pool_init<<<1, 1, 0, p->stream>>>(p->dev, p->nbuffers);
    p->ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(p->stream);
}

cudaError_t pool_pop_batch(Pool* p, uint32_t want, uint32_t timeout_us, uint32_t* got,
                           mgv_status* status) {
    // d_ids layout: [0 .. nbuffers) ids, then 2 words got/status
    uint32_t* d_gs = p->d_ids + p->nbuffers;
    k_pool_pop_batch<<<1, 1, 0, p->stream>>>(p->dev, want, (uint64_t)timeout_us * 1000ull, p->d_ids,
                                             d_gs);
    p->ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(p->h_ids, p->d_ids, sizeof(uint32_t) * (p->nbuffers + 2),
                        cudaMemcpyDeviceToHost, p->stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) return e;
    *got = p->h_ids[p->nbuffers];
    const uint32_t st = p->h_ids[p->nbuffers + 1];
    *status = st == 0 ? MGV_OK : st == 1 ? MGV_ETIMEDOUT : MGV_EDRAINED;
    return cudaSuccess;
}

cudaError_t pool_push_batch(Pool* p, const uint32_t* ids, uint32_t n) {
    if (n == 0) return cudaSuccess;
    for (uint32_t i = 0; i < n; ++i) p->h_ids[i] = ids[i];
    cudaError_t e = cudaMemcpyAsync(p->d_ids, p->h_ids, sizeof(uint32_t) * n,
                                    cudaMemcpyHostToDevice, p->stream);
    if (e != cudaSuccess) return e;
    k_pool_push_batch<<<1, 1, 0, p->stream>>>(p->dev, p->d_ids, n, p->ctx->d_err);
    p->ctx->launches++;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(p->stream);
}

cudaError_t pool_read_counters(Pool* p, uint32_t* available, uint32_t* producers) {
    PoolDev h{};
    cudaError_t e = cudaMemcpyAsync(&h, p->dev, offsetof(PoolDev, next), cudaMemcpyDeviceToHost,
                                    p->stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) return e;
    *available = h.available;
    *producers = h.producers;
    return cudaSuccess;
}

cudaError_t pool_add_producers(Pool* p, int delta) {
    k_pool_producers<<<1, 1, 0, p->stream>>>(p->dev, delta);
    p->ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(p->stream);
}

}  // namespace mgv
