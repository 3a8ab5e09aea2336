/*
 * mgv_device.cuh -- device-side buffer acquire / release for kernels that
 * use an mgv pool (include/mgv.h).
 *
 * Replaces the reference's device-side buffer_manager calls:
 *   get_buffer() on the device = pool->pop()      (src/buffer_manager.cuh:50-64),
 *   release_buffer(buff) on the device = push     (src/buffer_manager.cuh:96-129),
 *   acquire_buffer_blocked_to(...)                (src/buffer_manager.cuh:147-176)
 * whose stacks spin without limit (src/lockfree_stack.cuh:122,
 * src/threadsafe_device_stack.cuh:48).  Here every wait is bounded: a stack
 * operation gives up after a fixed number of compare-and-swap attempts, and
 * a blocked acquire gives up at a %globaltimer deadline, returning a status
 * the kernel can act on instead of hanging the GPU.
 *
 * Usage: the host fills an mgv_pool_device with mgv_pool_device_get() and
 * passes it to a kernel by value; a thread of the kernel then calls
 *   mgv_status s = mgv_dev_buffer_acquire(&p, timeout_ns, &id);
 *   int32_t* col0 = mgv_dev_buffer_col(&p, id, 0);   ... fill ...
 *   mgv_dev_buffer_release(&p, id);
 * Buffers a kernel acquires come off the pool's device free stack (not the
 * host-side cache of mgv_buffer_acquire) and go back to it on release; the
 * host does not track them, so a buffer acquired on the device is released
 * on the device.  The functions are per thread (not warp-collective).
 *
 * This header is the single implementation of the stack: the library's own
 * host batch operations (mgv_buffer_acquire / mgv_buffer_release) use it too.
 */
#ifndef MGV_DEVICE_CUH_
#define MGV_DEVICE_CUH_

#include <stdint.h>

#include "mgv.h"

#define MGV_DEV_NIL 0xffffffffu
/* Compare-and-swap attempts of one stack operation before it gives up. */
#define MGV_DEV_STACK_TRIES 4096

__device__ __forceinline__ unsigned long long mgv_dev_now_ns(void) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

/* Pops one free buffer id.  The stack head packs {top id (low word), tag
 * (high word)}; the tag changes on every successful operation, so a stale
 * head cannot be swapped in (ABA).  Returns 1 with *id set, 0 if the stack
 * was empty or the attempts ran out under contention. */
__device__ __forceinline__ int mgv_dev_stack_pop(const mgv_pool_device *p, uint32_t *id) {
    for (int i = 0; i < MGV_DEV_STACK_TRIES; ++i) {
        const unsigned long long h = atomicAdd(p->head, 0ull);
        const uint32_t top = (uint32_t)h;
        if (top == MGV_DEV_NIL) return 0;
        const uint32_t nxt = *((volatile uint32_t *)&p->next[top]);
        const unsigned long long nh = (((h >> 32) + 1ull) << 32) | nxt;
        if (atomicCAS(p->head, h, nh) == h) {
            atomicSub(p->available, 1u);
            *id = top;
            return 1;
        }
    }
    return 0;
}

/* Pushes buffer `id` back.  Returns 0 if the attempts ran out. */
__device__ __forceinline__ int mgv_dev_stack_push(const mgv_pool_device *p, uint32_t id) {
    for (int i = 0; i < MGV_DEV_STACK_TRIES; ++i) {
        const unsigned long long h = atomicAdd(p->head, 0ull);
        *((volatile uint32_t *)&p->next[id]) = (uint32_t)h;
        __threadfence();
        const unsigned long long nh = (((h >> 32) + 1ull) << 32) | id;
        if (atomicCAS(p->head, h, nh) == h) {
            atomicAdd(p->available, 1u);
            return 1;
        }
    }
    return 0;
}

/* Acquires one buffer, waiting at most timeout_ns for one to come back:
 * MGV_OK with *id set; MGV_EDRAINED at once when the pool is empty and no
 * producer is registered (nothing can come back); MGV_ETIMEDOUT when a
 * producer is registered but nothing was released before the deadline. */
__device__ __forceinline__ mgv_status mgv_dev_buffer_acquire(const mgv_pool_device *p, unsigned long long timeout_ns,
                                                             uint32_t *id) {
    const unsigned long long t0 = mgv_dev_now_ns();
    for (;;) {
        if (mgv_dev_stack_pop(p, id)) return MGV_OK;
        if (*((volatile uint32_t *)p->producers) == 0 && *((volatile uint32_t *)p->available) == 0)
            return MGV_EDRAINED;
        if (mgv_dev_now_ns() - t0 >= timeout_ns) return MGV_ETIMEDOUT;
        __nanosleep(1000);
    }
}

/* Returns buffer `id` to the pool: MGV_OK, MGV_EINVAL for an id outside the
 * pool, MGV_ETIMEDOUT if the stack stayed contended past its attempts. */
__device__ __forceinline__ mgv_status mgv_dev_buffer_release(const mgv_pool_device *p, uint32_t id) {
    if (id >= p->nbuffers) return MGV_EINVAL;
    return mgv_dev_stack_push(p, id) ? MGV_OK : MGV_ETIMEDOUT;
}

/* Column `col` of buffer `id`: `capacity` int32 rows. */
__device__ __forceinline__ int32_t *mgv_dev_buffer_col(const mgv_pool_device *p, uint32_t id, uint32_t col) {
    return p->slab + ((uint64_t)id * p->ncols + col) * p->capacity;
}

#endif /* MGV_DEVICE_CUH_ */
