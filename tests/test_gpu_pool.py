"""Device buffer pool: acquire / release, producers and bounded waits.

Mirrors buffer_pool::acquire_buffer_blocked_unsafe (src/buffer_pool.cuh:83-96):
an empty pool with no producer answers "drained" at once; with a producer
registered the acquire waits, bounded, and then reports a timeout.  The wait
runs out on the device (%globaltimer) and returns a status; nothing faults.
"""
import time

import numpy as np
import pytest

import mgv

pytestmark = pytest.mark.gpu


def test_acquire_release_roundtrip(ctx, torch_cuda):
    pool = mgv.Pool(ctx, 20, 1024, 2)
    st = pool.stats()
    assert (st.nbuffers, st.available, st.capacity, st.ncols) == (20, 20, 1024, 2)
    bufs = [pool.acquire() for _ in range(20)]
    assert len({b.contents.id for b in bufs}) == 20
    a = np.arange(1000, dtype=np.int32)
    mgv.buffer_write(bufs[3], 1, a.ctypes.data, 1000)
    back = np.zeros(1000, np.int32)
    mgv.buffer_read(bufs[3], 1, back.ctypes.data, 1000)
    assert np.array_equal(a, back) and bufs[3].contents.rows == 1000
    code, b = pool.try_acquire(0)
    assert code == mgv.EDRAINED and b is None
    for b in bufs:
        pool.release(b)
    st = pool.stats()
    assert st.available + st.host_cached == 20
    with pytest.raises(mgv.MgvError) as e:
        pool.release(bufs[0])
    assert e.value.status == mgv.ESTATE
    pool.destroy()


def test_bounded_wait_times_out_with_producer(ctx):
    pool = mgv.Pool(ctx, 2, 128, 1)
    held = [pool.acquire(), pool.acquire()]
    pool.register_producer()
    t0 = time.time()
    code, _ = pool.try_acquire(timeout_us=200000)
    dt = time.time() - t0
    assert code == mgv.ETIMEDOUT
    assert 0.15 < dt < 10.0
    pool.unregister_producer()
    code, _ = pool.try_acquire(timeout_us=200000)
    assert code == mgv.EDRAINED
    for b in held:
        pool.release(b)
    assert pool.acquire() is not None
    ctx.sync()
    pool.destroy()
