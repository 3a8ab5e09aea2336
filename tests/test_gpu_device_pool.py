"""Device-side buffer acquire / release from a caller's own kernels.

The reference's kernels take buffers with buffer_manager::get_buffer() (a
device pop, src/buffer_manager.cuh:50-64) and give them back with
release_buffer() (src/buffer_manager.cuh:96-129); acquire_buffer_blocked_to
(src/buffer_manager.cuh:147-176) waits for one.  Here a test library built
only against include/mgv_device.cuh (tests/native/user_pool_kernels.cu) plays
the caller: its kernels acquire, fill and release buffers of an mgv pool,
and a blocked acquire with a producer registered runs out at its deadline
and returns MGV_ETIMEDOUT (no kernel spins without limit)."""
import ctypes
import os
import subprocess
import time

import numpy as np
import pytest

import mgv

pytestmark = pytest.mark.gpu

NATIVE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "native")
LIB = os.path.join(NATIVE, "libuserpool.so")


@pytest.fixture(scope="module")
def user():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", NATIVE], check=True)
    lib = ctypes.CDLL(LIB)
    pv = ctypes.POINTER(mgv.PoolDevice)
    u32, u64, vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p
    lib.user_fill.argtypes = [pv, u32, u32, ctypes.c_int32, u64, vp, vp]
    lib.user_release.argtypes = [pv, vp, u32, vp]
    lib.user_churn.argtypes = [pv, u32, u32, u64, vp, vp]
    lib.user_read.argtypes = [vp, vp, ctypes.c_size_t]
    for f in (lib.user_fill, lib.user_release, lib.user_churn, lib.user_read):
        f.restype = ctypes.c_int
    return lib


def test_kernel_acquires_fills_and_releases(ctx, torch_cuda, user):
    torch = torch_cuda
    nbuf, cap = 8, 1024
    pool = mgv.Pool(ctx, nbuf, cap, 2)
    v = pool.device_view()
    assert (v.nbuffers, v.capacity, v.ncols) == (nbuf, cap, 2)
    ids = torch.zeros(nbuf, dtype=torch.int32, device="cuda")
    st = torch.zeros(nbuf, dtype=torch.int32, device="cuda")
    assert user.user_fill(ctypes.byref(v), nbuf, 1000, 7, 10**8, ids.data_ptr(), st.data_ptr()) == 0
    assert (st.cpu().numpy() == mgv.OK).all()
    got = ids.cpu().numpy().astype(np.int64)
    assert sorted(got.tolist()) == list(range(nbuf))  # every buffer, once
    assert pool.stats().available == 0
    # the rows each thread wrote, read from the slab: buffer i column 0 at slab + 2*i*cap
    h = np.empty((nbuf, 2, cap), np.int32)
    assert user.user_read(h.ctypes.data, v.slab, h.nbytes) == 0
    for t, bid in enumerate(got):
        assert np.array_equal(h[bid, 0, :1000], (7 + t) * (1 << 20) + np.arange(1000))
    # a full pool with no producer: drained at once
    st2 = torch.zeros(1, dtype=torch.int32, device="cuda")
    id2 = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert user.user_fill(ctypes.byref(v), 1, 0, 0, 10**9, id2.data_ptr(), st2.data_ptr()) == 0
    assert int(st2.item()) == mgv.EDRAINED
    # release from the kernel; the host then sees every buffer free
    assert user.user_release(ctypes.byref(v), ids.data_ptr(), nbuf, st.data_ptr()) == 0
    assert (st.cpu().numpy() == mgv.OK).all()
    s = pool.stats()
    assert s.available + s.host_cached == nbuf
    b = pool.acquire()
    pool.release(b)
    pool.destroy()


def test_kernel_blocked_acquire_times_out_with_producer(ctx, torch_cuda, user):
    """A producer is registered and nothing is released: the kernel's acquire
    waits until its deadline (0.2 s) and returns MGV_ETIMEDOUT."""
    torch = torch_cuda
    pool = mgv.Pool(ctx, 2, 128, 1)
    v = pool.device_view()
    ids = torch.zeros(2, dtype=torch.int32, device="cuda")
    st = torch.zeros(2, dtype=torch.int32, device="cuda")
    assert user.user_fill(ctypes.byref(v), 2, 16, 1, 10**8, ids.data_ptr(), st.data_ptr()) == 0
    assert (st.cpu().numpy() == mgv.OK).all()
    pool.register_producer()
    st1 = torch.zeros(1, dtype=torch.int32, device="cuda")
    id1 = torch.zeros(1, dtype=torch.int32, device="cuda")
    t0 = time.time()
    assert user.user_fill(ctypes.byref(v), 1, 0, 0, 200_000_000, id1.data_ptr(), st1.data_ptr()) == 0
    dt = time.time() - t0
    assert int(st1.item()) == mgv.ETIMEDOUT
    assert 0.15 < dt < 10.0
    pool.unregister_producer()
    assert user.user_release(ctypes.byref(v), ids.data_ptr(), 2, st.data_ptr()) == 0
    assert (st.cpu().numpy() == mgv.OK).all()
    assert pool.stats().available == 2
    ctx.sync()
    pool.destroy()


def test_kernel_release_rejects_foreign_id(ctx, torch_cuda, user):
    torch = torch_cuda
    pool = mgv.Pool(ctx, 4, 128, 1)
    v = pool.device_view()
    ids = torch.tensor([4, 1 << 30], dtype=torch.int32, device="cuda")
    st = torch.zeros(2, dtype=torch.int32, device="cuda")
    assert user.user_release(ctypes.byref(v), ids.data_ptr(), 2, st.data_ptr()) == 0
    assert (st.cpu().numpy() == mgv.EINVAL).all()
    assert pool.stats().available == 4
    pool.destroy()


def test_kernel_churn_keeps_buffers_exclusive(ctx, torch_cuda, user):
    """1024 threads acquire and release 8 buffers 50 times each: every
    acquisition succeeds within its deadline, no buffer is ever held twice,
    and all buffers are free at the end."""
    torch = torch_cuda
    pool = mgv.Pool(ctx, 8, 256, 1)
    v = pool.device_view()
    pool.register_producer()  # holders give buffers back: waiting is meaningful
    owner = torch.full((8,), -1, dtype=torch.int32, device="cuda")
    counters = torch.zeros(4, dtype=torch.int64, device="cuda")
    threads, iters = 1024, 50
    assert user.user_churn(ctypes.byref(v), threads, iters, 2_000_000_000, owner.data_ptr(),
                           counters.data_ptr()) == 0
    c = counters.cpu().numpy()
    assert c[1] == 0, "a buffer was held by two threads"
    assert c[3] == 0
    assert c[0] + c[2] == threads * iters
    assert c[2] == 0, f"{c[2]} acquisitions ran out"
    pool.unregister_producer()
    assert pool.stats().available == 8
    pool.destroy()
