"""Device generators equal the oracle's host generators row for row."""
import numpy as np
import pytest

import pyoracle as po
from gpu_util import host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [0, 1, 1000, (1 << 20) + 3])
def test_uniform_perm_probe_zipf(ctx, torch_cuda, n):
    torch = torch_cuda
    t = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    ctx.gen_uniform(t, n, 0x5EED0001, 4, -123, 1 << 31)
    assert np.array_equal(host(t)[:n], po.gen_uniform(n, 0x5EED0001, 4, -123, 1 << 31))
    if n:
        ctx.gen_perm(t, n, 0x5EED0002)
        p = host(t)[:n]
        assert np.array_equal(p, po.gen_perm(n, 0x5EED0002))
        assert np.array_equal(np.sort(p), np.arange(n, dtype=np.int32))
    hits = ctx.gen_probe_keys(t, n, 0x5EED0003, 0x5EED0002, 1 << 22, 3865470566, 1 << 22, (1 << 31) - (1 << 22))
    ref, ref_hits = po.gen_probe_keys(n, 0x5EED0003, 0x5EED0002, 1 << 22, 3865470566, 1 << 22, (1 << 31) - (1 << 22))
    assert np.array_equal(host(t)[:n], ref) and hits == ref_hits
    ctx.gen_zipf(t, n, 0x5EED0004, 5, 4096)
    assert np.array_equal(host(t)[:n], po.gen_zipf(n, 0x5EED0004, 5, 4096))
    ctx.sync()
