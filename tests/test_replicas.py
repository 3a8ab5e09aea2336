"""The N > 1 replica path of bench.py on CPU: two gloo processes.

Timing takes the slowest replica, the job rate counts every replica's
units, and a disagreeing replica is detected.  No GPU is involved."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "multigpu-vector_b200"))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "multigpu-vector_b200"))
    import replicas

    dist, w, r, local = replicas.init("gloo", timeout_s=60)
    slowest = replicas.max_over_ranks(dist, 1.0 + 0.5 * r)         # rank 1 is slower
    rate = replicas.job_rate(w, 1000, slowest)
    agree = replicas.same_on_all_ranks(dist, (12345, 678))
    differ = replicas.same_on_all_ranks(dist, (12345, 678 + r))     # rank 1 disagrees
    replicas.finish(dist)
    q.put((r, w, local, slowest, rate, agree, differ))


def test_two_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_replica, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, (rank, w, local, slowest, rate, agree, differ) in enumerate(out):
        assert (rank, w, local) == (r, 2, r)
        assert slowest == 1.5 and rate == pytest.approx(2 * 1000 / 1.5)
        assert agree is True and differ is False


def test_single_process_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    import replicas

    dist, w, r, local = replicas.init("gloo")
    assert dist is None and (w, r, local) == (1, 0, 0)
    assert replicas.max_over_ranks(dist, 2.5) == 2.5
    assert replicas.job_rate(1, 100, 2.0) == 50.0 and replicas.same_on_all_ranks(dist, 1)
    replicas.finish(dist)
