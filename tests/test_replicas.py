"""Multi-GPU bookkeeping of the bench, run as world-size-2 gloo process groups on
the CPU (the render path shards into independent replicas; ranks meet only to
time the job).

* the whole-job rate is every rank's samples over the slowest rank's time;
* max / sum reductions and the barrier agree on both ranks, rank 0 is the one
  that reports;
* a single process needs no process group;
* a rank that never joins makes the other one fail within the group timeout
  instead of waiting for good (failure made on the host, no GPU involved).
"""
import os
import socket
import time

import pytest
import torch.multiprocessing as mp

from lsystemeditor_b200.replicas import Replicas


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))


def _worker(rank, world, port, out):
    _env(rank, world, port)
    reps = Replicas(backend="gloo", device="cpu", timeout_s=30.0)
    try:
        reps.barrier()
        samples = 1000.0 * (rank + 1)       # rank 0: 1000, rank 1: 2000
        ms = 40.0 + 10.0 * rank             # the slowest rank takes 50 ms
        out[rank] = (reps.max(ms), reps.sum(samples), reps.job_rate(samples, ms, scale=1.0), reps.is_root)
        reps.barrier()
    finally:
        reps.close()


def test_two_ranks_time_the_job_together():
    world, port = 2, _port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        mx, total, rate, root = res[rank]
        assert mx == 50.0 and total == 3000.0
        assert rate == pytest.approx(3000.0 / 0.050)
        assert root == (rank == 0)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    reps = Replicas(backend="gloo", device="cpu")
    reps.barrier()
    assert reps.world == 1 and reps.is_root
    assert reps.max(7.0) == 7.0 and reps.sum(7.0) == 7.0
    assert reps.job_rate(100.0, 50.0, scale=1.0) == pytest.approx(2000.0)
    reps.close()


def _lonely(rank, world, port, out):
    _env(rank, world, port)
    if rank == 1:
        return  # this rank never joins the group
    t0 = time.monotonic()
    try:
        Replicas(backend="gloo", device="cpu", timeout_s=3.0).barrier()
        out[rank] = ("joined", time.monotonic() - t0)
    except Exception as e:  # the rendezvous or the barrier times out
        out[rank] = (type(e).__name__, time.monotonic() - t0)


def test_missing_rank_fails_within_the_timeout():
    world, port = 2, _port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_lonely, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    kind, elapsed = res[0]
    assert kind != "joined"
    assert elapsed < 60.0
