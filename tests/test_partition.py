"""Batch partitioning over GPUs (scene-granular, cost-balanced) and the one
image gather to rank 0, run as gloo process groups on the CPU with stand-in
images (no GPU): every scene is assigned exactly once, the load is balanced
within the greedy bound, and the gathered images equal a one-rank run bit for
bit."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from lsystemeditor_b200.partition import assign, gather_to_root, owners, scene_cost


def _sizes(n=64, seed=2):
    rng = np.random.default_rng(seed)
    tris = rng.integers(5_000, 3_000_000, n)
    res = rng.choice([256, 512, 768, 1024], n)
    return [(int(t), int(r), int(r)) for t, r in zip(tris, res)]


def _image(k, w, h):
    """Stand-in for scene k's rendered accumulation (float4 per pixel)."""
    rng = np.random.default_rng(1000 + k)
    return torch.from_numpy(rng.uniform(0, 1, (h * w, 4)).astype(np.float32))


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_assignment_covers_every_scene_once_and_balances_cost(world):
    sizes = _sizes()
    costs = [scene_cost(t, w * h, 512) for t, w, h in sizes]
    a = assign(costs, world)
    flat = sorted(k for ks in a for k in ks)
    assert flat == list(range(len(sizes)))
    assert all(ks == sorted(ks) for ks in a)
    loads = [sum(costs[k] for k in ks) for ks in a]
    lower = max(sum(costs) / world, max(costs))
    assert max(loads) <= 4.0 / 3.0 * lower + 1e-6 * lower
    assert assign(costs, world) == a  # every rank computes the same assignment


def test_cost_grows_with_pixels_samples_and_triangles():
    assert scene_cost(1000, 100, 16) < scene_cost(1000, 200, 16) < scene_cost(1000, 200, 32)
    assert scene_cost(1000, 100, 16) < scene_cost(1_000_000, 100, 16)


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from lsystemeditor_b200.replicas import Replicas
    reps = Replicas(backend="gloo", device="cpu", timeout_s=60.0)
    try:
        sizes = _sizes(24)
        costs = [scene_cost(t, w * h, 64) for t, w, h in sizes]
        a = assign(costs, world)
        local = {k: _image(k, sizes[k][1] // 8, sizes[k][2] // 8) for k in a[rank]}
        own = owners(a)
        recv = {}
        if rank == 0:
            recv = {k: torch.empty((sizes[k][1] // 8) * (sizes[k][2] // 8), 4) for k in own if own[k] != 0}
        gather_to_root(rank, a, local, recv)
        if rank == 0:
            images = {**local, **recv}
            out["images"] = {k: v.numpy().copy() for k, v in images.items()}
        reps.barrier()
    finally:
        reps.close()


@pytest.mark.parametrize("world", [2, 3])
def test_gather_to_rank0_equals_a_single_rank_run(world):
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _port(), out), nprocs=world, join=True)
        got = dict(out)["images"]
    sizes = _sizes(24)
    assert sorted(got) == list(range(len(sizes)))
    for k, (t, w, h) in enumerate(sizes):
        assert np.array_equal(got[k], _image(k, w // 8, h // 8).numpy()), k
