"""A batch of scenes split over GPUs, one process per GPU, and the one image
gather at the end.

Scenes are independent (every pixel accumulates on the GPU that renders it),
so a batch shards by whole scenes with no data-path collective: each rank
builds the BVHs of its own scenes and renders them in one batched pt_render,
and when the batch is done every image is gathered once to rank 0.

* ``scene_cost``: the estimated render cost of a scene -- its sample budget
  (pixels x spp) times the traversal depth of its BVH (1 + log2 triangles);
  the build cost, linear in the triangles and far smaller, is left out.
* ``assign``: greedy longest-processing-time assignment: scenes in order of
  decreasing cost, each to the rank with the least cost so far (ties to the
  lower rank), so the slowest rank carries at most 4/3 of the optimum.  Every
  rank computes the same assignment from the same costs.
* ``gather_to_root``: point-to-point sends of each remote scene's image (in
  scene order) into rank 0's buffers -- NCCL over NVLink between GPUs, gloo in
  the CPU tests.  Rank 0 posts all receives, the owners all sends; nothing
  else crosses between ranks.
"""
from __future__ import annotations

import math
from typing import Dict, List, Sequence


def scene_cost(triangles: int, pixels: int, spp: int) -> float:
    return float(pixels) * float(spp) * (1.0 + math.log2(max(int(triangles), 2)))


def assign(costs: Sequence[float], world: int) -> List[List[int]]:
    """Scene indices per rank (each rank's list in increasing scene order)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    owned: List[List[int]] = [[] for _ in range(world)]
    for k in sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i)):
        r = min(range(world), key=lambda q: (load[q], q))
        owned[r].append(k)
        load[r] += float(costs[k])
    return [sorted(o) for o in owned]


def owners(assignment: Sequence[Sequence[int]]) -> Dict[int, int]:
    return {k: r for r, ks in enumerate(assignment) for k in ks}


def gather_to_root(rank: int, assignment: Sequence[Sequence[int]], local: Dict[int, "object"],
                   recv_buffers: Dict[int, "object"]) -> None:
    """Sends this rank's scene images to rank 0, or (on rank 0) receives every
    other rank's.  `local`: scene -> tensor this rank rendered; `recv_buffers`
    (rank 0 only): scene -> preallocated tensor of the right shape, dtype and
    device for every scene rank 0 does not own.  Single-process runs return at once."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return
    own = owners(assignment)
    work = []
    for k in sorted(own):
        src = own[k]
        if src == 0:
            continue
        if rank == 0:
            work.append(dist.irecv(recv_buffers[k], src=src))
        elif rank == src:
            work.append(dist.isend(local[k].contiguous(), dst=0))
    for w in work:
        w.wait()
