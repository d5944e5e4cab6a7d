"""Ranks of a multi-GPU run: one process per GPU, each rendering its own replica.

The render path shards trivially -- pixels, samples and whole scenes are
independent and every pixel accumulates on its own GPU -- so a run on N GPUs
is N replicas of the workload (weak scaling) and no image data crosses between
ranks.  Ranks meet only to time the job: a barrier on both sides of the timed
region, the maximum of the ranks' device times and the sum of their samples
(the whole-job rate), and rank 0 reports.

`Replicas` wraps that bookkeeping over torch.distributed.  The collectives run
on `device` ("cuda" with NCCL on GPU boxes, "cpu" with gloo in the tests); a
single process (WORLD_SIZE unset or 1) needs no process group.
"""
from __future__ import annotations

import datetime
import os
from typing import Optional


class Replicas:
    def __init__(self, backend: Optional[str] = None, device: str = "cuda", timeout_s: float = 300.0,
                 local_device: Optional[int] = None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = device
        self._owns_group = False
        if self.world > 1:
            import torch
            import torch.distributed as dist
            if not dist.is_initialized():
                kw = {}
                if backend == "nccl" or (backend is None and device == "cuda"):
                    kw["device_id"] = torch.device("cuda", self.local if local_device is None else local_device)
                dist.init_process_group(backend or ("nccl" if device == "cuda" else "gloo"),
                                        timeout=datetime.timedelta(seconds=timeout_s), **kw)
                self._owns_group = True

    @property
    def is_root(self) -> bool:
        return self.rank == 0

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if self.world == 1:
            return float(x)
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(x)], device=self.device, dtype=torch.float64)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        """Largest value over the ranks (device times: the job ends with its slowest rank)."""
        import torch.distributed as dist
        return self._reduce(x, dist.ReduceOp.MAX if self.world > 1 else None)

    def sum(self, x: float) -> float:
        """Sum over the ranks (samples rendered by the whole job)."""
        import torch.distributed as dist
        return self._reduce(x, dist.ReduceOp.SUM if self.world > 1 else None)

    def job_rate(self, units: float, ms: float, scale: float = 1e-6) -> float:
        """Whole-job throughput: every rank's units over the slowest rank's time, in units/s x scale."""
        total_ms = self.max(ms)
        return self.sum(units) / (total_ms / 1e3) * scale if total_ms > 0 else 0.0

    def close(self):
        if self._owns_group:
            import torch.distributed as dist
            dist.destroy_process_group()
            self._owns_group = False
