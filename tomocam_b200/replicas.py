"""Replica plumbing for running independent reconstructions on several GPUs.

The MBIR path of one volume runs on one GPU; with N processes (one per GPU,
launched by torchrun) every rank reconstructs its own volume and the ranks
only synchronise for timing: a barrier before and after the timed region and
a maximum of the per-rank times.  No data crosses between ranks.

The same functions run over NCCL on GPUs and over gloo on CPU (tests).
"""
from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    """Rank, world size and the two collectives the timing needs."""

    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 600.0):
        import torch
        import torch.distributed as dist
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = device
        self._dist = dist
        self._torch = torch
        if self.world > 1 and not dist.is_initialized():
            kw = {"timeout": timedelta(seconds=timeout_s)}
            if backend == "nccl" and device is not None:
                kw["device_id"] = device
            dist.init_process_group(backend, **kw)

    def barrier(self):
        if self.world > 1:
            self._dist.barrier()

    def max_over_ranks(self, value: float) -> float:
        """The largest value over all ranks (every rank gets it)."""
        if self.world == 1:
            return float(value)
        dev = self.device if self.backend == "nccl" else "cpu"
        t = self._torch.tensor([float(value)], dtype=self._torch.float64, device=dev)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def aggregate_rate(self, units_per_rank: float, seconds_max: float) -> float:
        """Whole-job throughput: all ranks' units over the slowest rank's time."""
        return self.world * float(units_per_rank) / float(seconds_max)

    def close(self):
        if self.world > 1 and self._dist.is_initialized():
            self._dist.destroy_process_group()
