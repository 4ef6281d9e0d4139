"""One process per GPU, each an independent replica of the encoder.

Frames are independent (the reference's multi-GPU form is a host pull scheduler over
whole frames, src/core/pipeline.cpp:166-190), so replicas exchange no frame data: the
only collectives are the barrier around a timed region and the max over ranks of the
time it took. Rank, local rank and world size come from the launcher's environment
(torchrun sets RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT). NCCL between
GPUs; gloo on CPU, which is how the tests run two ranks without a GPU.
"""
from __future__ import annotations

import datetime
import os


def rank_info():
    """(rank, local rank, world size) from the launcher's environment."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class Replicas:
    """The process group of the replicas, or nothing when there is one."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0, device=None):
        self.rank, self.local, self.world = rank_info()
        self.backend = backend
        self.device = device
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    def _tensor(self, x):
        import torch
        dev = self.device if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def max(self, x: float) -> float:
        """The largest x over the ranks (every rank calls it, in the same order)."""
        if self._dist is None:
            return float(x)
        t = self._tensor(x)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if self._dist is None:
            return float(x)
        t = self._tensor(x)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def barrier(self):
        if self._dist is not None:
            if self.backend == "nccl":
                self._dist.barrier(device_ids=[self.local])
            else:
                self._dist.barrier()

    def frame_seed(self, base: int) -> int:
        """The seed of this replica's synthetic frames: each replica encodes its own frames."""
        return base + 1_000_003 * self.rank

    def close(self):
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None
