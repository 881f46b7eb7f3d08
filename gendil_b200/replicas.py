"""Multi-GPU runs of the operator path: independent replicas, one process per GPU.

The operator path does not shard across GPUs (every configuration fits one B200), so N GPUs run
N independent copies of the workload with no data-path collective; the only communication is
the timing reduction (the maximum over ranks) and barriers around the timed region.  Launched by
torchrun (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT from the environment) with
NCCL on GPUs; the same code runs with gloo on CPU processes, which is how it is tested.
"""
from __future__ import annotations

import datetime
import os


def env():
    """(world size, rank, local rank) from the launcher's environment (1, 0, 0 without one)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """Process group of the replicas (None for a single process) with the timing helpers."""

    def __init__(self, backend="nccl", timeout_s=120):
        import torch
        self.world, self.rank, self.local = env()
        self.backend = backend
        self.dist = None
        self.device = torch.device("cuda", self.local) if backend == "nccl" else torch.device("cpu")
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        """All ranks reach this point (and, on GPUs, their queued work is done)."""
        import torch
        if self.dist:
            self.dist.barrier()
        if self.device.type == "cuda":
            torch.cuda.synchronize()

    def max(self, value):
        """The maximum of a per-rank number over all ranks (every rank gets it)."""
        import torch
        if not self.dist:
            return float(value)
        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, units_per_rank, ms):
        """Whole-job rate (units / s) for weak scaling: every rank processed units_per_rank in at
        most `ms` milliseconds (the slowest rank's time)."""
        return self.world * units_per_rank / (ms * 1e-3)

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None
