"""Independent replicas over several GPUs (weak scaling).

One compressed product fits one GPU, so the multi-GPU form runs one
independent product stream per rank with no data exchange; the process
group only aligns the timed regions and reduces timings (max over ranks).
One process per GPU, launched by torchrun (RANK / WORLD_SIZE / LOCAL_RANK /
MASTER_ADDR / MASTER_PORT from the environment).  The backend is NCCL on
GPUs and gloo on the CPU, so this plumbing is testable without a GPU.
"""
from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    def __init__(self, backend=None, timeout_s=300):
        import torch
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.cuda = torch.cuda.is_available()
        if self.cuda:
            torch.cuda.set_device(self.local if self.world > 1 else 0)
        self.backend = backend or ("nccl" if self.cuda else "gloo")
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(self.backend, timeout=timedelta(seconds=timeout_s))
        self._dev = torch.device("cuda", torch.cuda.current_device()) if (self.cuda and self.backend == "nccl") \
            else torch.device("cpu")

    def barrier(self):
        """All ranks reach this point; pending device work is complete."""
        import torch
        if self.world > 1:
            torch.distributed.barrier()
        if self.cuda:
            torch.cuda.synchronize()

    def max(self, x):
        """Max of a float over ranks (timings: the slowest rank bounds the job)."""
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._dev)
        if self.world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._dev)
        if self.world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
        return float(t.item())

    def throughput(self, units_per_rank, seconds):
        """Whole-job rate: the units all ranks processed over the slowest rank's time."""
        return self.sum(units_per_rank) / self.max(seconds)

    def close(self):
        if self.world > 1:
            import torch.distributed as dist
            if dist.is_initialized():
                dist.destroy_process_group()
