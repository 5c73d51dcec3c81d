"""Multi-GPU replicas: one process per GPU, each advancing its own copy of the
workload with no data-path collective (weak scaling).  The process group only
brackets the timed region with barriers and takes the maximum device time
over the ranks; the job's rate is every rank's units over that time.

Launch (one node): python -m torch.distributed.run --nnodes=1
--nproc-per-node N --master-addr 127.0.0.1 --master-port P bench.py --gpus N
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    rank: int
    world: int
    local: int
    dist: object = None     # torch.distributed when world > 1
    device: str = "cpu"     # where reduction tensors live ("cuda" with NCCL)

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """Maximum of x over the ranks (x itself on one rank)."""
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def from_env(backend: str = "nccl", timeout_s: int = 600) -> Ranks:
    """Ranks from RANK / WORLD_SIZE / LOCAL_RANK; a process group (NCCL with
    one GPU per local rank, or gloo on the CPU) when more than one rank."""
    r = Ranks(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
              int(os.environ.get("LOCAL_RANK", "0")))
    if r.world > 1:
        import torch
        import torch.distributed as tdist
        if backend == "nccl":
            torch.cuda.set_device(r.local)
            tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                     device_id=torch.device("cuda", r.local))
            r.device = "cuda"
        else:
            tdist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
        r.dist = tdist
    return r


def job_rate(units_per_rank: float, world: int, seconds: float) -> float:
    """Job-wide rate of weak-scaled replicas: every rank's units over the
    slowest rank's time."""
    return world * units_per_rank / seconds
