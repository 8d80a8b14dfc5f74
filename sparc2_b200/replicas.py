"""Replica bookkeeping for runs on several GPUs of one node.

The SPARC time step does not shard here (the whole domain lives on one
GPU), so N GPUs run N independent simulations: no collective on the data
path.  torch.distributed is used only to line the ranks up (barrier) and to
take the maximum of their device-timed intervals.  Works with "nccl"
(GPU tensors) and "gloo" (CPU tensors, used by the CPU tests).
"""
import datetime
import os


class Replicas:
    def __init__(self, backend=None, timeout_s=300):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            if not dist.is_initialized():
                dist.init_process_group(
                    backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _device(self):
        if self.backend == "nccl":
            return f"cuda:{self.local}"
        return "cpu"

    def barrier(self):
        if self.dist is None:
            return
        import torch
        t = torch.zeros(1, device=self._device())
        self.dist.all_reduce(t)
        if self.backend == "nccl":
            torch.cuda.synchronize(self.local)

    def max(self, x):
        """Maximum of a float over all ranks (every rank gets it)."""
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def aggregate_rate(self, units_per_rank, seconds_per_rank):
        """Whole-job rate: all ranks' units over the slowest rank's time."""
        return self.world * units_per_rank / self.max(seconds_per_rank)

    def close(self):
        if self.dist is not None and self.dist.is_initialized():
            self.dist.destroy_process_group()
        self.dist = None
