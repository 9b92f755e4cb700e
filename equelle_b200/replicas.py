"""Several GPUs of one node: one process per GPU, each running an
independent replica of the workload.

The generated simulators have no exchange step between processes (the
reference's runtime is serial: one grid, one process), so nothing crosses
between ranks on the data path.  What the ranks share is timing plumbing
only: a barrier before the timed region, the maximum of the per-rank times
after it, and a barrier before the group is torn down.  The group uses
NCCL when the ranks own GPUs and gloo otherwise (the CPU tests run the
oracle's simulators as replicas through the same code).

Ranks read RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT from
the environment, as torchrun sets them.  A group is created only when
WORLD_SIZE > 1.  Its timeout is short enough that ranks waiting on one that
left end with an error instead of waiting for good.
"""
import datetime
import os


class Replicas:
    def __init__(self, backend=None, timeout_s=600.0, group=True):
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.dist = None
        self.backend = None
        if self.world > 1 and group:
            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist
            self.backend = backend

    @property
    def leader(self):
        return self.rank == 0

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, x):
        """The maximum of the float `x` over all ranks (every rank gets it)."""
        if not self.dist:
            return float(x)
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, units_per_rank, ms):
        """Whole-job rate: the units all ranks processed over the slowest
        rank's time (`ms` already the maximum over ranks)."""
        return self.world * units_per_rank / (ms / 1000.0)

    def close(self, sync=True):
        """Tears the group down (after a barrier unless `sync` is False, as
        for ranks that leave before any collective)."""
        if self.dist:
            if sync:
                self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
