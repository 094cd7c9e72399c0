"""Host-side bookkeeping for running the likelihood on several GPUs of one
node, one process per GPU (launched by torchrun).

The path shards by proposal: every rank evaluates its own batches of
proposals (its own walkers' proposals, the way the reference's MPI farm hands
each slave its own parameter sets) and there is no exchange on the data path;
the process group carries only the barriers around timed regions and the
max-over-ranks of their durations.  Throughput is then weak-scaled: the units
all ranks processed over the slowest rank's time.
"""
import datetime
import os


class Ranks:
    """rank / world / local rank from the torchrun environment, and the
    process group (NCCL on GPUs, gloo for host-only runs) when world > 1."""

    def __init__(self, backend="nccl", timeout_s=120):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend,
                                    timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _device(self):
        return "cuda" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max_over_ranks(self, x):
        """The largest of every rank's x (a duration): the job's time."""
        if not self.dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(self, x):
        if not self.dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def proposal_seed(self, k):
        """Seed of this rank's k-th proposal batch: disjoint across ranks for
        k < 100, so no two ranks evaluate the same proposals."""
        return 100 * self.rank + k

    def throughput(self, units_per_rank, seconds):
        """Weak-scaled whole-job rate: all ranks' units over the slowest
        rank's time (seconds already reduced with max_over_ranks)."""
        return self.world * units_per_rank / seconds

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
