"""Multi-process plumbing for running one engine per GPU.

One process per GPU (torchrun sets RANK / LOCAL_RANK / WORLD_SIZE /
MASTER_*).  Each rank integrates its own independent clusters -- clusters are
independent units, so there is no collective on the data path; the process
group only provides barriers and the max-over-ranks of timings.
"""
import datetime
import os


class Dist:
    def __init__(self, use_cuda, timeout_s=300):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.use_cuda = use_cuda
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            if use_cuda:
                import torch
                torch.cuda.set_device(self.local)
            dist.init_process_group("nccl" if use_cuda else "gloo",
                                    timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x):
        """Maximum of x over all ranks (x itself on one rank)."""
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if self.use_cuda else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if self.use_cuda else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def cluster_seed(base, rank):
    """Seed of the cluster a rank integrates (independent units per rank)."""
    return base + 97 * rank


def weak_scaling_value(world, interactions_per_step, steps, max_total_ms):
    """Whole-job interactions/s: all ranks' work over the slowest rank's time."""
    return world * interactions_per_step * steps / (max_total_ms * 1e-3)
