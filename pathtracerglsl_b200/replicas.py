"""Multi-GPU replicas: one process per GPU, each rendering its own sample stream.

Pixels, samples and scenes are independent, so the transport loop shards without any
exchange: every rank renders the same frame with its own reset salt (decorrelated random
streams), and ranks meet only at a barrier and a max over ranks of their device time (the
job's time).  The one optional exchange combines the ranks' float64 films into the image of
all their samples (a sum over ranks of film sums and sample counts), outside any timed loop.

``torch.distributed`` is the plumbing: NCCL on GPUs, gloo on CPU (the multi-process tests).
"""
import datetime
import os


class Replicas:
    def __init__(self, rank=0, local=0, world=1, dist=None, device="cpu"):
        self.rank, self.local, self.world, self.dist, self.device = rank, local, world, dist, device

    @classmethod
    def from_env(cls, backend="nccl", timeout_s=120):
        """torchrun's environment (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_*); world 1 = no group."""
        world = int(os.environ.get("WORLD_SIZE", "1"))
        if world <= 1:
            return cls()
        import torch
        import torch.distributed as dist
        local = int(os.environ.get("LOCAL_RANK", "0"))
        kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
        device = "cpu"
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
            device = f"cuda:{local}"
        dist.init_process_group(backend, **kw)
        return cls(dist.get_rank(), local, world, dist, device)

    def salt(self, base):
        """The reset salt of this rank's sample stream (distinct per rank)."""
        return base + self.rank

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x):
        """Max over ranks of a host scalar (the job's device time)."""
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def combine_film(self, film_sum, film_sumsq, nsamples):
        """Sum the ranks' float64 film sums and sample counts: (mean, sumsq, n) of every
        rank's samples together (arrays are host numpy float64)."""
        if self.dist is None:
            return film_sum / nsamples, film_sumsq, nsamples
        import numpy as np
        import torch
        flat = np.concatenate([film_sum.ravel(), film_sumsq.ravel(), [float(nsamples)]])
        t = torch.from_numpy(flat).to(self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        out = t.cpu().numpy()
        n = out[-1]
        k = film_sum.size
        return (out[:k] / n).reshape(film_sum.shape), out[k:2 * k].reshape(film_sumsq.shape), n

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
