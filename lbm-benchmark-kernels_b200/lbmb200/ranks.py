"""One process per GPU: rank bookkeeping for runs over several GPUs.

Every rank works on its own domains -- nothing on the data path crosses
GPUs -- so torch.distributed only provides the barrier around timed regions
and the max / sum of per-rank numbers. The process group uses NCCL on GPUs
and gloo for CPU-only use (tests), with a short timeout so that a rank that
never arrives ends the others with an error instead of a hang.
"""
import datetime
import os


class Ranks:
    def __init__(self, backend=None, timeout_s=120):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.device = "cpu"
        if self.world > 1:
            import torch
            import torch.distributed as dist
            self.torch, self.dist = torch, dist
            backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = "cuda"
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def _reduce(self, v, op):
        if self.dist is None:
            return float(v)
        t = self.torch.tensor([float(v)], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, v):
        return self._reduce(v, self.dist.ReduceOp.MAX if self.dist else None)

    def sum(self, v):
        return self._reduce(v, self.dist.ReduceOp.SUM if self.dist else None)

    def sum_vec(self, values):
        """Element-wise FP64 sum over ranks of a short vector (conservation
        sums of a decomposed lattice)."""
        vals = [float(v) for v in values]
        if self.dist is None:
            return vals
        t = self.torch.tensor(vals, dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return [float(v) for v in t.tolist()]

    def share(self, items):
        """This rank's share of a list (round robin)."""
        return list(items)[self.rank::self.world]

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
