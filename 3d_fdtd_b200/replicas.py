"""One process per GPU running independent simulations (replicas).

The hot path does not shard one domain across GPUs: taper candidates are
independent, so N GPUs run N simulations with no collective on the data path.
What ranks share is host plumbing -- a barrier around timed regions, the
maximum of the per-rank device times (the whole job is as slow as its slowest
rank), a deterministic split of candidates over ranks and a gather of the
per-candidate results (T(lambda), gradients) to every rank.

The process group comes from the usual torchrun environment (RANK,
WORLD_SIZE, LOCAL_RANK, MASTER_ADDR, MASTER_PORT).  Backend "nccl" on GPUs;
"gloo" runs the same logic on CPU.  A short timeout turns a rank that died or
never joined into an error on the others' next collective instead of a hang.
"""
from __future__ import annotations

import datetime
import os


class Ranks:
    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.local_rank = int(os.environ.get("LOCAL_RANK", 0))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            if not dist.is_initialized():
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    @property
    def on_cuda(self) -> bool:
        return self.backend == "nccl"

    def _sync(self):
        if self.on_cuda:
            import torch

            torch.cuda.synchronize()

    def barrier(self) -> None:
        """Device synchronise, barrier over ranks, device synchronise."""
        self._sync()
        if self.dist is not None:
            self.dist.barrier()
        self._sync()

    def max(self, x: float) -> float:
        """Maximum of x over ranks (every rank gets it)."""
        if self.dist is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda" if self.on_cuda else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def shard(self, n: int) -> list[int]:
        """Candidate indices of this rank: rank, rank + world, ... (disjoint, covering 0..n-1)."""
        return list(range(self.rank, n, self.world))

    def gather(self, obj) -> list:
        """obj of every rank, in rank order, on every rank."""
        if self.dist is None:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out

    def gather_shards(self, n: int, results: dict) -> list:
        """Per-candidate results of every rank, indexed 0..n-1 (results: index -> value)."""
        merged = {}
        for part in self.gather(results):
            merged.update(part)
        missing = [i for i in range(n) if i not in merged]
        if missing:
            raise RuntimeError(f"candidates without a result: {missing[:8]}")
        return [merged[i] for i in range(n)]

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
