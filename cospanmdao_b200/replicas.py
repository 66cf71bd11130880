"""Several GPUs of one node: one process per GPU, independent units, no collective on the data path.

The path shards as independent objects (GEMVER instances, ragged-batch instances, serving requests), so a job on N
GPUs is N ranks that each run their own units. The only cross-rank steps are host-side bookkeeping:

  - the timing of a step is the MAX over ranks of each rank's device time (`Ranks.max`);
  - the whole-job rate is every rank's units over that max time (`whole_job_rate`);
  - a ragged column split across ranks (`shard_by_cost`) gets its global offsets from ONE exchange of the shard
    totals: rank r adds the exclusive scan of the totals of ranks < r to its local offsets (`global_offsets`).

`Ranks` reads RANK / WORLD_SIZE / LOCAL_RANK (torchrun's variables) and runs the collectives over torch.distributed:
NCCL on GPUs, gloo on the CPU (the tests run two gloo ranks).
"""
from __future__ import annotations

import datetime
import os

import numpy as np


class Ranks:
    """This process's place in the job, and the few collectives the host side needs."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self._device = None

    def init(self, backend: str = "nccl", timeout_s: float = 120.0):
        """Joins the process group (when WORLD_SIZE > 1). With NCCL, binds this process to GPU LOCAL_RANK first."""
        import torch
        if backend == "nccl":
            torch.cuda.set_device(self.local)
            self._device = torch.device("cuda", self.local)
        else:
            self._device = torch.device("cpu")
        if self.world > 1:
            import torch.distributed as dist
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl":
                kw["device_id"] = self._device
            dist.init_process_group(backend, rank=self.rank, world_size=self.world, **kw)
            self.pg = dist
        return self

    def barrier(self):
        import torch
        if self.pg:
            self.pg.barrier()
        if self._device is not None and self._device.type == "cuda":
            torch.cuda.synchronize()

    def _reduce(self, x: float, op) -> float:
        if not self.pg:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device)
        self.pg.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, self.pg.ReduceOp.MAX if self.pg else None)

    def sum(self, x: float) -> float:
        return self._reduce(x, self.pg.ReduceOp.SUM if self.pg else None)

    def gather_ints(self, x: int) -> list[int]:
        """Every rank's value of an integer, in rank order (exact for any 64-bit value)."""
        if not self.pg:
            return [int(x)]
        import torch
        t = torch.tensor([int(x)], dtype=torch.int64, device=self._device)
        out = [torch.empty_like(t) for _ in range(self.world)]
        self.pg.all_gather(out, t)
        return [int(o.item()) for o in out]

    def all_gather_tensor(self, t):
        """Every rank's copy of the tensor `t` (same shape and dtype on every rank), in rank order."""
        if not self.pg:
            return [t]
        import torch
        out = [torch.empty_like(t) for _ in range(self.world)]
        self.pg.all_gather(out, t.contiguous())
        return out

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()
            self.pg = None


def rank_seed(seed: int, rank: int) -> int:
    """The workload seed of rank `rank`: every rank runs its own units (weak scaling), rank 0 the single-GPU ones."""
    return int(seed) + 1_000_003 * int(rank)


def whole_job_rate(units_per_rank: list[float], seconds_max: float) -> float:
    """Units of every rank over the job's time (the max over ranks)."""
    return float(sum(units_per_rank)) / float(seconds_max)


def shard_by_cost(costs, world: int) -> list[np.ndarray]:
    """Splits units 0..len(costs)-1 into `world` CONTIGUOUS shards of near-equal total cost (cut where the prefix sum
    crosses r/world of the total). Contiguous shards keep a ragged column's order, so global offsets need only the
    shard totals. Every unit lands in exactly one shard; a shard may be empty when there are fewer units than ranks."""
    c = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    if c.ndim != 1 or (c < 0).any():
        raise ValueError("costs must be a 1-d array of non-negative values")
    pre = np.concatenate([[0.0], np.cumsum(c)])
    total = pre[-1]
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(pre, total * r / world, side="left")) if total > 0 else len(c) * r // world)
    cuts.append(len(c))
    cuts = np.maximum.accumulate(np.minimum(np.array(cuts), len(c)))
    return [np.arange(cuts[r], cuts[r + 1], dtype=np.int64) for r in range(world)]


def global_offsets(local_offsets: np.ndarray, ranks: Ranks) -> np.ndarray:
    """A contiguous shard's exclusive-scan offsets (count + 1 entries, local_offsets[0] == 0) moved to the global
    column: every rank adds the total of the shards before it (one exchange of the shard totals)."""
    totals = ranks.gather_ints(int(local_offsets[-1]))
    base = sum(totals[:ranks.rank])
    return np.asarray(local_offsets, dtype=np.uint64) + np.uint64(base)
