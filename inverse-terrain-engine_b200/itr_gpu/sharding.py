"""Design sharding across GPUs: one process per GPU, torch.distributed for the plumbing.

A population's designs are independent (the batch axis of BatchBackend::run,
crates/itr-opt/src/evaluator.rs:131-135): each rank runs a contiguous shard of the designs
on its own GPU with the same terrain, and one all-gather of the per-design results after
the batch gives every rank the whole population's results, in population order. There is
no exchange during the run.

The collective moves a fixed-width float64 record per design (steps, cell_updates, bad,
status, j, feasible, monitor maxima), so it runs on NCCL (CUDA tensors) and on gloo (CPU
tensors) alike.
"""
from __future__ import annotations

import numpy as np

from .solver import BatchRun


def shard_bounds(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced shard [lo, hi) of n designs for `rank` of `world` (the first
    n % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


_HEAD = 3   # steps, cell_updates, bad


def _pack(runs: list[BatchRun], n_mon: int, rows: int) -> np.ndarray:
    out = np.zeros((rows, _HEAD + n_mon), dtype=np.float64)
    for i, r in enumerate(runs):
        out[i, 0] = r.steps
        out[i, 1] = r.cell_updates
        out[i, 2] = 1.0 if r.bad else 0.0
        out[i, _HEAD:] = r.monitor_max[:n_mon]
    return out


def _unpack(rec: np.ndarray, n_mon: int) -> BatchRun:
    return BatchRun(monitor_max=rec[_HEAD:_HEAD + n_mon].copy(), steps=int(rec[0]), cell_updates=int(rec[1]),
                    bad=bool(rec[2] != 0.0))


class ShardedBackend:
    """BatchBackend<f32> over the ranks of a torch.distributed process group.

    `backend` is this rank's evaluator (normally a GpuBackend on the rank's own GPU). run()
    takes the whole population on every rank, evaluates this rank's shard and returns every
    design's BatchRun on every rank. All ranks must call run() with the same population, as
    with any collective.
    """

    def __init__(self, backend, group=None):
        import torch.distributed as dist
        self.backend = backend
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"

    def name(self) -> str:
        return f"sharded x{self.world} [{self.backend.name()}]"

    def run(self, p, terrains, monitors) -> list[BatchRun]:
        import torch
        import torch.distributed as dist
        n = len(terrains)
        n_mon = len(monitors.cells)
        lo, hi = shard_bounds(n, self.world, self.rank)
        local = self.backend.run(p, terrains[lo:hi], monitors) if hi > lo else []
        if len(local) != hi - lo:
            raise RuntimeError(f"backend returned {len(local)} results for {hi - lo} designs")
        rows = shard_bounds(n, self.world, 0)[1]          # the largest shard
        mine = torch.from_numpy(_pack(local, n_mon, rows)).to(self.device)
        parts = [torch.empty_like(mine) for _ in range(self.world)]
        dist.all_gather(parts, mine, group=self.group)
        out: list[BatchRun] = []
        for r, part in enumerate(parts):
            a, b = shard_bounds(n, self.world, r)
            rec = part.cpu().numpy()
            out.extend(_unpack(rec[i], n_mon) for i in range(b - a))
        return out
