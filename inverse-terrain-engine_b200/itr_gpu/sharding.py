"""Design sharding across GPUs: one process per GPU, torch.distributed for the plumbing.

A population's designs are independent (the batch axis of BatchBackend::run,
crates/itr-opt/src/evaluator.rs:131-135): each rank runs a contiguous shard of the designs
on its own GPU with the same terrain, and one all-gather of the per-design results after
the batch gives every rank the whole population's results, in population order. There is
no exchange during the run.

Two entry points:
  * ShardedBackend.run(p, terrains, monitors) is BatchBackend::run: it returns BatchRun
    {monitor_max, steps, cell_updates, bad} per design, the reference's batch record;
  * ShardedBackend.run_batch(p, terrains, monitors, objective=..., baseline_max=...,
    guard_abort=..., incumbent=...) is GpuSolver.run_batch with the objective and aborts live:
    every design's whole outcome comes back (status, J, feasibility, guard breach cell, sync
    and exceedance, incumbent lower bound, end time, volume, residual, monitor maxima).
Both move one fixed-width float64 record per design (the fields of _FIELDS, then the monitor
maxima), so the collective runs on NCCL (CUDA tensors) and on gloo (CPU tensors) alike.
Integer fields (steps, cell ids) stay below 2^53 and pass through float64 exactly.
"""
from __future__ import annotations

import numpy as np

from .solver import BatchRun, GpuRun


def shard_bounds(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced shard [lo, hi) of n designs for `rank` of `world` (the first
    n % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


# Scalar fields of a design's record, in order; the monitor maxima follow.
_FIELDS = ("steps", "cell_updates", "bad", "status", "j", "feasible", "breach_cell", "breach_sync", "violation",
           "lower_bound", "t_end", "volume_m3", "rel_residual", "sync_count")
_HEAD = len(_FIELDS)


def _pack(runs: list, n_mon: int, rows: int) -> np.ndarray:
    out = np.zeros((rows, _HEAD + n_mon), dtype=np.float64)
    for i, r in enumerate(runs):
        for k, f in enumerate(_FIELDS):
            v = getattr(r, f, 0.0)
            out[i, k] = float(v) if not isinstance(v, bool) else (1.0 if v else 0.0)
        out[i, _HEAD:] = np.asarray(r.monitor_max, dtype=np.float64)[:n_mon]
    return out


def _unpack_batch(rec: np.ndarray, n_mon: int) -> BatchRun:
    return BatchRun(monitor_max=rec[_HEAD:_HEAD + n_mon].copy(), steps=int(rec[0]), cell_updates=int(rec[1]),
                    bad=bool(rec[2] != 0.0))


def _unpack_full(rec: np.ndarray, n_mon: int) -> GpuRun:
    v = dict(zip(_FIELDS, rec[:_HEAD]))
    return GpuRun(monitor_max=rec[_HEAD:_HEAD + n_mon].copy(), steps=int(v["steps"]), t_end=float(v["t_end"]),
                  volume_m3=float(v["volume_m3"]), depth=None, bad=bool(v["bad"] != 0.0), status=int(v["status"]),
                  breach_cell=int(v["breach_cell"]), breach_sync=int(v["breach_sync"]), violation=float(v["violation"]),
                  lower_bound=float(v["lower_bound"]), j=float(v["j"]), feasible=bool(v["feasible"] != 0.0),
                  sync_count=int(v["sync_count"]), rel_residual=float(v["rel_residual"]),
                  cell_updates=int(v["cell_updates"]))


class ShardedBackend:
    """BatchBackend<f32> over the ranks of a torch.distributed process group.

    `backend` is this rank's evaluator (normally a GpuBackend on the rank's own GPU; for
    run_batch it needs a `solver` with GpuSolver.run_batch's signature). Every call takes the
    whole population on every rank, evaluates this rank's shard and returns every design's
    result on every rank. All ranks must make the same calls with the same population, as
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

    def _gather(self, n, n_mon, local, unpack):
        import torch
        import torch.distributed as dist
        lo, hi = shard_bounds(n, self.world, self.rank)
        if len(local) != hi - lo:
            raise RuntimeError(f"backend returned {len(local)} results for {hi - lo} designs")
        rows = shard_bounds(n, self.world, 0)[1]          # the largest shard
        mine = torch.from_numpy(_pack(local, n_mon, rows)).to(self.device)
        parts = [torch.empty_like(mine) for _ in range(self.world)]
        dist.all_gather(parts, mine, group=self.group)
        out = []
        for r, part in enumerate(parts):
            a, b = shard_bounds(n, self.world, r)
            rec = part.cpu().numpy()
            out.extend(unpack(rec[i], n_mon) for i in range(b - a))
        return out

    def run(self, p, terrains, monitors) -> list[BatchRun]:
        """BatchBackend::run over the shards: BatchRun per design, population order."""
        n = len(terrains)
        lo, hi = shard_bounds(n, self.world, self.rank)
        local = self.backend.run(p, terrains[lo:hi], monitors) if hi > lo else []
        return self._gather(n, len(monitors.cells), local, _unpack_batch)

    def run_batch(self, p, terrains, monitors, objective=None, baseline_max=None, guard_abort=False,
                  incumbent=None) -> list[GpuRun]:
        """GpuSolver.run_batch over the shards with the objective and aborts live: every
        design's outcome (status, J, feasible, breach, exceedance, lower bound, ...) on every
        rank, population order. Depths and peaks stay on the rank that ran the design."""
        n = len(terrains)
        lo, hi = shard_bounds(n, self.world, self.rank)
        local = []
        if hi > lo:
            local = self.backend.solver.run_batch(p, terrains[lo:hi], monitors, objective=objective,
                                                  baseline_max=baseline_max, guard_abort=guard_abort,
                                                  incumbent=incumbent, want_depth=False)
        return self._gather(n, len(monitors.cells), local, _unpack_full)
