"""Design sharding across ranks (CPU, gloo, world size 2).

Each rank evaluates a contiguous shard of the population and one all-gather returns every
design's result on every rank, in population order (the multi-GPU layout of the batch
axis, crates/itr-opt/src/evaluator.rs:131-135). The per-rank evaluator here is the CPU
oracle, so the host logic is tested without a GPU; on GPUs it is a GpuBackend per rank.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from itr_gpu.sharding import shard_bounds


def test_shard_bounds_cover_the_population_once():
    for n in range(0, 23):
        for world in range(1, 6):
            spans = [shard_bounds(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for (a, b), (c, _) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(4, 2, 2)


class OracleBackend:
    """BatchBackend over the f32 CPU oracle (test stand-in for a rank's GPU)."""

    def name(self):
        return "oracle-f32"

    def run(self, p, terrains, monitors):
        import oracle_ref as orc
        from helpers import base_arrays, design_dict
        from itr_gpu import BatchRun
        out = []
        for t in terrains:
            o = orc.flat_run(base_arrays(t.base), design_dict(t, p), p, monitors)
            n = t.base.nx * t.base.ny
            out.append(BatchRun(monitor_max=np.asarray(o["monitor_max"], np.float64), steps=int(o["steps"]),
                                cell_updates=int(o["steps"]) * n, bad=bool(o.get("bad", False))))
        return out


class OracleSolver:
    """GpuSolver.run_batch over the f32 CPU oracle, aborts live (stand-in for a rank's GPU):
    status, breach, exceedance and lower bound from the oracle's observer, J and feasibility
    from the host objective, as itr_gpu_run_batch reports them."""

    def run_batch(self, p, terrains, monitors, objective=None, baseline_max=None, guard_abort=False, incumbent=None,
                  want_depth=True):
        import oracle_ref as orc
        from helpers import base_arrays, design_dict
        from itr_gpu import GpuRun
        out = []
        for t in terrains:
            o = orc.flat_run(base_arrays(t.base), design_dict(t, p), p, monitors, objective=objective,
                             baseline=baseline_max if guard_abort else None, incumbent=incumbent)
            rep = objective.evaluate(o["monitor_max"], t.cut_m3, t.fill_m3, baseline_max)
            n = t.base.nx * t.base.ny
            out.append(GpuRun(monitor_max=np.asarray(o["monitor_max"], np.float64), steps=int(o["steps"]), t_end=o["t_end"],
                              volume_m3=0.0, depth=None, bad=o["abort"] == orc.ABORT_UNHEALTHY, status=o["abort"],
                              breach_cell=o["abort_cell"], breach_sync=o["abort_sync"], violation=o["abort_exceed"],
                              lower_bound=o["abort_lb"], j=rep["j"], feasible=rep["feasible"], sync_count=o["sync_count"],
                              rel_residual=o["rel_residual"], cell_updates=int(o["steps"]) * n))
        return out


class OracleFullBackend(OracleBackend):
    solver = OracleSolver()


def _guarded():
    """The population with guard aborts live: the baseline is the unedited terrain's run and
    the tolerance is tight, so some designs stop at a breached sync point."""
    import oracle_ref as orc
    from helpers import base_arrays, design_dict
    from itr_gpu import PreparedTerrain
    sc, terrs = _population()
    sc.params.duration_s = 1200.0
    sc.objective.d.guard_tolerance_m = 1e-5   # two of the five designs worsen the guard by 2.5e-5 and 3.9e-5 m
    b = orc.flat_run(base_arrays(sc.base), design_dict(PreparedTerrain(sc.base), sc.params), sc.params, sc.monitors)
    return sc, terrs, b["monitor_max"]


def _population():
    from itr_gpu.scenes import valley_scene
    sc = valley_scene(10.0)          # 45 x 35
    sc.params.duration_s = 240.0
    return sc, [t for _, _, t in sc.designs(5)]   # odd count: shards of 3 and 2


def _rank_main(rank, world, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [os.path.join(os.path.dirname(here), "inverse-terrain-engine_b200"), here]
    import datetime
    import torch.distributed as dist
    from itr_gpu.sharding import ShardedBackend
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sc, terrs = _population()
        runs = ShardedBackend(OracleBackend()).run(sc.params, terrs, sc.monitors)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), steps=np.array([r.steps for r in runs]),
                 cu=np.array([r.cell_updates for r in runs]), bad=np.array([r.bad for r in runs]),
                 mm=np.stack([r.monitor_max for r in runs]))
        sc, terrs, baseline = _guarded()
        full = ShardedBackend(OracleFullBackend()).run_batch(sc.params, terrs, sc.monitors, objective=sc.objective,
                                                            baseline_max=baseline, guard_abort=True)
        np.savez(os.path.join(out_dir, f"full{rank}.npz"), **{f: np.array([getattr(r, f) for r in full]) for f in FULL_FIELDS},
                 mm=np.stack([r.monitor_max for r in full]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_population_matches_single_process(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    sc, terrs = _population()
    ref = OracleBackend().run(sc.params, terrs, sc.monitors)
    for rank in range(world):
        got = np.load(tmp_path / f"rank{rank}.npz")
        assert list(got["steps"]) == [r.steps for r in ref]
        assert list(got["cu"]) == [r.cell_updates for r in ref]
        assert list(got["bad"]) == [r.bad for r in ref]
        np.testing.assert_array_equal(got["mm"], np.stack([r.monitor_max for r in ref]))
    # the whole outcome of every design crosses the gather, guard aborts included
    sc, terrs, baseline = _guarded()
    ref = OracleSolver().run_batch(sc.params, terrs, sc.monitors, objective=sc.objective, baseline_max=baseline,
                                   guard_abort=True)
    assert any(r.status == 1 for r in ref) and any(r.status == 0 for r in ref), [r.status for r in ref]
    for rank in range(world):
        got = np.load(tmp_path / f"full{rank}.npz")
        for f in FULL_FIELDS:
            assert list(got[f]) == [getattr(r, f) for r in ref], f
        np.testing.assert_array_equal(got["mm"], np.stack([r.monitor_max for r in ref]))


FULL_FIELDS = ("steps", "cell_updates", "bad", "status", "j", "feasible", "breach_cell", "breach_sync", "violation",
               "lower_bound", "t_end", "rel_residual", "sync_count")
