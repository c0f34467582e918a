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
