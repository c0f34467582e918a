"""Design sharding over NCCL on the device (itr_gpu/sharding.py).

The gloo test (tests/test_sharding.py) covers two ranks on the CPU. Here the same backend runs
over an NCCL process group of one rank on the GPU, in a child process: the fixed-width records
cross NCCL's all-gather as CUDA tensors, and every design's outcome (BatchBackend::run's record,
and run_batch's with the objective and guard aborts live) equals the direct GpuSolver call.
"""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ("steps", "cell_updates", "bad", "status", "j", "feasible", "breach_cell", "breach_sync", "violation",
          "lower_bound", "t_end", "rel_residual", "sync_count")

CHILD = r'''
import datetime, os, sys
import numpy as np
here, out = sys.argv[1], sys.argv[2]
sys.path[:0] = [os.path.join(os.path.dirname(here), "inverse-terrain-engine_b200"), here]
import torch
import torch.distributed as dist
from itr_gpu import GpuSolver
from itr_gpu.solver import GpuBackend
from itr_gpu.sharding import ShardedBackend
from test_sharding_nccl import population
torch.cuda.set_device(0)
dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                        device_id=torch.device("cuda", 0))
g = GpuSolver(0)
try:
    sb = ShardedBackend(GpuBackend(g))
    assert sb.device == "cuda"
    sc, terrs, baseline = population()
    batch = sb.run(sc.params, terrs, sc.monitors)
    full = sb.run_batch(sc.params, terrs, sc.monitors, objective=sc.objective, baseline_max=baseline, guard_abort=True)
    fields = %r
    np.savez(out, b_steps=np.array([r.steps for r in batch]), b_cu=np.array([r.cell_updates for r in batch]),
             b_bad=np.array([r.bad for r in batch]), b_mm=np.stack([r.monitor_max for r in batch]),
             mm=np.stack([r.monitor_max for r in full]), **{f: np.array([getattr(r, f) for r in full]) for f in fields})
finally:
    g.close()
    dist.destroy_process_group()
''' % (FIELDS,)


def population():
    """Five valley designs (45 x 35 at 10 m) over 1200 s with guard aborts live: the baseline
    is the unedited terrain's device run, the guard tolerance tight."""
    from itr_gpu import GpuSolver, PreparedTerrain
    from itr_gpu.scenes import valley_scene
    sc = valley_scene(10.0)
    sc.params.duration_s = 1200.0
    sc.objective.d.guard_tolerance_m = 1e-5
    terrs = [t for _, _, t in sc.designs(5)]
    g = GpuSolver(0)
    try:
        baseline = g.run_batch(sc.params, [PreparedTerrain(sc.base)], sc.monitors, want_depth=False)[0].monitor_max
    finally:
        g.close()
    return sc, terrs, np.asarray(baseline, np.float64)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_backend_over_nccl_matches_direct_call(tmp_path):
    out = str(tmp_path / "nccl.npz")
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()), NCCL_NVLS_ENABLE="0")
    r = subprocess.run([sys.executable, "-c", CHILD, HERE, out], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got = np.load(out)
    from itr_gpu import GpuSolver
    sc, terrs, baseline = population()
    g = GpuSolver(0)
    try:
        ref = g.run_batch(sc.params, terrs, sc.monitors, objective=sc.objective, baseline_max=baseline, guard_abort=True,
                          want_depth=False)
        plain = g.run_batch(sc.params, terrs, sc.monitors, want_depth=False)
    finally:
        g.close()
    n = sc.base.nx * sc.base.ny
    assert list(got["b_steps"]) == [x.steps for x in plain]
    assert list(got["b_cu"]) == [x.steps * n for x in plain]
    assert list(got["b_bad"]) == [x.bad for x in plain]
    np.testing.assert_array_equal(got["b_mm"], np.stack([x.monitor_max for x in plain]))
    assert any(x.status == 1 for x in ref), [x.status for x in ref]
    for f in FIELDS:
        assert list(got[f]) == [getattr(x, f) for x in ref], f
    np.testing.assert_array_equal(got["mm"], np.stack([x.monitor_max for x in ref]))
