"""Uneven batch (itr_gpu_run_ladder): the fidelity ladder's grids in one CUDA graph launch.

Every group's results must equal the same group run alone through itr_gpu_run_batch (bit
for bit: steps, end time, monitor maxima, status, J), including live guard and incumbent
aborts (the reference runs one batch per ladder level, evaluator.rs:218-266).
"""
from __future__ import annotations

import numpy as np
import pytest

from itr_gpu import GpuSolver, PreparedTerrain
from itr_gpu.scenes import valley_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = GpuSolver()
    yield g
    g.close()


def ladder(duration=600.0, counts=(5, 3, 2)):
    groups = []
    for cell, n in zip((10.0, 5.0, 2.5), counts):
        sc = valley_scene(cell)
        sc.params.duration_s = duration
        groups.append((sc, [t for _, _, t in sc.designs(n)]))
    return groups


def same(a, b, what):
    assert a.steps == b.steps and a.t_end == b.t_end and a.status == b.status, what
    np.testing.assert_array_equal(a.monitor_max, b.monitor_max, err_msg=what)
    assert a.j == b.j and a.feasible == b.feasible, what


def test_ladder_matches_separate_batches(gpu):
    groups = ladder()
    p = groups[0][0].params
    spec = [dict(terrains=ts, monitors=sc.monitors, objective=sc.objective) for sc, ts in groups]
    out = gpu.run_ladder(p, spec)
    assert [len(o) for o in out] == [len(ts) for _, ts in groups]
    for gi, (sc, ts) in enumerate(groups):
        ref = gpu.run_batch(p, ts, sc.monitors, objective=sc.objective, want_depth=False)
        for i, (a, b) in enumerate(zip(out[gi], ref)):
            same(a, b, f"group {gi} design {i}")


def test_ladder_with_live_aborts(gpu):
    groups = ladder(duration=1200.0, counts=(6, 4, 2))
    p = groups[0][0].params
    spec = []
    for sc, ts in groups:
        base = gpu.run_batch(p, [PreparedTerrain(sc.base)], sc.monitors)[0]
        sc.objective.d.guard_tolerance_m = 0.0005
        full = gpu.run_batch(p, ts, sc.monitors, objective=sc.objective)
        inc = sorted(r.j for r in full)[len(full) // 2]
        spec.append(dict(terrains=ts, monitors=sc.monitors, objective=sc.objective, baseline_max=base.monitor_max,
                         guard_abort=True, incumbent=inc))
    out = gpu.run_ladder(p, spec)
    statuses = []
    for gi, ((sc, ts), g) in enumerate(zip(groups, spec)):
        ref = gpu.run_batch(p, ts, sc.monitors, objective=sc.objective, baseline_max=g["baseline_max"], guard_abort=True,
                            incumbent=g["incumbent"], want_depth=False)
        for i, (a, b) in enumerate(zip(out[gi], ref)):
            same(a, b, f"group {gi} design {i}")
            assert a.breach_cell == b.breach_cell and a.violation == b.violation and a.lower_bound == b.lower_bound
            statuses.append(a.status)
    assert any(s != 0 for s in statuses), "no abort was exercised"
