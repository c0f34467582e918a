"""Guard-abort soundness (crates/itr-opt/tests/search.rs:144-171): every candidate stopped by
the guard test, re-run to completion without aborts, is infeasible. The whole map outside
the assets is guarded (`guard_whole_map`), so most edits move water somewhere.

The converse holds as well and is checked: a candidate that runs to the end with the guard
live is feasible, because the end of the storm is itself a sync point (the last sync
instant is min((k+1) sync, duration), solver.rs:449) and the running maxima only grow.
CPU: the oracle's GuardObserver restatement. GPU: the device's guard abort on the batched
cluster kernel and on the tiled path.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle_ref as orc
from helpers import base_arrays, design_dict
from itr_gpu import Objective, ObjectiveDef, PreparedTerrain
from itr_gpu.scenes import valley_scene

N_DESIGNS = 24


def whole_map_problem():
    sc = valley_scene(10.0, design_seed=11)
    sc.params.duration_s = 1500.0
    nx, ny = sc.base.nx, sc.base.ny
    d = sc.objective.d
    asset_cells = {c for a in d.assets for c in a.cells}
    guard = [c for c in range(nx * ny) if c not in asset_cells]
    obj = Objective(ObjectiveDef(d.assets, guard, guard_tolerance_m=0.002))
    o = orc.flat_run(base_arrays(sc.base), design_dict(PreparedTerrain(sc.base), sc.params), sc.params, obj.monitors)
    return sc, obj, o["monitor_max"].copy()


def test_oracle_guard_abort_is_sound():
    sc, obj, baseline = whole_map_problem()
    n_abort = 0
    for prims, e, t in sc.designs(N_DESIGNS):
        live = orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, obj.monitors, objective=obj,
                            baseline=baseline)
        full = orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, obj.monitors)
        feasible = obj.evaluate(full["monitor_max"], e.cut_m3, e.fill_m3, baseline)["feasible"]
        aborted = live["abort"] == orc.ABORT_GUARD
        n_abort += aborted
        assert aborted == (not feasible), (aborted, feasible)
    assert 0 < n_abort < N_DESIGNS   # the problem yields both outcomes


@pytest.mark.gpu
@pytest.mark.parametrize("impl", [0, 2])
def test_device_guard_abort_is_sound(impl):
    from itr_gpu import GpuSolver
    sc, obj, baseline = whole_map_problem()
    terrs = [t for _, _, t in sc.designs(N_DESIGNS)]
    g = GpuSolver()
    try:
        g.set_option("impl", impl)
        live = g.run_batch(sc.params, terrs, obj.monitors, objective=obj, baseline_max=baseline, guard_abort=True)
        full = g.run_batch(sc.params, terrs, obj.monitors, objective=obj, baseline_max=baseline, guard_abort=False)
    finally:
        g.close()
    n_abort = 0
    for a, f in zip(live, full):
        aborted = a.status == 1   # ITR_RUN_GUARD_ABORT
        n_abort += aborted
        assert f.status == 0
        assert aborted == (not f.feasible), (aborted, f.feasible, f.violation)
        if aborted:
            assert a.steps <= f.steps and a.violation > 0.0
    assert 0 < n_abort < N_DESIGNS
