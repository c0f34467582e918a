"""Warm starts from a recorded baseline (BaselineRecord, crates/itr-hydro/src/solver.rs:95-118,
Evaluator's record.best_for, crates/itr-opt/src/evaluator.rs:423).

A rain-free storm that enters from part of the north edge: the southern rows stay dry for a
while, so designs edited there start from a late checkpoint of the baseline. A warm-started
run must equal the cold run of the same design bit for bit (steps, end time, depth, peaks,
monitor maxima, J; the f64 ledger to rounding), on every forward path, for designs given as
jump arrays and as primitives.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import assert_bitwise
from itr_gpu import GpuSolver, Hyetograph, PreparedTerrain, Segment, TerrainBase
from itr_gpu.design import BERM, SWALE, Primitive, materialize
from itr_gpu.scenes import valley_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = GpuSolver()
    yield g
    g.close()


def north_inflow_scene():
    sc = valley_scene(10.0)   # 45 x 35, valley along x, outlet east
    fine = sc.base.fine
    sc.base = TerrainBase(fine, 1, [Segment("transmissive", "east"),
                                    Segment("inflow", "north", (100.0, 160.0), hydrograph=[(0.0, 0.0), (300.0, 4.0), (1200.0, 2.0)])])
    sc.params.rain = Hyetograph.from_mm_h([(0, 0)])
    sc.params.infil_capacity = 0.0
    sc.params.duration_s = 1200.0
    return sc


def prim_sets(sc):
    south = [Primitive(BERM, 200.0, 30.0, 80.0, 8.0, 0.0, 0.4)]                 # rows near the south edge
    south2 = [Primitive(SWALE, 330.0, 45.0, 60.0, 10.0, 20.0, -0.3), Primitive(BERM, 120.0, 25.0, 40.0, 6.0, 90.0, 0.3)]
    north = [Primitive(BERM, 130.0, 343.0, 40.0, 8.0, 0.0, 0.3)]                # row 0, beside the inflow edge: cold
    return [south, south2, north] + [p for p, _, _ in sc.designs(3)] + [[]]


def terrains(sc, sets):
    b = sc.base
    return [PreparedTerrain(b).apply_edit(materialize(s, sc.geo, b.fine.nx, b.fine.ny, sc.editable, sc.max_abs_dz)) for s in sets]


def same(a, b, what):
    assert a.steps == b.steps and a.t_end == b.t_end, f"{what}: steps {a.steps} vs {b.steps}"
    assert_bitwise(a.depth, b.depth, f"{what}: depth")
    assert_bitwise(a.peak, b.peak, f"{what}: peak")
    np.testing.assert_array_equal(a.monitor_max, b.monitor_max, err_msg=what)
    assert a.j == b.j and a.status == b.status, what
    assert len(a.ledger) == len(b.ledger), what
    np.testing.assert_allclose(a.ledger, b.ledger, rtol=1e-12, atol=1e-9, err_msg=f"{what}: ledger")


@pytest.mark.parametrize("impl", [0, 1, 2])
def test_warm_start_equals_cold_start(gpu, impl):
    sc = north_inflow_scene()
    sets = prim_sets(sc)
    ts = terrains(sc, sets)
    base = gpu.record_baseline(sc.params, PreparedTerrain(sc.base), sc.monitors, checkpoint_interval=16, want_peak=True,
                               ledger_rows=64)
    cold_base = gpu.run_batch(sc.params, [PreparedTerrain(sc.base)], sc.monitors, want_peak=True, ledger_rows=64)[0]
    same(base, cold_base, "record vs cold baseline")
    gpu.set_option("impl", impl)
    try:
        cold = gpu.run_batch(sc.params, ts, sc.monitors, objective=sc.objective, want_peak=True, ledger_rows=64)
        gpu.set_option("warm_start", 1)
        warm = gpu.run_batch(sc.params, ts, sc.monitors, objective=sc.objective, want_peak=True, ledger_rows=64)
    finally:
        gpu.set_option("warm_start", 0)
        gpu.set_option("impl", 0)
    for i, (w, c) in enumerate(zip(warm, cold)):
        same(w, c, f"impl {impl} design {i} (warm from step {w.warm_start_steps})")
    ws = [w.warm_start_steps for w in warm]
    assert ws[0] > 0 and ws[1] > 0, ws     # the southern edits start late
    assert ws[2] == 0, ws                  # beside the inflow edge: cold
    assert ws[-1] > 0, ws                  # no edit: the last checkpoint


def test_warm_start_primitives_and_fallbacks(gpu):
    sc = north_inflow_scene()
    sets = prim_sets(sc)
    gpu.record_baseline(sc.params, PreparedTerrain(sc.base), sc.monitors, checkpoint_interval=16)
    cold, _, _ = gpu.run_primitives(sc.params, sc.base, sets, sc.monitors, sc.editable, sc.max_abs_dz, objective=sc.objective,
                                    want_peak=True, ledger_rows=64)
    gpu.set_option("warm_start", 1)
    try:
        warm, _, _ = gpu.run_primitives(sc.params, sc.base, sets, sc.monitors, sc.editable, sc.max_abs_dz,
                                        objective=sc.objective, want_peak=True, ledger_rows=64)
        # an incumbent abort, or other params, start cold
        ts = terrains(sc, sets)
        inc = gpu.run_batch(sc.params, ts, sc.monitors, objective=sc.objective, incumbent=1e9)
        p2 = north_inflow_scene().params
        p2.duration_s = 900.0
        other = gpu.run_batch(p2, ts, sc.monitors)
    finally:
        gpu.set_option("warm_start", 0)
    for i, (w, c) in enumerate(zip(warm, cold)):
        same(w, c, f"primitives design {i}")
    assert warm[0].warm_start_steps > 0
    assert all(r.warm_start_steps == 0 for r in inc) and all(r.warm_start_steps == 0 for r in other)
