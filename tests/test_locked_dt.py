"""Baseline-locked dt (SolverParams::locked_dt / cfl_hard, crates/itr-hydro/src/solver.rs:42-46,
run loop :436-483, snapshot at every sync :611-614).

Every step takes the baseline's recorded dt when dt * smax of the current state stays within
cfl_hard; at the first step where it would not, the run goes back to the last sync snapshot and
continues with the adaptive dt from there, reporting the time of the fallback
(RunSummary::dt_fallback_t).

CPU: the oracle keeps the reference's own properties (crates/itr-hydro/tests/replay.rs:40-80):
a zero edit under its own locked schedule is the baseline bit for bit with no fallback; an
edit that speeds the flow up past a tight cfl_hard falls back and stays healthy, its ledger
closing to 1e-4 (f32) and 1e-10 (f64) of the gross input.
GPU: the batched cluster kernel and the tiled path under a locked schedule against the f32
oracle under the same schedule, bit for bit (steps, end time, depth, peaks, monitor maxima,
fallback time), for a zero edit, an edit that stays locked and an edit that falls back.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle_ref as orc
from helpers import assert_bitwise, base_arrays, design_dict
from itr_gpu import GpuSolver, Hyetograph, MonitorSet, PreparedTerrain, Segment, SolverParams, UnsupportedError, synthetic_terrain
from itr_gpu.terrain import TerrainEdit

NX, NY = 72, 56


def base():
    """The scene of replay.rs:15-21: a gentle slope with ripples, an inflow on part of the west
    edge, a transmissive east edge."""
    segs = [Segment("inflow", "west", (40.0, 70.0), hydrograph=[(0.0, 0.0), (200.0, 2.0), (600.0, 0.3)]),
            Segment("transmissive", "east")]
    return synthetic_terrain(NX, NY, 2.0, lambda x, y: 50.0 + 0.004 * (150.0 - x) + 0.3 * math.sin(x / 11.0) * math.cos(y / 9.0),
                             n=0.035, segments=segs)


def params(cfl_hard=0.5):
    """validation::params(800, 40) with the storm of replay.rs:23-27."""
    p = SolverParams(duration_s=800.0, sync_interval_s=40.0,
                     rain=Hyetograph.from_mm_h([(0.0, 0.0), (100.0, 0.0), (200.0, 60.0), (500.0, 0.0)]))
    p.cfl_hard = cfl_hard
    return p


def monitors():
    return MonitorSet(np.array([c for c in range(NX * NY) if c % 5 == 1], dtype=np.uint32))


def fast_edit():
    """replay.rs:72-75: a cut deepening toward the east over the western 30 columns, which
    speeds the flow up."""
    w = 30
    dz = np.array([-0.6 * ((k % w) / w) for k in range(w * NY)])
    return TerrainEdit(0, 0, w, NY, dz)


def small_edit():
    """A 3 x 3 bump of 2 cm well inside the domain: the flow barely changes."""
    return TerrainEdit(34, 26, 3, 3, np.full(9, 0.02))


def run(b, t, p, prec=32, locked=None, record=False):
    mon = monitors()
    if prec == 32:
        f = lambda: orc.flat_run(base_arrays(b), design_dict(t, p), p, mon, want_peak=True, bnd=orc.bnd_dict(b, t), max_rows=64)
    else:
        f = lambda: orc.flat_run64(base_arrays(b), design_dict(t, p), p, mon, want_peak=True, bnd=orc.bnd_dict(b, t), max_rows=64)
    return orc.locked(f, locked, p.cfl_hard, record)


@pytest.mark.parametrize("prec", [32, 64])
def test_oracle_locked_schedule(prec):
    b = base()
    zero = PreparedTerrain(b)
    s0 = run(b, zero, params(), prec, record=True)
    dts = s0["dts"]
    assert len(dts) == s0["steps"] and s0["dt_fallback_t"] == -1.0

    # zero edit under its own schedule: the baseline bit for bit, no fallback
    s1 = run(b, zero, params(), prec, locked=dts, record=True)
    assert s1["steps"] == s0["steps"] and s1["t_end"] == s0["t_end"]
    assert s1["dt_fallback_t"] == -1.0
    np.testing.assert_array_equal(s1["dts"], dts)
    for k in ("h", "qx", "qy", "peak", "monitor_max"):
        np.testing.assert_array_equal(s1[k], s0[k], err_msg=k)

    # an edit that speeds the flow past a tight cfl_hard: falls back at a step start, restarts
    # from a sync snapshot (a multiple of the sync interval), stays healthy, ledger closes
    fast = PreparedTerrain(b).apply_edit(fast_edit())
    sf = run(b, fast, params(cfl_hard=0.36), prec, locked=dts, record=True)
    assert sf["abort"] == orc.ABORT_NONE
    assert sf["dt_fallback_t"] >= 0.0
    tol = 1e-4 if prec == 32 else 1e-10
    assert sf["rel_residual"] < tol, sf["rel_residual"]
    t_snap = max(t for t in (40.0 * k for k in range(21)) if t <= sf["dt_fallback_t"])
    n_locked = int(np.searchsorted(np.cumsum(sf["dts"]), t_snap - 1e-9 * 40.0, side="left")) + 1 if t_snap > 0 else 0
    # before the snapshot the run stepped with the baseline's dts
    np.testing.assert_array_equal(sf["dts"][:n_locked], dts[:n_locked])
    # the ledger rows end at the run's end: one per sync
    assert len(sf["ledger"]) == sf["sync_count"] == 20

    # an edit that stays within cfl_hard keeps the schedule to the end
    sm = PreparedTerrain(b).apply_edit(small_edit())
    ss = run(b, sm, params(), prec, locked=dts, record=True)
    assert ss["dt_fallback_t"] == -1.0 and ss["steps"] == s0["steps"]
    np.testing.assert_array_equal(ss["dts"], dts)


def test_oracle_locked_schedule_too_short():
    """A schedule shorter than the run falls back when it runs out (solver.rs:454-456: no
    entry for the step)."""
    b = base()
    zero = PreparedTerrain(b)
    s0 = run(b, zero, params(), 32, record=True)
    dts = s0["dts"]
    s1 = run(b, zero, params(), 32, locked=dts[: len(dts) // 2])
    assert s1["dt_fallback_t"] >= 0.0
    # the adaptive continuation of a zero edit from a snapshot of the baseline is the baseline
    assert s1["steps"] == s0["steps"]
    np.testing.assert_array_equal(s1["h"], s0["h"])


# ---------------------------------------------------------------------------- GPU ----------

@pytest.fixture(scope="module")
def gpu():
    g = GpuSolver()
    yield g
    g.close()


def same(g, o, what):
    assert g.steps == o["steps"] and g.t_end == o["t_end"], f"{what}: steps {g.steps} vs {o['steps']}"
    assert g.dt_fallback_t == o["dt_fallback_t"], f"{what}: fallback {g.dt_fallback_t} vs {o['dt_fallback_t']}"
    assert_bitwise(g.depth.ravel(), o["h"].ravel(), f"{what}: depth")
    assert_bitwise(g.peak.ravel(), o["peak"].ravel(), f"{what}: peak")
    np.testing.assert_array_equal(g.monitor_max, o["monitor_max"], err_msg=what)
    assert len(g.ledger) == len(o["ledger"]), what
    # f64 ledger (t, V, rain, in, out, infil, fix, residual): the device sums the same f32
    # fluxes and depths in another order, so its totals agree to rounding, not bit for bit
    np.testing.assert_array_equal(g.ledger[:, 0], o["ledger"][:, 0], err_msg=f"{what}: ledger t")
    np.testing.assert_allclose(g.ledger[:, 3:5], o["ledger"][:, 3:5], rtol=1e-9, err_msg=f"{what}: ledger in/out")
    np.testing.assert_allclose(g.ledger[:, [1, 2, 5, 6]], o["ledger"][:, [1, 2, 5, 6]], rtol=1e-6, atol=1e-9,
                               err_msg=f"{what}: ledger V, rain, infil, fix")


@pytest.mark.gpu
def test_gpu_locked_matches_oracle(gpu):
    b = base()
    zero = PreparedTerrain(b)
    dts = run(b, zero, params(), 32, record=True)["dts"]
    terrs = [zero, PreparedTerrain(b).apply_edit(small_edit()), PreparedTerrain(b).apply_edit(fast_edit())]
    for cfl_hard in (0.5, 0.36):
        p = params(cfl_hard)
        p.locked_dt = dts
        runs = gpu.run_batch(p, terrs, monitors(), want_peak=True, want_depth=True, ledger_rows=64)
        for i, t in enumerate(terrs):
            o = run(b, t, params(cfl_hard), 32, locked=dts)
            same(runs[i], o, f"cfl_hard {cfl_hard} design {i}")
        if cfl_hard == 0.36:
            assert runs[2].dt_fallback_t >= 0.0   # the fast edit fell back
    # the zero edit under its own schedule is the adaptive device run, ledger included
    free = gpu.run_batch(params(), [zero], monitors(), want_peak=True, want_depth=True, ledger_rows=64)[0]
    p = params()
    p.locked_dt = dts
    lk = gpu.run_batch(p, [zero], monitors(), want_peak=True, want_depth=True, ledger_rows=64)[0]
    assert lk.steps == free.steps and lk.t_end == free.t_end and lk.dt_fallback_t == -1.0
    assert_bitwise(lk.depth, free.depth, "locked zero edit vs adaptive: depth")
    assert_bitwise(lk.peak, free.peak, "locked zero edit vs adaptive: peak")
    np.testing.assert_array_equal(lk.ledger, free.ledger)
    # twice in a row on the same context: the snapshot buffers are reused
    p = params(0.36)
    p.locked_dt = dts
    again = gpu.run_batch(p, terrs, monitors(), want_peak=True, want_depth=True, ledger_rows=64)
    o = run(b, terrs[2], params(0.36), 32, locked=dts)
    same(again[2], o, "second call, fast edit")


@pytest.mark.gpu
def test_gpu_locked_tiled_path(gpu):
    """The tiled path (state in HBM; the path of grids too large for a cluster) under the same
    schedules: the same bits as the oracle, fallback included, twice on one context."""
    b = base()
    zero = PreparedTerrain(b)
    dts = run(b, zero, params(), 32, record=True)["dts"]
    terrs = [zero, PreparedTerrain(b).apply_edit(small_edit()), PreparedTerrain(b).apply_edit(fast_edit())]
    gpu.set_option("impl", 2)
    try:
        for cfl_hard in (0.5, 0.36, 0.36):
            p = params(cfl_hard)
            p.locked_dt = dts
            runs = gpu.run_batch(p, terrs, monitors(), want_peak=True, want_depth=True, ledger_rows=64)
            for i, t in enumerate(terrs):
                o = run(b, t, params(cfl_hard), 32, locked=dts)
                same(runs[i], o, f"tiled, cfl_hard {cfl_hard} design {i}")
            if cfl_hard == 0.36:
                assert runs[2].dt_fallback_t >= 0.0
        # a schedule cut short falls back when it runs out
        p = params()
        p.locked_dt = dts[: len(dts) // 3]
        r = gpu.run_batch(p, [zero], monitors(), want_peak=True, want_depth=True, ledger_rows=64)[0]
        same(r, run(b, zero, params(), 32, locked=dts[: len(dts) // 3]), "tiled, short schedule")
        assert r.dt_fallback_t >= 0.0
    finally:
        gpu.set_option("impl", 0)


@pytest.mark.gpu
def test_gpu_locked_unsupported_paths(gpu):
    """Paths without a locked schedule say so (ITR_UNSUPPORTED, the reference's Err from
    run_batch, evaluator.rs:231-238) instead of running adaptively: the plain one-design path."""
    b = base()
    zero = PreparedTerrain(b)
    p = params()
    p.locked_dt = np.full(10, 0.1)
    gpu.set_option("impl", 1)
    try:
        with pytest.raises(UnsupportedError):
            gpu.run_batch(p, [zero], monitors())
    finally:
        gpu.set_option("impl", 0)
