"""GPU parity: the CUDA batched (and plain) forward against the f32 CPU oracle.

The oracle restates the reference's f32 fused kernel; with IEEE arithmetic and no FMA on
both sides the results are expected bit for bit: same step count and end time, same final
depth and same per-cell peak depth. The required tolerances (<= 1e-4 m peak depth,
<= 1e-5 relative J) are asserted too, so a failure says which bar broke.
Mirrors crates/itr-gpu/tests/gpu.rs (lake at rest, rain volume, CPU comparison, batch vs
single). gpu.rs:112-125's stage, inflow and inflow_scale cases, which the reference's GPU
backend rejects, run here: tests/test_boundaries.py.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle_ref as orc
from helpers import assert_bitwise, base_arrays, design_dict
from itr_gpu import GpuSolver, Hyetograph, MonitorSet, PreparedTerrain, Segment, SolverParams, synthetic_terrain
from itr_gpu.scenes import valley_scene

pytestmark = pytest.mark.gpu

PEAK_TOL_M = 1e-4      # required: per-cell peak depth vs the reference's f32 kernel
J_REL_TOL = 1e-5       # required: relative J


@pytest.fixture(scope="module")
def gpu():
    g = GpuSolver()
    yield g
    g.close()


def small_valley(duration=600.0):
    sc = valley_scene(10.0)   # 45 x 35
    sc.params.duration_s = duration
    return sc


def compare_run(g_run, o_run, what):
    assert g_run.steps == o_run["steps"], f"{what}: steps {g_run.steps} vs {o_run['steps']}"
    assert g_run.t_end == o_run["t_end"], f"{what}: t_end {g_run.t_end} vs {o_run['t_end']}"
    assert_bitwise(g_run.depth.ravel(), o_run["h"].ravel(), f"{what}: final depth")
    if g_run.peak is not None and o_run["peak"] is not None:
        assert np.max(np.abs(g_run.peak.astype(np.float64) - o_run["peak"])) <= PEAK_TOL_M
        assert_bitwise(g_run.peak.ravel(), o_run["peak"].ravel(), f"{what}: per-cell peak")
    np.testing.assert_array_equal(g_run.monitor_max, o_run["monitor_max"], err_msg=f"{what}: monitor maxima")


IMPL = {"batched": 0, "plain": 1, "tiled": 2}


@pytest.mark.parametrize("impl", ["batched", "plain", "tiled"])
def test_valley_designs_bitwise_vs_oracle(gpu, impl):
    sc = small_valley()
    designs = sc.designs(3)
    terrs = [t for _, _, t in designs]
    gpu.set_option("impl", IMPL[impl])
    try:
        runs = gpu.run_batch(sc.params, terrs, sc.monitors, want_peak=True)
    finally:
        gpu.set_option("impl", 0)
    for i, t in enumerate(terrs):
        o = orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, sc.monitors, want_peak=True)
        compare_run(runs[i], o, f"{impl} design {i}")


@pytest.mark.parametrize("cluster,threads", [(1, 256), (1, 512), (2, 256), (4, 512), (8, 256)])
def test_cluster_shapes_bitwise(gpu, cluster, threads):
    sc = valley_scene(5.0)   # 90 x 70
    sc.params.duration_s = 300.0
    t = [t for _, _, t in sc.designs(2)]
    gpu.set_option("cluster", cluster)
    gpu.set_option("threads", threads)
    try:
        runs = gpu.run_batch(sc.params, t, sc.monitors, want_peak=True)
    finally:
        gpu.set_option("cluster", 0)
        gpu.set_option("threads", 0)
    for i in range(2):
        o = orc.flat_run(base_arrays(sc.base), design_dict(t[i], sc.params), sc.params, sc.monitors, want_peak=True)
        compare_run(runs[i], o, f"cluster={cluster} threads={threads} design {i}")


def test_fast_reciprocal_matches_ieee_path(gpu):
    """The batched kernel's branch-free reciprocal and its IEEE fallback (option
    exact_special forces the fallback on every call) give the same bits, and both the
    oracle's."""
    sc = valley_scene(5.0)   # 90 x 70
    sc.params.duration_s = 600.0
    t = [t for _, _, t in sc.designs(2)]
    runs = {}
    for exact in (0, 1):
        gpu.set_option("exact_special", exact)
        try:
            runs[exact] = gpu.run_batch(sc.params, t, sc.monitors, want_peak=True)
        finally:
            gpu.set_option("exact_special", 0)
    for i in range(2):
        o = orc.flat_run(base_arrays(sc.base), design_dict(t[i], sc.params), sc.params, sc.monitors, want_peak=True)
        compare_run(runs[0][i], o, f"fast reciprocal design {i}")
        compare_run(runs[1][i], o, f"IEEE reciprocal design {i}")


def test_large_grid_takes_tiled_path(gpu):
    """A design too large for 8 CTAs' shared memory (400 x 300 cells, 3.4 MB of state) runs
    on the tiled batched path, bit for bit with the oracle."""
    base = synthetic_terrain(400, 300, 2.0, lambda x, y: 3.0 - 0.004 * x + 0.3 * math.sin(y / 40.0), n=0.035,
                             segments=[Segment("transmissive", "east")])
    p = SolverParams(90.0, 30.0, rain=Hyetograph.from_mm_h([(0, 0), (30, 200), (90, 0)]))
    mon = MonitorSet(np.arange(0, 400 * 300, 997))
    t = [PreparedTerrain(base), PreparedTerrain(base)]
    runs = gpu.run_batch(p, t, mon, want_peak=True)
    o = orc.flat_run(base_arrays(base), design_dict(t[0]), p, mon, want_peak=True)
    for i in range(2):
        compare_run(runs[i], o, f"large grid design {i}")


def test_lake_at_rest(gpu):
    # gpu.rs:21-38
    base = synthetic_terrain(64, 48, 1.0, lambda x, y: 0.3 * math.sin(x / 7.0) * math.cos(y / 5.0) + (0.4 if x > 30.0 else 0.0),
                             n=0.03)
    p = SolverParams(60.0, 10.0, initial_stage=1.5)
    t = PreparedTerrain(base)
    r = gpu.run_batch(p, [t], MonitorSet())[0]
    assert not r.bad
    eta = r.depth.astype(np.float64) + base.z + base.fine.z_ref
    err = np.max(np.abs(eta - 1.5))
    assert err < 1e-4
    assert r.steps == 1446   # itr-gpu README: "64x48 variable bed, 1446 steps"


def test_rain_closed_plain_volume(gpu):
    # gpu.rs:40-53
    base = synthetic_terrain(40, 30, 2.0, lambda x, y: 10.0, n=0.04)
    p = SolverParams(600.0, 60.0, rain=Hyetograph.from_mm_h([(0, 0), (100, 50), (400, 10), (500, 0)]))
    r = gpu.run_batch(p, [PreparedTerrain(base)], MonitorSet(), ledger_rows=16)[0]
    expect = p.rain.integral(0.0, 600.0) * 4.0 * (40 * 30)
    assert abs(r.volume_m3 / expect - 1.0) < 1e-4
    assert abs(r.t_end - 600.0) < 1e-3
    assert r.rel_residual < 1e-6   # f64 ledger on the device


def test_cpu_comparison_tilted_rain_outflow(gpu):
    # gpu.rs:55-79; the reference's CPU f32 run takes 1718 steps (itr-gpu README, D3 row)
    nx, ny = 100, 8
    base = synthetic_terrain(nx, ny, 2.0, lambda x, y: 5.0 - 0.01 * x + 0.002 * y, n=0.03,
                             segments=[Segment("transmissive", "east")])
    p = SolverParams(900.0, 100.0, rain=Hyetograph.from_mm_h([(0, 120), (600, 60), (800, 0)]))
    cells = [r * nx + c for c, r in [(10, 2), (30, 4), (50, 1), (70, 6), (90, 3), (99, 5), (99, 0)]]
    mon = MonitorSet(np.array(cells))
    t = PreparedTerrain(base)
    gr = gpu.run_batch(p, [t], mon)[0]
    o = orc.flat_run(base_arrays(base), design_dict(t), p, mon)
    assert o["steps"] == 1718
    assert gr.steps == o["steps"]
    rel = np.abs(gr.monitor_max - o["monitor_max"]) / np.maximum(np.abs(o["monitor_max"]), 1e-6)
    assert rel.max() < 0.02
    np.testing.assert_array_equal(gr.monitor_max, o["monitor_max"])
    assert not gr.bad


def test_batch_matches_single_bitwise(gpu):
    # gpu.rs:81-110
    from itr_gpu.terrain import TerrainEdit
    nx, ny = 48, 40
    base = synthetic_terrain(nx, ny, 2.0, lambda x, y: 3.0 - 0.01 * y + 0.2 * math.sin(x / 9.0), n=0.035,
                             segments=[Segment("transmissive", "south")])
    p = SolverParams(300.0, 50.0, rain=Hyetograph.from_mm_h([(0, 90), (200, 90), (250, 0)]))

    def mk(c0, r0, w, h, amp):
        dz = np.array([amp * (1.0 + (i % 5) * 0.1) for i in range(w * h)])
        return PreparedTerrain(base).apply_edit(TerrainEdit(c0, r0, w, h, dz))
    ts = [PreparedTerrain(base), mk(10, 10, 8, 6, 0.3), mk(25, 18, 10, 4, -0.15)]
    mon = MonitorSet(np.array([35 * nx + 5, 20 * nx + 20, 39 * nx + 30]))
    batch = gpu.run_batch(p, ts, mon)
    for i, t in enumerate(ts):
        single = gpu.run_batch(p, [t], mon)[0]
        assert batch[i].steps == single.steps
        assert batch[i].t_end == single.t_end
        assert_bitwise(batch[i].depth, single.depth, f"cand {i} depth")
        np.testing.assert_array_equal(batch[i].monitor_max, single.monitor_max)
    assert not np.array_equal(batch[0].depth, batch[1].depth)


@pytest.mark.parametrize("impl", ["batched", "tiled"])
def test_crest_mode_level2_bitwise(gpu, impl):
    # coarse fidelity level (FaceMode::Crest, terrain.rs:12-18), which the reference GPU path rejects
    sc = valley_scene(5.0)
    from itr_gpu.terrain import TerrainBase
    base2 = TerrainBase(sc.base.fine, 2, [Segment("transmissive", "east")])
    p = sc.params
    p.duration_s = 600.0
    t = PreparedTerrain(base2)
    mon = MonitorSet(np.arange(0, base2.nx * base2.ny, 7))
    gpu.set_option("impl", IMPL[impl])
    try:
        r = gpu.run_batch(p, [t], mon, want_peak=True)[0]
    finally:
        gpu.set_option("impl", 0)
    o = orc.flat_run(base_arrays(base2), design_dict(t), p, mon, want_peak=True)
    compare_run(r, o, f"crest level 2 ({impl})")


@pytest.fixture(params=["batched", "tiled"])
def impl_gpu(gpu, request):
    gpu.set_option("impl", IMPL[request.param])
    yield gpu
    gpu.set_option("impl", 0)


def test_guard_and_incumbent_aborts_identical(impl_gpu):
    gpu = impl_gpu
    sc = small_valley(1200.0)
    designs = sc.designs(6)
    terrs = [t for _, _, t in designs]
    # baseline = the unedited terrain's maxima
    base_run = gpu.run_batch(sc.params, [PreparedTerrain(sc.base)], sc.monitors)[0]
    baseline = base_run.monitor_max
    obj = sc.objective
    obj.d.guard_tolerance_m = 0.0005
    runs = gpu.run_batch(sc.params, terrs, sc.monitors, objective=obj, baseline_max=baseline, guard_abort=True)
    for i, t in enumerate(terrs):
        o = orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, sc.monitors, objective=obj,
                         baseline=baseline)
        assert runs[i].status == o["abort"], f"design {i}: status {runs[i].status} vs oracle {o['abort']}"
        assert runs[i].steps == o["steps"]
        if o["abort"] == orc.ABORT_GUARD:
            assert runs[i].breach_cell == o["abort_cell"]
            assert runs[i].breach_sync == o["abort_sync"]
            assert runs[i].violation == o["abort_exceed"]
    # incumbent: the median full-run J of the batch
    full = gpu.run_batch(sc.params, terrs, sc.monitors, objective=obj)
    js = sorted(r.j for r in full)
    inc = js[len(js) // 2]
    runs = gpu.run_batch(sc.params, terrs, sc.monitors, objective=obj, incumbent=inc)
    n_abort = 0
    for i, t in enumerate(terrs):
        o = orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, sc.monitors, objective=obj,
                         incumbent=inc)
        assert runs[i].status == o["abort"]
        assert runs[i].steps == o["steps"]
        if o["abort"] == orc.ABORT_INCUMBENT:
            n_abort += 1
            assert runs[i].lower_bound == o["abort_lb"]
    assert n_abort >= 1


def test_objective_j_matches_oracle(gpu):
    sc = small_valley(900.0)
    terrs = [t for _, _, t in sc.designs(4)]
    runs = gpu.run_batch(sc.params, terrs, sc.monitors, objective=sc.objective)
    for r, t in zip(runs, terrs):
        o = orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, sc.monitors)
        rep = sc.objective.evaluate(o["monitor_max"], t.cut_m3, t.fill_m3)
        assert abs(r.j - rep["j"]) <= J_REL_TOL * abs(rep["j"])
        assert r.j == rep["j"]


def test_ledger_vs_f64_oracle(gpu):
    sc = small_valley(1200.0)
    t = PreparedTerrain(sc.base)
    r = gpu.run_batch(sc.params, [t], sc.monitors, ledger_rows=64)[0]
    assert r.ledger is not None and len(r.ledger) == r.sync_count
    assert r.rel_residual < 1e-6
    geo = sc.geo
    s = orc.Scene(sc.base.fine.z + sc.base.fine.z_ref, sc.base.fine.wall, 0.035, geo, 1, [Segment("transmissive", "east")])
    o64 = s.run(sc.params, sc.monitors, prec=1)
    # storage and outflow against the f64 oracle (f32 state vs f64 state: 1e-3 relative)
    np.testing.assert_allclose(r.ledger[-1, 1], o64["ledger"][-1, 1], rtol=1e-3)
    np.testing.assert_allclose(r.ledger[-1, 2], o64["ledger"][-1, 2], rtol=1e-9)


@pytest.mark.parametrize("impl", ["batched", "tiled"])
def test_outputs_do_not_change_the_trajectory(gpu, impl):
    """crates/itr-hydro/tests/equivalence.rs:177: asking for the per-cell peak, the final
    depth and the ledger rows changes nothing of the run (steps, end time, monitor maxima)."""
    sc = small_valley(900.0)
    terrs = [t for _, _, t in sc.designs(3)]
    gpu.set_option("impl", IMPL[impl])
    try:
        bare = gpu.run_batch(sc.params, terrs, sc.monitors, want_peak=False, want_depth=False, ledger_rows=0)
        full = gpu.run_batch(sc.params, terrs, sc.monitors, want_peak=True, want_depth=True, ledger_rows=64)
    finally:
        gpu.set_option("impl", 0)
    for a, b in zip(bare, full):
        assert a.steps == b.steps and a.t_end == b.t_end and a.status == b.status
        np.testing.assert_array_equal(a.monitor_max, b.monitor_max)
        assert len(b.ledger) == b.sync_count
