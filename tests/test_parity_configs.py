"""Device vs oracle at the benchmark configurations themselves, not at smaller stand-ins.

* configuration 2 as the bench runs it: rolling hills 120 x 96 at 5 m, 64 designs of 4
  primitives, the whole 60 min storm, autotuned launch shape: every design bit for bit
  against the f32 oracle (steps, end time, final depth, per-cell peak, monitor maxima, J),
  and a sample against the f64 oracle (<= 1e-4 m peak depth, <= 1e-5 relative J);
* configuration 1 as specified: valley 90 x 70 at 5 m, 16 designs of 2 primitives, 40 min
  storm: bit for bit against the f32 oracle, and all 16 against the f64 oracle;
* configuration 5's tiled path: fractal 1024 x 1024 at 2 m, 2 designs of 6 primitives, the
  first 600 s of the storm, bit for bit against the f32 oracle;
* configuration 3's ladder: valley at 10, 5 and 2.5 m (45 x 35, 90 x 70, 180 x 140), 128 / 96 /
  32 designs of 3 primitives, guard and incumbent aborts live, all groups in one graph launch
  with autotuned shapes: every design's status, breach, exceedance, lower bound, steps, end
  time, depth and monitor maxima equal the oracle's, which runs each design alone.

The oracle legs run on every host thread (ctypes releases the GIL during a run). Mirrors
crates/itr-gpu/tests/gpu.rs:56-110 (CPU comparison, batch == single) and
crates/itr-opt/tests/search.rs:227-256 (f32 against f64 on seeded random designs).
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle_ref as orc
from helpers import assert_bitwise, base_arrays, design_dict
from itr_gpu import GpuSolver, PreparedTerrain
from itr_gpu.scenes import config, valley_scene

pytestmark = pytest.mark.gpu

PEAK_TOL_M = 1e-4   # per-cell peak depth against the f64 oracle
J_REL_TOL = 1e-5    # relative J against the f64 oracle


def pmap(fn, items):
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        return list(ex.map(fn, items))


@pytest.fixture(scope="module")
def gpu():
    g = GpuSolver()
    yield g
    g.close()


def check_bitwise(r, o, what, peak=True):
    assert r.steps == o["steps"], f"{what}: steps {r.steps} vs {o['steps']}"
    assert r.t_end == o["t_end"], f"{what}: t_end {r.t_end} vs {o['t_end']}"
    if r.depth is not None:
        assert_bitwise(r.depth, o["h"], f"{what}: final depth")
    if peak:
        assert_bitwise(r.peak, o["peak"], f"{what}: per-cell peak")
    np.testing.assert_array_equal(r.monitor_max, o["monitor_max"], err_msg=f"{what}: monitor maxima")


def check_f64(sc, t, r32, what):
    o64 = orc.flat_run64(base_arrays(sc.base), design_dict(t, sc.params), sc.params, sc.monitors, want_peak=True)
    dpk = float(np.max(np.abs(r32.peak.astype(np.float64) - o64["peak"])))
    j32 = sc.objective.evaluate(r32.monitor_max, t.cut_m3, t.fill_m3)["j"]
    j64 = sc.objective.evaluate(o64["monitor_max"], t.cut_m3, t.fill_m3)["j"]
    dj = abs(j32 - j64) / max(abs(j64), 1e-300)
    assert dpk <= PEAK_TOL_M, f"{what}: peak depth {dpk:.3g} m from the f64 oracle"
    assert dj <= J_REL_TOL, f"{what}: J {j32!r} vs f64 {j64!r} (rel {dj:.3g})"
    return dpk, dj, abs(r32.steps - o64["steps"])


def test_config2_as_benched_bitwise_and_f64(gpu):
    sc = config(2)
    terrs = [t for _, _, t in sc.designs(64, seed=sc.design_seed)]   # the bench's rank-0 population
    runs = gpu.run_batch(sc.params, terrs, sc.monitors, objective=sc.objective, want_peak=True)
    orcs = pmap(lambda t: orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, sc.monitors,
                                       want_peak=True), terrs)
    for i, (r, o, t) in enumerate(zip(runs, orcs, terrs)):
        check_bitwise(r, o, f"config 2 design {i}")
        assert r.j == sc.objective.evaluate(o["monitor_max"], t.cut_m3, t.fill_m3)["j"], f"config 2 design {i}: J"
    assert sum(r.steps for r in runs) > 64 * 10000   # the whole storm ran
    sample = [0, 21, 42, 63]
    res = pmap(lambda i: check_f64(sc, terrs[i], runs[i], f"config 2 design {i}"), sample)
    print(f"\nconfig 2 vs f64 oracle on designs {sample}: max peak err {max(x[0] for x in res):.3g} m, "
          f"max rel J err {max(x[1] for x in res):.3g}, max step-count diff {max(x[2] for x in res)}")


def test_config1_as_specified_bitwise_and_f64(gpu):
    sc = config(1)
    terrs = [t for _, _, t in sc.designs(16)]
    runs = gpu.run_batch(sc.params, terrs, sc.monitors, objective=sc.objective, want_peak=True)
    orcs = pmap(lambda t: orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, sc.monitors,
                                       want_peak=True), terrs)
    for i, (r, o, t) in enumerate(zip(runs, orcs, terrs)):
        check_bitwise(r, o, f"config 1 design {i}")
        assert r.j == sc.objective.evaluate(o["monitor_max"], t.cut_m3, t.fill_m3)["j"], f"config 1 design {i}: J"
    res = pmap(lambda i: check_f64(sc, terrs[i], runs[i], f"config 1 design {i}"), range(16))
    print(f"\nconfig 1 vs f64 oracle, 16 designs: max peak err {max(x[0] for x in res):.3g} m, "
          f"max rel J err {max(x[1] for x in res):.3g}")


def test_config5_tiled_path_bitwise(gpu):
    sc = config(5)
    sc.params.duration_s = 600.0
    terrs = [t for _, _, t in sc.designs(2)]
    runs = gpu.run_batch(sc.params, terrs, sc.monitors, objective=sc.objective, want_peak=True)
    orcs = pmap(lambda t: orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, sc.monitors,
                                       want_peak=True), terrs)
    for i, (r, o) in enumerate(zip(runs, orcs)):
        check_bitwise(r, o, f"config 5 design {i}")
    assert all(r.steps > 300 for r in runs)


def test_config3_ladder_groups_vs_oracle(gpu):
    spec, scenes, p = [], [], None
    for cell, n in ((10.0, 128), (5.0, 96), (2.5, 32)):
        sc = valley_scene(cell, n_prims=3)
        sc.params.duration_s = 2400.0
        p = sc.params
        ts = [t for _, _, t in sc.designs(n)]
        prev = [t for _, _, t in sc.designs(n, seed=sc.design_seed + 500)]
        base = gpu.run_batch(p, [PreparedTerrain(sc.base)], sc.monitors)[0]
        ob = orc.flat_run(base_arrays(sc.base), design_dict(PreparedTerrain(sc.base), p), p, sc.monitors)
        np.testing.assert_array_equal(base.monitor_max, ob["monitor_max"])
        inc = min(r.j for r in gpu.run_batch(p, prev, sc.monitors, objective=sc.objective, want_depth=False))
        spec.append(dict(terrains=ts, monitors=sc.monitors, objective=sc.objective, baseline_max=base.monitor_max,
                         guard_abort=True, incumbent=inc))
        scenes.append(sc)
    out = gpu.run_ladder(p, spec, want_peak=False, want_depth=True)
    counts = {}
    for sc, g, runs in zip(scenes, spec, out):
        def one(t, sc=sc, g=g):
            return orc.flat_run(base_arrays(sc.base), design_dict(t, p), p, g["monitors"], objective=g["objective"],
                                baseline=g["baseline_max"], incumbent=g["incumbent"])
        orcs = pmap(one, g["terrains"])
        for i, (r, o) in enumerate(zip(runs, orcs)):
            what = f"ladder {sc.base.nx}x{sc.base.ny} design {i}"
            assert r.status == o["abort"], f"{what}: status {r.status} vs {o['abort']}"
            check_bitwise(r, o, what, peak=False)
            if o["abort"] == orc.ABORT_GUARD:
                assert (r.breach_cell, r.breach_sync, r.violation) == (o["abort_cell"], o["abort_sync"], o["abort_exceed"]), what
            if o["abort"] == orc.ABORT_INCUMBENT:
                assert r.lower_bound == o["abort_lb"], what
            counts[r.status] = counts.get(r.status, 0) + 1
    print(f"\nladder statuses (0 ok, 1 guard, 2 incumbent): {counts}")
