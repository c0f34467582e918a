"""Designs as primitives materialised on the device (itr_gpu_run_primitives): the device
restates DesignSpace::materialize (crates/itr-core/src/design.rs:316-385) and
PreparedTerrain::apply_edit at level 1 (crates/itr-hydro/src/terrain.rs:460-505), the steps
the reference runs on the host before uploading per-design jump arrays (crates/itr-gpu/src/
lib.rs:177-194). Everything must equal the host path bit for bit: the run (steps, depth,
peaks, monitor maxima, J) and the earthwork volumes.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import assert_bitwise
from itr_gpu import GpuSolver, PreparedTerrain, UnsupportedError
from itr_gpu.design import CUT, MOUND, Primitive, materialize
from itr_gpu.scenes import hills_scene, inflow_valley_scene, valley_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = GpuSolver()
    yield g
    g.close()


def host_path(sc, prim_sets):
    b = sc.base
    ts, vols = [], []
    for prims in prim_sets:
        e = materialize(prims, sc.geo, b.fine.nx, b.fine.ny, sc.editable, sc.max_abs_dz)
        ts.append(PreparedTerrain(b).apply_edit(e))
        vols.append((e.cut_m3, e.fill_m3))
    return ts, vols


def check(gpu, sc, prim_sets, impl=0, what=""):
    ts, vols = host_path(sc, prim_sets)
    gpu.set_option("impl", impl)
    try:
        ref = gpu.run_batch(sc.params, ts, sc.monitors, objective=sc.objective, want_peak=True)
        got, cut, fill = gpu.run_primitives(sc.params, sc.base, prim_sets, sc.monitors, sc.editable, sc.max_abs_dz,
                                            objective=sc.objective, want_peak=True)
    finally:
        gpu.set_option("impl", 0)
    for i, (r, g) in enumerate(zip(ref, got)):
        w = f"{what} design {i}"
        assert g.steps == r.steps and g.t_end == r.t_end, w
        assert_bitwise(g.depth, r.depth, f"{w}: final depth")
        assert_bitwise(g.peak, r.peak, f"{w}: per-cell peak")
        np.testing.assert_array_equal(g.monitor_max, r.monitor_max, err_msg=w)
        assert g.j == r.j, f"{w}: J {g.j} vs {r.j}"
        assert cut[i] == vols[i][0] and fill[i] == vols[i][1], f"{w}: volumes {cut[i]}, {fill[i]} vs {vols[i]}"


@pytest.mark.parametrize("impl", [0, 2])
def test_valley_designs_match_host_materialize(gpu, impl):
    sc = valley_scene(10.0)
    sc.params.duration_s = 900.0
    prim_sets = [p for p, _, _ in sc.designs(6)]
    # every kind, a primitive straddling the domain edge, an empty design, a zero height
    prim_sets.append([Primitive(CUT, 150.0, 170.0, 60.0, 12.0, 30.0, -0.4), Primitive(MOUND, 5.0, 175.0, 0.0, 30.0, 0.0, 0.6)])
    prim_sets.append([])
    prim_sets.append([Primitive(0, 200.0, 100.0, 50.0, 6.0, 45.0, 0.0)])
    check(gpu, sc, prim_sets, impl, f"valley impl {impl}")


def test_hills_designs_match_host_materialize(gpu):
    sc = hills_scene()
    sc.params.duration_s = 600.0
    check(gpu, sc, [p for p, _, _ in sc.designs(8)], 0, "hills")


def test_stage_edge_designs_match_host_materialize(gpu):
    """The stage ghosts' depths are rebuilt from each design's edited levels on the device."""
    sc = inflow_valley_scene(10.0)
    sc.params.duration_s = 600.0
    prim_sets = [p for p, _, _ in sc.designs(3)]
    prim_sets.append([Primitive(0, 440.0, 200.0, 80.0, 20.0, 90.0, 0.5)])   # a berm along the east stage edge
    check(gpu, sc, prim_sets, 0, "stage edge")


def test_coarse_level_rejected(gpu):
    from itr_gpu import TerrainBase
    sc = valley_scene(10.0)
    coarse = TerrainBase(sc.base.fine, 2, [])
    with pytest.raises(UnsupportedError):
        gpu.run_primitives(sc.params, coarse, [[]], sc.monitors, np.ones((coarse.ny, coarse.nx), bool), 1.0)
