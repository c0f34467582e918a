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


def test_design_chain_on_device_matches_host_chain(gpu):
    """itr_gpu_vjp_primitives: the forward on the device-materialised designs, its adjoint,
    and dJ/d(height, width, length) contracted on the device equal the host chain
    (itr_gpu/adjoint.py primitive_gradient) on the same face-jump gradients, up to the order
    of the f64 sums."""
    import math
    from itr_gpu import Asset, Hyetograph, Objective, ObjectiveDef, Segment, SolverParams, synthetic_terrain
    from itr_gpu.adjoint import primitive_gradient
    from itr_gpu.design import BERM, SWALE
    nx, ny = 24, 16
    base = synthetic_terrain(nx, ny, 5.0, lambda x, y: 2.0 - 0.01 * x + 0.2 * math.sin(y / 15.0) + 0.1 * math.cos(x / 20.0),
                             n=0.03, segments=[Segment("transmissive", "east")])
    p = SolverParams(120.0, 30.0, rain=Hyetograph.from_mm_h([(0, 50), (60, 120), (120, 0)]), initial_depth=0.3)
    cells = [5 * nx + 8, 9 * nx + 15, 12 * nx + 20]
    probe = Objective(ObjectiveDef([Asset(f"a{i}", [c], 10.0) for i, c in enumerate(cells)], []))
    r0 = gpu.run_batch(p, [PreparedTerrain(base)], probe.monitors)[0]
    odef = ObjectiveDef([Asset(f"a{i}", [c], float(r0.monitor_max[probe.monitors.position(c)]) - 0.004, 1.0 + i)
                         for i, c in enumerate(cells)], [], earth_weight=1e-3)
    obj = Objective(odef)
    editable = np.ones((ny, nx), dtype=bool)
    designs = [[Primitive(BERM, 55.0, 45.0, 40.0, 10.0, 30.0, 0.20), Primitive(SWALE, 85.0, 30.0, 30.0, 8.0, 110.0, -0.15)],
               [Primitive(CUT, 60.0, 40.0, 30.0, 12.0, 0.0, -0.2)],
               [Primitive(MOUND, 70.0, 50.0, 0.0, 20.0, 0.0, 0.3), Primitive(BERM, 40.0, 20.0, 25.0, 6.0, 80.0, 0.1)]]
    runs, grads = gpu.vjp_primitives(p, base, designs, obj.monitors, obj, editable, 1.0, checkpoint_interval=16)
    for d, prims in enumerate(designs):
        host = primitive_gradient(base, base.fine.geo, editable, 1.0, prims, runs[d].dj_ddzx, runs[d].dj_ddzy, odef)
        scale = max(np.abs(host).max(), 1e-30)
        np.testing.assert_allclose(grads[d], host, rtol=1e-9, atol=1e-12 * scale, err_msg=f"design {d}")
        assert np.any(grads[d] != 0.0)
    # the forward part equals the device-materialised forward
    fw, _, _ = gpu.run_primitives(p, base, designs, obj.monitors, editable, 1.0, objective=obj)
    for a, b in zip(runs, fw):
        assert a.steps == b.steps and np.array_equal(a.monitor_max, b.monitor_max) and a.j == b.j
