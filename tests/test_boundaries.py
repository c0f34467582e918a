"""Stage and inflow ghost boundaries (Ghost::Stage / Ghost::Inflow, crates/itr-hydro/src/
boundary.rs:43-50,66-71) and inflow_scale (boundary.rs:27), which the reference's GPU
backend declined (crates/itr-gpu/src/lib.rs:166-176, crates/itr-cli/src/backend.rs:53-55).

CPU: the packed boundary tables the host mirror hands the C ABI (codes, stage levels,
hydrograph indices, 1 / segment length, z behind each boundary cell) reproduce, through
the flat oracle, the run of the scene oracle, whose boundaries the C++ restatement of
Boundaries::from_segments builds itself (terrain.rs:151-187): same steps, same bits.
GPU: every forward path against the flat oracle, bit for bit, with a design that edits the
cells behind a stage edge (its ghost depths differ from the base's).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle_ref as orc
from helpers import assert_bitwise, base_arrays, design_dict
from itr_gpu import GpuSolver, Hyetograph, MonitorSet, PreparedTerrain, Segment, SolverParams, UnsupportedError, synthetic_terrain
from itr_gpu.terrain import TerrainEdit
from itr_gpu.scenes import inflow_valley_scene


def edge_edit(base, rows, cols, dz):
    """A TerrainEdit raising a block of cells by dz (cut/fill volumes as materialize counts)."""
    r0, r1 = rows
    c0, c1 = cols
    h, w = r1 - r0, c1 - c0
    d = np.full(h * w, float(dz))
    area = base.fine.geo.dx * base.fine.geo.dy
    return TerrainEdit(c0, r0, w, h, d, max(-dz, 0.0) * h * w * area, max(dz, 0.0) * h * w * area)


def scene_case(duration=900.0, scale=1.0):
    sc = inflow_valley_scene(10.0)   # 45 x 35
    sc.params.duration_s = duration
    sc.params.inflow_scale = scale
    terrs = [t for _, _, t in sc.designs(2)]
    b = sc.base
    # a berm along the east (stage) edge and a cut at the west inflow mouth
    e = edge_edit(b, (5, 30), (b.nx - 2, b.nx), -0.15)
    terrs.append(PreparedTerrain(b).apply_edit(e))
    terrs.append(PreparedTerrain(b).apply_edit(edge_edit(b, (10, 25), (0, 3), 0.2)))
    return sc, terrs


def oracle_run(sc, t, want_peak=True):
    return orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, sc.monitors, want_peak=want_peak,
                        bnd=orc.bnd_dict(sc.base, t), max_rows=64)


def test_boundary_tables_match_scene_oracle():
    sc, terrs = scene_case(duration=600.0)
    b = sc.base
    fine = b.fine
    segs = [Segment("inflow", "west", (125.0, 225.0), hydrograph=[(0.0, 0.0), (600.0, 6.0), (1800.0, 2.0), (2400.0, 0.5)]),
            Segment("inflow", "south", (200.0, 260.0), hydrograph=[(0.0, 1.0), (1200.0, 3.0), (2400.0, 0.0)]),
            Segment("stage", "east", stage_m=10.2),
            Segment("stage", "north", (300.0, 450.0), stage_m=11.8),
            Segment("transmissive", "south", (350.0, 450.0))]
    s = orc.Scene(fine.z + fine.z_ref, fine.wall, 0.035, fine.geo, 1, segs)
    np.testing.assert_array_equal(s.pack()["bc"], b.bc)
    # the unedited terrain and the two edge edits
    for t, e in [(PreparedTerrain(b), None), (terrs[2], edge_edit(b, (5, 30), (b.nx - 2, b.nx), -0.15)),
                 (terrs[3], edge_edit(b, (10, 25), (0, 3), 0.2))]:
        a = s.run(sc.params, sc.monitors, prec=0, kernel=1, edit=e, max_rows=64)
        f = oracle_run(sc, t, want_peak=False)
        assert a["steps"] == f["steps"] and a["t_end"] == f["t_end"]
        assert_bitwise(f["h"], a["h"], "flat vs scene oracle: depth")
        np.testing.assert_array_equal(f["monitor_max"], a["monitor_max"])
        np.testing.assert_array_equal(f["ledger"], a["ledger"])
        assert f["ledger"][-1, 3] > 0.0   # the inflow column (ledger: t, V, rain, in, out, ...)
    # the edits reach the stage edge: a different ghost depth, a different run
    assert not np.array_equal(oracle_run(sc, terrs[2], want_peak=False)["h"], oracle_run(sc, PreparedTerrain(b), want_peak=False)["h"])


def test_inflow_scale_scales_the_inflow():
    """inflow_scale multiplies every hydrograph (boundary.rs:27): the same run with the
    hydrographs doubled in the scene, or with inflow_scale 2, is the same run."""
    sc1, _ = scene_case(600.0, 2.0)
    sc2 = inflow_valley_scene(10.0, scale=2.0)
    sc2.params.duration_s = 600.0
    a = oracle_run(sc1, PreparedTerrain(sc1.base), want_peak=False)
    b = oracle_run(sc2, PreparedTerrain(sc2.base), want_peak=False)
    assert a["steps"] == b["steps"]
    assert_bitwise(a["h"], b["h"], "inflow_scale 2 vs doubled hydrographs")
    c = oracle_run(*scene_case(600.0, 1.0)[:1], PreparedTerrain(sc1.base), want_peak=False)
    assert a["ledger"][-1, 3] > c["ledger"][-1, 3]   # inflow volume (the stage edges add their own)


@pytest.fixture(scope="module")
def gpu():
    g = GpuSolver()
    yield g
    g.close()


IMPL = {"batched": 0, "plain": 1, "tiled": 2}


def compare(g, o, what):
    assert g.steps == o["steps"], f"{what}: steps {g.steps} vs {o['steps']}"
    assert g.t_end == o["t_end"], what
    assert_bitwise(g.depth, o["h"], f"{what}: final depth")
    assert_bitwise(g.peak, o["peak"], f"{what}: per-cell peak")
    np.testing.assert_array_equal(g.monitor_max, o["monitor_max"], err_msg=f"{what}: monitor maxima")
    assert len(g.ledger) == len(o["ledger"]), what
    # f64 ledger (t, V, rain, in, out, infil, fix, residual). The boundary volumes are f64
    # sums of the same f32 face fluxes in another order; volume, infiltration and fix are
    # summed from f32 partials in another order (relative 1e-6)
    np.testing.assert_allclose(g.ledger[:, 3:5], o["ledger"][:, 3:5], rtol=1e-9, err_msg=f"{what}: ledger in/out")
    np.testing.assert_allclose(g.ledger[:, [1, 2, 5, 6]], o["ledger"][:, [1, 2, 5, 6]], rtol=1e-6, atol=1e-9,
                               err_msg=f"{what}: ledger V, rain, infil, fix")


@pytest.mark.gpu
@pytest.mark.parametrize("impl", ["batched", "plain", "tiled"])
@pytest.mark.parametrize("scale", [1.0, 1.7])
def test_stage_inflow_bitwise_vs_oracle(gpu, impl, scale):
    sc, terrs = scene_case(scale=scale)
    gpu.set_option("impl", IMPL[impl])
    try:
        runs = gpu.run_batch(sc.params, terrs, sc.monitors, want_peak=True, ledger_rows=64)
    finally:
        gpu.set_option("impl", 0)
    for i, t in enumerate(terrs):
        compare(runs[i], oracle_run(sc, t), f"{impl} scale {scale} design {i}")
    assert runs[0].ledger[-1, 3] > 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("cluster,threads", [(1, 256), (2, 512), (8, 256)])
def test_stage_inflow_cluster_shapes(gpu, cluster, threads):
    sc, terrs = scene_case(duration=600.0)
    gpu.set_option("cluster", cluster)
    gpu.set_option("threads", threads)
    try:
        runs = gpu.run_batch(sc.params, terrs[2:], sc.monitors, want_peak=True, ledger_rows=64)
    finally:
        gpu.set_option("cluster", 0)
        gpu.set_option("threads", 0)
    for i, t in enumerate(terrs[2:]):
        compare(runs[i], oracle_run(sc, t), f"C={cluster} T={threads} design {i}")


@pytest.mark.gpu
@pytest.mark.parametrize("impl", ["batched", "tiled"])
def test_inflow_east_north_crest_level2(gpu, impl):
    """Inward-negative inflow (east) and a y-normal inflow from the north on a coarse
    fidelity level (crest faces), stage on the west and south."""
    z = lambda x, y: 3.0 + 0.004 * x - 0.003 * y + 0.2 * np.sin(x / 17.0) * np.cos(y / 23.0)
    segs = [Segment("inflow", "east", (20.0, 60.0), hydrograph=[(0.0, 0.5), (300.0, 2.0), (600.0, 0.2)]),
            Segment("inflow", "north", (10.0, 50.0), hydrograph=[(0.0, 0.0), (400.0, 1.5)]),
            Segment("stage", "west", stage_m=3.05), Segment("stage", "south", (0.0, 40.0), stage_m=3.3)]
    base = synthetic_terrain(40, 32, 2.5, z, n=0.03, segments=segs, level=2)
    p = SolverParams(600.0, 60.0, rain=Hyetograph.from_mm_h([(0, 10), (600, 0)]))
    t = PreparedTerrain(base)
    mon = MonitorSet(np.arange(0, base.nx * base.ny, 7, dtype=np.uint32))
    gpu.set_option("impl", IMPL[impl])
    try:
        r = gpu.run_batch(p, [t], mon, want_peak=True, ledger_rows=16)[0]
    finally:
        gpu.set_option("impl", 0)
    o = orc.flat_run(base_arrays(base), design_dict(t, p), p, mon, want_peak=True, bnd=orc.bnd_dict(base, t), max_rows=16)
    assert base.mode == 1
    compare(r, o, f"{impl} crest")


@pytest.mark.gpu
def test_stage_inflow_ladder(gpu):
    """Two fidelity groups with stage and inflow cells in one graph launch."""
    groups, cases = [], []
    for cell in (10.0, 5.0):
        sc = inflow_valley_scene(cell)
        sc.params.duration_s = 600.0
        ts = [t for _, _, t in sc.designs(2)]
        groups.append(dict(terrains=ts, monitors=sc.monitors))
        cases.append((sc, ts))
    out = gpu.run_ladder(cases[0][0].params, groups, want_peak=True, want_depth=True)
    for (sc, ts), runs in zip(cases, out):
        for i, t in enumerate(ts):
            o = oracle_run(sc, t)
            assert runs[i].steps == o["steps"]
            assert_bitwise(runs[i].depth, o["h"], f"ladder {sc.base.nx}x{sc.base.ny} design {i}")
            np.testing.assert_array_equal(runs[i].monitor_max, o["monitor_max"])


@pytest.mark.gpu
def test_too_many_inflow_groups_rejected(gpu):
    """More inflow groups than the device table holds is declined ("unsupported here",
    evaluator.rs:232-238), so the evaluator's CPU fallback takes the level."""
    segs = [Segment("inflow", "north", (4.0 * k, 4.0 * k + 4.0), hydrograph=[(0.0, 0.1 * (k + 1))]) for k in range(9)]
    base = synthetic_terrain(40, 16, 1.0, lambda x, y: 0.0, n=0.03, segments=segs)
    with pytest.raises(UnsupportedError):
        gpu.run_batch(SolverParams(10.0, 5.0), [PreparedTerrain(base)], MonitorSet())
