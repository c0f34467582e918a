"""The adjoint's row-band kernels against its 16x16-tile kernels, bit for bit.

itr_gpu_vjp replays each checkpoint segment and steps the adjoint back through it, each part on
row-band sweeps or on 16x16 tiles (option adj_band: bit 0 the replay, the forward's own k_band
in TAPE mode instead of k_adj_replay; bit 1 the backward step, k_adj_band instead of
k_adj_step).
Both replays are the forward step bit for bit, and k_adj_band evaluates k_adj_step's arithmetic
in the same order, so every gradient must be identical: walls and transmissive edges, stage
and inflow ghosts, crest faces, a dry start, and configuration 4's grid with several designs
(several segments and bands per design, designs that stop at different steps).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from itr_gpu import (Asset, GpuSolver, Hyetograph, Objective, ObjectiveDef, PreparedTerrain, Segment, SolverParams,
                     synthetic_terrain)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = GpuSolver()
    yield g
    g.close()


def _objective(gpu, p, terrains, cells):
    probe = Objective(ObjectiveDef([Asset(f"a{i}", [c], 10.0) for i, c in enumerate(cells)], []))
    r = gpu.run_batch(p, terrains[:1], probe.monitors)[0]
    return Objective(ObjectiveDef([Asset(f"a{i}", [c], float(r.monitor_max[probe.monitors.position(c)]) - 0.004, 1.0 + i)
                                   for i, c in enumerate(cells)], []))


def _z(x, y):
    return 2.0 - 0.01 * x + 0.2 * math.sin(y / 15.0) + 0.1 * math.cos(x / 20.0)


def case_smooth(gpu):
    base = synthetic_terrain(24, 16, 5.0, _z, n=0.03, segments=[Segment("transmissive", "east")])
    p = SolverParams(120.0, 30.0, rain=Hyetograph.from_mm_h([(0, 50), (60, 120), (120, 0)]), initial_depth=0.3)
    t = [PreparedTerrain(base)]
    return p, t, _objective(gpu, p, t, [5 * 24 + 8, 9 * 24 + 15, 12 * 24 + 20]), 7


def case_dry_start(gpu):
    base = synthetic_terrain(70, 45, 5.0, _z, n=0.03, segments=[Segment("transmissive", "east")])
    p = SolverParams(240.0, 30.0, rain=Hyetograph.from_mm_h([(0, 50), (60, 120), (240, 0)]))
    t = [PreparedTerrain(base)]
    return p, t, _objective(gpu, p, t, [5 * 70 + 8, 30 * 70 + 61, 40 * 70 + 33]), 32


def case_stage_inflow(gpu):
    segs = [Segment("inflow", "west", (20.0, 60.0), hydrograph=[(0.0, 0.2), (60.0, 0.6), (120.0, 0.3)]),
            Segment("inflow", "north", (30.0, 80.0), hydrograph=[(0.0, 0.1), (120.0, 0.4)]),
            Segment("stage", "east", stage_m=1.5), Segment("stage", "south", (10.0, 40.0), stage_m=1.9)]
    base = synthetic_terrain(40, 33, 5.0, _z, n=0.03, segments=segs)
    p = SolverParams(120.0, 30.0, rain=Hyetograph.from_mm_h([(0, 50), (60, 120), (120, 0)]), initial_depth=0.3)
    t = [PreparedTerrain(base)]
    return p, t, _objective(gpu, p, t, [5 * 40 + 8, 9 * 40 + 15, 12 * 40 + 20, 2 * 40 + 3]), 16


def case_crest(gpu):
    base = synthetic_terrain(48, 32, 2.5, lambda x, y: _z(x, y) + 0.05 * math.sin(x / 3.0) * math.cos(y / 4.0), n=0.03,
                             segments=[Segment("transmissive", "east")], level=2)
    assert base.mode == 1
    p = SolverParams(120.0, 30.0, rain=Hyetograph.from_mm_h([(0, 50), (60, 120), (120, 0)]), initial_depth=0.3)
    t = [PreparedTerrain(base)]
    nx = base.nx
    return p, t, _objective(gpu, p, t, [5 * nx + 8, 9 * nx + 15, 12 * nx + 20]), 16


def case_config4(gpu):
    from itr_gpu.scenes import hills_scene
    sc = hills_scene(2.5, seed=20261203 + 2, design_seed=7 + 4)
    sc.params.duration_s = 300.0
    t = [x for _, _, x in sc.designs(3)]
    return sc.params, t, sc.objective, 64


CASES = {"smooth": case_smooth, "dry_start": case_dry_start, "stage_inflow": case_stage_inflow, "crest": case_crest,
         "config4": case_config4}


@pytest.mark.parametrize("name", list(CASES))
def test_band_backward_equals_tile_backward(gpu, name):
    p, terrains, obj, K = CASES[name](gpu)
    runs = {}
    try:
        for band in (3, 1, 0):
            gpu.set_option("adj_band", band)
            runs[band] = gpu.vjp(p, terrains, obj.monitors, obj, checkpoint_interval=K)
    finally:
        gpu.set_option("adj_band", -1)
    nonzero = 0
    pairs = [(i, a, b) for band in (3, 1) for i, (a, b) in enumerate(zip(runs[band], runs[0]))]
    for i, a, b in pairs:
        assert a.steps == b.steps and a.j == b.j, (name, i)
        for f in ("dj_ddzx", "dj_ddzy", "dj_ddzx2", "dj_ddzy2"):
            ga, gb = getattr(a, f, None), getattr(b, f, None)
            if ga is None and gb is None:
                continue
            assert np.all(np.isfinite(ga)), (name, i, f)
            assert np.array_equal(np.asarray(ga).view(np.uint64), np.asarray(gb).view(np.uint64)), \
                (name, i, f, int(np.count_nonzero(ga != gb)), float(np.max(np.abs(ga - gb))))
            nonzero += int(np.count_nonzero(ga))
    assert nonzero > 0, name


@pytest.mark.parametrize("name", ["smooth", "stage_inflow", "config4"])
def test_trimmed_sweep_equals_full_sweep(gpu, name):
    """The backward sweep stops at each design's latest asset maximum (option adj_trim): past it
    the adjoint is zero, so the gradients equal the full sweep's bit for bit."""
    p, terrains, obj, K = CASES[name](gpu)
    runs = {}
    try:
        for trim in (1, 0):
            gpu.set_option("adj_trim", trim)
            runs[trim] = gpu.vjp(p, terrains, obj.monitors, obj, checkpoint_interval=K)
    finally:
        gpu.set_option("adj_trim", 1)
    for i, (a, b) in enumerate(zip(runs[1], runs[0])):
        for f in ("dj_ddzx", "dj_ddzy"):
            ga, gb = np.asarray(getattr(a, f)), np.asarray(getattr(b, f))
            assert np.array_equal(ga.view(np.uint64), gb.view(np.uint64)), (name, i, f, int(np.count_nonzero(ga != gb)))


def test_default_kernels_on_a_large_grid_equal_the_tiles(gpu):
    """From 2^18 cells on, the default (adj_band = -1) runs the backward step on row bands too:
    on a 512 x 512 grid (configuration 5's fractal terrain at 4 m, 0.3 m of water everywhere at
    the start so every asset has a peak to differentiate, two designs, the first 120 s) its
    gradients equal the all-tile sweep's bit for bit."""
    from itr_gpu.scenes import fractal_scene
    sc = fractal_scene(512, 4.0)
    sc.params.duration_s = 120.0
    sc.params.initial_depth = 0.3
    terrs = [t for _, _, t in sc.designs(2)]
    runs = {}
    try:
        for band in (-1, 0):
            gpu.set_option("adj_band", band)
            runs[band] = gpu.vjp(sc.params, terrs, sc.monitors, sc.objective, checkpoint_interval=64)
    finally:
        gpu.set_option("adj_band", -1)
    nonzero = 0
    for i, (a, b) in enumerate(zip(runs[-1], runs[0])):
        assert a.steps == b.steps and a.j == b.j, i
        for f in ("dj_ddzx", "dj_ddzy"):
            ga, gb = np.asarray(getattr(a, f)), np.asarray(getattr(b, f))
            assert np.all(np.isfinite(ga)), (i, f)
            assert np.array_equal(ga.view(np.uint64), gb.view(np.uint64)), (i, f, int(np.count_nonzero(ga != gb)))
            nonzero += int(np.count_nonzero(ga))
    assert nonzero > 0
