"""Adjoint (itr_gpu_vjp): dJ/d(face jump) against central finite differences of the f64 oracle.

Required: <= 1% relative error against finite differences on a fully wet, smooth case
(initial depth 0.3 m, no dry cells). The adjoint is the derivative of the discrete f32 step
with the recorded dt sequence held fixed; the finite differences rerun the f64 oracle with
its own adaptive dt, so agreement also bounds the effect of freezing dt.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle_ref as orc
from helpers import base_arrays, design_dict
from itr_gpu import (Asset, GpuSolver, Hyetograph, Objective, ObjectiveDef, PreparedTerrain, Segment, SolverParams,
                     synthetic_terrain)

pytestmark = pytest.mark.gpu

FD_REL_TOL = 0.01      # required: adjoint vs finite differences
FD_STEP_M = 1e-3       # central difference step on one face jump


@pytest.fixture(scope="module")
def gpu():
    g = GpuSolver()
    yield g
    g.close()


def smooth_case(gpu, initial_depth=0.3, duration=120.0):
    nx, ny = 24, 16
    base = synthetic_terrain(nx, ny, 5.0, lambda x, y: 2.0 - 0.01 * x + 0.2 * math.sin(y / 15.0) + 0.1 * math.cos(x / 20.0),
                             n=0.03, segments=[Segment("transmissive", "east")])
    p = SolverParams(duration, 30.0, rain=Hyetograph.from_mm_h([(0, 50), (60, 120), (120, 0)]), initial_depth=initial_depth)
    t = PreparedTerrain(base)
    cells = [5 * nx + 8, 9 * nx + 15, 12 * nx + 20]
    # thresholds just under each cell's peak, so every asset term has a slope of order one
    probe = Objective(ObjectiveDef([Asset(f"a{i}", [c], 10.0) for i, c in enumerate(cells)], []))
    r = gpu.run_batch(p, [t], probe.monitors)[0]
    assets = [Asset(f"a{i}", [c], float(r.monitor_max[probe.monitors.position(c)]) - 0.004, 1.0 + i) for i, c in enumerate(cells)]
    obj = Objective(ObjectiveDef(assets, []))
    return base, p, t, obj


def j_f64(base, p, t, obj, dzx=None, dzy=None):
    d = design_dict(t, p)
    if dzx is not None:
        d["dzx"] = dzx
    if dzy is not None:
        d["dzy"] = dzy
    o = orc.flat_run64(base_arrays(base), d, p, obj.monitors)
    return obj.evaluate(o["monitor_max"], 0.0, 0.0)["j_risk"]


def test_gradient_independent_of_checkpoint_interval(gpu):
    """Segments are recomputed bit for bit from their checkpoints, so the gradient cannot
    depend on the interval."""
    base, p, t, obj = smooth_case(gpu)
    a = gpu.vjp(p, [t], obj.monitors, obj, checkpoint_interval=7)[0]
    b = gpu.vjp(p, [t], obj.monitors, obj, checkpoint_interval=4096)[0]
    assert np.array_equal(a.dj_ddzx, b.dj_ddzx) and np.array_equal(a.dj_ddzy, b.dj_ddzy)
    assert np.any(a.dj_ddzx != 0.0) and np.all(np.isfinite(a.dj_ddzx)) and np.all(np.isfinite(a.dj_ddzy))
    # the forward part is the ordinary forward
    r = gpu.run_batch(p, [t], obj.monitors, objective=obj)[0]
    assert a.steps == r.steps and np.array_equal(a.monitor_max, r.monitor_max) and a.j == r.j


def test_gradient_vs_f64_finite_differences_smooth(gpu):
    base, p, t, obj = smooth_case(gpu)
    run = gpu.vjp(p, [t], obj.monitors, obj, checkpoint_interval=16)[0]
    gx, gy = run.dj_ddzx, run.dj_ddzy
    nx, ny = base.nx, base.ny
    dzx0 = np.asarray(t.dzx, np.float64).reshape(ny, nx + 1)
    dzy0 = np.asarray(t.dzy, np.float64).reshape(ny + 1, nx)
    # the faces with the largest sensitivity (interior faces only: edge jumps are fixed at 0)
    gxi = np.abs(gx.copy()); gxi[:, 0] = 0; gxi[:, nx] = 0
    gyi = np.abs(gy.copy()); gyi[0, :] = 0; gyi[ny, :] = 0
    picks = [("x", np.unravel_index(i, gx.shape)) for i in np.argsort(gxi, axis=None)[-3:]]
    picks += [("y", np.unravel_index(i, gy.shape)) for i in np.argsort(gyi, axis=None)[-3:]]
    worst = 0.0
    for kind, idx in picks:
        if kind == "x":
            up, dn = dzx0.copy(), dzx0.copy()
            up[idx] += FD_STEP_M; dn[idx] -= FD_STEP_M
            fd = (j_f64(base, p, t, obj, dzx=up) - j_f64(base, p, t, obj, dzx=dn)) / (2 * FD_STEP_M)
            ad = gx[idx]
        else:
            up, dn = dzy0.copy(), dzy0.copy()
            up[idx] += FD_STEP_M; dn[idx] -= FD_STEP_M
            fd = (j_f64(base, p, t, obj, dzy=up) - j_f64(base, p, t, obj, dzy=dn)) / (2 * FD_STEP_M)
            ad = gy[idx]
        rel = abs(ad - fd) / abs(fd)
        worst = max(worst, rel)
        assert rel <= FD_REL_TOL, f"{kind}-face {idx}: adjoint {ad:.6e} vs finite difference {fd:.6e} (rel {rel:.3%})"
    print(f"worst relative error vs f64 central differences: {worst:.3%}")


def _fd_check_faces(base, p, t, obj, gx, gy, n_per_dir=3, threads=None):
    """Central differences of the f64 oracle's J on the faces of largest |gradient| (interior
    faces; n_per_dir per direction), the runs spread over the host threads. Returns
    [(kind, index, adjoint, finite difference)]."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    nx, ny = base.nx, base.ny
    dzx0 = np.asarray(t.dzx, np.float64).reshape(ny, nx + 1)
    dzy0 = np.asarray(t.dzy, np.float64).reshape(ny + 1, nx)
    gxi = np.abs(gx.copy()); gxi[:, 0] = 0; gxi[:, nx] = 0
    gyi = np.abs(gy.copy()); gyi[0, :] = 0; gyi[ny, :] = 0
    picks = [("x", np.unravel_index(i, gx.shape)) for i in np.argsort(gxi, axis=None)[-n_per_dir:]]
    picks += [("y", np.unravel_index(i, gy.shape)) for i in np.argsort(gyi, axis=None)[-n_per_dir:]]
    jobs = []
    for kind, idx in picks:
        for sgn in (1.0, -1.0):
            a = (dzx0 if kind == "x" else dzy0).copy()
            a[idx] += sgn * FD_STEP_M
            jobs.append(dict(dzx=a) if kind == "x" else dict(dzy=a))
    with ThreadPoolExecutor(max_workers=threads or os.cpu_count() or 1) as ex:
        js = list(ex.map(lambda kw: j_f64(base, p, t, obj, **kw), jobs))
    out = []
    for k, (kind, idx) in enumerate(picks):
        fd = (js[2 * k] - js[2 * k + 1]) / (2 * FD_STEP_M)
        out.append((kind, idx, (gx if kind == "x" else gy)[idx], fd))
    return out


def config4_case(initial_depth, duration=300.0):
    """Configuration 4's scene (rolling hills 240 x 192 at 2.5 m, its assets and storm) for the
    first `duration` seconds of the storm, from `initial_depth` everywhere, one design."""
    from itr_gpu.scenes import hills_scene
    sc = hills_scene(2.5, seed=20261203 + 2, design_seed=7 + 4, initial_depth=initial_depth)
    sc.params.duration_s = duration
    return sc, sc.designs(1)[0][2]


def test_gradient_vs_f64_finite_differences_config4_smooth(gpu):
    """The required bar at the configured scale: configuration 4's grid (240 x 192), the fully
    wet smooth sub-case (initial depth 0.3 m, no dry cells), the first 300 s of its storm
    (3646 steps): dJ/d(face jump) on the six most sensitive faces within 1% of f64 central
    differences."""
    sc, t = config4_case(0.3)
    run = gpu.vjp(sc.params, [t], sc.monitors, sc.objective, checkpoint_interval=128)[0]
    assert run.status == 0 and run.steps > 3000
    res = _fd_check_faces(sc.base, sc.params, t, sc.objective, run.dj_ddzx, run.dj_ddzy)
    worst = 0.0
    for kind, idx, ad, fd in res:
        rel = abs(ad - fd) / abs(fd)
        worst = max(worst, rel)
        assert rel <= FD_REL_TOL, f"{kind}-face {idx}: adjoint {ad:.6e} vs finite difference {fd:.6e} (rel {rel:.3%})"
    print(f"\nconfig 4 smooth (240x192, 300 s, {run.steps} steps): worst relative error vs f64 central "
          f"differences on {len(res)} faces {worst:.3%}")


def test_gradient_config4_mixed_wet_dry_reported(gpu):
    """The mixed wet/dry case at configuration 4's scale (dry start, rain on dry hills, the
    first 1200 s of the storm), reported beside the smooth one: through wetting fronts the
    frozen-dt discrete adjoint and f64 finite differences of the adaptive-dt run may part, so
    only finiteness and the sign on the dominant faces are asserted."""
    sc, t = config4_case(0.0, 1200.0)
    run = gpu.vjp(sc.params, [t], sc.monitors, sc.objective, checkpoint_interval=128)[0]
    assert np.all(np.isfinite(run.dj_ddzx)) and np.all(np.isfinite(run.dj_ddzy))
    res = _fd_check_faces(sc.base, sc.params, t, sc.objective, run.dj_ddzx, run.dj_ddzy, n_per_dir=2)
    rels = [abs(ad - fd) / max(abs(fd), 1e-300) for _, _, ad, fd in res]
    print(f"\nconfig 4 mixed wet/dry (1200 s, {run.steps} steps): relative errors vs f64 central differences "
          + ", ".join(f"{r:.2%}" for r in rels))
    assert sum(np.sign(ad) == np.sign(fd) for _, _, ad, fd in res) >= len(res) - 1


def test_mixed_wet_dry_gradient_finite(gpu):
    """Dry start (rain on dry ground): the wet/dry branches still give a finite gradient."""
    base, p, t, obj = smooth_case(gpu, initial_depth=0.0, duration=240.0)
    run = gpu.vjp(p, [t], obj.monitors, obj, checkpoint_interval=32)[0]
    assert np.all(np.isfinite(run.dj_ddzx)) and np.all(np.isfinite(run.dj_ddzy))


def test_primitive_gradient_vs_f64_finite_differences(gpu):
    """dJ/d(height, width, length) of each primitive through the design chain (materialize,
    bed, face jumps) against central differences of the whole chain on the f64 oracle, on the
    smooth fully wet case (small steps: J is only piecewise smooth, and a wide stencil can
    straddle a kink of the upwinding or wet/dry branches)."""
    import dataclasses
    from itr_gpu.adjoint import PARAMS, face_jumps_f64, primitive_gradient
    from itr_gpu.design import BERM, SWALE, materialize, Primitive
    base, p, t0, obj = smooth_case(gpu)
    geo = base.fine.geo
    editable = np.ones((base.ny, base.nx), dtype=bool)
    prims = [Primitive(BERM, 55.0, 45.0, 40.0, 10.0, 30.0, 0.20), Primitive(SWALE, 85.0, 30.0, 30.0, 8.0, 110.0, -0.15)]

    def terrain(ps):
        return PreparedTerrain(base).apply_edit(materialize(ps, geo, base.nx, base.ny, editable, 1.0))

    t = terrain(prims)
    run = gpu.vjp(p, [t], obj.monitors, obj, checkpoint_interval=16)[0]
    grad = primitive_gradient(base, geo, editable, 1.0, prims, run.dj_ddzx, run.dj_ddzy)

    def j_of(ps):
        ee = materialize(ps, geo, base.nx, base.ny, editable, 1.0)
        full = np.zeros((base.ny, base.nx))
        full[ee.r0:ee.r0 + ee.h, ee.c0:ee.c0 + ee.w] = ee.dz.reshape(ee.h, ee.w)
        dzx, dzy = face_jumps_f64(base, full)
        return j_f64(base, p, t, obj, dzx=dzx, dzy=dzy)

    steps = {"height": 5e-4, "width": 2e-3, "length": 2e-3}
    worst = 0.0
    for i in range(len(prims)):
        for k, name in enumerate(PARAMS):
            h = steps[name]
            up = [dataclasses.replace(q, **{name: getattr(q, name) + h}) if j == i else q for j, q in enumerate(prims)]
            dn = [dataclasses.replace(q, **{name: getattr(q, name) - h}) if j == i else q for j, q in enumerate(prims)]
            fd = (j_of(up) - j_of(dn)) / (2 * h)
            rel = abs(grad[i, k] - fd) / abs(fd)
            worst = max(worst, rel)
            assert rel <= FD_REL_TOL, f"primitive {i} {name}: adjoint {grad[i, k]:.6e} vs finite difference {fd:.6e} ({rel:.3%})"
    print(f"worst relative error of dJ/d(height, width, length) vs f64 central differences: {worst:.3%}")


def test_gradient_with_stage_and_inflow_vs_f64_finite_differences(gpu):
    """Stage (east) and inflow (west, north) ghosts on the smooth fully wet case: the ghost
    adjoints fold onto the interior cells (a stage ghost's momentum, an inflow ghost's depth
    above the critical depth). The stage depths are held fixed, as the finite differences,
    which perturb face jumps only, hold them."""
    nx, ny = 24, 16
    segs = [Segment("inflow", "west", (20.0, 60.0), hydrograph=[(0.0, 0.2), (60.0, 0.6), (120.0, 0.3)]),
            Segment("inflow", "north", (30.0, 80.0), hydrograph=[(0.0, 0.1), (120.0, 0.4)]),
            Segment("stage", "east", stage_m=1.5)]
    base = synthetic_terrain(nx, ny, 5.0, lambda x, y: 2.0 - 0.01 * x + 0.2 * math.sin(y / 15.0) + 0.1 * math.cos(x / 20.0),
                             n=0.03, segments=segs)
    p = SolverParams(120.0, 30.0, rain=Hyetograph.from_mm_h([(0, 50), (60, 120), (120, 0)]), initial_depth=0.3)
    t = PreparedTerrain(base)
    cells = [5 * nx + 8, 9 * nx + 15, 12 * nx + 20, 2 * nx + 3]
    probe = Objective(ObjectiveDef([Asset(f"a{i}", [c], 10.0) for i, c in enumerate(cells)], []))
    r = gpu.run_batch(p, [t], probe.monitors)[0]
    obj = Objective(ObjectiveDef([Asset(f"a{i}", [c], float(r.monitor_max[probe.monitors.position(c)]) - 0.004, 1.0 + i)
                                  for i, c in enumerate(cells)], []))
    run = gpu.vjp(p, [t], obj.monitors, obj, checkpoint_interval=16)[0]
    gx, gy = run.dj_ddzx, run.dj_ddzy
    assert np.all(np.isfinite(gx)) and np.all(np.isfinite(gy))
    bnd = orc.bnd_dict(base, t)

    def j(dzx=None, dzy=None):
        d = design_dict(t, p)
        if dzx is not None:
            d["dzx"] = dzx
        if dzy is not None:
            d["dzy"] = dzy
        o = orc.flat_run64(base_arrays(base), d, p, obj.monitors, bnd=bnd)
        return obj.evaluate(o["monitor_max"], 0.0, 0.0)["j_risk"]

    dzx0 = np.asarray(t.dzx, np.float64).reshape(ny, nx + 1)
    dzy0 = np.asarray(t.dzy, np.float64).reshape(ny + 1, nx)
    gxi = np.abs(gx.copy()); gxi[:, 0] = 0; gxi[:, nx] = 0
    gyi = np.abs(gy.copy()); gyi[0, :] = 0; gyi[ny, :] = 0
    picks = [("x", np.unravel_index(i, gx.shape)) for i in np.argsort(gxi, axis=None)[-3:]]
    picks += [("y", np.unravel_index(i, gy.shape)) for i in np.argsort(gyi, axis=None)[-3:]]
    # and the faces next to the ghost edges
    picks += [("x", (8, 1)), ("x", (8, nx - 1)), ("y", (1, 10))]
    worst = 0.0
    for kind, idx in picks:
        base_a = dzx0 if kind == "x" else dzy0
        up, dn = base_a.copy(), base_a.copy()
        up[idx] += FD_STEP_M; dn[idx] -= FD_STEP_M
        fd = ((j(dzx=up) - j(dzx=dn)) if kind == "x" else (j(dzy=up) - j(dzy=dn))) / (2 * FD_STEP_M)
        ad = gx[idx] if kind == "x" else gy[idx]
        if abs(fd) < 1e-6 * max(np.abs(gx).max(), np.abs(gy).max()):
            continue   # a face with no influence on J
        rel = abs(ad - fd) / abs(fd)
        worst = max(worst, rel)
        assert rel <= FD_REL_TOL, f"{kind}-face {idx}: adjoint {ad:.6e} vs finite difference {fd:.6e} (rel {rel:.3%})"
    print(f"stage/inflow case: worst relative error vs f64 central differences: {worst:.3%}")


def test_crest_gradient_vs_f64_finite_differences(gpu):
    """Crest faces (a coarse fidelity level, face_crest: each side reduced by its own jump):
    itr_gpu_vjp_crest gives dJ/d(first jump) and dJ/d(second jump) of every face, against
    central differences of the f64 oracle on jumps well away from the d > 0 switch."""
    base = synthetic_terrain(48, 32, 2.5, lambda x, y: 2.0 - 0.01 * x + 0.2 * math.sin(y / 15.0) + 0.1 * math.cos(x / 20.0)
                             + 0.05 * math.sin(x / 3.0) * math.cos(y / 4.0), n=0.03,
                             segments=[Segment("transmissive", "east")], level=2)
    assert base.mode == 1
    nx, ny = base.nx, base.ny
    p = SolverParams(120.0, 30.0, rain=Hyetograph.from_mm_h([(0, 50), (60, 120), (120, 0)]), initial_depth=0.3)
    t = PreparedTerrain(base)
    cells = [5 * nx + 8, 9 * nx + 15, 12 * nx + 20]
    probe = Objective(ObjectiveDef([Asset(f"a{i}", [c], 10.0) for i, c in enumerate(cells)], []))
    r = gpu.run_batch(p, [t], probe.monitors)[0]
    obj = Objective(ObjectiveDef([Asset(f"a{i}", [c], float(r.monitor_max[probe.monitors.position(c)]) - 0.004, 1.0 + i)
                                  for i, c in enumerate(cells)], []))
    run = gpu.vjp(p, [t], obj.monitors, obj, checkpoint_interval=16)[0]
    grads = {"dzx": run.dj_ddzx, "dzy": run.dj_ddzy, "dzx2": run.dj_ddzx2, "dzy2": run.dj_ddzy2}
    jumps = {"dzx": np.asarray(t.dzx, np.float64).reshape(ny, nx + 1), "dzy": np.asarray(t.dzy, np.float64).reshape(ny + 1, nx),
             "dzx2": np.asarray(t.dzx2, np.float64).reshape(ny, nx + 1), "dzy2": np.asarray(t.dzy2, np.float64).reshape(ny + 1, nx)}
    for a in grads.values():
        assert np.all(np.isfinite(a))

    def j(name, arr):
        d = design_dict(t, p)
        d[name] = arr
        o = orc.flat_run64(base_arrays(base), d, p, obj.monitors)
        return obj.evaluate(o["monitor_max"], 0.0, 0.0)["j_risk"]

    worst, checked = 0.0, 0
    for name, g in grads.items():
        cand = np.abs(g) * (jumps[name] > 10 * FD_STEP_M)
        for i in np.argsort(cand, axis=None)[-2:]:
            idx = np.unravel_index(i, g.shape)
            if cand[idx] == 0.0:
                continue
            up, dn = jumps[name].copy(), jumps[name].copy()
            up[idx] += FD_STEP_M; dn[idx] -= FD_STEP_M
            fd = (j(name, up) - j(name, dn)) / (2 * FD_STEP_M)
            rel = abs(g[idx] - fd) / abs(fd)
            worst = max(worst, rel)
            checked += 1
            assert rel <= FD_REL_TOL, f"{name} {idx}: adjoint {g[idx]:.6e} vs finite difference {fd:.6e} ({rel:.3%})"
    assert checked >= 6
    print(f"crest faces: worst relative error vs f64 central differences: {worst:.3%}")
