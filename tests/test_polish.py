"""Gradient polishing of an incumbent (itr_gpu/polish.py): the adjoint proposes, the exact
forward decides.

CPU: the host logic against a stand-in solver with a known J and guard: steps follow the
gradient inside the trust region, every proposal is snapped onto the quantisation grid
(DesignSpace::q, crates/itr-core/src/design.rs:259-261) and the bounds, a step that breaks
the guard or raises J is never kept, a berm whose height turns negative becomes a swale.
GPU: a real incumbent on a small wet scene with assets and a guard area: J goes down, the
result is feasible, its J is the exact forward's (a fresh itr_gpu_run_primitives gives the
same bits), the f32 CPU oracle rerun of the polished design gives the same monitor maxima
bit for bit, and the f64 oracle rerun agrees to 1e-3 relative in J.
"""
from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np
import pytest

import oracle_ref as orc
from helpers import base_arrays, design_dict
from itr_gpu import (Asset, Hyetograph, MonitorSet, Objective, ObjectiveDef, PreparedTerrain, Segment, SolverParams,
                     synthetic_terrain)
from itr_gpu.design import BERM, SWALE, Primitive, materialize
from itr_gpu.polish import polish


class QuadSolver:
    """J = sum_i (h_i - 0.22)^2 + (w_i - 6)^2 / 10 + (L_i - 47)^2 / 100; feasible while every
    height stays <= 0.3 (a stand-in guard)."""

    def __init__(self):
        self.calls = 0

    @staticmethod
    def j(prims):
        return sum((p.height - 0.22) ** 2 + (p.width - 6.0) ** 2 / 10 + (p.length - 47.0) ** 2 / 100 for p in prims)

    def run_primitives(self, params, base, designs, monitors, editable, max_abs_dz, objective=None, baseline_max=None):
        self.calls += 1
        prims = designs[0]
        ok = all(p.height <= 0.3 for p in prims)
        return [SimpleNamespace(j=self.j(prims), feasible=ok, status=0)], [0.0], [0.0]

    def vjp_primitives(self, params, base, designs, monitors, objective, editable, max_abs_dz, checkpoint_interval=128):
        g = [[2 * (p.height - 0.22), (p.width - 6.0) / 5, (p.length - 47.0) / 50] for p in designs[0]]
        return None, [np.array(g)]


def quantised(v, step):
    return abs(v / step - round(v / step)) < 1e-9


def test_polish_host_logic():
    s = QuadSolver()
    obj = SimpleNamespace(monitors=MonitorSet())
    start = [Primitive(SWALE, 10.0, 10.0, 80.0, 3.5, 30.0, -0.12), Primitive(BERM, 30.0, 20.0, 25.0, 7.5, 0.0, 0.05)]
    res = polish(s, None, None, start, obj, None, 1.0, iters=40, radius=(0.1, 1.0, 10.0))
    assert res.j < res.j_start and res.accepted > 0 and res.feasible
    assert all(b <= a for a, b in zip([res.j_start] + res.history, res.history))   # J never goes up
    for p in res.prims:
        assert quantised(p.height, 0.01) and quantised(p.width, 0.5) and quantised(p.length, 0.5)
        assert -0.5 <= p.height <= 0.3 and 3.0 <= p.width <= 8.0 and 20.0 <= p.length <= 100.0
        assert (p.kind == BERM) == (p.height > 0.0)                 # the swale turned into a berm
        assert abs(p.height - 0.22) <= 0.011 and abs(p.width - 6.0) <= 0.5 and abs(p.length - 47.0) <= 0.5
    assert res.evaluations == s.calls


def test_polish_never_keeps_an_infeasible_step():
    """Optimum beyond the guard (h = 0.5 > 0.3): heights stop at or below 0.3."""
    class Beyond(QuadSolver):
        @staticmethod
        def j(prims):
            return sum((p.height - 0.5) ** 2 for p in prims)

        def vjp_primitives(self, *a, **k):
            return None, [np.array([[2 * (p.height - 0.5), 0.0, 0.0] for p in a[2][0]])]
    s = Beyond()
    obj = SimpleNamespace(monitors=MonitorSet())
    res = polish(s, None, None, [Primitive(BERM, 0, 0, 40.0, 5.0, 0.0, 0.1)], obj, None, 1.0, iters=30)
    assert res.feasible and res.accepted > 0
    assert 0.25 <= res.prims[0].height <= 0.3


# ---------------------------------------------------------------------------- GPU ----------

def wet_scene():
    nx, ny = 24, 16
    base = synthetic_terrain(nx, ny, 5.0, lambda x, y: 2.0 - 0.01 * x + 0.2 * math.sin(y / 15.0) + 0.1 * math.cos(x / 20.0),
                             n=0.03, segments=[Segment("transmissive", "east")])
    p = SolverParams(180.0, 30.0, rain=Hyetograph.from_mm_h([(0, 50), (60, 120), (180, 0)]), initial_depth=0.3)
    return base, p


@pytest.mark.gpu
def test_polish_incumbent_on_device():
    from itr_gpu import GpuSolver
    base, p = wet_scene()
    nx, ny = base.nx, base.ny
    assets = [5 * nx + 8, 9 * nx + 15, 12 * nx + 20]
    guard = [3 * nx + 21, 4 * nx + 21]
    probe = Objective(ObjectiveDef([Asset(f"a{i}", [c], 10.0) for i, c in enumerate(assets)], guard))
    g = GpuSolver()
    try:
        r0 = g.run_batch(p, [PreparedTerrain(base)], probe.monitors)[0]
        peaks = {c: float(r0.monitor_max[probe.monitors.position(c)]) for c in assets + guard}
        odef = ObjectiveDef([Asset(f"a{i}", [c], peaks[c] - 0.004, 1.0 + i) for i, c in enumerate(assets)], guard,
                            guard_tolerance_m=0.002, earth_weight=1e-4)
        obj = Objective(odef)
        baseline = np.array([peaks[int(c)] for c in obj.monitors.cells])
        editable = np.ones((ny, nx), dtype=bool)
        start = [Primitive(BERM, 55.0, 45.0, 40.0, 6.0, 30.0, 0.10), Primitive(SWALE, 85.0, 30.0, 30.0, 5.0, 110.0, -0.10)]
        res = polish(g, p, base, start, obj, editable, 1.0, baseline_max=baseline, iters=6, checkpoint_interval=16)
        assert res.feasible and res.accepted > 0 and res.j < res.j_start, (res.j_start, res.history)
        # the exact forward: a fresh device run of the polished design gives the same J bits
        runs, cut, fill = g.run_primitives(p, base, [res.prims], obj.monitors, editable, 1.0, objective=obj,
                                           baseline_max=baseline)
        assert runs[0].j == res.j and runs[0].feasible
    finally:
        g.close()
    # the CPU oracle reruns of the polished design: f32 bit for bit, f64 to 1e-3 in J
    e = materialize(res.prims, base.fine.geo, nx, ny, editable, 1.0)
    t = PreparedTerrain(base).apply_edit(e)
    o32 = orc.flat_run(base_arrays(base), design_dict(t, p), p, obj.monitors)
    np.testing.assert_array_equal(o32["monitor_max"].astype(np.float32), runs[0].monitor_max.astype(np.float32))
    o64 = orc.flat_run64(base_arrays(base), design_dict(t, p), p, obj.monitors)
    j64 = obj.evaluate(o64["monitor_max"], e.cut_m3, e.fill_m3, baseline)["j"]
    assert abs(j64 - res.j) <= 1e-3 * abs(j64), (j64, res.j)


@pytest.mark.gpu
def test_polish_config5_incumbent_exact_and_oracle_reruns():
    """Configuration 5's polish workflow (fractal 1024 x 1024 at 2 m, 6 primitives per design,
    the first 900 s of its storm, when the assets around their 0.05 m threshold are wet): the
    best feasible design of a 16-design generation is polished with the device adjoint, every
    proposal re-evaluated exactly on the device. Then the polished incumbent is rerun: a fresh
    device run gives its J bits, the f32 oracle its monitor maxima bit for bit, the f64 oracle
    its J to 1e-3 relative, and it is feasible against the baseline."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    from itr_gpu import GpuSolver
    from itr_gpu.polish import polish_population
    from itr_gpu.scenes import config
    sc = config(5)
    p = sc.params
    p.duration_s = 900.0
    g = GpuSolver()
    try:
        r = polish_population(g, p, sc.base, sc.primitive_designs(16), sc.objective, sc.editable, sc.max_abs_dz,
                              max_volume=sc.max_volume, iters=4)
        res = r.result
        assert res.feasible and res.j <= res.j_start, (res.j_start, res.history)
        runs, cut, fill = g.run_primitives(p, sc.base, [res.prims], sc.objective.monitors, sc.editable, sc.max_abs_dz,
                                           objective=sc.objective, baseline_max=r.baseline_max)
        assert runs[0].j == res.j and runs[0].feasible
    finally:
        g.close()
    e = materialize(res.prims, sc.geo, sc.base.nx, sc.base.ny, sc.editable, sc.max_abs_dz)
    t = PreparedTerrain(sc.base).apply_edit(e)
    with ThreadPoolExecutor(max_workers=2) as ex:
        f32 = ex.submit(orc.flat_run, base_arrays(sc.base), design_dict(t, p), p, sc.objective.monitors)
        f64 = ex.submit(orc.flat_run64, base_arrays(sc.base), design_dict(t, p), p, sc.objective.monitors)
        o32, o64 = f32.result(), f64.result()
    np.testing.assert_array_equal(o32["monitor_max"].astype(np.float32), runs[0].monitor_max.astype(np.float32))
    rep64 = sc.objective.evaluate(o64["monitor_max"], e.cut_m3, e.fill_m3, r.baseline_max)
    assert abs(rep64["j"] - res.j) <= 1e-3 * abs(rep64["j"]), (rep64["j"], res.j)
    assert rep64["guard_violation_m"] == 0.0
    print(f"\nconfig 5 polish: J {res.j_start:.6g} -> {res.j:.6g} ({res.accepted} of {res.evaluations - 1} proposals kept), "
          f"f64 rerun J {rep64['j']:.6g}; wall {r.wall_s}")


def test_quantize_rounds_half_away_from_zero():
    """DesignSpace::q (crates/itr-core/src/design.rs:259-261) rounds with Rust's f64::round,
    half-way cases away from zero (Python's round() would take the even neighbour)."""
    from itr_gpu.design import quantize
    assert quantize(0.125, 0.25) == 0.25 and quantize(-0.125, 0.25) == -0.25
    assert quantize(0.375, 0.25) == 0.5 and quantize(0.625, 0.25) == 0.75
    assert quantize(2.6, 0.5) == 2.5 and quantize(-2.76, 0.5) == -3.0
    assert quantize(1.2345, 0.0) == 1.2345
    from itr_gpu.design import round_half_away
    # x + 0.5 would round these wrongly: 0.49999999999999994 + 0.5 rounds to 1.0, and an odd
    # integer above 2^52 plus 0.5 rounds to the even neighbour
    assert round_half_away(0.49999999999999994) == 0.0 and round_half_away(-0.49999999999999994) == 0.0
    assert round_half_away(2.0 ** 52 + 1) == 2.0 ** 52 + 1 and round_half_away(-(2.0 ** 52 + 1)) == -(2.0 ** 52 + 1)
    assert round_half_away(0.5) == 1.0 and round_half_away(-0.5) == -1.0 and round_half_away(-2.5) == -3.0
