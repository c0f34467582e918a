"""The reference's eight validation cases (crates/itr-hydro/src/validation.rs:80-258) built
through the host mirror, so the same inputs can run on the device (itr_gpu_run_batch), on
the flat f32 oracle and on the flat f64 oracle.

Each builder returns a Case: the TerrainBase, SolverParams, per-design initial depths (None:
the params' initial depth / stage), the monitors, the ledger rows wanted, and `metric`, the
case's own measure computed from one run's outputs (depth, ledger rows, rel_residual, steps,
t_end), with the suite's threshold for f32 (validation.rs; docs/validation.md:60-69).

Differences from the reference's own run of a case, by design of the batch API:
  * dam_break_ritter: the reference starts with dt = 0.4 dx / sqrt(g h0) (validation.rs:
    141-146, a Start with dt_next); a batch run starts from the initial-smax pre-pass
    (solver.rs:314-332), dt = cfl / (2 sqrt(g h0) / dx), half of it. The Ritter error is
    measured the same way on the resulting state.
  * lake_at_rest: the device returns depths, not momenta, so the device-side metric is
    max |eta - 1.5| (the reference's adds |qx|, |qy|; the flat oracle reports both).
Everything else is the reference's case.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from itr_gpu import Hyetograph, MonitorSet, PreparedTerrain, Segment, SolverParams, synthetic_terrain

G = 9.81


@dataclass
class Case:
    name: str
    base: object
    params: SolverParams
    h0: list | None = None
    monitors: MonitorSet = field(default_factory=MonitorSet)
    ledger_rows: int = 64
    threshold: float = 0.0
    # metric(depth (ny, nx) f64, ledger rows (k, 8), rel_residual, steps, t_end) -> value
    metric: object = None
    # extra pass/fail condition beyond value <= threshold
    check: object = None
    terrains: list = field(default_factory=list)


def _vparams(duration, sync, **kw):
    """validation::params (validation.rs:23-41): the reference defaults, skip_dry on."""
    return SolverParams(duration, sync, cfl=kw.pop("cfl", 0.35), **kw)


def lake_at_rest():
    def zf(x, y):
        return 0.3 * math.sin(x / 7.0) * math.cos(y / 5.0) + (0.4 if x > 30.0 else 0.0)
    base = synthetic_terrain(64, 48, 1.0, zf, n=0.03)
    p = _vparams(60.0, 10.0, initial_stage=1.5)

    def metric(h, led, rr, steps, t_end):
        eta = h + base.z + base.fine.z_ref
        return float(np.max(np.abs(eta - 1.5)))
    return Case("lake_at_rest", base, p, threshold=1e-4, metric=metric, terrains=[PreparedTerrain(base)])


def rain_closed_plain():
    base = synthetic_terrain(40, 30, 2.0, lambda x, y: 10.0, n=0.04)
    p = _vparams(600.0, 60.0, rain=Hyetograph.from_mm_h([(0, 0), (100, 50), (400, 10), (500, 0)]))
    return Case("rain_closed_plain", base, p, threshold=1e-6, metric=lambda h, led, rr, s, t: rr,
                terrains=[PreparedTerrain(base)])


def dam_break_ritter():
    nx, dx, h0v, x0 = 800, 0.25, 1.0, 100.0
    base = synthetic_terrain(nx, 3, dx, lambda x, y: 0.0, n=0.0)
    p = _vparams(10.0, 10.0, cfl=0.4)
    x = (np.arange(nx) + 0.5) * dx
    h0 = np.zeros((3, nx), np.float32)
    h0[:, x < x0] = h0v

    def metric(h, led, rr, steps, t):
        c0 = math.sqrt(G * h0v)
        xs = x - x0
        a = 2.0 * c0 - xs / t
        exact = np.where(xs <= -c0 * t, h0v, np.where(xs >= 2.0 * c0 * t, 0.0, a * a / (9.0 * G)))
        l1 = float(np.sum(np.abs(h[1] - exact) * dx))   # the middle row (validation.rs: row j = 2 of 3)
        return l1 / (h0v * 3.0 * c0 * t)
    return Case("dam_break_ritter", base, p, h0=[h0], threshold=0.03, metric=metric, terrains=[PreparedTerrain(base)])


def wet_dry_step():
    base = synthetic_terrain(80, 20, 1.0, lambda x, y: (0.8 if x > 40.0 else 0.0) + 0.01 * x, n=0.02)
    p = _vparams(120.0, 20.0, initial_stage=1.0)
    return Case("wet_dry_step", base, p, threshold=1e-6, metric=lambda h, led, rr, s, t: rr,
                check=lambda h, led, rr, s, t: float(np.min(h)) >= 0.0, terrains=[PreparedTerrain(base)])


def tilted_plane_kinematic():
    nx, ny, dx, slope, rate = 100, 4, 2.0, 0.01, 100.0
    base = synthetic_terrain(nx, ny, dx, lambda x, y: 5.0 - slope * x, n=0.03, segments=[Segment("transmissive", "east")])
    p = _vparams(3600.0, 300.0, rain=Hyetograph.from_mm_h([(0.0, rate), (1e9, rate)]))

    def metric(h, led, rr, s, t):
        q_out = (led[-1, 4] - led[-2, 4]) / (led[-1, 0] - led[-2, 0])
        q_in = rate / 1000.0 / 3600.0 * nx * ny * dx * dx
        return abs(q_out / q_in - 1.0)
    return Case("tilted_plane_kinematic", base, p, threshold=0.02, metric=metric, terrains=[PreparedTerrain(base)])


def gauge_invariance(offset=0.0):
    def zf(x, y):
        v = 0.2 * math.sin(x / 6.0) + 0.01 * y
        return offset + round(v * 1024.0) / 1024.0
    base = synthetic_terrain(40, 30, 1.0, zf, n=0.03)
    p = _vparams(60.0, 30.0, initial_stage=offset + 0.5, rain=Hyetograph.from_mm_h([(0.0, 40.0), (60.0, 0.0)]))
    return Case(f"gauge_invariance@{offset:g}", base, p, threshold=0.0, metric=None, terrains=[PreparedTerrain(base)])


def walls_under_rain():
    base = synthetic_terrain(30, 30, 1.0, lambda x, y: 0.01 * x, wallfun=lambda c, r: 10 <= c < 20 and 10 <= r < 20, n=0.03)
    p = _vparams(300.0, 60.0, rain=Hyetograph.from_mm_h([(0.0, 80.0), (300.0, 80.0)]))
    return Case("walls_under_rain", base, p, threshold=1e-6, metric=lambda h, led, rr, s, t: rr,
                check=lambda h, led, rr, s, t: float(np.max(h[10:20, 10:20])) == 0.0, terrains=[PreparedTerrain(base)])


def inflow_ledger():
    seg = Segment("inflow", "west", (10.0, 20.0), hydrograph=[(0.0, 0.0), (100.0, 2.0), (300.0, 0.0)])
    base = synthetic_terrain(60, 30, 1.0, lambda x, y: 1.0 - 0.005 * x, n=0.03, segments=[seg])
    p = _vparams(400.0, 50.0)
    return Case("inflow_ledger", base, p, threshold=1e-6, metric=lambda h, led, rr, s, t: rr,
                check=lambda h, led, rr, s, t: abs((led[-1, 3] - led[-1, 4]) / 300.0 - 1.0) < 0.02,
                terrains=[PreparedTerrain(base)])


BUILDERS = {"lake_at_rest": lake_at_rest, "rain_closed_plain": rain_closed_plain, "dam_break_ritter": dam_break_ritter,
            "wet_dry_step": wet_dry_step, "tilted_plane_kinematic": tilted_plane_kinematic,
            "gauge_invariance": gauge_invariance, "walls_under_rain": walls_under_rain, "inflow_ledger": inflow_ledger}
