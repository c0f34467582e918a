"""Seeded synthetic scenes for the five benchmark configurations of the batched path.

The reference measures on no public dataset; these stand in for its example scenarios
(examples/*/scenario.toml shapes) with the sizes, storms, roughness, infiltration, assets
and guards of each configuration. Elevations are analytic functions of (x, y) so one scene
can be sampled at any cell size (the fidelity ladder of configuration 3 resamples without
resampling error):
  * a random Fourier-feature field stands in for the FFT-filtered Gaussian random field of
    scripts/make_rolling_hills.py:77-82 (same Gaussian covariance, sigma and length),
  * Gaussian hills and polyline-distance gullies follow make_rolling_hills.py:68-97,
  * the fractal field of configuration 5 is a spectral sum with amplitude ~ k^-(H+1).
Seeds: scene 20261203 + config index, designs 7 + config index.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .design import Primitive, materialize, random_design
from .solver import Asset, Hyetograph, MonitorSet, Objective, ObjectiveDef, SolverParams
from .terrain import FineTerrain, GeoTransform, PreparedTerrain, Segment, TerrainBase


def _fourier_field(rng, sigma, length, k=64):
    """Gaussian-covariance random field as a sum of k random cosines (resolution-free)."""
    w = rng.normal(0.0, 1.0 / length, size=(k, 2))
    ph = rng.uniform(0.0, 2 * math.pi, size=k)
    amp = sigma * math.sqrt(2.0 / k)

    def f(x, y):
        return amp * np.cos(x[..., None] * w[:, 0] + y[..., None] * w[:, 1] + ph).sum(-1)
    return f


def _polyline_dist(px, py, pts):
    d = np.full(np.shape(px), np.inf)
    for (ax, ay), (bx, by) in zip(pts[:-1], pts[1:]):
        vx, vy = bx - ax, by - ay
        t = np.clip(((px - ax) * vx + (py - ay) * vy) / (vx * vx + vy * vy), 0, 1)
        d = np.minimum(d, np.hypot(px - ax - t * vx, py - ay - t * vy))
    return d


def _rect_cells(geo, nx, ny, x0, y0, w, h):
    """Cells whose centres fall inside the world rectangle [x0, x0+w] x [y0, y0+h]."""
    out = []
    for r in range(ny):
        for c in range(nx):
            x, y = geo.cell_center(c, r)
            if x0 <= x <= x0 + w and y0 <= y <= y0 + h:
                out.append(r * nx + c)
    return out


@dataclass
class Scene:
    name: str
    base: TerrainBase
    params: SolverParams
    objective: Objective
    editable: np.ndarray
    geo: GeoTransform
    design_box: tuple
    n_prims: int
    max_volume: float
    max_abs_dz: float = 1.0
    design_seed: int = 7

    @property
    def monitors(self) -> MonitorSet:
        return self.objective.monitors

    def designs(self, n: int, seed: int | None = None, length=(20.0, 100.0), width=(3.0, 8.0), height=(-0.5, 0.5)):
        """n seeded random designs (materialized, prepared); over-volume ones are resampled
        (max_static_attempts, crates/itr-opt/src/driver.rs:207-218)."""
        rng = np.random.default_rng(self.design_seed if seed is None else seed)
        out = []
        b = self.base
        while len(out) < n:
            prims = random_design(rng, self.n_prims, self.design_box, length=length, width=width, height=height)
            e = materialize(prims, self.geo, b.fine.nx, b.fine.ny, self.editable, self.max_abs_dz)
            if e.cut_m3 + e.fill_m3 > self.max_volume:
                continue
            t = PreparedTerrain(b).apply_edit(e)
            out.append((prims, e, t))
        return out


    def primitive_designs(self, n: int, seed: int | None = None, length=(20.0, 100.0), width=(3.0, 8.0),
                          height=(-0.5, 0.5)):
        """n seeded random designs as primitive lists, not materialised on the host (the
        device does it, itr_gpu_run_primitives; the volume limit is applied to the volumes it
        returns)."""
        rng = np.random.default_rng(self.design_seed if seed is None else seed)
        return [random_design(rng, self.n_prims, self.design_box, length=length, width=width, height=height)
                for _ in range(n)]


def _objective(geo, nx, ny, assets, guards, tol, thr=0.05):
    A = [Asset(f"asset{i}", _rect_cells(geo, nx, ny, *r), thr) for i, r in enumerate(assets)]
    G = sorted(set(c for g in guards for c in _rect_cells(geo, nx, ny, *g)))
    return Objective(ObjectiveDef(A, G, guard_tolerance_m=tol))


def valley_field(seed: int):
    """Configuration-1 DEM as a function of (x, y) on a 450 x 350 m domain."""
    rng = np.random.default_rng(seed)
    grf = _fourier_field(rng, 0.4, 40.0)
    yc, W = 175.0, 150.0

    def z(x, y):
        x = np.asarray(x, float); y = np.asarray(y, float)
        v = 20.0 - 0.02 * x + grf(x, y)
        s = np.abs(y - yc) < W / 2
        v = v - np.where(s, 1.5 * 0.5 * (1.0 + np.cos(2 * math.pi * (y - yc) / W)), 0.0)
        return v
    return z


def valley_scene(cell: float, seed: int = 20261203 + 1, design_seed: int = 7 + 1, n_prims: int = 2, name="valley") -> Scene:
    Lx, Ly = 450.0, 350.0
    nx, ny = int(round(Lx / cell)), int(round(Ly / cell))
    geo = GeoTransform(0.0, Ly, cell, cell)
    zf = valley_field(seed)
    cols, rows = np.meshgrid(np.arange(nx), np.arange(ny))
    x = (cols + 0.5) * cell
    y = Ly - (rows + 0.5) * cell
    dem = zf(x, y)
    fine = FineTerrain(dem, np.zeros((ny, nx), bool), np.full((ny, nx), 0.035), geo)
    base = TerrainBase(fine, 1, [Segment("transmissive", "east")])
    params = SolverParams(duration_s=2400.0, sync_interval_s=60.0, rain=Hyetograph.from_mm_h([(0, 0), (720, 80), (2400, 0)]),
                          infil_capacity=5.0 / 1000.0 / 3600.0)
    assets = [(250.0, 160.0, 15.0, 10.0), (300.0, 180.0, 15.0, 10.0)]
    guards = [(380.0, 165.0, 30.0, 20.0)]
    obj = _objective(geo, nx, ny, assets, guards, tol=0.01)
    editable = np.ones((ny, nx), bool)
    for c in obj.monitors.cells:
        editable[c // nx, c % nx] = False
    return Scene(name, base, params, obj, editable, geo, (80.0, 100.0, 240.0, 250.0), n_prims, 300.0, 1.0, design_seed)


def inflow_valley_scene(cell: float, seed: int = 20261203 + 1, design_seed: int = 7 + 1, n_prims: int = 2,
                        scale: float = 1.0) -> Scene:
    """The configuration-1 valley driven from its boundaries, the case the reference's GPU
    backend declined (lib.rs:166-176): an upstream inflow hydrograph across the valley floor
    on the west edge, a side-channel inflow on part of the south edge, a tailwater stage on
    the east edge and a stage on part of the north edge; light rain. Every kind of ghost
    (wall, transmissive, stage, inflow; x- and y-normal) occurs."""
    sc = valley_scene(cell, seed, design_seed, n_prims, name="inflow-valley")
    fine = sc.base.fine
    segs = [Segment("inflow", "west", (125.0, 225.0), hydrograph=[(0.0, 0.0), (600.0, 6.0 * scale), (1800.0, 2.0 * scale),
                                                                    (2400.0, 0.5 * scale)]),
            Segment("inflow", "south", (200.0, 260.0), hydrograph=[(0.0, 1.0 * scale), (1200.0, 3.0 * scale), (2400.0, 0.0)]),
            Segment("stage", "east", stage_m=10.2),
            Segment("stage", "north", (300.0, 450.0), stage_m=11.8),
            Segment("transmissive", "south", (350.0, 450.0))]
    base = TerrainBase(fine, 1, segs)
    sc.base = base
    sc.params.rain = Hyetograph.from_mm_h([(0, 0), (720, 20), (2400, 0)])
    return sc


def hills_field(seed: int):
    """Configuration-2 DEM as a function of (x, y) on a 600 x 480 m domain."""
    rng = np.random.default_rng(seed)
    hills = [(rng.uniform(100, 500), rng.uniform(120, 420), rng.uniform(2, 6), rng.uniform(30, 60)) for _ in range(3)]
    gullies = []
    for _ in range(2):
        x0 = rng.uniform(120, 480)
        pts = [(x0 + rng.uniform(-30, 30), 470.0), (x0 + rng.uniform(-40, 40), 320.0), (x0 + rng.uniform(-50, 50), 160.0),
               (x0 + rng.uniform(-50, 50), 20.0)]
        gullies.append((pts, rng.uniform(1.5, 2.5), rng.uniform(10, 16)))
    noise = _fourier_field(rng, 0.3, 30.0)

    def z(x, y):
        x = np.asarray(x, float); y = np.asarray(y, float)
        v = 50.0 + 0.03 * y + noise(x, y)
        for hx, hy, a, s in hills:
            v = v + a * np.exp(-((x - hx) ** 2 + (y - hy) ** 2) / (2 * s * s))
        for pts, depth, w in gullies:
            v = v - depth * np.exp(-(_polyline_dist(x, y, pts) / w) ** 2)
        return v
    return z, hills, gullies


def hills_scene(cell: float = 5.0, seed: int = 20261203 + 2, design_seed: int = 7 + 2, n_prims: int = 4, name="hills",
                initial_depth: float = 0.0) -> Scene:
    Lx, Ly = 600.0, 480.0
    nx, ny = int(round(Lx / cell)), int(round(Ly / cell))
    geo = GeoTransform(0.0, Ly, cell, cell)
    zf, hills, gullies = hills_field(seed)
    cols, rows = np.meshgrid(np.arange(nx), np.arange(ny))
    x = (cols + 0.5) * cell
    y = Ly - (rows + 0.5) * cell
    fine = FineTerrain(zf(x, y), np.zeros((ny, nx), bool), np.full((ny, nx), 0.045), geo)
    base = TerrainBase(fine, 1, [Segment("transmissive", "south")])
    params = SolverParams(duration_s=3600.0, sync_interval_s=60.0, rain=Hyetograph.from_mm_h([(0, 0), (1200, 100), (3600, 0)]),
                          infil_capacity=8.0 / 1000.0 / 3600.0, initial_depth=initial_depth)
    # houses near the gully outlets, the guard downstream by the southern edge
    gx = [g[0][2][0] for g in gullies]
    assets = [(gx[0] - 20.0, 140.0, 12.0, 12.0), (gx[0] + 10.0, 110.0, 12.0, 12.0), (gx[1] - 15.0, 130.0, 12.0, 12.0),
              (gx[1] + 12.0, 100.0, 12.0, 12.0)]
    guards = [(0.5 * (gx[0] + gx[1]) - 20.0, 25.0, 40.0, 25.0)]
    obj = _objective(geo, nx, ny, assets, guards, tol=0.02)
    editable = np.ones((ny, nx), bool)
    for c in obj.monitors.cells:
        editable[c // nx, c % nx] = False
    return Scene(name, base, params, obj, editable, geo, (80.0, 150.0, 520.0, 420.0), n_prims, 1000.0, 1.0, design_seed)


def fractal_scene(n: int = 1024, cell: float = 2.0, seed: int = 20261203 + 5, design_seed: int = 7 + 5, n_prims: int = 6) -> Scene:
    """Configuration 5: n x n at `cell` m, spectral fractal (Hurst 0.8, relief 15 m) + channel."""
    rng = np.random.default_rng(seed)
    L = n * cell
    geo = GeoTransform(0.0, L, cell, cell)
    kx = np.fft.fftfreq(n)[None, :]
    ky = np.fft.fftfreq(n)[:, None]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    H = 0.8
    spec = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) * k ** (-(H + 1.0))
    spec[0, 0] = 0.0
    f = np.real(np.fft.ifft2(spec))
    f = (f - f.min()) / (f.max() - f.min()) * 15.0
    cols, rows = np.meshgrid(np.arange(n), np.arange(n))
    x = (cols + 0.5) * cell
    y = L - (rows + 0.5) * cell
    chan = [(0.1 * L, 0.95 * L), (0.35 * L, 0.6 * L), (0.6 * L, 0.45 * L), (0.95 * L, 0.05 * L)]
    dem = 30.0 + f + 0.004 * y - 2.0 * np.exp(-(_polyline_dist(x, y, chan) / 12.0) ** 2)
    fine = FineTerrain(dem, np.zeros((n, n), bool), np.full((n, n), 0.04), geo)
    base = TerrainBase(fine, 1, [Segment("transmissive", "south"), Segment("transmissive", "east")])
    params = SolverParams(duration_s=5400.0, sync_interval_s=60.0,
                          rain=Hyetograph.from_mm_h([(0, 0), (1200, 60), (2100, 30), (3300, 120), (5400, 0)]),
                          infil_capacity=5.0 / 1000.0 / 3600.0)
    pts = [(0.3 + 0.05 * i) * L for i in range(8)]
    assets = [(p, (0.62 - 0.04 * i) * L, 12.0, 12.0) for i, p in enumerate(pts)]
    guards = [(0.75 * L, 0.25 * L, 40.0, 25.0), (0.85 * L, 0.15 * L, 40.0, 25.0), (0.5 * L, 0.3 * L, 40.0, 25.0)]
    obj = _objective(geo, n, n, assets, guards, tol=0.02)
    editable = np.ones((n, n), bool)
    for c in obj.monitors.cells:
        editable[c // n, c % n] = False
    return Scene("fractal", base, params, obj, editable, geo, (0.2 * L, 0.4 * L, 0.6 * L, 0.8 * L), n_prims, 3000.0, 1.0,
                 design_seed)


def river_scene(n: int = 1024, cell: float = 2.0, duration_s: float = 900.0) -> Scene:
    """Rain-free and inflow-driven: configuration 5's fractal terrain fed by a river that enters
    through 60 m of the north edge at the head of the terrain's channel (0 to 40 m^3/s over the
    first 10 min, then steady) and leaves through the transmissive south and east edges. Rows
    far from the river stay dry for the whole run (the case dry-row skipping is for)."""
    sc = fractal_scene(n, cell)
    L = n * cell
    x0 = 0.1 * L
    segs = [Segment("inflow", "north", (x0 - 30.0, x0 + 30.0), hydrograph=[(0.0, 0.0), (600.0, 40.0), (duration_s, 40.0)]),
            Segment("transmissive", "south"), Segment("transmissive", "east")]
    sc.base = TerrainBase(sc.base.fine, 1, segs)
    sc.params.rain = Hyetograph.from_mm_h([(0.0, 0.0), (duration_s, 0.0)])
    sc.params.duration_s = duration_s
    sc.name = "river"
    return sc


def config(i: int) -> Scene:
    """Scene of configuration i (1-based) at its native resolution."""
    if i == 1:
        return valley_scene(5.0, name="config1-valley-90x70")
    if i == 2:
        return hills_scene(5.0, name="config2-hills-120x96")
    if i == 3:
        return valley_scene(5.0, seed=20261203 + 3, design_seed=7 + 3, n_prims=3, name="config3-valley-ladder")
    if i == 4:
        return hills_scene(2.5, seed=20261203 + 2, design_seed=7 + 4, name="config4-hills-240x192")
    if i == 5:
        return fractal_scene()
    raise ValueError(i)
