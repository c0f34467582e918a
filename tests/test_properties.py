"""Property tests after crates/itr-hydro/tests/properties.rs:39,60 (24 random cases each) and
the mirror test of crates/itr-hydro/tests/equivalence.rs:210-240, for the HLL path.

Beds as properties.rs:22-31 draws them: 12-39 x 10-31 cells at 2 m, three sinusoids of
random amplitude and wavelength, a step of +-0.5 m half-way across, and in half the cases a
wall segment along a column; all edges closed. Seeded draws stand in for proptest's.
  * Lake at rest: a random stage (9-11.5 m) over the bed, 60 s. f64 oracle (jumps and
    initial depth in f64, as PreparedTerrain<f64> holds them): |q| < 1e-10, the reference's
    bound. f32 oracle and device: |q| and |h - h0| <= 1e-4 (the reference's GPU lake bound,
    crates/itr-gpu/tests/gpu.rs:22-38), and the device equals the f32 oracle bit for bit.
  * Positivity and ledger: random rain (1-4 hyetograph points up to 150 mm/h, 80 s apart)
    and a random 4 x 4 edit of +-0.6 m, 400 s. f64: h >= -1e-10 and relative ledger residual
    < 1e-10 (the reference's bounds); f32 and device: h >= 0 and residual < 1e-4 (the f64
    ledger over f32 state; gpu.rs:41-53's rain-volume bound), device bitwise equal to f32.
  * Mirror: an east-west mirrored bed with walls only, 200 s of rain: mirrored depths within
    1e-9 (f64; the reference's bound) and 1e-6 (f32 and device).
  * Crest lake at rest (equivalence.rs:245-268): a 1-cell berm kept by level-4 crest faces,
    still water below its crest: |q| < 1e-10 and ledger residual < 1e-12 in f64; the device
    keeps the depth to 1e-4 and equals the f32 oracle bit for bit.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle_ref as orc
from helpers import assert_bitwise, base_arrays, design_dict
from itr_gpu import Hyetograph, MonitorSet, PreparedTerrain, SolverParams, synthetic_terrain
from itr_gpu.adjoint import face_jumps_f64
from itr_gpu.terrain import TerrainEdit

CASES = 24


def beds(seed=20261204):
    """The 24 cases: (base, lake params, initial stage, rain params, edit)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(CASES):
        nx, ny = int(rng.integers(12, 40)), int(rng.integers(10, 32))
        amp, freq, step = rng.uniform(0, 0.8, 3), rng.uniform(2, 15, 3), rng.uniform(-0.5, 0.5)
        wall = (int(rng.integers(2, 8)), int(rng.integers(2, 8))) if rng.random() < 0.5 else None

        def z(x, y, amp=amp, freq=freq, step=step, nx=nx):
            return (10.0 + amp[0] * np.sin(x / freq[0]) + amp[1] * np.cos(y / freq[1]) + amp[2] * np.sin((x + y) / freq[2])
                    + np.where(x > nx, step, 0.0))
        z.vectorized = True
        wf = None if wall is None else (lambda c, r, w=wall: (c == w[0]) & (r >= w[1]))
        base = synthetic_terrain(nx, ny, 2.0, z, wf, n=0.03, segments=[])
        stage = float(rng.uniform(9.0, 11.5))
        lake = SolverParams(60.0, 30.0, initial_stage=stage)
        rain = rng.uniform(0, 150, int(rng.integers(1, 5)))
        dz = rng.uniform(-0.6, 0.6, 16)
        at = (int(rng.integers(0, 8)), int(rng.integers(0, 6)))
        wet = SolverParams(400.0, 50.0, rain=Hyetograph.from_mm_h([(k * 80.0, r) for k, r in enumerate(rain)]))
        out.append((base, lake, stage, wet, TerrainEdit(at[0], at[1], 4, 4, dz)))
    return out


def lake_f64_design(base, t, stage):
    h = np.maximum(stage - base.fine.z_ref - t.z, 0.0)
    h[base.wall] = 0.0
    dzx, dzy = face_jumps_f64(base, np.zeros((base.ny, base.nx)))
    return dict(dzx=dzx, dzy=dzy, h0=h)


def test_lake_at_rest_random_beds_oracle():
    for base, p, stage, _, _ in beds():
        t = PreparedTerrain(base)
        o64 = orc.flat_run64(base_arrays(base), lake_f64_design(base, t, stage), p, MonitorSet())
        assert max(np.abs(o64["qx"]).max(), np.abs(o64["qy"]).max()) < 1e-10
        d = design_dict(t, p)
        o32 = orc.flat_run(base_arrays(base), d, p, MonitorSet())
        assert max(np.abs(o32["qx"]).max(), np.abs(o32["qy"]).max()) <= 1e-4
        assert np.abs(o32["h"] - d["h0"]).max() <= 1e-4


def test_positivity_and_ledger_random_rain_and_edits_oracle():
    for base, _, _, p, e in beds():
        t = PreparedTerrain(base).apply_edit(e)
        o64 = orc.flat_run64(base_arrays(base), design_dict(t, p), p, MonitorSet())
        assert o64["abort"] == orc.ABORT_NONE
        assert o64["h"].min() >= -1e-10 and o64["rel_residual"] < 1e-10
        o32 = orc.flat_run(base_arrays(base), design_dict(t, p), p, MonitorSet())
        assert o32["abort"] == orc.ABORT_NONE
        assert o32["h"].min() >= 0.0 and o32["rel_residual"] < 1e-4


def mirror_case(mirrored: bool):
    def z(x, y):
        x = 40.0 - x if mirrored else x
        return 0.3 * math.sin(x / 5.0) + 0.02 * x + 0.01 * y
    base = synthetic_terrain(40, 20, 1.0, z, n=0.03, segments=[])
    p = SolverParams(200.0, 50.0, rain=Hyetograph.from_mm_h([(0.0, 60.0), (100.0, 0.0)]))
    return base, p


def test_mirror_metamorphic_oracle():
    for f, tol in ((orc.flat_run64, 1e-9), (orc.flat_run, 1e-6)):
        hs = []
        for m in (False, True):
            base, p = mirror_case(m)
            h = f(base_arrays(base), design_dict(PreparedTerrain(base), p), p, MonitorSet())["h"]
            hs.append(h[:, ::-1] if m else h)
        assert np.abs(hs[0] - hs[1]).max() < tol


@pytest.fixture(scope="module")
def gpu():
    from itr_gpu import GpuSolver
    g = GpuSolver()
    yield g
    g.close()


@pytest.mark.gpu
def test_lake_at_rest_random_beds_device(gpu):
    for i, (base, p, stage, _, _) in enumerate(beds()):
        t = PreparedTerrain(base)
        d = design_dict(t, p)
        r = gpu.run_batch(p, [t], MonitorSet(), want_peak=True)[0]
        assert np.abs(r.depth - d["h0"]).max() <= 1e-4, i
        o = orc.flat_run(base_arrays(base), d, p, MonitorSet())
        assert r.steps == o["steps"]
        assert_bitwise(r.depth.ravel(), o["h"].ravel(), f"lake case {i}")


@pytest.mark.gpu
def test_positivity_and_ledger_random_rain_and_edits_device(gpu):
    for i, (base, _, _, p, e) in enumerate(beds()):
        t = PreparedTerrain(base).apply_edit(e)
        r = gpu.run_batch(p, [t], MonitorSet(), ledger_rows=16)[0]
        assert r.status == 0 and r.depth.min() >= 0.0 and r.rel_residual < 1e-4, (i, r.rel_residual)
        o = orc.flat_run(base_arrays(base), design_dict(t, p), p, MonitorSet())
        assert r.steps == o["steps"]
        assert_bitwise(r.depth.ravel(), o["h"].ravel(), f"rain case {i}")


@pytest.mark.gpu
def test_mirror_metamorphic_device(gpu):
    hs = []
    for m in (False, True):
        base, p = mirror_case(m)
        h = gpu.run_batch(p, [PreparedTerrain(base)], MonitorSet())[0].depth.astype(np.float64)
        hs.append(h[:, ::-1] if m else h)
    assert np.abs(hs[0] - hs[1]).max() < 1e-6


def crest_case():
    """equivalence.rs:245-268: 64 x 48 at 1 m, 0.2 sin(col / 9) plus a 1-cell berm of 1 m at
    column 30, coarsened 4x (crest faces keep the berm); still water at stage 0.6 m, 120 s."""
    from itr_gpu.terrain import FineTerrain, GeoTransform, TerrainBase
    nx, ny = 64, 48
    cols = np.arange(nx)
    dem = np.tile(0.2 * np.sin(cols / 9.0) + np.where(cols == 30, 1.0, 0.0), (ny, 1))
    geo = GeoTransform(0.0, float(ny), 1.0, 1.0)
    walls = np.zeros((ny, nx), bool)
    base = TerrainBase(FineTerrain(dem, walls, np.full((ny, nx), 0.03), geo), 4, [])
    p = SolverParams(120.0, 30.0, initial_stage=0.6)
    return dem, walls, geo, base, p


def test_crest_level_lake_at_rest_oracle():
    dem, walls, geo, base, p = crest_case()
    s = orc.Scene(dem, walls, 0.03, geo, 4, [])
    assert s.mode == 1   # crest faces at level 4
    o = s.run(p, MonitorSet(), prec=1)
    assert max(np.abs(o["qx"]).max(), np.abs(o["qy"]).max()) < 1e-10
    assert o["rel_residual"] < 1e-12


@pytest.mark.gpu
def test_crest_level_lake_at_rest_device(gpu):
    _, _, _, base, p = crest_case()
    t = PreparedTerrain(base)
    d = design_dict(t, p)
    r = gpu.run_batch(p, [t], MonitorSet(), ledger_rows=8)[0]
    assert np.abs(r.depth - d["h0"]).max() <= 1e-4
    o = orc.flat_run(base_arrays(base), d, p, MonitorSet())
    assert r.steps == o["steps"]
    assert_bitwise(r.depth.ravel(), o["h"].ravel(), "crest lake")
