"""Dry-row skipping (crates/itr-hydro/src/kernel.rs:605-612, 649-657) on the device.

The scene is crates/itr-hydro/tests/equivalence.rs:35-53: 57 x 43 cells at 2 m, an inflow
hydrograph on part of the west edge, a transmissive east edge, a stage on part of the south
edge, a block of wall cells, and a storm with a rain-free lead-in (no rain until 300 s, none
after 700 s), so rows between dry rows are skipped while the inflow and stage edges keep
their rows computed. Skipping must not change a single bit (equivalence.rs:108-128 checks the
same on the CPU): every forward path gives the same steps, depths, peaks, monitor maxima and
ledger with params.skip_dry on and off, equal to the f32 oracle's, and reports the oracle's
count of skipped rows; cell_updates leaves the skipped rows out.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle_ref as orc
from helpers import assert_bitwise, base_arrays, design_dict
from itr_gpu import Hyetograph, MonitorSet, PreparedTerrain, Segment, SolverParams, synthetic_terrain

NX, NY = 57, 43


def scene(skip=True):
    segs = [Segment("inflow", "west", (20.0, 40.0), hydrograph=[(0.0, 0.0), (200.0, 1.5), (500.0, 0.2)]),
            Segment("transmissive", "east"),
            Segment("stage", "south", (5.0, 25.0), stage_m=100.3)]

    def z(x, y):
        return 100.0 + 0.5 * math.sin(x / 9.0) * math.cos(y / 7.0) + 0.004 * (120.0 - x) + (0.6 if 60.0 <= x < 64.0 else 0.0)
    base = synthetic_terrain(NX, NY, 2.0, z, wallfun=lambda c, r: 30 <= c < 34 and 10 <= r < 18, n=0.035, segments=segs)
    p = SolverParams(900.0, 60.0, rain=Hyetograph.from_mm_h([(0, 0), (300, 0), (400, 80), (700, 0)]),
                     infil_capacity=10.0 / 1000.0 / 3600.0, skip_dry=skip)
    mon = MonitorSet(np.array([c for c in range(NX * NY) if c % 7 == 3]))
    return base, p, mon


def oracle(base, p, mon, t):
    return orc.flat_run(base_arrays(base), design_dict(t, p), p, mon, want_peak=True, max_rows=32, bnd=orc.bnd_dict(base, t))


def test_oracle_skips_rows_on_the_scene():
    base, p, mon = scene(True)
    t = PreparedTerrain(base)
    on = oracle(base, p, mon, t)
    p.skip_dry = False
    off = oracle(base, p, mon, t)
    assert on["rows_skipped"] > 0 and off["rows_skipped"] == 0
    assert on["steps"] == off["steps"]
    assert_bitwise(on["h"], off["h"], "oracle depth, skipping on vs off")
    np.testing.assert_array_equal(on["ledger"], off["ledger"])


IMPL = {"batched": 0, "tiled": 2}


@pytest.mark.gpu
@pytest.mark.parametrize("impl", ["batched", "tiled"])
def test_skipping_is_bitwise_neutral_and_counts_rows(impl):
    from itr_gpu import GpuSolver
    base, p, mon = scene(True)
    t = PreparedTerrain(base)
    o = oracle(base, p, mon, t)
    g = GpuSolver()
    try:
        g.set_option("impl", IMPL[impl])
        runs = {}
        for skip in (True, False):
            p.skip_dry = skip
            runs[skip] = g.run_batch(p, [t, t], mon, want_peak=True, ledger_rows=32)
    finally:
        g.close()
    for i in range(2):
        on, off = runs[True][i], runs[False][i]
        what = f"{impl} design {i}"
        assert on.steps == off.steps == o["steps"], what
        assert on.t_end == off.t_end == o["t_end"], what
        for r in (on, off):
            assert_bitwise(r.depth, o["h"], f"{what}: depth")
            assert_bitwise(r.peak, o["peak"], f"{what}: peak")
            np.testing.assert_array_equal(r.monitor_max, o["monitor_max"], err_msg=what)
        np.testing.assert_array_equal(on.ledger, off.ledger, err_msg=f"{what}: ledger, skipping on vs off")
        assert on.rows_skipped == o["rows_skipped"] > 0, (what, on.rows_skipped, o["rows_skipped"])
        assert off.rows_skipped == 0, what
        assert on.cell_updates == on.steps * NX * NY - on.rows_skipped * NX, what
