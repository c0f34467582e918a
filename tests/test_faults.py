"""Failure detection with corrupted inputs, made on the host (no GPU fault): the solver's health
test (`bad`: a depth that is NaN or below -h_dry after the positivity fix, numerics.rs:163-193)
ends a design as Unhealthy (solver.rs:541-544; status 3, `bad` in BatchRun, evaluator.rs:249-256).

A cell of NaN or negative initial depth makes its design unhealthy at the first step, on the
oracle and on the device; the device stops that design alone: the healthy designs of the same
batch give the oracle's bits. An infinite initial depth (whose first CFL dt would be zero) is
refused at the C boundary before any device work.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle_ref as orc
from helpers import assert_bitwise, base_arrays, design_dict
from itr_gpu import DeviceError
from itr_gpu.scenes import valley_scene


def scene():
    sc = valley_scene(10.0)   # 45 x 35
    sc.params.duration_s = 600.0
    sc.params.initial_stage = None
    return sc


def corrupted(sc, value):
    h0 = np.zeros((sc.base.ny, sc.base.nx), np.float32)
    h0[10, 20] = value
    return h0


def test_oracle_corrupted_initial_depth_is_unhealthy():
    sc = scene()
    t = sc.designs(1)[0][2]
    for v in (np.nan, -0.5):
        d = design_dict(t, sc.params)
        d["h0"] = corrupted(sc, v)
        o = orc.flat_run(base_arrays(sc.base), d, sc.params, sc.monitors)
        assert o["abort"] == orc.ABORT_UNHEALTHY and o["steps"] == 1, (v, o["abort"], o["steps"])


@pytest.mark.gpu
@pytest.mark.parametrize("impl", [0, 2])
def test_device_unhealthy_design_leaves_its_batch_alone(impl):
    from itr_gpu import GpuSolver
    sc = scene()
    terrs = [t for _, _, t in sc.designs(4)]
    zero = np.zeros((sc.base.ny, sc.base.nx), np.float32)
    h0s = [zero, corrupted(sc, np.nan), zero, corrupted(sc, -0.5)]
    g = GpuSolver()
    try:
        g.set_option("impl", impl)
        runs = g.run_arrays(sc.params, sc.base, [t.dzx for t in terrs], [t.dzy for t in terrs], [None] * 4, [None] * 4,
                            h0s, [(t.cut_m3, t.fill_m3) for t in terrs], sc.monitors, objective=sc.objective,
                            want_peak=True)
    finally:
        g.close()
    for i, (r, t, h0) in enumerate(zip(runs, terrs, h0s)):
        d = design_dict(t, sc.params)
        d["h0"] = h0
        o = orc.flat_run(base_arrays(sc.base), d, sc.params, sc.monitors, want_peak=True)
        assert r.steps == o["steps"], (i, r.steps, o["steps"])
        if i in (1, 3):
            assert r.status == 3 and r.bad and not r.feasible and o["abort"] == orc.ABORT_UNHEALTHY
        else:
            assert r.status == 0 and not r.bad
            assert_bitwise(r.depth.ravel(), o["h"].ravel(), f"healthy design {i}")
            assert_bitwise(r.peak.ravel(), o["peak"].ravel(), f"healthy design {i} peak")


@pytest.mark.gpu
def test_infinite_initial_depth_refused():
    from itr_gpu import GpuSolver
    sc = scene()
    t = sc.designs(1)[0][2]
    g = GpuSolver()
    try:
        with pytest.raises(DeviceError, match="infinite"):
            g.run_arrays(sc.params, sc.base, [t.dzx], [t.dzy], [None], [None], [corrupted(sc, np.inf)],
                         [(0.0, 0.0)], sc.monitors)
    finally:
        g.close()
