"""Failure detection with corrupted inputs, made on the host (no GPU fault): the solver's health
test (`bad`: a depth that is NaN or below -h_dry after the positivity fix, numerics.rs:163-193)
ends a design as Unhealthy (solver.rs:541-544; status 3, `bad` in BatchRun, evaluator.rs:249-256).

A cell of NaN or negative initial depth makes its design unhealthy at the first step, on the
oracle and on the device; the device stops that design alone: the healthy designs of the same
batch give the oracle's bits. An infinite initial depth (whose first CFL dt would be zero) is
refused at the C boundary before any device work.

A barrier wait that never completes (a single-CTA design's barrier expecting one arrival
more than its CTA makes: option stall_wait_test) runs to its bounded limit; the kernel leaves
its step loop with the whole CTA and the call returns ITR_DEVICE_TIMEOUT, after which the same
context runs the batch again normally. No GPU fault is involved: the wait is a bounded
try_wait loop.
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


@pytest.mark.gpu
def test_stalled_barrier_wait_times_out_and_context_recovers():
    from itr_gpu import GpuSolver
    sc = scene()
    sc.params.duration_s = 300.0
    terrs = [t for _, _, t in sc.designs(2)]
    g = GpuSolver()
    try:
        for k, v in (("autotune", 0), ("cluster", 1), ("threads", 256), ("wait_limit", 2000), ("stall_wait_test", 1)):
            g.set_option(k, v)
        with pytest.raises(DeviceError, match="wait limit"):
            g.run_batch(sc.params, terrs, sc.monitors, want_peak=True)
        g.set_option("stall_wait_test", 0)
        runs = g.run_batch(sc.params, terrs, sc.monitors, want_peak=True)
    finally:
        g.close()
    for r, t in zip(runs, terrs):
        o = orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, sc.monitors, want_peak=True)
        assert r.steps == o["steps"] and r.status == 0
        assert_bitwise(r.peak.ravel(), o["peak"].ravel(), "after the timeout: per-cell peak")
