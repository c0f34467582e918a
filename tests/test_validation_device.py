"""The reference's validation suite (crates/itr-hydro/src/validation.rs:80-258, run by
crates/itr-hydro/tests/validation.rs:4-19) through the device's public call.

CPU: the host-mirror builders of tests/validation_cases.py reproduce the oracle's own case
runs: the flat f32 and f64 oracles on the builders' packed inputs give the same case values as
orc.validation (the C++ restatement of validation.rs, pinned to the reference README's table
in tests/test_oracle_golden.py), bit for bit where the start is the same.
GPU: every case through itr_gpu_run_batch on the three forward paths (batched cluster kernel,
plain one-design-per-launch, tiled): steps, end time, final depth and per-cell peak equal the
flat f32 oracle bit for bit, the ledger to f64 summation order, and the case's value meets the
suite's f32 threshold. Each case's device value is printed beside the f64 oracle's.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle_ref as orc
import validation_cases as vc
from helpers import assert_bitwise, base_arrays

CASES = list(vc.BUILDERS)


def design_of(case, i=0):
    t = case.terrains[i]
    h0 = case.h0[i] if case.h0 is not None else None
    if h0 is None and case.params.initial_stage is not None:
        h0 = t.initial_depth(case.params.initial_depth, case.params.initial_stage)
    return dict(dzx=t.dzx, dzy=t.dzy, dzx2=t.dzx2, dzy2=t.dzy2, h0=h0, cut=0.0, fill=0.0)


def oracle(case, prec=0):
    run = orc.flat_run if prec == 0 else orc.flat_run64
    return run(base_arrays(case.base), design_of(case), case.params, case.monitors, want_peak=True,
               max_rows=case.ledger_rows, bnd=orc.bnd_dict(case.base, case.terrains[0]))


def value_of(case, r):
    """The case's measure from a run dict (oracle) — depth, ledger, rel_residual."""
    h = np.asarray(r["h"], np.float64)
    return case.metric(h, r["ledger"], r["rel_residual"], r["steps"], r["t_end"])


def gauge_diff(a, b):
    return int(np.count_nonzero(np.asarray(a, np.float32).view(np.uint32) != np.asarray(b, np.float32).view(np.uint32)))


@pytest.mark.parametrize("name", CASES)
def test_builders_reproduce_oracle_cases(name):
    ref32 = orc.validation(0, orc.VALIDATION_CASES.index(name))
    if name == "gauge_invariance":
        a, b = oracle(vc.gauge_invariance(0.0)), oracle(vc.gauge_invariance(1000.0))
        assert gauge_diff(a["h"], b["h"]) == 0 == ref32["value"]
        return
    case = vc.BUILDERS[name]()
    o = oracle(case)
    v = value_of(case, o)
    if name == "lake_at_rest":
        # the reference's measure adds |qx| and |qy|, which the flat oracle reports
        full = max(v, float(np.max(np.abs(o["qx"]))), float(np.max(np.abs(o["qy"]))))
        assert full == ref32["value"], (full, ref32)
    elif name == "dam_break_ritter":
        # another first dt (module docstring): a different, equally valid trajectory
        assert v <= case.threshold and abs(v - ref32["value"]) < 0.1 * ref32["value"], (v, ref32)
    else:
        assert v == ref32["value"], (v, ref32)
    if case.check is not None:
        assert case.check(np.asarray(o["h"]), o["ledger"], o["rel_residual"], o["steps"], o["t_end"])


@pytest.mark.parametrize("name", ["rain_closed_plain", "tilted_plane_kinematic", "walls_under_rain", "inflow_ledger"])
def test_builders_f64_case_values(name):
    """The f64 flat oracle on the builders' (f32-rounded) jumps stays at the f64 case's level."""
    case = vc.BUILDERS[name]()
    o = oracle(case, prec=1)
    ref64 = orc.validation(1, orc.VALIDATION_CASES.index(name))
    v = value_of(case, o)
    assert v <= max(1e3 * ref64["value"], 1e-12), (v, ref64)


# ------------------------------------------------------------------------------ GPU ----

@pytest.fixture(scope="module")
def gpu():
    from itr_gpu import GpuSolver
    g = GpuSolver()
    yield g
    g.close()


IMPL = {"batched": 0, "plain": 1, "tiled": 2}


def device_run(g, case, impl):
    g.set_option("impl", IMPL[impl])
    try:
        t = case.terrains
        h0 = case.h0 if case.h0 is not None else [x.initial_depth(case.params.initial_depth, case.params.initial_stage)
                                                   if case.params.initial_stage is not None else None for x in t]
        return g.run_arrays(case.params, case.base, [x.dzx for x in t], [x.dzy for x in t], [x.dzx2 for x in t],
                            [x.dzy2 for x in t], h0, [(0.0, 0.0) for _ in t], case.monitors, want_peak=True, want_depth=True,
                            ledger_rows=case.ledger_rows, z_edge=[x.z_edge() for x in t] if case.base.has_stage else None)[0]
    finally:
        g.set_option("impl", 0)


def compare(r, o, what):
    assert r.steps == o["steps"], f"{what}: steps {r.steps} vs {o['steps']}"
    assert r.t_end == o["t_end"], what
    assert_bitwise(r.depth, o["h"], f"{what}: final depth")
    assert_bitwise(r.peak, o["peak"], f"{what}: per-cell peak")
    assert len(r.ledger) == len(o["ledger"]), what
    # f64 ledger (t, V, rain, in, out, infil, fix, residual): time and rain are the same f64
    # arithmetic; the boundary volumes are f64 sums of the same f32 face fluxes in another
    # order; volume, infiltration and fix are summed from f32 values in another order
    np.testing.assert_array_equal(r.ledger[:, [0, 2]], o["ledger"][:, [0, 2]], err_msg=f"{what}: ledger t, rain")
    np.testing.assert_allclose(r.ledger[:, 3:5], o["ledger"][:, 3:5], rtol=1e-9, atol=1e-12, err_msg=f"{what}: ledger in/out")
    np.testing.assert_allclose(r.ledger[:, [1, 5, 6]], o["ledger"][:, [1, 5, 6]], rtol=1e-6, atol=1e-12,
                               err_msg=f"{what}: ledger V, infil, fix")


@pytest.mark.gpu
@pytest.mark.parametrize("impl", ["batched", "plain", "tiled"])
@pytest.mark.parametrize("name", CASES)
def test_validation_case_on_device(gpu, name, impl):
    if name == "gauge_invariance":
        runs = []
        for off in (0.0, 1000.0):
            case = vc.gauge_invariance(off)
            r = device_run(gpu, case, impl)
            compare(r, oracle(case), f"{name}@{off:g} [{impl}]")
            runs.append(r)
        d = gauge_diff(runs[0].depth, runs[1].depth)
        print(f"\n{name} [{impl}]: device {d} cells differ; f64 oracle {orc.validation(1, 5)['value']:g}")
        assert d == 0
        return
    case = vc.BUILDERS[name]()
    r = device_run(gpu, case, impl)
    o = oracle(case)
    compare(r, o, f"{name} [{impl}]")
    h = np.asarray(r.depth, np.float64)
    v = case.metric(h, r.ledger, r.rel_residual, r.steps, r.t_end)
    ref64 = orc.validation(1, orc.VALIDATION_CASES.index(name))["value"]
    print(f"\n{name} [{impl}]: device f32 {v:.3g} (threshold {case.threshold:g}); f64 oracle {ref64:.3g}; steps {r.steps}")
    assert v <= case.threshold, (name, impl, v)
    if case.check is not None:
        assert case.check(h, r.ledger, r.rel_residual, r.steps, r.t_end), (name, impl)
