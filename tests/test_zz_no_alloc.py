"""itr_gpu_run_plain_static: the allocation-free plain forward (static device scratch).

Two consecutive calls must each reproduce the context entry point (itr_gpu_run_batch) bit
for bit on the same design: everything, ledger included, against its plain path (the same
kernels), and the state (depth, peaks, monitor maxima, steps) against its default batched
path and against the f32 oracle. The second call checks that nothing of the first survives
in the static scratch, and that it takes no device memory: the device's free memory
(cudaMemGetInfo) is the same before and after it. A grid of more than 32 tiles checks the
ledger's summation order against the context path. The size limit and the start check are
on the host, before any device work. The entry point exists for callers that cannot
allocate device memory when they run a design (a device committed to their own pool,
other streams that cudaMalloc's device-wide synchronisation would stall).
This file sorts last so that it also runs after every other GPU test in one process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle_ref as orc
from helpers import assert_bitwise, base_arrays, design_dict
from itr_gpu import GpuSolver, _lib
from itr_gpu.scenes import valley_scene


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


def static_call(lib, device, p, base, t, h0, monitors, ledger_rows=0):
    """One itr_gpu_run_plain_static call from host buffers; returns (status, err, result, arrays)."""
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a

    rain_t = arr([q[0] for q in p.rain.pts] or [0.0], np.float64)
    rain_r = arr([q[1] for q in p.rain.pts] or [0.0], np.float64)
    P = _lib.Params(p.duration_s, p.sync_interval_s, p.cfl, p.dt_max_s, p.h_dry, p.h_eps,
                    _ptr(rain_t, C.c_double), _ptr(rain_r, C.c_double), len(p.rain.pts), p.infil_capacity,
                    p.initial_depth, 1 if p.skip_dry else 0, p.inflow_scale)
    wet, gn2, bc = arr(base.wet, np.float32), arr(base.gn2, np.float32), arr(base.bc, np.uint8)
    G = _lib.Grid(base.nx, base.ny, base.dx, base.dy, base.g, base.mode, _ptr(wet, C.c_float), _ptr(gn2, C.c_float),
                  _ptr(bc, C.c_uint8), base.wet_count)
    a, b = arr(t.dzx, np.float32), arr(t.dzy, np.float32)
    a2 = arr(t.dzx2, np.float32) if t.dzx2 is not None else None
    b2 = arr(t.dzy2, np.float32) if t.dzy2 is not None else None
    hh = arr(h0, np.float32) if h0 is not None else None
    D = _lib.Design(_ptr(a, C.c_float), _ptr(b, C.c_float), _ptr(a2, C.c_float), _ptr(b2, C.c_float), _ptr(hh, C.c_float),
                    t.cut_m3, t.fill_m3)
    mon = arr(monitors.cells, np.uint32)
    n = base.nx * base.ny
    mm = np.zeros(max(len(mon), 1), np.float64)
    pk = np.zeros(n, np.float32)
    dp = np.zeros(n, np.float32)
    lg = np.zeros((max(ledger_rows, 1), 8), np.float64)
    R = _lib.Result()
    R.monitor_max = _ptr(mm, C.c_double)
    R.peak = _ptr(pk, C.c_float)
    R.depth = _ptr(dp, C.c_float)
    R.ledger = _ptr(lg, C.c_double) if ledger_rows else None
    R.max_rows = ledger_rows
    err = C.create_string_buffer(512)
    rc = lib.itr_gpu_run_plain_static(device, C.byref(P), C.byref(G), C.byref(D), _ptr(mon, C.c_uint32), len(mon),
                                      C.byref(R), err, len(err))
    return rc, err.value.decode(), R, dict(monitor_max=mm[:len(mon)], peak=pk.reshape(base.ny, base.nx),
                                          depth=dp.reshape(base.ny, base.nx), ledger=lg[:R.n_rows])


def test_oversize_grid_rejected_before_device_work():
    """A grid beyond the static scratch is refused with ITR_INVALID_ARG and a message; the
    check runs on the host, so it holds without a GPU too."""
    lib = _lib.load()
    sc = valley_scene(10.0)

    class Big:
        nx, ny, dx, dy, g, mode, wet_count = 600, 600, 5.0, 5.0, 9.81, 0, 0
        wet = np.zeros(1, np.float32)
        gn2 = np.zeros(1, np.float32)
        bc = np.zeros(1, np.uint8)

    class NoDesign:
        dzx = np.zeros(1, np.float32)
        dzy = np.zeros(1, np.float32)
        dzx2 = dzy2 = None
        cut_m3 = fill_m3 = 0.0

    rc, err, _, _ = static_call(lib, 0, sc.params, Big, NoDesign, None, sc.monitors)
    assert rc == _lib.ITR_INVALID_ARG
    assert "600x600" in err and "static scratch" in err, err


def test_infinite_initial_depth_rejected_before_device_work():
    """An infinite or absurd start depth would make the first dt vanish and the run crawl
    to its step limit: refused on the host like itr_gpu_run_batch refuses it."""
    lib = _lib.load()
    sc = valley_scene(10.0)
    t = [t for _, _, t in sc.designs(1)][0]
    h0 = np.zeros((sc.base.ny, sc.base.nx), np.float32)
    for bad in (np.inf, 2e4):
        h0[3, 4] = bad
        rc, err, _, _ = static_call(lib, 0, sc.params, t.base, t, h0, sc.monitors)
        assert rc == _lib.ITR_INVALID_ARG, (bad, rc, err)
        assert "initial depth" in err, err


def _free_bytes():
    import torch
    torch.cuda.synchronize(0)
    return torch.cuda.mem_get_info(0)[0]


@pytest.mark.gpu
@pytest.mark.parametrize("cell,duration", [(10.0, 900.0), (4.0, 600.0)])
def test_static_entry_matches_run_batch_twice(cell, duration):
    """45 x 35 (9 tiles) and 112 x 88 (42 tiles, more than one finalize warp's 32)."""
    sc = valley_scene(cell)   # rain, transmissive outlet
    sc.params.duration_s = duration
    terrs = [t for _, _, t in sc.designs(2)]
    g = GpuSolver(0)
    try:
        batched = g.run_batch(sc.params, terrs, sc.monitors, want_peak=True, want_depth=True, ledger_rows=64)
        g.set_option("impl", 1)
        plain = g.run_batch(sc.params, terrs, sc.monitors, want_peak=True, want_depth=True, ledger_rows=64)
    finally:
        g.close()
    lib = _lib.load()
    orcs = [orc.flat_run(base_arrays(sc.base), design_dict(t, sc.params), sc.params, sc.monitors, want_peak=True)
            for t in terrs]
    # two consecutive calls per design, designs alternating: each must equal run_batch
    for call in range(2):
        for t, r, rb, o in zip(terrs, plain, batched, orcs):
            p = sc.params   # h0 as run_batch passes it: explicit only for an initial stage
            h0 = t.initial_depth(p.initial_depth, p.initial_stage) if p.initial_stage is not None else None
            free0 = _free_bytes()
            rc, err, R, out = static_call(lib, 0, sc.params, t.base, t, h0, sc.monitors, ledger_rows=64)
            free1 = _free_bytes()
            assert rc == _lib.ITR_OK, err
            if call == 1:   # the first call may load the module (and with it the static array)
                assert free1 == free0, f"the call changed free device memory by {free0 - free1} bytes"
            what = f"static call {call}"
            assert R.steps == r.steps, f"{what}: steps {R.steps} vs {r.steps}"
            assert R.t_end == r.t_end and R.sync_count == r.sync_count and R.status == r.status, what
            assert R.cell_updates == r.cell_updates, what
            assert_bitwise(out["depth"], r.depth, f"{what}: final depth")
            assert_bitwise(out["peak"], r.peak, f"{what}: per-cell peak")
            np.testing.assert_array_equal(out["monitor_max"], r.monitor_max, err_msg=f"{what}: monitor maxima")
            assert R.rel_residual == r.rel_residual, what
            assert R.n_rows == len(r.ledger), what
            np.testing.assert_array_equal(out["ledger"], r.ledger, err_msg=f"{what}: ledger")
            assert R.steps == rb.steps and R.t_end == rb.t_end, f"{what}: vs batched"
            assert_bitwise(out["depth"], rb.depth, f"{what}: final depth vs batched")
            assert_bitwise(out["peak"], rb.peak, f"{what}: per-cell peak vs batched")
            np.testing.assert_array_equal(out["monitor_max"], rb.monitor_max, err_msg=f"{what}: monitor maxima vs batched")
            assert R.steps == o["steps"] and R.t_end == o["t_end"], f"{what}: vs oracle"
            assert_bitwise(out["depth"], o["h"], f"{what}: final depth vs oracle")
            assert_bitwise(out["peak"], o["peak"], f"{what}: per-cell peak vs oracle")
            np.testing.assert_array_equal(out["monitor_max"], o["monitor_max"], err_msg=f"{what}: monitor maxima vs oracle")
