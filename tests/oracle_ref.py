"""ctypes wrapper of oracle/liboracle.so — the CPU oracle (test infrastructure only).

Builds the library on first use if it is missing (make -C oracle). Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE_DIR, "liboracle.so")

_d = C.POINTER(C.c_double)
_f = C.POINTER(C.c_float)
_u8 = C.POINTER(C.c_uint8)
_i64 = C.POINTER(C.c_int64)
_u32 = C.POINTER(C.c_uint32)

_lib = None

VALIDATION_CASES = ["lake_at_rest", "rain_closed_plain", "dam_break_ritter", "wet_dry_step", "tilted_plane_kinematic",
                    "gauge_invariance", "walls_under_rain", "inflow_ledger"]

ABORT_NONE, ABORT_GUARD, ABORT_INCUMBENT, ABORT_UNHEALTHY = 0, 1, 2, 3


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    L = C.CDLL(LIB)
    L.orc_rcbrt32.restype = C.c_float; L.orc_rcbrt32.argtypes = [C.c_float]
    L.orc_rcbrt64.restype = C.c_double; L.orc_rcbrt64.argtypes = [C.c_double]
    for n in ("orc_exp", "orc_log1p", "orc_softplus"):
        getattr(L, n).restype = C.c_double
        getattr(L, n).argtypes = [C.c_double]
    L.orc_hyeto_integral.restype = C.c_double
    L.orc_hyeto_integral.argtypes = [_d, _d, C.c_int, C.c_double, C.c_double]
    L.orc_hyeto_rate.restype = C.c_double
    L.orc_hyeto_rate.argtypes = [_d, _d, C.c_int, C.c_double]
    L.orc_fixedsum32.restype = C.c_float; L.orc_fixedsum32.argtypes = [_f, C.c_int]
    L.orc_fixedsum64.restype = C.c_double; L.orc_fixedsum64.argtypes = [_d, C.c_int]
    L.orc_profile.restype = C.c_double; L.orc_profile.argtypes = [_d, C.c_double, C.c_double]
    L.orc_materialize.restype = C.c_int64
    L.orc_materialize.argtypes = [_d, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int64, C.c_int64, _u8,
                                  C.c_double, _i64, _d, _d]
    L.orc_scene_new.restype = C.c_void_p
    L.orc_scene_new.argtypes = [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double, _d, _u8, _d, C.c_int64,
                                C.c_int, _d, _d, _i64, _d, _d]
    L.orc_scene_free.argtypes = [C.c_void_p]
    L.orc_scene_info.argtypes = [C.c_void_p, _i64, _d]
    L.orc_scene_pack32.argtypes = [C.c_void_p, _i64, _d, _f, _f, _f, _f, _f, _f, _d]
    L.orc_scene_bc.argtypes = [C.c_void_p, _u8]
    run_args = [_d, _d, _d, C.c_int, C.c_int, _u32, C.c_int, _i64, _d, C.c_int, _i64, _i64, _d, _d, _d]
    out_args = [C.c_int, _d, _d, _d, _d, C.c_int, _d, _d, _d, _d, _d]
    L.orc_scene_run.argtypes = [C.c_void_p, C.c_int, C.c_int, _i64, _d, C.c_double, C.c_double] + run_args + [_d] + out_args
    _i32 = C.POINTER(C.c_int32)
    bnd_args = [_d, _i32, _d, C.c_int, _i32, _d, _d, _d]
    L.orc_flat_run.argtypes = ([C.c_int, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int, _f, _f, _u8, _f, _f, _f, _f, _f]
                               + run_args + out_args + bnd_args)
    L.orc_flat_run64.argtypes = ([C.c_int, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int, _d, _d, _u8, _d, _d, _d, _d, _d]
                                 + run_args + out_args + bnd_args)
    L.orc_flat_batch.restype = C.c_double
    L.orc_flat_batch.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_double, C.c_double, _f, _f, _u8, _f, _f, _f, _d, _d,
                                 _d, C.c_int, C.c_int, _u32, _d, _d]
    L.orc_validation.argtypes = [C.c_int, C.c_int, _d]
    L.orc_render_map.argtypes = [C.c_int, C.c_int, C.c_double, _f, _f, _f, C.c_int, C.c_float, C.c_int, _u8]
    L.orc_set_locked_dt.argtypes = [_d, C.c_int64, C.c_double, C.c_int]
    L.orc_render_scene.argtypes = [_u8, C.c_int, C.c_int, _u8, _u8, C.c_int, C.c_int, _f, C.c_int, C.c_int, C.c_int,
                                   C.c_int, _u8]
    L.orc_sin_ref.restype = C.c_double
    L.orc_sin_ref.argtypes = [C.c_double]
    L.orc_powf_ref.restype = C.c_float
    L.orc_powf_ref.argtypes = [C.c_float, C.c_float]
    L.orc_last_locked.restype = C.c_int64
    L.orc_last_locked.argtypes = [_d, _d, C.c_int64]
    _lib = L
    return L


def P(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def validation(prec: int, case: int):
    o = np.zeros(4)
    lib().orc_validation(prec, case, P(o, C.c_double))
    return {"value": o[0], "threshold": o[1], "passed": bool(o[2]), "extra": o[3]}


class Scene:
    """A DEM-described terrain built by the oracle itself (terrain.rs restatement)."""

    def __init__(self, dem, walls, manning, geo, level=1, segments=()):
        L = lib()
        self.ny, self.nx = dem.shape
        dem = np.ascontiguousarray(dem, dtype=np.float64)
        walls = np.ascontiguousarray(walls, dtype=np.uint8)
        man = np.ascontiguousarray(np.broadcast_to(manning, dem.shape), dtype=np.float64)
        sides = {"north": 0, "south": 1, "west": 2, "east": 3}
        kinds = {"stage": 0, "inflow": 1, "transmissive": 2}
        segf, stage, off, ht, hq = [], [], [0], [], []
        for s in segments:
            segf += [kinds[s.kind], sides[s.side], 1.0 if s.range_m else 0.0, *(s.range_m or (0.0, 0.0))]
            stage.append(s.stage_m)
            for t, q in s.hydrograph:
                ht.append(t); hq.append(q)
            off.append(len(ht))
        self._keep = [np.array(segf or [0.0], dtype=np.float64), np.array(stage or [0.0]), np.array(off, dtype=np.int64),
                      np.array(ht or [0.0]), np.array(hq or [0.0])]
        self.h = L.orc_scene_new(self.nx, self.ny, geo.origin_x, geo.origin_y, geo.dx, geo.dy, P(dem, C.c_double),
                                 P(walls, C.c_uint8), P(man, C.c_double), level, len(segments), P(self._keep[0], C.c_double),
                                 P(self._keep[1], C.c_double), P(self._keep[2], C.c_int64), P(self._keep[3], C.c_double),
                                 P(self._keep[4], C.c_double))
        info = np.zeros(4, dtype=np.int64)
        infod = np.zeros(4)
        L.orc_scene_info(self.h, P(info, C.c_int64), P(infod, C.c_double))
        self.lnx, self.lny, self.mode, self.wet_count = (int(v) for v in info)
        self.dx, self.dy, self.z_ref, self.z_wall = infod

    def __del__(self):
        try:
            lib().orc_scene_free(self.h)
        except Exception:
            pass

    def pack(self, edit=None):
        nx, ny = self.lnx, self.lny
        dzx = np.zeros((ny, nx + 1), np.float32); dzy = np.zeros((ny + 1, nx), np.float32)
        dzx2 = np.zeros_like(dzx); dzy2 = np.zeros_like(dzy)
        wet = np.zeros((ny, nx), np.float32); gn2 = np.zeros((ny, nx), np.float32); z = np.zeros((ny, nx))
        bbox, dz = _edit_args(edit)
        lib().orc_scene_pack32(self.h, P(bbox, C.c_int64), P(dz, C.c_double), P(dzx, C.c_float), P(dzy, C.c_float),
                               P(dzx2, C.c_float), P(dzy2, C.c_float), P(wet, C.c_float), P(gn2, C.c_float), P(z, C.c_double))
        bc = np.zeros(2 * nx + 2 * ny, np.uint8)
        lib().orc_scene_bc(self.h, P(bc, C.c_uint8))
        return dict(dzx=dzx, dzy=dzy, dzx2=dzx2, dzy2=dzy2, wet=wet, gn2=gn2, z=z, bc=bc)

    def run(self, params, monitors, prec=0, kernel=1, edit=None, objective=None, baseline=None, incumbent=None,
            h0=None, want_peak=False, max_rows=256):
        bbox, dz = _edit_args(edit)
        cut = edit.cut_m3 if edit is not None else 0.0
        fill = edit.fill_m3 if edit is not None else 0.0
        return _run(lambda *a: lib().orc_scene_run(self.h, prec, kernel, P(bbox, C.c_int64), P(dz, C.c_double), cut, fill, *a),
                    self.lnx, self.lny, params, monitors, objective, baseline, incumbent, cut, fill, h0, want_peak, max_rows,
                    scene=True)


def _edit_args(edit):
    if edit is None or edit.w == 0 or edit.h == 0:
        return None, None
    return np.array([edit.c0, edit.r0, edit.w, edit.h], dtype=np.int64), np.ascontiguousarray(edit.dz, dtype=np.float64)


def _obj_arrays(objective, baseline, incumbent, cut, fill):
    d = objective.d
    off = np.cumsum([0] + [len(a) for a in objective.asset_pos]).astype(np.int64)
    pos = np.array([k for a in objective.asset_pos for k in a] or [0], dtype=np.int64)
    thr = np.array([a.threshold_m for a in d.assets] or [0.0])
    w = np.array([a.weight for a in d.assets] or [0.0])
    gp = np.array(objective.guard_pos or [0], dtype=np.int64)
    objf = np.array([d.guard_tolerance_m, d.tau_m, d.cut_cost, d.fill_cost, d.earth_weight,
                     1.0 if d.require_no_offsite_worsening else 0.0, 1.0 if incumbent is not None else 0.0,
                     float(incumbent or 0.0), cut, fill])
    bl = None if baseline is None else np.ascontiguousarray(baseline, dtype=np.float64)
    return len(objective.guard_pos), gp, bl, len(d.assets), off, pos, thr, w, objf


def _run(call, nx, ny, params, monitors, objective, baseline, incumbent, cut, fill, h0, want_peak, max_rows, scene):
    rain_t = np.array([q[0] for q in params.rain.pts] or [0.0])
    rain_r = np.array([q[1] for q in params.rain.pts] or [0.0])
    pv = params.vector()
    mon = np.ascontiguousarray(monitors.cells, dtype=np.uint32)
    nm = len(mon)
    if objective is not None:
        ng, gp, bl, na, off, pos, thr, w, objf = _obj_arrays(objective, baseline, incumbent, cut, fill)
    else:
        ng, gp, bl, na, off, pos, thr, w, objf = 0, None, None, 0, None, None, None, None, None
    out_s = np.zeros(16)
    mm = np.zeros(max(nm, 1)); mt = np.zeros(max(nm, 1))
    led = np.zeros((max_rows, 8))
    h = np.zeros((ny, nx)); qx = np.zeros((ny, nx)); qy = np.zeros((ny, nx))
    pk = np.zeros((ny, nx)) if want_peak else None
    ps = np.zeros((ny, nx)) if want_peak else None
    if scene:
        h0a = None if h0 is None else np.ascontiguousarray(h0, dtype=np.float64)
        call(P(pv, C.c_double), P(rain_t, C.c_double), P(rain_r, C.c_double), len(params.rain.pts), nm, P(mon, C.c_uint32),
             ng, P(gp, C.c_int64), P(bl, C.c_double), na, P(off, C.c_int64), P(pos, C.c_int64), P(thr, C.c_double),
             P(w, C.c_double), P(objf, C.c_double), P(h0a, C.c_double), 1 if want_peak else 0, P(out_s, C.c_double),
             P(mm, C.c_double), P(mt, C.c_double), P(led, C.c_double), max_rows, P(h, C.c_double), P(qx, C.c_double),
             P(qy, C.c_double), P(pk, C.c_double), P(ps, C.c_double))
    else:
        call(P(pv, C.c_double), P(rain_t, C.c_double), P(rain_r, C.c_double), len(params.rain.pts), nm, P(mon, C.c_uint32),
             ng, P(gp, C.c_int64), P(bl, C.c_double), na, P(off, C.c_int64), P(pos, C.c_int64), P(thr, C.c_double),
             P(w, C.c_double), P(objf, C.c_double), 1 if want_peak else 0, P(out_s, C.c_double),
             P(mm, C.c_double), P(mt, C.c_double), P(led, C.c_double), max_rows, P(h, C.c_double), P(qx, C.c_double),
             P(qy, C.c_double), P(pk, C.c_double), P(ps, C.c_double))
    n_rows = int(out_s[15])
    return dict(t_end=out_s[0], steps=int(out_s[1]), sync_count=int(out_s[2]), abort=int(out_s[3]), abort_cell=int(out_s[4]),
                abort_exceed=out_s[5], abort_sync=int(out_s[6]), abort_lb=out_s[7], v0=out_s[8], rel_residual=out_s[9],
                dt_min=out_s[10], dt_max=out_s[11], dt_mean=out_s[12], cell_updates=int(out_s[13]),
                rows_skipped=int(out_s[14]), monitor_max=mm[:nm].copy(), monitor_tmax=mt[:nm].copy(),
                ledger=led[:min(n_rows, max_rows)].copy(), h=h, qx=qx, qy=qy, peak=pk, peak_step=ps)


def locked(run, locked_dt=None, cfl_hard=0.5, record_dts=False):
    """Calls run() (one oracle run) with SolverParams::locked_dt / cfl_hard set (solver.rs:42-46), and
    adds to its result dict dt_fallback_t (RunSummary::dt_fallback_t, -1 for none) and, with record_dts,
    dts: the dt of every step (BaselineRecord::dts)."""
    L = lib()
    sched = None if locked_dt is None else np.ascontiguousarray(locked_dt, dtype=np.float64)
    L.orc_set_locked_dt(P(sched, C.c_double), 0 if sched is None else len(sched), cfl_hard, 1 if record_dts else 0)
    try:
        r = run()
    finally:
        L.orc_set_locked_dt(None, 0, 0.5, 0)
    fb = C.c_double(-1.0)
    n = L.orc_last_locked(C.byref(fb), None, 0)
    dts = np.zeros(n)
    L.orc_last_locked(C.byref(fb), P(dts, C.c_double), n)
    r["dt_fallback_t"] = fb.value
    if record_dts:
        r["dts"] = dts
    return r


def render_scene(terrain_rgba, depth_rgba, vel_rgba, view, width, height):
    """The video's ray-marched frame restated on the CPU (RGBA uint8, (height, width, 4))."""
    t = np.ascontiguousarray(terrain_rgba, dtype=np.uint8)
    d = np.ascontiguousarray(depth_rgba, dtype=np.uint8)
    v = np.ascontiguousarray(vel_rgba, dtype=np.uint8)
    vf = np.ascontiguousarray(view.floats(), dtype=np.float32)
    out = np.zeros((height, width, 4), dtype=np.uint8)
    lib().orc_render_scene(P(t, C.c_uint8), t.shape[1], t.shape[0], P(d, C.c_uint8), P(v, C.c_uint8), d.shape[1], d.shape[0],
                           P(vf, C.c_float), 1 if view.ortho else 0, int(view.debug), width, height, P(out, C.c_uint8))
    return out


def render_map(z, value, cell_size, mode=0, vex=1.0, scale=1, worse_dz=None):
    """The viewer's map image restated on the CPU (RGBA uint8, (scale ny, scale nx, 4))."""
    z = np.ascontiguousarray(z, dtype=np.float32)
    ny, nx = z.shape
    v = np.ascontiguousarray(value, dtype=np.float32).reshape(ny, nx)
    w = None if worse_dz is None else np.ascontiguousarray(worse_dz, dtype=np.float32).reshape(ny, nx)
    out = np.zeros((ny * scale, nx * scale, 4), dtype=np.uint8)
    lib().orc_render_map(nx, ny, float(cell_size), P(z, C.c_float), P(v, C.c_float), P(w, C.c_float), int(mode), float(vex),
                         int(scale), P(out, C.c_uint8))
    return out


def bnd_dict(base, terrain):
    """Stage and inflow tables of a TerrainBase (itr_grid) with one design's z_edge, or None
    when the grid has walls and transmissive edges only."""
    if not (getattr(base, "has_stage", False) or getattr(base, "has_inflow", False)):
        return None
    return dict(stage=base.bc_stage, hydro=base.bc_inflow, inv_len=base.bc_inv_len, hydros=base.hydrographs,
                z_edge=terrain.z_edge())


def _bnd_args(bnd, keep):
    if bnd is None:
        return (None, None, None, 0, None, None, None, None)
    i32 = C.POINTER(C.c_int32)

    def a(x, dt):
        x = np.ascontiguousarray(x, dtype=dt)
        keep.append(x)
        return x
    hy = bnd["hydros"]
    off = a(np.cumsum([0] + [len(h) for h in hy]), np.int32)
    ht = a([q[0] for h in hy for q in h] or [0.0], np.float64)
    hq = a([q[1] for h in hy for q in h] or [0.0], np.float64)
    return (P(a(bnd["stage"], np.float64), C.c_double), P(a(bnd["hydro"], np.int32), C.c_int32),
            P(a(bnd["inv_len"], np.float64), C.c_double), len(hy), off.ctypes.data_as(i32), P(ht, C.c_double),
            P(hq, C.c_double), P(a(bnd["z_edge"], np.float64), C.c_double))


def flat_run(base_arrays, design, params, monitors, kernel=1, objective=None, baseline=None, incumbent=None,
             want_peak=False, max_rows=256, bnd=None):
    """f32 run on the packed arrays of the GPU ABI: base_arrays = (nx, ny, dx, dy, mode, wet, gn2, bc),
    design = dict(dzx, dzy, dzx2, dzy2, h0, cut, fill), bnd = bnd_dict(...) for stage / inflow cells."""
    nx, ny, dx, dy, mode, wet, gn2, bc = base_arrays
    keep = []

    def f32(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float32)
        keep.append(a)
        return a

    wet, gn2 = f32(wet), f32(gn2)
    bc = np.ascontiguousarray(bc, dtype=np.uint8)
    dzx, dzy, dzx2, dzy2, h0 = (f32(design.get(k)) for k in ("dzx", "dzy", "dzx2", "dzy2", "h0"))
    cut, fill = design.get("cut", 0.0), design.get("fill", 0.0)
    ba = _bnd_args(bnd, keep)
    return _run(lambda *a: lib().orc_flat_run(kernel, nx, ny, dx, dy, mode, P(wet, C.c_float), P(gn2, C.c_float),
                                              P(bc, C.c_uint8), P(dzx, C.c_float), P(dzy, C.c_float), P(dzx2, C.c_float),
                                              P(dzy2, C.c_float), P(h0, C.c_float), *a, *ba),
                nx, ny, params, monitors, objective, baseline, incumbent, cut, fill, None, want_peak, max_rows, scene=False)


def flat_run64(base_arrays, design, params, monitors, kernel=1, objective=None, want_peak=False, max_rows=256, bnd=None):
    """The f64 scalar oracle on the same packed arrays (face jumps taken as f64)."""
    nx, ny, dx, dy, mode, wet, gn2, bc = base_arrays
    keep = []

    def f64(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return a

    wet, gn2 = f64(wet), f64(gn2)
    bc = np.ascontiguousarray(bc, dtype=np.uint8)
    dzx, dzy, dzx2, dzy2, h0 = (f64(design.get(k)) for k in ("dzx", "dzy", "dzx2", "dzy2", "h0"))
    cut, fill = design.get("cut", 0.0), design.get("fill", 0.0)
    ba = _bnd_args(bnd, keep)
    return _run(lambda *a: lib().orc_flat_run64(kernel, nx, ny, dx, dy, mode, P(wet, C.c_double), P(gn2, C.c_double),
                                                P(bc, C.c_uint8), P(dzx, C.c_double), P(dzy, C.c_double), P(dzx2, C.c_double),
                                                P(dzy2, C.c_double), P(h0, C.c_double), *a, *ba),
                nx, ny, params, monitors, objective, None, None, cut, fill, None, want_peak, max_rows, scene=False)


def flat_batch(threads, base_arrays, dzx_all, dzy_all, h0_all, params, monitors):
    """Candidate-parallel f32 fused runs (CPU baseline timing). Returns (wall_s, steps, monitor_max)."""
    nx, ny, dx, dy, mode, wet, gn2, bc = base_arrays
    n = len(dzx_all)
    dzx = np.ascontiguousarray(np.stack(dzx_all), dtype=np.float32)
    dzy = np.ascontiguousarray(np.stack(dzy_all), dtype=np.float32)
    h0 = np.ascontiguousarray(np.stack(h0_all), dtype=np.float32) if h0_all is not None else None
    wet = np.ascontiguousarray(wet, dtype=np.float32); gn2 = np.ascontiguousarray(gn2, dtype=np.float32)
    bc = np.ascontiguousarray(bc, dtype=np.uint8)
    rain_t = np.array([q[0] for q in params.rain.pts] or [0.0]); rain_r = np.array([q[1] for q in params.rain.pts] or [0.0])
    pv = params.vector()
    mon = np.ascontiguousarray(monitors.cells, dtype=np.uint32)
    steps = np.zeros(n); mm = np.zeros(n * max(len(mon), 1))
    wall = lib().orc_flat_batch(threads, n, nx, ny, dx, dy, P(wet, C.c_float), P(gn2, C.c_float), P(bc, C.c_uint8),
                                P(dzx, C.c_float), P(dzy, C.c_float), P(h0, C.c_float), P(pv, C.c_double),
                                P(rain_t, C.c_double), P(rain_r, C.c_double), len(params.rain.pts), len(mon),
                                P(mon, C.c_uint32), P(steps, C.c_double), P(mm, C.c_double))
    return wall, steps.astype(np.int64), mm.reshape(n, max(len(mon), 1))[:, :len(mon)]
