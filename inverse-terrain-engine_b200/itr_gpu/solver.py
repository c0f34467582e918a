"""Host side of the drop-in boundary: GpuSolver / BatchBackend over the C ABI.

Mirrors the reference's interface for the batch evaluator path:
  GpuSolver::new / adapter_info / run_batch      crates/itr-gpu/src/lib.rs:85,126,149
  GpuRun {monitor_max, steps, t_end, volume_m3, depth, bad}   lib.rs:49-60
  trait BatchBackend<f32> {name, run} -> BatchRun              crates/itr-opt/src/evaluator.rs:117-135
  Gpu(GpuSolver) as BatchBackend                               crates/itr-cli/src/backend.rs:44-63
`run_batch` raises UnsupportedError where the reference returns Err(String) ("unsupported
here": the evaluator then runs that level on the CPU, evaluator.rs:231-238).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .terrain import PreparedTerrain, TerrainBase


class UnsupportedError(RuntimeError):
    """run_batch declined the inputs (the reference's Err(String))."""


class DeviceError(RuntimeError):
    pass


@dataclass
class Hyetograph:
    """Piecewise-linear rate (scenario.rs:526-586); pts are (t [s], rate [m/s])."""
    pts: list[tuple[float, float]] = field(default_factory=list)

    @staticmethod
    def from_mm_h(pairs) -> "Hyetograph":
        return Hyetograph([(float(t), float(r) / 1000.0 / 3600.0) for t, r in pairs])

    def rate(self, t: float) -> float:
        p = self.pts
        if not p:
            return 0.0
        if t <= p[0][0]:
            return p[0][1]
        for (t0, r0), (t1, r1) in zip(p[:-1], p[1:]):
            if t <= t1:
                if t1 == t0:
                    return r1
                return r0 + (r1 - r0) * (t - t0) / (t1 - t0)
        return p[-1][1]

    def integral(self, a: float, b: float) -> float:
        if b <= a or not self.pts:
            return 0.0
        total, tt, rr = 0.0, a, self.rate(a)
        for tk, _ in self.pts:
            if a < tk < b:
                rk = self.rate(tk)
                total += 0.5 * (rr + rk) * (tk - tt)
                tt, rr = tk, rk
        rb = self.rate(b)
        return total + 0.5 * (rr + rb) * (b - tt)


@dataclass
class SolverParams:
    """SolverParams (crates/itr-hydro/src/solver.rs:27-49), reference defaults (scenario.rs:334-345)."""
    duration_s: float
    sync_interval_s: float = 60.0
    cfl: float = 0.35
    dt_max_s: float = 5.0
    h_dry: float = 1e-6
    h_eps: float = 1e-5
    rain: Hyetograph = field(default_factory=Hyetograph)
    infil_capacity: float = 0.0
    initial_depth: float = 0.0
    initial_stage: float | None = None
    skip_dry: bool = True
    inflow_scale: float = 1.0
    # Baseline-locked dt (solver.rs:42-46): the baseline's dt per step, each verified against
    # cfl_hard; on a violation the run restarts adaptively from the last sync snapshot.
    locked_dt: np.ndarray | None = None
    cfl_hard: float = 0.5

    def vector(self) -> np.ndarray:
        """The 12-number parameter vector the CPU oracle takes."""
        return np.array([self.duration_s, self.sync_interval_s, self.cfl, self.dt_max_s, self.h_dry, self.h_eps,
                         self.infil_capacity, self.initial_depth, 1.0 if self.initial_stage is not None else 0.0,
                         self.initial_stage or 0.0, 1.0 if self.skip_dry else 0.0, self.inflow_scale], dtype=np.float64)


@dataclass
class MonitorSet:
    """Sorted unique interior cell ids, row * nx + col (model.rs:6-24)."""
    cells: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.uint32))

    def __post_init__(self):
        self.cells = np.unique(np.asarray(self.cells, dtype=np.uint32))

    @staticmethod
    def all(nx, ny) -> "MonitorSet":
        return MonitorSet(np.arange(nx * ny, dtype=np.uint32))

    def position(self, cell: int) -> int:
        i = int(np.searchsorted(self.cells, cell))
        if i < len(self.cells) and self.cells[i] == cell:
            return i
        raise KeyError(cell)


@dataclass
class Asset:
    name: str
    cells: list[int]
    threshold_m: float
    weight: float = 1.0


@dataclass
class ObjectiveDef:
    """ObjectiveDef (objective.rs:17-30) with the scenario defaults (scenario.rs:234-265)."""
    assets: list[Asset]
    guard_cells: list[int]
    guard_tolerance_m: float = 0.02
    tau_m: float = 0.02
    cut_cost: float = 1.0
    fill_cost: float = 1.0
    earth_weight: float = 1e-5
    require_no_offsite_worsening: bool = True


class Objective:
    """Objective (objective.rs:32-150): asset/guard positions in the monitor list."""

    def __init__(self, d: ObjectiveDef):
        self.d = d
        cells = [c for a in d.assets for c in a.cells] + list(d.guard_cells)
        self.monitors = MonitorSet(np.array(cells, dtype=np.uint32))
        self.asset_pos = [[self.monitors.position(c) for c in a.cells] for a in d.assets]
        self.guard_pos = [self.monitors.position(c) for c in d.guard_cells]

    def softplus(self, x: float) -> float:
        from .mathref import softplus
        return softplus(x)

    def evaluate(self, monitor_max, cut_m3: float, fill_m3: float, baseline_max=None) -> dict:
        """Objective::evaluate (objective.rs:94-128)."""
        d = self.d
        j_risk = 0.0
        peaks = []
        for a, pos in zip(d.assets, self.asset_pos):
            pk = 0.0
            for k in pos:
                pk = max(pk, float(monitor_max[k]))
            peaks.append(pk)
            j_risk += a.weight * d.tau_m * self.softplus((pk - a.threshold_m) / d.tau_m)
        j_earth = d.cut_cost * cut_m3 + d.fill_cost * fill_m3
        rep = {"j": j_risk + d.earth_weight * j_earth, "j_risk": j_risk, "j_earth": j_earth, "peaks": peaks,
               "guard_violation_m": 0.0, "guard_max_worsening_m": 0.0}
        if baseline_max is not None:
            worst = 0.0
            for k in self.guard_pos:
                worst = max(worst, float(monitor_max[k]) - float(baseline_max[k]))
            rep["guard_max_worsening_m"] = worst
            if d.require_no_offsite_worsening and worst > d.guard_tolerance_m:
                rep["guard_violation_m"] = worst - d.guard_tolerance_m
        rep["feasible"] = rep["guard_violation_m"] == 0.0
        return rep


@dataclass
class GpuRun:
    """GpuRun (lib.rs:49-60) plus the outputs the reference's GPU path lacks."""
    monitor_max: np.ndarray
    steps: int
    t_end: float
    volume_m3: float
    depth: np.ndarray | None
    bad: bool
    status: int = 0
    peak: np.ndarray | None = None
    ledger: np.ndarray | None = None
    breach_cell: int = 0
    breach_sync: int = 0
    violation: float = 0.0
    lower_bound: float = 0.0
    j: float = 0.0
    feasible: bool = True
    sync_count: int = 0
    rel_residual: float = 0.0
    cell_updates: int = 0
    dj_ddzx: np.ndarray | None = None   # itr_gpu_vjp: dJ/d(x-face jump), (ny, nx+1)
    dj_ddzy: np.ndarray | None = None   # itr_gpu_vjp: dJ/d(y-face jump), (ny+1, nx)
    warm_start_steps: int = 0           # steps taken over from the baseline record
    dj_ddzx2: np.ndarray | None = None  # itr_gpu_vjp_crest: dJ/d(second x-face jump)
    dj_ddzy2: np.ndarray | None = None
    dt_fallback_t: float = -1.0         # locked dt: time of the snapshot the run fell back to (-1: none)
    rows_skipped: int = 0               # dry rows skipped (RunSummary::rows_skipped)


@dataclass
class BatchRun:
    """BatchRun (evaluator.rs:117-125)."""
    monitor_max: np.ndarray
    steps: int
    cell_updates: int
    bad: bool


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


def _z_edges(base, terrains):
    """Per-design z levels behind the boundary cells, needed when the grid has stage cells."""
    return [t.z_edge() for t in terrains] if getattr(base, "has_stage", False) else None


class GpuSolver:
    """GpuSolver (lib.rs:62-373) on a B200 through libitr_gpu.so."""

    def __init__(self, device: int = -1, impl: str = "batched"):
        self.lib = _lib.load()
        err = C.create_string_buffer(512)
        self.ctx = self.lib.itr_gpu_create(device, err, 512)
        if not self.ctx:
            raise DeviceError(f"itr_gpu_create failed: {err.value.decode()}")
        self.set_option("impl", 0 if impl == "batched" else 1)
        self.last_cell_updates = 0

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.itr_gpu_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def adapter_info(self) -> str:
        buf = C.create_string_buffer(512)
        self.lib.itr_gpu_info(self.ctx, buf, 512)
        return buf.value.decode()

    def set_option(self, key: str, value: int):
        rc = self.lib.itr_gpu_set_option(self.ctx, key.encode(), int(value))
        if rc != 0:
            raise ValueError(self.lib.itr_gpu_last_error(self.ctx).decode())

    def last_timing(self):
        k, t = C.c_double(), C.c_double()
        cu, nl = C.c_uint64(), C.c_int32()
        self.lib.itr_gpu_last_timing(self.ctx, C.byref(k), C.byref(t), C.byref(cu), C.byref(nl))
        return {"kernel_ms": k.value, "total_ms": t.value, "cell_updates": cu.value, "launches": nl.value}

    def rerun_resident(self):
        rc = self.lib.itr_gpu_rerun_resident(self.ctx)
        if rc != 0:
            raise DeviceError(self.lib.itr_gpu_last_error(self.ctx).decode())

    def run_batch(self, p: SolverParams, terrains: list[PreparedTerrain], monitors: MonitorSet, objective: Objective | None = None,
                  baseline_max=None, guard_abort: bool = False, incumbent: float | None = None, want_peak: bool = False,
                  want_depth: bool = True, ledger_rows: int = 0) -> list[GpuRun]:
        """GpuSolver::run_batch (lib.rs:149): all candidates share one TerrainBase."""
        if not terrains:
            return []
        base: TerrainBase = terrains[0].base
        for t in terrains:
            if t.base is not base:
                raise UnsupportedError("all candidates must share the same TerrainBase")
        return self.run_arrays(p, base, [t.dzx for t in terrains], [t.dzy for t in terrains],
                               [t.dzx2 for t in terrains], [t.dzy2 for t in terrains],
                               [t.initial_depth(p.initial_depth, p.initial_stage) if p.initial_stage is not None else None for t in terrains],
                               [(t.cut_m3, t.fill_m3) for t in terrains], monitors, objective, baseline_max, guard_abort,
                               incumbent, want_peak, want_depth, ledger_rows, z_edge=_z_edges(base, terrains))

    def vjp(self, p: SolverParams, terrains: list[PreparedTerrain], monitors: MonitorSet, objective: Objective,
            checkpoint_interval: int = 128, want_peak: bool = False) -> list[GpuRun]:
        """Forward runs plus dJ/d(face jump) per design (itr_gpu_vjp)."""
        base: TerrainBase = terrains[0].base
        return self.run_arrays(p, base, [t.dzx for t in terrains], [t.dzy for t in terrains],
                               [t.dzx2 for t in terrains], [t.dzy2 for t in terrains],
                               [t.initial_depth(p.initial_depth, p.initial_stage) if p.initial_stage is not None else None for t in terrains],
                               [(t.cut_m3, t.fill_m3) for t in terrains], monitors, objective, want_peak=want_peak,
                               want_depth=True, vjp_interval=checkpoint_interval, z_edge=_z_edges(base, terrains))

    def last_vjp_timing(self) -> dict:
        f, b = C.c_double(), C.c_double()
        self.lib.itr_gpu_last_vjp_timing(self.ctx, C.byref(f), C.byref(b))
        return {"forward_ms": f.value, "backward_ms": b.value}

    def _params(self, p: SolverParams, keep: list):
        # the locked dt schedule lives on the context: set (or clear) it for this call
        sched = None if p.locked_dt is None else np.ascontiguousarray(p.locked_dt, dtype=np.float64)
        keep.append(sched)
        rc = self.lib.itr_gpu_set_locked_dt(self.ctx, _ptr(sched, C.c_double) if sched is not None and len(sched) else None,
                                            0 if sched is None else len(sched), float(p.cfl_hard))
        self._check(rc, "itr_gpu_set_locked_dt")
        rain_t = np.ascontiguousarray([q[0] for q in p.rain.pts] or [0.0], dtype=np.float64)
        rain_r = np.ascontiguousarray([q[1] for q in p.rain.pts] or [0.0], dtype=np.float64)
        keep += [rain_t, rain_r]
        return _lib.Params(p.duration_s, p.sync_interval_s, p.cfl, p.dt_max_s, p.h_dry, p.h_eps,
                           _ptr(rain_t, C.c_double), _ptr(rain_r, C.c_double), len(p.rain.pts), p.infil_capacity,
                           p.initial_depth, 1 if p.skip_dry else 0, p.inflow_scale)

    @staticmethod
    def _grid(base, arr) -> "_lib.Grid":
        """itr_grid of a TerrainBase, with its stage and inflow tables when it has such cells."""
        wet, gn2, bc = arr(base.wet, np.float32), arr(base.gn2, np.float32), arr(base.bc, np.uint8)
        Gd = _lib.Grid(base.nx, base.ny, base.dx, base.dy, base.g, base.mode, _ptr(wet, C.c_float), _ptr(gn2, C.c_float),
                       _ptr(bc, C.c_uint8), base.wet_count)
        if getattr(base, "has_stage", False):
            Gd.bc_stage = _ptr(arr(base.bc_stage, np.float64), C.c_double)
        if getattr(base, "has_inflow", False):
            hy = base.hydrographs
            Gd.bc_hydro = _ptr(arr(base.bc_inflow, np.int32), C.c_int32)
            Gd.bc_inv_len = _ptr(arr(base.bc_inv_len, np.float64), C.c_double)
            Gd.n_hydro = len(hy)
            Gd.hydro_off = _ptr(arr(np.cumsum([0] + [len(h) for h in hy]), np.int32), C.c_int32)
            Gd.hydro_t = _ptr(arr([q[0] for h in hy for q in h] or [0.0], np.float64), C.c_double)
            Gd.hydro_q = _ptr(arr([q[1] for h in hy for q in h] or [0.0], np.float64), C.c_double)
        return Gd

    def _pack(self, base, dzx, dzy, dzx2, dzy2, h0, vols, monitors: MonitorSet, objective, baseline_max, guard_abort,
              incumbent, want_peak, want_depth, ledger_rows, keep: list, z_edge=None) -> dict:
        """ctypes views of one batch (grid, designs, monitors, objective, result slots)."""
        n = len(dzx)
        nx, ny = base.nx, base.ny

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a

        Gd = self._grid(base, arr)
        D = (_lib.Design * max(n, 1))()
        for i in range(n):
            a = arr(dzx[i], np.float32) if dzx[i] is not None else None
            b = arr(dzy[i], np.float32) if dzy[i] is not None else None
            a2 = arr(dzx2[i], np.float32) if dzx2 and dzx2[i] is not None else None
            b2 = arr(dzy2[i], np.float32) if dzy2 and dzy2[i] is not None else None
            hh = arr(h0[i], np.float32) if h0 and h0[i] is not None else None
            cut, fill = vols[i] if vols else (0.0, 0.0)
            ze = arr(z_edge[i], np.float64) if z_edge and z_edge[i] is not None else None
            D[i] = _lib.Design(_ptr(a, C.c_float), _ptr(b, C.c_float), _ptr(a2, C.c_float), _ptr(b2, C.c_float),
                               _ptr(hh, C.c_float), cut, fill, _ptr(ze, C.c_double))
        mon = arr(monitors.cells, np.uint32)
        nm = len(mon)
        O = None
        if objective is not None:
            d = objective.d
            off = arr(np.cumsum([0] + [len(a) for a in objective.asset_pos]), np.int32)
            pos = arr([k for a in objective.asset_pos for k in a] or [0], np.int32)
            thr = arr([a.threshold_m for a in d.assets] or [0.0], np.float64)
            wts = arr([a.weight for a in d.assets] or [0.0], np.float64)
            gp = arr(objective.guard_pos or [0], np.int32)
            bl = arr(baseline_max, np.float64) if baseline_max is not None else None
            O = _lib.Objective(len(d.assets), _ptr(off, C.c_int32), _ptr(pos, C.c_int32), _ptr(thr, C.c_double),
                               _ptr(wts, C.c_double), len(objective.guard_pos), _ptr(gp, C.c_int32), _ptr(bl, C.c_double),
                               d.guard_tolerance_m, d.tau_m, d.cut_cost, d.fill_cost, d.earth_weight,
                               1 if d.require_no_offsite_worsening else 0, 1 if guard_abort else 0,
                               1 if incumbent is not None else 0, float(incumbent or 0.0))
            keep.append(O)
        R = (_lib.Result * max(n, 1))()
        outs = []
        for i in range(n):
            mm = np.zeros(max(nm, 1), dtype=np.float64)
            pk = np.zeros(nx * ny, dtype=np.float32) if want_peak else None
            dp = np.zeros(nx * ny, dtype=np.float32) if want_depth else None
            lg = np.zeros((max(ledger_rows, 1), 8), dtype=np.float64) if ledger_rows else None
            outs.append((mm, pk, dp, lg))
            R[i].monitor_max = _ptr(mm, C.c_double)
            R[i].peak = _ptr(pk, C.c_float)
            R[i].depth = _ptr(dp, C.c_float)
            R[i].ledger = _ptr(lg, C.c_double)
            R[i].max_rows = ledger_rows
        keep += [Gd, D, R]
        return dict(n=n, nx=nx, ny=ny, base=base, Gd=Gd, D=D, mon=mon, nm=nm, O=O, R=R, outs=outs)

    def _check(self, rc, what):
        if rc == _lib.ITR_UNSUPPORTED:
            raise UnsupportedError(self.lib.itr_gpu_last_error(self.ctx).decode())
        if rc != _lib.ITR_OK:
            raise DeviceError(f"{what} failed ({rc}): {self.lib.itr_gpu_last_error(self.ctx).decode()}")

    @staticmethod
    def _unpack(b: dict, R, gx=None, gy=None) -> list[GpuRun]:
        n, nx, ny, nm, base = b["n"], b["nx"], b["ny"], b["nm"], b["base"]
        area = base.dx * base.dy
        runs = []
        for i in range(n):
            mm, pk, dp, lg = b["outs"][i]
            r = R[i]
            depth = dp.reshape(ny, nx) if dp is not None else None
            runs.append(GpuRun(monitor_max=mm[:nm].copy(), steps=int(r.steps), t_end=float(r.t_end),
                               volume_m3=float(r.volume_m3) if depth is None else float(depth.astype(np.float64).sum() * area),
                               depth=depth, bad=r.status == _lib.RUN_UNHEALTHY, status=int(r.status),
                               peak=pk.reshape(ny, nx) if pk is not None else None,
                               ledger=lg[:r.n_rows].copy() if lg is not None else None, breach_cell=int(r.breach_cell),
                               breach_sync=int(r.breach_sync), violation=float(r.violation), lower_bound=float(r.lower_bound),
                               j=float(r.j), feasible=bool(r.feasible), sync_count=int(r.sync_count),
                               rel_residual=float(r.rel_residual), cell_updates=int(r.cell_updates),
                               warm_start_steps=int(r.warm_start_steps), dt_fallback_t=float(r.dt_fallback_t),
                               rows_skipped=int(r.rows_skipped),
                               dj_ddzx=gx[i] if gx is not None else None, dj_ddzy=gy[i] if gy is not None else None))
        return runs

    def run_arrays(self, p: SolverParams, base, dzx, dzy, dzx2, dzy2, h0, vols, monitors: MonitorSet, objective=None,
                   baseline_max=None, guard_abort=False, incumbent=None, want_peak=False, want_depth=True, ledger_rows=0,
                   vjp_interval: int | None = None, z_edge=None):
        """run_batch on packed per-design arrays (the C ABI's own view); with vjp_interval,
        itr_gpu_vjp instead (the runs then carry dj_ddzx / dj_ddzy)."""
        keep = []   # keep numpy buffers alive for the call
        P = self._params(p, keep)
        b = self._pack(base, dzx, dzy, dzx2, dzy2, h0, vols, monitors, objective, baseline_max, guard_abort, incumbent,
                       want_peak, want_depth, ledger_rows, keep, z_edge)
        n, nx, ny, O, R = b["n"], b["nx"], b["ny"], b["O"], b["R"]
        gx = gy = None
        if vjp_interval:
            if O is None:
                raise ValueError("the adjoint needs an objective")
            gx = np.zeros((n, ny, nx + 1), dtype=np.float64)
            gy = np.zeros((n, ny + 1, nx), dtype=np.float64)
            if base.mode == _lib.FACE_CREST:   # itr_gpu_vjp_crest: both jumps of every face
                gx2 = np.zeros_like(gx)
                gy2 = np.zeros_like(gy)
                rc = self.lib.itr_gpu_vjp_crest(self.ctx, C.byref(P), C.byref(b["Gd"]), n, b["D"], _ptr(b["mon"], C.c_uint32),
                                                b["nm"], C.byref(O), int(vjp_interval), R, _ptr(gx, C.c_double),
                                                _ptr(gy, C.c_double), _ptr(gx2, C.c_double), _ptr(gy2, C.c_double))
            else:
                rc = self.lib.itr_gpu_vjp(self.ctx, C.byref(P), C.byref(b["Gd"]), n, b["D"], _ptr(b["mon"], C.c_uint32),
                                          b["nm"], C.byref(O), int(vjp_interval), R, _ptr(gx, C.c_double), _ptr(gy, C.c_double))
        else:
            rc = self.lib.itr_gpu_run_batch(self.ctx, C.byref(P), C.byref(b["Gd"]), n, b["D"], _ptr(b["mon"], C.c_uint32),
                                            b["nm"], C.byref(O) if O is not None else None, R)
        self._check(rc, "itr_gpu_run_batch")
        runs = self._unpack(b, R, gx, gy)
        if vjp_interval and base.mode == _lib.FACE_CREST:
            for i, r in enumerate(runs):
                r.dj_ddzx2, r.dj_ddzy2 = gx2[i], gy2[i]
        self.last_cell_updates = sum(r.cell_updates for r in runs)
        return runs

    def _space(self, base, designs, editable, max_abs_dz, keep):
        if base.level != 1:
            raise UnsupportedError("designs as primitives need a fidelity level 1 terrain")
        flat = [q for d in designs for q in d]
        prims = (_lib.Primitive * max(len(flat), 1))()
        for k, q in enumerate(flat):
            prims[k] = _lib.Primitive(int(q.kind), q.cx, q.cy, q.length, q.width, q.angle_deg, q.height)
        off = np.ascontiguousarray(np.cumsum([0] + [len(d) for d in designs]), dtype=np.int32)
        fine = base.fine
        z = np.ascontiguousarray(base.z, dtype=np.float64)
        wall = np.ascontiguousarray(base.wall, dtype=np.uint8)
        ed = np.ascontiguousarray(editable, dtype=np.uint8)
        keep += [off, z, wall, ed, prims]
        S = _lib.DesignSpace(fine.geo.origin_x, fine.geo.origin_y, _ptr(z, C.c_double), _ptr(wall, C.c_uint8),
                             _ptr(ed, C.c_uint8), fine.z_wall, max_abs_dz)
        keep.append(S)
        return S, off, prims

    def vjp_primitives(self, p: SolverParams, base, designs, monitors: MonitorSet, objective, editable, max_abs_dz: float,
                       checkpoint_interval: int = 128):
        """itr_gpu_vjp_primitives: forward runs of designs given as primitives, and
        dJ/d(height, width, length) of every primitive from the design chain on the device.
        Returns (runs with dj_ddzx / dj_ddzy, [per design an array (n_prims, 3)])."""
        if p.initial_stage is not None:
            raise UnsupportedError("designs as primitives start from initial_depth (no initial stage)")
        keep = []
        P = self._params(p, keep)
        n = len(designs)
        S, off, prims = self._space(base, designs, editable, max_abs_dz, keep)
        b = self._pack(base, [None] * n, [None] * n, None, None, None, None, monitors, objective, None, False, None,
                       False, True, 0, keep)
        nx, ny = base.nx, base.ny
        gx = np.zeros((n, ny, nx + 1))
        gy = np.zeros((n, ny + 1, nx))
        gp = np.zeros(max(3 * int(off[-1]), 1))
        rc = self.lib.itr_gpu_vjp_primitives(self.ctx, C.byref(P), C.byref(b["Gd"]), C.byref(S), n, _ptr(off, C.c_int32), prims,
                                             _ptr(b["mon"], C.c_uint32), b["nm"], C.byref(b["O"]), int(checkpoint_interval),
                                             b["R"], _ptr(gp, C.c_double), _ptr(gx, C.c_double), _ptr(gy, C.c_double))
        self._check(rc, "itr_gpu_vjp_primitives")
        runs = self._unpack(b, b["R"], gx, gy)
        return runs, [gp[3 * off[d]:3 * off[d + 1]].reshape(-1, 3) for d in range(n)]

    def render_map(self, z, value, cell_size: float, mode: int = 0, vex: float = 1.0, scale: int = 1, worse_dz=None):
        """itr_gpu_render_map: the result viewer's map of `value` (depth, mode 0, or depth
        difference, mode 1) over the hillshaded terrain z, as an RGBA uint8 image of shape
        (scale ny, scale nx, 4), row 0 north."""
        z = np.ascontiguousarray(z, dtype=np.float32)
        ny, nx = z.shape
        v = np.ascontiguousarray(value, dtype=np.float32).reshape(ny, nx)
        w = None if worse_dz is None else np.ascontiguousarray(worse_dz, dtype=np.float32).reshape(ny, nx)
        out = np.zeros((ny * scale, nx * scale, 4), dtype=np.uint8)
        rc = self.lib.itr_gpu_render_map(self.ctx, nx, ny, float(cell_size), _ptr(z, C.c_float), _ptr(v, C.c_float),
                                         _ptr(w, C.c_float), int(mode), float(vex), int(scale), _ptr(out, C.c_uint8))
        self._check(rc, "itr_gpu_render_map")
        return out

    def render_scene(self, terrain_rgba, depth_rgba, vel_rgba, view, width: int, height: int) -> np.ndarray:
        """itr_gpu_render_scene: the video's ray-marched frame (video/src/shaders/terrain.sksl) of
        the textures (itr_gpu.scene_render builds them) under `view` (a SceneView), as an RGBA
        uint8 image of shape (height, width, 4), row 0 the top."""
        t = np.ascontiguousarray(terrain_rgba, dtype=np.uint8)
        d = np.ascontiguousarray(depth_rgba, dtype=np.uint8)
        v = np.ascontiguousarray(vel_rgba, dtype=np.uint8)
        th, tw = t.shape[:2]
        ny, nx = d.shape[:2]
        if v.shape[:2] != (ny, nx):
            raise ValueError("depth and velocity textures must have the same size")
        out = np.zeros((height, width, 4), dtype=np.uint8)
        V = view.to_c()
        rc = self.lib.itr_gpu_render_scene(self.ctx, _ptr(t, C.c_uint8), tw, th, _ptr(d, C.c_uint8), _ptr(v, C.c_uint8),
                                           nx, ny, C.byref(V), int(width), int(height), _ptr(out, C.c_uint8))
        self._check(rc, "itr_gpu_render_scene")
        return out

    def record_baseline(self, p: SolverParams, terrain: PreparedTerrain, monitors: MonitorSet, checkpoint_interval: int = 64,
                        want_peak: bool = False, ledger_rows: int = 0) -> GpuRun:
        """itr_gpu_record_baseline: run the unedited terrain with checkpoints every
        checkpoint_interval steps; with set_option("warm_start", 1) later batches on the same
        grid and params start each design from the latest checkpoint where that is exact."""
        keep = []
        P = self._params(p, keep)
        h0 = [terrain.initial_depth(p.initial_depth, p.initial_stage)] if p.initial_stage is not None else None
        b = self._pack(terrain.base, [terrain.dzx], [terrain.dzy], [terrain.dzx2], [terrain.dzy2], h0,
                       [(terrain.cut_m3, terrain.fill_m3)], monitors, None, None, False, None, want_peak, True, ledger_rows,
                       keep, _z_edges(terrain.base, [terrain]))
        rc = self.lib.itr_gpu_record_baseline(self.ctx, C.byref(P), C.byref(b["Gd"]), b["D"], _ptr(b["mon"], C.c_uint32),
                                              b["nm"], int(checkpoint_interval), b["R"])
        self._check(rc, "itr_gpu_record_baseline")
        return self._unpack(b, b["R"])[0]

    def run_primitives(self, p: SolverParams, base, designs, monitors: MonitorSet, editable, max_abs_dz: float,
                       objective=None, baseline_max=None, guard_abort=False, incumbent=None, want_peak=False,
                       want_depth=True, ledger_rows=0):
        """run_batch with every design given as its primitives (itr_gpu_run_primitives): the
        device materialises dz, the edited levels, the face jumps and the earthwork volumes
        (DesignSpace::materialize + PreparedTerrain::apply_edit) for a level-1 TerrainBase.
        Returns (runs, cut_m3, fill_m3)."""
        if p.initial_stage is not None:
            raise UnsupportedError("designs as primitives start from initial_depth (no initial stage)")
        keep = []
        P = self._params(p, keep)
        n = len(designs)
        S, off, prims = self._space(base, designs, editable, max_abs_dz, keep)
        b = self._pack(base, [None] * n, [None] * n, None, None, None, None, monitors, objective, baseline_max, guard_abort,
                       incumbent, want_peak, want_depth, ledger_rows, keep)
        cut = np.zeros(max(n, 1))
        fill = np.zeros(max(n, 1))
        O = b["O"]
        rc = self.lib.itr_gpu_run_primitives(self.ctx, C.byref(P), C.byref(b["Gd"]), C.byref(S), n, _ptr(off, C.c_int32),
                                             prims, _ptr(b["mon"], C.c_uint32), b["nm"],
                                             C.byref(O) if O is not None else None, b["R"], _ptr(cut, C.c_double),
                                             _ptr(fill, C.c_double))
        self._check(rc, "itr_gpu_run_primitives")
        runs = self._unpack(b, b["R"])
        self.last_cell_updates = sum(r.cell_updates for r in runs)
        return runs, cut[:n], fill[:n]

    def run_ladder(self, p: SolverParams, groups: list[dict], want_peak=False, want_depth=False) -> list[list[GpuRun]]:
        """itr_gpu_run_ladder: several grid groups (each a dict with terrains, monitors and
        optionally objective, baseline_max, guard_abort, incumbent) in one graph launch."""
        keep = []
        P = self._params(p, keep)
        packs = []
        for g in groups:
            ts = g["terrains"]
            base = ts[0].base
            packs.append(self._pack(base, [t.dzx for t in ts], [t.dzy for t in ts], [t.dzx2 for t in ts], [t.dzy2 for t in ts],
                                    [t.initial_depth(p.initial_depth, p.initial_stage) if p.initial_stage is not None else None for t in ts],
                                    [(t.cut_m3, t.fill_m3) for t in ts], g["monitors"], g.get("objective"), g.get("baseline_max"),
                                    g.get("guard_abort", False), g.get("incumbent"), want_peak, want_depth, 0, keep,
                                    _z_edges(base, ts)))
        total = sum(b["n"] for b in packs)
        R = (_lib.Result * total)()
        k = 0
        for b in packs:                       # the result slots of each group, contiguous
            for i in range(b["n"]):
                R[k + i] = b["R"][i]
            k += b["n"]
        G = (_lib.Group * len(packs))()
        for gi, b in enumerate(packs):
            G[gi] = _lib.Group(C.pointer(b["Gd"]), b["n"], b["D"], _ptr(b["mon"], C.c_uint32), b["nm"],
                               C.pointer(b["O"]) if b["O"] is not None else None)
        rc = self.lib.itr_gpu_run_ladder(self.ctx, C.byref(P), len(packs), G, R)
        self._check(rc, "itr_gpu_run_ladder")
        out, k = [], 0
        for b in packs:
            out.append(self._unpack(b, R[k:k + b["n"]]))
            k += b["n"]
        self.last_cell_updates = sum(r.cell_updates for g in out for r in g)
        return out


class GpuBackend:
    """BatchBackend<f32> over GpuSolver, as the CLI's Gpu wrapper (backend.rs:44-63)."""

    def __init__(self, solver: GpuSolver | None = None):
        self.solver = solver or GpuSolver()

    def name(self) -> str:
        return f"gpu ({self.solver.adapter_info()})"

    def run(self, p: SolverParams, terrains: list[PreparedTerrain], monitors: MonitorSet) -> list[BatchRun]:
        cells = terrains[0].base.nx * terrains[0].base.ny if terrains else 0
        return [BatchRun(r.monitor_max, r.steps, r.steps * cells, r.bad)
                for r in self.solver.run_batch(p, terrains, monitors, want_depth=False)]
