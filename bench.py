#!/usr/bin/env python3
"""Benchmark of the batched forward operator (one JSON line on rank 0).

Workload (one "step"): one population evaluation of the plain batched configuration:
120 x 96 cells at 5 m (rolling hills, 3 Gaussian hills + 2 gullies on a 3% slope), 60 min
storm peaking at 100 mm/h at 20 min, 64 designs of 4 primitives each, run to completion
(abort off), f32 state with f64 time/rain/ledgers. Synthetic, seeded inputs.

  value    cell-steps/s of the batched kernel over inputs already resident in HBM (CUDA
           events on the launching stream, L2 flushed between iterations)
  e2e      the same metric through the public C ABI call (itr_gpu_run_batch) from host
           buffers: packing, host->device copies, kernel, device->host results
  roofline the batched kernel's bound: instruction issue (its state stays in shared memory,
           so DRAM carries only the inputs once). achieved = warp-instructions per
           cell-step (ncu counters of the same kernel, profiles/) x cell-steps/s; peak = SMs x
           4 schedulers x the median SM clock sampled during the timed region. The 32 B/cell-
           step HBM model is reported beside it (roofline.hbm).
  cpu_baseline  the f32 CPU port of the reference's fused kernel (oracle/), candidate-parallel
           on the host cores, on a bounded sample of the same workload

Multi-GPU (torchrun): designs are sharded across ranks with no data-path collective (weak
scaling: every rank runs 64 designs of the population); a barrier brackets the timed
region and the max time over ranks is reported. The e2e leg evaluates the whole population
through itr_gpu.sharding.ShardedBackend, whose one all-gather returns every design's
results to every rank.

--impl reference: the reference cannot be built here (Rust workspace; no cargo/rustc), so
its CPU path is timed through the restatement in oracle/ (f32 fused kernel, all host cores).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "inverse-terrain-engine_b200")
sys.path[:0] = [PKG, os.path.join(ROOT, "tests")]

METRIC = "cell-steps/s (batched forward, 1 design per cluster)"
BYTES_PER_CELL_STEP = 32          # read h,qx,qy + write h,qx,qy (24 B) + dzx,dzy (8 B), spec.md:620
BYTES_PER_CELL_STEP_REF_MODEL = 40  # the reference bench's model incl. wet and gn2, main.rs:696-697


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        import statistics
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) >= 9:
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


COUNTERS = os.path.join(ROOT, "profiles", "k_batched_config2_counters.json")


def kernel_counters():
    """ncu counters of the batched kernel on this workload, committed under profiles/:
    DRAM bytes per launch and warp-instructions issued per cell-step."""
    try:
        with open(COUNTERS) as f:
            return json.load(f)
    except Exception:
        return {}


def issue_roofline(cell_steps, avg_ms, counters, clocks, hbm_achieved, hbm_peak, hbm_src):
    """The batched kernel keeps a design's state in shared memory for the whole storm, so it
    is bound by instruction issue, not HBM: achieved warp-instructions/s = (warp-instructions
    per cell-step, from ncu) x cell-steps/s; peak = SMs x 4 schedulers x 1 instruction per
    clock at the median SM clock of the timed region. The HBM model rides along."""
    import torch
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    ipc = counters.get("warp_inst_per_cell_step")
    rate = cell_steps / (avg_ms / 1e3)
    peak = sms * 4 * mhz * 1e6
    line = {"bound": "issue", "unit": "warp-instr/s", "peak": peak,
            "achieved": ipc * rate if ipc else None, "frac": ipc * rate / peak if ipc else None,
            "traffic": counters.get("dram_bytes_per_launch"),
            "model": (f"{ipc} warp-instructions per cell-step (ncu, {os.path.relpath(COUNTERS, ROOT)}) x "
                      f"{rate:.4g} cell-steps/s; peak {sms} SMs x 4 issue slots x {mhz:.0f} MHz"),
            "sms_used": counters.get("sms_used"),
            "hbm": {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s", "frac": hbm_achieved / hbm_peak,
                    "peak_source": hbm_src,
                    "model": f"{BYTES_PER_CELL_STEP} B/cell-step x {cell_steps:.4g} cell-steps per launch"}}
    if ipc and counters.get("sms_used"):
        line["frac_of_used_sms"] = ipc * rate / (counters["sms_used"] * 4 * mhz * 1e6)
    return line


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        rank = int(os.environ["RANK"])
        local = int(os.environ.get("LOCAL_RANK", rank))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        return rank, world, local
    return 0, 1, 0


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.zeros(1, device="cuda")
        dist.all_reduce(t)
        torch.cuda.synchronize()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def workload(rank=0, n_designs=64, which=2):
    from itr_gpu.scenes import config
    sc = config(which)
    ds = sc.designs(n_designs, seed=sc.design_seed + 1000 * rank)
    return sc, [t for _, _, t in ds]


def cpu_baseline(sc, terrs, budget_s=20.0):
    """f32 fused CPU port, one design per thread on every host core, on a bounded sample:
    the first `dur` seconds of the storm for one design per thread."""
    import oracle_ref as orc
    from helpers import base_arrays
    import copy
    threads = os.cpu_count() or 1
    p = copy.deepcopy(sc.params)
    # calibrate on one design for a short stretch, then size the sample to the budget
    p.duration_s = 240.0
    t0 = time.perf_counter()
    w, steps, _ = orc.flat_batch(1, base_arrays(sc.base), [terrs[0].dzx], [terrs[0].dzy], None, p, sc.monitors)
    rate1 = steps[0] * sc.base.nx * sc.base.ny / max(w, 1e-9)
    n = min(len(terrs), threads)
    # cell-steps the sample may take: budget * threads * single-thread rate
    want = budget_s * rate1 * n * 0.8
    per_design = want / n
    full_steps_guess = 4.0 * steps[0] * (sc.params.duration_s / p.duration_s)
    frac = min(1.0, per_design / max(full_steps_guess * sc.base.nx * sc.base.ny, 1.0))
    p.duration_s = max(120.0, min(sc.params.duration_s, sc.params.duration_s * frac))
    wall, steps, _ = orc.flat_batch(threads, base_arrays(sc.base), [t.dzx for t in terrs[:n]], [t.dzy for t in terrs[:n]], None,
                                    p, sc.monitors)
    cs = float(steps.sum()) * sc.base.nx * sc.base.ny
    return {"value": cs / wall, "unit": "cell-steps/s", "cores": threads, "kind": "port", "value_1_thread": rate1,
            "sample": f"{n} designs x first {p.duration_s:.0f} s of the storm (of {sc.params.duration_s:.0f} s), "
                      f"f32 fused CPU port, candidate-parallel on {threads} threads, {wall:.1f} s wall",
            "cell_steps": cs, "wall_s": wall}


def plain_comparison(g, sc, terrs, n_sample=2):
    """The plain one-design-per-launch CUDA forward (impl 1: per step one tiled update and one
    finalize launch, designs one after another) on the first designs of the same workload,
    full storm; its cell-steps/s does not depend on how many designs it runs in sequence."""
    g.set_option("impl", 1)
    try:
        runs = g.run_batch(sc.params, terrs[:n_sample], sc.monitors, want_depth=False)
        g.rerun_resident()
        tm = g.last_timing()
    finally:
        g.set_option("impl", 0)
    cs = float(sum(r.steps for r in runs)) * sc.base.nx * sc.base.ny
    return {"value": cs / (tm["kernel_ms"] / 1e3), "unit": "cell-steps/s", "designs_sampled": n_sample,
            "launches": tm["launches"], "kernel_ms": tm["kernel_ms"]}


def adjoint_summary(g, K=128, duration=None, which=4, sweep=()):
    """Config 4 (rolling hills 240x192 @2.5 m, 60 min storm, 32 designs x 4 primitives), or
    config 5 (fractal 1024x1024 @2 m, 90 min storm, 16 designs x 6 primitives): the autotuned
    forward against itr_gpu_vjp (taped forward + checkpointed backward), device time, both on
    the second call (the first autotunes and sizes the buffers)."""
    from itr_gpu.scenes import config
    sc = config(which)
    if duration is not None:
        sc.params.duration_s = float(duration)
    n = 32 if which == 4 else 16
    N = sc.base.nx * sc.base.ny
    if which == 5:   # 1024^2: designs as primitives, materialised on the device (same forward)
        prims = sc.primitive_designs(n)
        fwd_call = lambda: g.run_primitives(sc.params, sc.base, prims, sc.monitors, sc.editable, sc.max_abs_dz,  # noqa: E731
                                            objective=sc.objective, want_depth=False)
        vjp_call = lambda k: g.vjp_primitives(sc.params, sc.base, prims, sc.monitors, sc.objective, sc.editable,  # noqa: E731
                                              sc.max_abs_dz, checkpoint_interval=k)[0]
    else:
        terrs = [t for _, _, t in sc.designs(n)]
        fwd_call = lambda: g.run_batch(sc.params, terrs, sc.monitors, objective=sc.objective, want_depth=False)  # noqa: E731
        vjp_call = lambda k: g.vjp(sc.params, terrs, sc.monitors, sc.objective, checkpoint_interval=k)  # noqa: E731
    fwd_call()   # autotune
    fwd_call()
    fwd = g.last_timing()["kernel_ms"]

    def one(k):
        # the first call sizes the context's checkpoint and tape buffers; a search loop reuses them
        vjp_call(k)
        runs = vjp_call(k)
        v = g.last_vjp_timing()
        steps = max(r.steps for r in runs)
        # device memory of the adjoint: a checkpoint of (h, qx, qy) per design every k steps and
        # two tapes of k states (replay of one segment beside the backward of the next)
        ck = -(-steps // k) * n * 12 * N
        tape = 2 * k * n * 12 * N
        return runs, {"checkpoint_interval": k, "vjp_taped_forward_ms": v["forward_ms"], "vjp_backward_ms": v["backward_ms"],
                      "adjoint_over_forward": (v["forward_ms"] + v["backward_ms"]) / fwd,
                      "checkpoint_bytes": ck, "tape_bytes": tape}
    runs, main = one(K)
    cs = float(sum(r.steps for r in runs)) * N
    label = ("config4 rolling hills 240x192 @2.5 m" if which == 4 else "config5 fractal 1024x1024 @2 m")
    out = {"workload": f"{label}, {sc.params.duration_s:.0f} s storm, {n} designs x {sc.n_prims} primitives",
           "forward_ms": fwd, "forward_cell_steps_per_s": cs / (fwd / 1e3), **main,
           "gradient": ("dJ/d(face jump), f32 discrete adjoint with frozen dt; within 1% of f64 central differences on "
                        "config 4's grid, smooth sub-case (tests/test_adjoint.py)")}
    if sweep:
        out["interval_sweep"] = [one(k)[1] for k in sweep]
    return out


def polish_summary(g, duration=900.0, n_pop=16, iters=4):
    """Config 5's search use of the adjoint (fractal 1024x1024 @2 m, the first `duration` s of
    its double-peak storm): a generation of 16 seeded designs of 6 primitives evaluated on the
    device, its best feasible design (the incumbent) polished with itr_gpu_vjp_primitives
    gradients in a trust region, each proposal re-evaluated exactly with itr_gpu_run_primitives
    (guard against the unedited baseline, volume limit). The f32 and f64 oracle reruns of the
    polished incumbent are in tests/test_polish.py (about 2 CPU-minutes each)."""
    from itr_gpu.polish import polish_population
    from itr_gpu.scenes import config
    sc = config(5)
    sc.params.duration_s = float(duration)
    designs = sc.primitive_designs(n_pop)
    r = polish_population(g, sc.params, sc.base, designs, sc.objective, sc.editable, sc.max_abs_dz, max_volume=sc.max_volume,
                          iters=iters)
    res = r.result
    return {"workload": f"config5 fractal 1024x1024 @2 m, first {duration:.0f} s of the storm, {n_pop} designs x 6 primitives",
            "population_feasible": r.feasible, "j_incumbent": res.j_start, "j_polished": res.j, "delta_j": res.j - res.j_start,
            "feasible": res.feasible, "accepted": res.accepted, "exact_evaluations": res.evaluations,
            "history": res.history, "wall_s": r.wall_s}


def ladder_summary(g):
    """Config 3 (uneven batching with early abort): the valley scene at 10, 5 and 2.5 m
    (45x35, 90x70, 180x140), 40 min storm, 3 primitives per design, 256 designs split
    128 / 96 / 32, guard and incumbent abort live (incumbent = best J of the previous batch,
    frozen for this one), all groups in one CUDA graph launch (itr_gpu_run_ladder)."""
    from itr_gpu import PreparedTerrain
    from itr_gpu.scenes import valley_scene
    spec, p = [], None
    for cell, n in ((10.0, 128), (5.0, 96), (2.5, 32)):
        sc = valley_scene(cell, n_prims=3)
        sc.params.duration_s = 2400.0
        p = sc.params
        ts = [t for _, _, t in sc.designs(n)]
        prev = [t for _, _, t in sc.designs(n, seed=sc.design_seed + 500)]   # the previous batch
        base = g.run_batch(p, [PreparedTerrain(sc.base)], sc.monitors)[0]
        inc = min(r.j for r in g.run_batch(p, prev, sc.monitors, objective=sc.objective, want_depth=False))
        spec.append(dict(terrains=ts, monitors=sc.monitors, objective=sc.objective, baseline_max=base.monitor_max,
                         guard_abort=True, incumbent=inc))
    g.run_ladder(p, spec)                                        # autotunes each group's shape
    out = g.run_ladder(p, spec)
    t = g.last_timing()
    cs = sum(r.cell_updates for o in out for r in o)
    st = [r.status for o in out for r in o]
    return {"workload": "config3 valley ladder 45x35/90x70/180x140, 2400 s storm, 128/96/32 designs x 3 primitives, aborts live",
            "ms": t["kernel_ms"], "cell_steps_per_s": cs / (t["kernel_ms"] / 1e3), "designs_per_s": len(st) / (t["kernel_ms"] / 1e3),
            "status_counts": {"ok": st.count(0), "guard_abort": st.count(1), "incumbent_abort": st.count(2), "unhealthy": st.count(3)},
            "launch": "one CUDA graph, one persistent cluster kernel per grid as parallel branches"}


def boundary_summary(g):
    """Stage and inflow ghosts (the boundaries the reference's GPU backend declined): the
    inflow-driven valley at 5 m (90x70; inflow hydrographs on the west and south edges,
    stage on the east and north), 40 min storm, 64 designs on the batched path, beside the
    same designs on the valley with its plain transmissive outlet. Both run twice; the
    second run (autotuned shape) is timed."""
    from itr_gpu.scenes import inflow_valley_scene, valley_scene
    out = {}
    for name, sc in (("stage_inflow", inflow_valley_scene(5.0)), ("transmissive_only", valley_scene(5.0))):
        ts = [t for _, _, t in sc.designs(64)]
        g.run_batch(sc.params, ts, sc.monitors, want_depth=False)
        runs = g.run_batch(sc.params, ts, sc.monitors, want_depth=False)
        t = g.last_timing()
        cs = sum(r.cell_updates for r in runs)
        out[name] = {"ms": t["kernel_ms"], "cell_steps_per_s": cs / (t["kernel_ms"] / 1e3),
                     "steps_per_design_mean": sum(r.steps for r in runs) / len(runs)}
    out["workload"] = "valley 90x70 @5 m, 2400 s storm, 64 designs x 2 primitives, batched path"
    return out


def dry_rows_summary(g):
    """Dry-row skipping (kernel.rs:605-612) on rain-free, inflow-driven scenes, each run once with
    params.skip_dry on and once off (the same bits either way: the final depths are compared).
    * tiled path: the river scene (configuration 5's fractal terrain, 1024^2 @2 m, fed through
      60 m of the north edge, 900 s, 8 designs): the row bands of a step run independently, so
      the step costs what its computed rows cost;
    * batched path: the inflow valley (90x70 @5 m, inflows on the west and south edges, stages on
      the east and north, 2400 s, 64 designs): a step ends at the cluster barrier, so it is as
      long as its wettest strip, and skipping shortens it only where every strip skips.
    cell-steps/s counts the cells actually advanced (cell_updates)."""
    import numpy as np

    from itr_gpu import Hyetograph
    from itr_gpu.scenes import inflow_valley_scene, river_scene

    def leg(name, run, ncells):
        out = {"workload": name}
        depth = {}
        for skip in (True, False):
            run(skip)
            runs, ms = run(skip)
            steps = sum(r.steps for r in runs)
            upd = sum(r.cell_updates for r in runs)
            depth[skip] = [np.asarray(r.depth) for r in runs]
            out["skip_on" if skip else "skip_off"] = {
                "ms": ms, "rows_skipped_fraction": 1.0 - upd / max(steps * ncells, 1),
                "cell_steps_advanced_per_s": upd / (ms / 1e3), "steps_x_cells_per_s": steps * ncells / (ms / 1e3)}
        out["speedup"] = out["skip_off"]["ms"] / out["skip_on"]["ms"]
        out["identical"] = all(np.array_equal(a.view(np.uint32), b.view(np.uint32)) for a, b in zip(depth[True], depth[False]))
        return out

    rv = river_scene()
    ds = rv.primitive_designs(8)

    def run_river(skip):
        rv.params.skip_dry = skip
        runs, _, _ = g.run_primitives(rv.params, rv.base, ds, rv.monitors, rv.editable, rv.max_abs_dz, want_depth=True)
        return runs, g.last_timing()["kernel_ms"]

    iv = inflow_valley_scene(5.0)
    iv.params.rain = Hyetograph.from_mm_h([(0, 0), (2400, 0)])
    ts = [t for _, _, t in iv.designs(64)]

    def run_valley(skip):
        iv.params.skip_dry = skip
        runs = g.run_batch(iv.params, ts, iv.monitors, want_depth=True)
        return runs, g.last_timing()["kernel_ms"]

    return {"tiled": leg("river 1024x1024 @2 m, no rain, 900 s of inflow through the north edge, 8 designs x 6 primitives, "
                         "tiled path", run_river, rv.base.nx * rv.base.ny),
            "batched": leg("inflow valley 90x70 @5 m, no rain, 2400 s of inflow, 64 designs x 2 primitives, batched path",
                           run_valley, iv.base.nx * iv.base.ny)}


# The reference's own GPU throughput cases and its published numbers for them (wgpu on an
# Apple M4 Pro through Metal, crates/itr-gpu/README.md:62-65): (label, n, designs, duration s,
# useful cell-updates/s).
GPUBENCH_CASES = (("512^2 x1", 512, 1, 120.0, 1.35e9), ("128^2 x16", 128, 16, 120.0, 0.66e9),
                  ("128^2 x64", 128, 64, 120.0, 1.15e9), ("1024^2 x1", 1024, 1, 40.0, 1.40e9))


def gpubench_summary(g):
    """crates/itr-gpu/examples/gpubench.rs:17-33 on this operator: a plane 5 - 0.01 x +
    0.3 sin(y / 40) at 2 m, closed walls, still water at stage 2 m, 100 mm/h of rain, sync every
    quarter of the run; one warm-up call, then one run_batch call timed from the host as the
    reference times it (packing, copies, kernels and results included): useful cell-updates/s
    = steps x n^2 x designs / wall. Beside each, the reference's published number (other
    hardware, for context)."""
    import math

    import numpy as np

    from itr_gpu import Hyetograph, MonitorSet, PreparedTerrain, SolverParams, synthetic_terrain

    def plane(x, y):
        return 5.0 - 0.01 * x + 0.3 * np.sin(y / 40.0)
    plane.vectorized = True
    out = {}
    for label, n, cands, dur, ref in GPUBENCH_CASES:
        base = synthetic_terrain(n, n, 2.0, plane, n=0.03, segments=[])
        p = SolverParams(dur, dur / 4.0, rain=Hyetograph.from_mm_h([(0.0, 100.0), (1e9, 100.0)]), initial_stage=2.0)
        ts = [PreparedTerrain(base) for _ in range(cands)]
        g.run_batch(p, ts, MonitorSet(), want_depth=False)
        t0 = time.perf_counter()
        runs = g.run_batch(p, ts, MonitorSet(), want_depth=False)
        wall = time.perf_counter() - t0
        upd = float(sum(r.steps for r in runs)) * n * n
        out[label] = {"steps": int(runs[0].steps), "wall_s": wall, "cell_updates_per_s": upd / wall,
                      "reference_m4pro_metal": ref, "over_reference": upd / wall / ref}
        assert math.isfinite(out[label]["cell_updates_per_s"])
    out["note"] = ("the reference's numbers are wgpu on an Apple M4 Pro (Metal); running them here is unavailable on "
                   "this box. Ours: host-timed run_batch, as gpubench.rs times it")
    return out


def guarded(fn, *a):
    """A side summary must not cost the bench line: its failure is reported in its place."""
    try:
        return fn(*a)
    except Exception as e:  # noqa: BLE001
        return {"error": f"{type(e).__name__}: {e}"}


def run_reference(args):
    rank, world, _ = dist_setup(args.gpus)
    if rank != 0:
        barrier(world)
        return 0
    sc, terrs = workload(0)
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(sc, terrs, budget_s=max(5.0, 60.0 / max(args.steps + args.warmup, 1)))
        if i >= args.warmup:
            vals.append(r)
    v = sum(x["cell_steps"] for x in vals) / sum(x["wall_s"] for x in vals)
    line = {"metric": METRIC, "value": v, "unit": "cell-steps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(x["wall_s"] for x in vals) / len(vals), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded), reference CPU path via oracle/ restatement",
            "config": {"workload": "config2 rolling hills 120x96 @5 m, 64 designs x 4 primitives, 3600 s storm (bounded sample)",
                       "impl_note": "reference Rust workspace not buildable here (no cargo/rustc); its f32 fused kernel is timed through the C++ restatement"},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": vals[0]["cores"], "kind": "port", "sample": vals[0]["sample"]},
            "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    barrier(world)
    return 0


def _case_tiled5(g):
    """Config 5 on the tiled path (row bands): 1024^2 x 16 designs as primitives, first 300 s."""
    from itr_gpu.scenes import config
    sc = config(5)
    sc.params.duration_s = 300.0
    ds = sc.primitive_designs(16)
    for _ in range(2):
        g.run_primitives(sc.params, sc.base, ds, sc.monitors, sc.editable, sc.max_abs_dz, want_depth=False)


def _case_mat4(g):
    """Config 4's design chain: device materialisation and its adjoint, 32 designs, first 120 s."""
    from itr_gpu.scenes import config
    sc = config(4)
    sc.params.duration_s = 120.0
    ds = sc.primitive_designs(32)
    for _ in range(2):
        g.vjp_primitives(sc.params, sc.base, ds, sc.monitors, sc.objective, sc.editable, sc.max_abs_dz, checkpoint_interval=64)


def _case_plain2(g):
    """Config 2 on the plain one-design-per-launch path, 2 designs, first 300 s."""
    from itr_gpu.scenes import config
    sc = config(2)
    sc.params.duration_s = 300.0
    ts = [t for _, _, t in sc.designs(2)]
    g.set_option("impl", 1)
    for _ in range(2):
        g.run_batch(sc.params, ts, sc.monitors, want_depth=False)


def _case_adj4(g):
    """Config 4's adjoint: 32 designs, first 300 s of the storm, checkpoint interval 64."""
    from itr_gpu.scenes import config
    sc = config(4)
    sc.params.duration_s = 300.0
    ts = [t for _, _, t in sc.designs(32)]
    for _ in range(2):
        g.vjp(sc.params, ts, sc.monitors, sc.objective, checkpoint_interval=64)


def _case_render(g):
    """The presentation kernels: a 1920x1080 perspective frame of the 45x35 valley scene at 10 m
    (terrain refined twice, water, flow), and a map image of a seeded 1024^2 field at scale 2."""
    import numpy as np
    from itr_gpu.scene_render import SceneView, depth_texture, look, terrain_texture, velocity_texture
    from itr_gpu.scenes import valley_field
    nx, ny, cell, up = 45, 35, 10.0, 2
    zf = valley_field(20261203 + 1)
    x = (np.arange(nx * up) + 0.5) * cell / up
    y = ny * cell - (np.arange(ny * up) + 0.5) * cell / up
    trgba, z_lo, z_span = terrain_texture(zf(*np.meshgrid(x, y)), np.zeros((ny * up, nx * up), np.uint8))
    zc = zf(*np.meshgrid((np.arange(nx) + 0.5) * cell, ny * cell - (np.arange(ny) + 0.5) * cell))
    depth = np.clip(zc.min() + 1.4 - zc, 0.0, None)
    drgba = depth_texture(depth, 4.0)
    vrgba = velocity_texture(np.where(depth > 0, 0.7, 0.0), np.where(depth > 0, 0.15, 0.0), 2.0)
    top = z_span * 2.0
    fwd, right, upv, focal = look((520.0, 420.0, top + 60.0), (200.0, 160.0, 0.2 * top), 60.0)
    view = SceneView(cam_pos=(520.0, 420.0, top + 60.0), cam_fwd=fwd, cam_right=right, cam_up=upv, focal=focal,
                     domain=(nx * cell, ny * cell, cell), z_lo=z_lo, z_span=z_span, up=float(up), depth_span=4.0, ve=2.0,
                     vel_max=2.0, time=1200.0, rain=1.0, wet=1.0, overcast=0.98)
    for _ in range(2):
        g.render_scene(trgba, drgba, vrgba, view, 1920, 1080)
    rng = np.random.default_rng(3)
    z = (rng.random((1024, 1024)) * 10.0).astype(np.float32)
    val = rng.random((1024, 1024)).astype(np.float32)
    for _ in range(2):
        g.render_map(z, val, 2.0, mode=0, vex=3.0, scale=2)


PROFILE_CASES = {"tiled5": _case_tiled5, "mat4": _case_mat4, "plain2": _case_plain2, "adj4": _case_adj4,
                 "render": _case_render}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--designs", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain one-design-per-launch comparison")
    ap.add_argument("--cluster", type=int, default=0, help="pin the cluster size (profiling; 0 = autotune)")
    ap.add_argument("--threads", type=int, default=0, help="pin the threads per CTA (profiling; 0 = autotune)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the config-4 adjoint summary")
    ap.add_argument("--no-ladder", action="store_true", help="skip the config-3 uneven-batch and stage/inflow summaries")
    ap.add_argument("--workload", type=int, default=2, choices=[2, 4, 5],
                    help="2: the bench workload; 4: the 240x192 scene (32 designs); 5: the 1024x1024 scene (16 designs) "
                         "(4 and 5: measurement / profiling only)")
    ap.add_argument("--impl-path", default="auto", choices=["auto", "tiled", "plain"],
                    help="profiling: run the main workload on the tiled or plain path instead of the autotuned one")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="profiling: only the config-4 adjoint (forward + VJP) for --duration seconds of storm; prints its summary")
    ap.add_argument("--set", action="append", default=[], metavar="KEY=VALUE",
                    help="profiling: itr_gpu_set_option(KEY, VALUE) on the context before the run (repeatable)")
    ap.add_argument("--profile-case", default=None, choices=sorted(PROFILE_CASES),
                    help="profiling: run one small case of one path twice (the second run is the one to capture) and exit")
    ap.add_argument("--duration", type=float, default=None,
                    help="simulate only the first DURATION s of the storm (profiling case; not a bench line)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    rank, world, local = dist_setup(args.gpus)
    import torch
    torch.cuda.set_device(local)
    from itr_gpu import GpuSolver
    def apply_options(g):
        for kv in args.set:
            key, val = kv.split("=", 1)
            g.set_option(key, int(val))

    if args.profile_case:
        g = GpuSolver(local)
        apply_options(g)
        PROFILE_CASES[args.profile_case](g)
        g.close()
        print(json.dumps({"profile_case": args.profile_case, "ok": True}))
        return 0
    if args.adjoint_only:
        g = GpuSolver(local)
        apply_options(g)
        print(json.dumps({"adjoint": adjoint_summary(g, duration=args.duration, which=4 if args.workload == 2 else 5)}))
        g.close()
        return 0
    sc, terrs = workload(rank, {2: args.designs, 4: 32, 5: 16}[args.workload], args.workload)
    if args.duration is not None:
        sc.params.duration_s = float(args.duration)
    g = GpuSolver(local)
    apply_options(g)
    if args.cluster or args.threads:
        g.set_option("cluster", args.cluster)
        g.set_option("threads", args.threads)
    if args.impl_path != "auto":
        g.set_option("impl", 2 if args.impl_path == "tiled" else 1)
    N = sc.base.nx * sc.base.ny
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # warm-up through the public call (also autotunes the launch shape)
    for _ in range(max(args.warmup, 3)):
        runs = g.run_batch(sc.params, terrs, sc.monitors, want_depth=False)
    steps_per_design = [r.steps for r in runs]
    cell_steps = float(sum(steps_per_design)) * N

    # ---- value: kernel over resident inputs ----
    barrier(world)
    torch.cuda.synchronize()
    kern_ms = []
    launches = 0
    with ClockSampler(local) as clk:
        t_wall0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()                       # L2 flush (256 MB > 126 MB L2) between iterations
            torch.cuda.synchronize()
            g.rerun_resident()
            tm = g.last_timing()
            kern_ms.append(tm["kernel_ms"])
            launches += tm["launches"]
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall0
    barrier(world)
    launch_shape = g.adapter_info().split("; last batch: ")[-1] if "; last batch: " in g.adapter_info() else None
    k_total_ms = max_over_ranks(sum(kern_ms), world)
    total_cs = sum_over_ranks(cell_steps * args.steps, world)
    value = total_cs / (k_total_ms / 1e3)
    designs_per_s = sum_over_ranks(len(terrs) * args.steps, world) / (k_total_ms / 1e3)

    # ---- e2e: the public C ABI call from host buffers ----
    # N > 1: the whole population (every rank's designs) goes through ShardedBackend, so
    # each step also gathers every design's results on every rank (one all-gather).
    if world > 1:
        from itr_gpu import GpuBackend
        from itr_gpu.sharding import ShardedBackend
        population = []
        for r in range(world):
            population += terrs if r == rank else workload(r, args.designs)[1]
        evaluator = ShardedBackend(GpuBackend(g))
        step_fn = lambda: evaluator.run(sc.params, population, sc.monitors)  # noqa: E731
    else:
        step_fn = lambda: g.run_batch(sc.params, terrs, sc.monitors, want_depth=False)  # noqa: E731
    barrier(world)
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step_fn()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    barrier(world)
    e2e_total = max_over_ranks(sum(e2e_ms), world)
    e2e_value = total_cs / (e2e_total / 1e3)
    nx, ny = sc.base.nx, sc.base.ny
    h2d = len(terrs) * (ny * (nx + 1) + (ny + 1) * nx + nx * ny) * 4 + 2 * N * 4 + 2 * (nx + ny) + len(terrs) * 16 \
        + len(sc.monitors.cells) * 4
    from itr_gpu.solver import GpuRun  # noqa: F401
    d2h = len(terrs) * (len(sc.monitors.cells) * 4 + 96)

    if rank == 0:
        hbm, src = peaks()
        per_launch_bytes = cell_steps * BYTES_PER_CELL_STEP
        avg_ms = sum(kern_ms) / len(kern_ms)
        achieved = per_launch_bytes / (avg_ms / 1e3) / 1e9
        counters = kernel_counters()
        clocks = clk.summary()
        # single-GPU only: the other ranks would wait on the closing barrier meanwhile
        plain = None if args.no_plain or world > 1 else plain_comparison(g, sc, terrs)
        adj = None if args.no_adjoint or world > 1 or args.duration is not None else guarded(adjoint_summary, g, 128, None, 4,
                                                                                              (32, 512))
        adj5 = None if args.no_adjoint or world > 1 or args.duration is not None else guarded(adjoint_summary, g, 128, None, 5)
        lad = None if args.no_ladder or world > 1 or args.duration is not None else ladder_summary(g)
        bnd = None if args.no_ladder or world > 1 or args.duration is not None else boundary_summary(g)
        gpb = None if args.no_ladder or world > 1 or args.duration is not None else guarded(gpubench_summary, g)
        pol = None if args.no_adjoint or world > 1 or args.duration is not None else guarded(polish_summary, g)
        dry = None if args.no_ladder or world > 1 or args.duration is not None else guarded(dry_rows_summary, g)
        cpu = None
        if not args.no_cpu_baseline:
            cpu = cpu_baseline(sc, terrs)
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample", "value_1_thread")}
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": k_total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes and designs)",
            "config": {"workload": {2: ("config2: rolling hills 120x96 @5 m, 60 min storm (100 mm/h peak at 20 min), "
                                        f"{len(terrs)} designs x 4 primitives per GPU, run to completion"),
                                    4: (f"config4: rolling hills 240x192 @2.5 m, {sc.params.duration_s:.0f} s of the 60 min storm, "
                                        f"{len(terrs)} designs x 4 primitives"),
                                    5: (f"config5: fractal 1024x1024 @2 m, {sc.params.duration_s:.0f} s of the 90 min double-peak "
                                        f"storm, {len(terrs)} designs x 6 primitives")}[args.workload],
                       "path": args.impl_path,
                       "designs_per_gpu": len(terrs), "cells": N, "steps_per_design_mean": sum(steps_per_design) / len(steps_per_design),
                       "parallelism": f"designs sharded over {world} GPU(s), 1 design per thread-block cluster",
                       "launch": launch_shape,
                       "l2": "flushed between timed iterations (256 MB write)"},
            "designs_per_s": designs_per_s,
            "precision": ("device path bit-identical to the f32 CPU port (tests/test_gpu_parity.py); that port's "
                          "per-cell peak depth within 2.0e-6 m of the f64 oracle on config 1, J within 3e-7 "
                          "relative (tests/test_precision.py; bar 1e-4 m)"),
            "roofline": issue_roofline(cell_steps, avg_ms, counters, clocks, achieved, hbm, src),
            "cpu_baseline": cpu,
            "plain": plain,
            "batched_over_plain": (value / world / plain["value"]) if plain else None,
            "adjoint": adj,
            "ladder": lad,
            "boundaries": bnd,
            "reference_gpubench": gpb,
            "polish": pol,
            "dry_rows": dry,
            "adjoint_config5": adj5,
            "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": launches,
            "clocks": clocks,
            "wall_s_timed": t_wall,
        }
        print(json.dumps(line))
    g.close()
    if world > 1:
        import torch.distributed as dist
        barrier(world)
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
