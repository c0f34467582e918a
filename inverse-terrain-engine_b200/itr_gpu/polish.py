"""Gradient polishing of an incumbent design: the adjoint's use in the search loop.

The reference's optimisers are derivative-free (CMA-ES / IPOP, crates/itr-opt/src/cmaes.rs;
random, Sobol, compass, crates/itr-opt/src/search.rs). Here the device adjoint gives
dJ/d(height, width, length) of every primitive at fixed quantised centre and angle
(itr_gpu_vjp_primitives), and polish() uses it on an incumbent, the best design a batch
returned: it steps the continuous parameters down the gradient inside a trust region, snaps
them back onto the design space's quantisation grid (DesignSpace::q, design.rs:259-261), and
keeps a step only when the EXACT forward re-evaluation of the snapped design
(itr_gpu_run_primitives with the objective, the guard test against the baseline maxima and
the volume limit) lowers J and stays feasible (objective.rs:126-145, design.rs:388-410). The
gradient proposes, the forward decides: the guard constraint is enforced exactly as the
evaluator enforces it.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field

import numpy as np

from .design import BERM, SWALE, Primitive, quantize

PARAMS = ("height", "width", "length")


@dataclass
class PolishResult:
    prims: list            # the polished design (quantised primitives)
    j: float               # its J from the exact forward re-evaluation
    j_start: float         # J of the incumbent
    feasible: bool
    accepted: int          # steps kept
    evaluations: int       # exact forward re-evaluations of proposals
    history: list = field(default_factory=list)   # J after every iteration


def _snap(p: Primitive, quant, bounds) -> Primitive:
    qh, qw, ql = quant
    (hlo, hhi), (wlo, whi), (llo, lhi) = bounds
    h = quantize(min(max(p.height, hlo), hhi), qh)
    w = quantize(min(max(p.width, wlo), whi), qw)
    ln = quantize(min(max(p.length, llo), lhi), ql)
    kind = p.kind
    if kind in (BERM, SWALE) and h != 0.0:   # berm when raising, swale when lowering (prepare_prims)
        kind = BERM if h > 0.0 else SWALE
    return dataclasses.replace(p, kind=kind, height=h, width=w, length=ln)


def polish(solver, params, base, prims, objective, editable, max_abs_dz: float, baseline_max=None, iters: int = 8,
           radius=(0.05, 1.0, 5.0), quant=(0.01, 0.5, 0.5), bounds=((-0.5, 0.5), (3.0, 8.0), (20.0, 100.0)),
           max_volume: float | None = None, checkpoint_interval: int = 128) -> PolishResult:
    """Polish one incumbent. radius: the trust region per parameter (height, width, length in
    m): the largest move of a parameter over the primitives in one proposal; it grows by 1.5
    after a kept step and halves after a rejected one, and the search ends after `iters`
    proposals or when every radius is below its quantisation step."""
    monitors = objective.monitors
    prims = [_snap(p, quant, bounds) for p in prims]
    r = np.array(radius, dtype=np.float64)
    q = np.array(quant, dtype=np.float64)

    def exact(ps):
        runs, cut, fill = solver.run_primitives(params, base, [ps], monitors, editable, max_abs_dz, objective=objective,
                                                baseline_max=baseline_max)
        ok = bool(runs[0].feasible) and runs[0].status == 0
        if max_volume is not None and cut[0] + fill[0] > max_volume:
            ok = False
        return float(runs[0].j), ok

    j, feasible = exact(prims)
    res = PolishResult(prims=prims, j=j, j_start=j, feasible=feasible, accepted=0, evaluations=1)
    for _ in range(iters):
        if np.all(r < q):
            break
        _, grads = solver.vjp_primitives(params, base, [prims], monitors, objective, editable, max_abs_dz,
                                         checkpoint_interval=checkpoint_interval)
        g = np.asarray(grads[0], dtype=np.float64).reshape(len(prims), 3)
        scale = np.abs(g).max(axis=0)
        step = np.where(scale > 0.0, -r * g / np.where(scale > 0.0, scale, 1.0), 0.0)
        cand = [_snap(dataclasses.replace(p, **{k: getattr(p, k) + step[i, n] for n, k in enumerate(PARAMS)}), quant, bounds)
                for i, p in enumerate(prims)]
        if cand == prims:          # the step rounds away: a finer one cannot move either
            r *= 0.5
            res.history.append(res.j)
            continue
        jc, okc = exact(cand)
        res.evaluations += 1
        if okc and jc < res.j:
            prims, res.prims, res.j, res.feasible = cand, cand, jc, True
            res.accepted += 1
            r = np.minimum(r * 1.5, np.array(radius) * 4.0)
        else:
            r *= 0.5
        res.history.append(res.j)
    return res


@dataclass
class IncumbentPolish:
    """One search generation's incumbent, polished: what polish_population() reports."""
    population: int              # designs evaluated
    feasible: int                # of which feasible (guard, volume limit)
    incumbent: list              # the best feasible design of the population
    result: PolishResult         # its polish
    baseline_max: np.ndarray     # the unedited terrain's monitor maxima (guard reference)
    wall_s: dict                 # wall time of the population run and of the polish


def polish_population(solver, params, base, designs, objective, editable, max_abs_dz: float, max_volume=None,
                      iters: int = 4, checkpoint_interval: int = 256, **kw) -> IncumbentPolish:
    """The search loop's use of the adjoint for one generation: run the unedited terrain for
    the guard baseline (Problem::build, crates/itr-opt/src/problem.rs:183-190), evaluate the
    population of designs (given as primitives) exactly on the device, take the best feasible
    one (lowest J with no guard violation and within the volume limit: the incumbent an
    elitist method keeps, crates/itr-opt/src/driver.rs:169) and polish it (polish())."""
    import time
    from .terrain import PreparedTerrain
    monitors = objective.monitors
    t0 = time.perf_counter()
    base_run = solver.run_batch(params, [PreparedTerrain(base)], monitors)[0]
    baseline = np.asarray(base_run.monitor_max, dtype=np.float64)
    runs, cut, fill = solver.run_primitives(params, base, designs, monitors, editable, max_abs_dz, objective=objective,
                                            baseline_max=baseline, want_depth=False)
    t1 = time.perf_counter()
    ok = [i for i, r in enumerate(runs) if r.feasible and r.status == 0
          and (max_volume is None or cut[i] + fill[i] <= max_volume)]
    if not ok:
        raise RuntimeError("no feasible design in the population")
    best = min(ok, key=lambda i: runs[i].j)
    res = polish(solver, params, base, designs[best], objective, editable, max_abs_dz, baseline_max=baseline, iters=iters,
                 max_volume=max_volume, checkpoint_interval=checkpoint_interval, **kw)
    t2 = time.perf_counter()
    return IncumbentPolish(population=len(designs), feasible=len(ok), incumbent=designs[best], result=res,
                           baseline_max=baseline, wall_s={"population": t1 - t0, "polish": t2 - t1})
