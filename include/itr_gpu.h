/* itr_gpu.h — C ABI of the B200 batched forward operator (and its adjoint) for itr.
 *
 * This is the drop-in boundary for the reference's batch evaluator path:
 *   trait BatchBackend<f32>::run(&SolverParams, &[&PreparedTerrain<f32>], &MonitorSet)
 *       crates/itr-opt/src/evaluator.rs:131-135
 *   GpuSolver::{new, run_batch, adapter_info}      crates/itr-gpu/src/lib.rs:85,149,126
 *   CLI wiring Gpu(GpuSolver) -> BatchRun          crates/itr-cli/src/backend.rs:44-63
 * Plain pointers and sizes only. A context owns its device memory and one CUDA stream; a
 * context is not thread-safe (the reference backend is `&mut self`), several contexts may
 * coexist. Every entry point returns an itr_status; itr_gpu_last_error() has the text.
 *
 * Units and layouts follow the reference: depths in m, rates in m/s, row-major grids with
 * row 0 the northern row, linear cell id = row * nx + col (MonitorSet, model.rs:6-24).
 */
#ifndef ITR_GPU_H
#define ITR_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ITR_GPU_ABI_VERSION 4

typedef struct itr_ctx itr_ctx;

/* Status codes. ITR_UNSUPPORTED plays the role of the reference's Err(String) from
 * run_batch: "unsupported here", the evaluator then falls back to the CPU for that level
 * (evaluator.rs:231-238). */
enum itr_status {
  ITR_OK = 0,
  ITR_UNSUPPORTED = 1,
  ITR_INVALID_ARG = 2,
  ITR_DEVICE_ERROR = 3,
  ITR_DEVICE_TIMEOUT = 4
};

/* Ghost-cell kinds per boundary side cell (terrain.rs:121-129, boundary.rs:12-87). */
enum itr_bc { ITR_BC_WALL = 0, ITR_BC_TRANSMISSIVE = 1, ITR_BC_STAGE = 2, ITR_BC_INFLOW = 3 };

/* Face modes (terrain.rs:12-18): one signed jump per face (fidelity level 1) or two
 * non-negative jumps to a face crest (coarse levels). */
enum itr_face_mode { ITR_FACE_SIGNED = 0, ITR_FACE_CREST = 1 };

/* Per-design outcome (evaluator.rs:20-28 Status, reduced to what a batch run can yield). */
enum itr_run_status {
  ITR_RUN_OK = 0,
  ITR_RUN_GUARD_ABORT = 1,     /* AbortReason::GuardViolation (objective.rs:130-145) */
  ITR_RUN_INCUMBENT_ABORT = 2, /* AbortReason::Incumbent (evaluator.rs:100-104)       */
  ITR_RUN_UNHEALTHY = 3        /* negative depth beyond h_dry or NaN (numerics.rs:163) */
};

/* SolverParams (crates/itr-hydro/src/solver.rs:27-49). locked_dt and cfl_hard are set on the
 * context with itr_gpu_set_locked_dt (one schedule per grid, shared by the batch). inflow_scale
 * multiplies every inflow hydrograph as in fill_ghosts (boundary.rs:27); the reference GPU
 * backend rejected values other than 1 (backend.rs:53-55), this one takes any. */
typedef struct itr_params {
  double duration_s;
  double sync_interval_s;
  double cfl;
  double dt_max_s;
  double h_dry;
  double h_eps;
  const double* rain_t;     /* Hyetograph points: time [s]            (scenario.rs:526) */
  const double* rain_rate;  /*                    rate [m/s]                             */
  int32_t n_rain;
  double infil_capacity;    /* constant infiltration capacity [m/s]                      */
  double initial_depth;     /* used for designs whose h0 is NULL (init_state, solver.rs:287) */
  int32_t skip_dry;         /* dry-row skipping (kernel.rs:605-612): with no rain in a step, a row
                               between dry rows (and dry ghosts) is not computed; results are
                               the same bits. Done by the cluster kernel and the tiled path;
                               a storm without a rain-free stretch inside the run has no step
                               to skip, and such runs leave the bookkeeping out             */
  double inflow_scale;      /* factor on every inflow hydrograph (1.0 = as given)        */
} itr_params;

/* The shared TerrainBase<f32> of one call (terrain.rs:237-257): every design in a call
 * shares it, as run_batch requires (Arc::ptr_eq, lib.rs:154-159). */
typedef struct itr_grid {
  int32_t nx, ny;
  double dx, dy;
  double g;                 /* 9.81 (terrain.rs:259) */
  int32_t mode;             /* itr_face_mode */
  const float* wet;         /* nx*ny, 1 = open cell, 0 = wall (TerrainBase::wet)      */
  const float* gn2;         /* nx*ny, g*n^2 (TerrainBase::gn2)                        */
  const uint8_t* bc;        /* 2*nx + 2*ny codes: north[nx], south[nx], west[ny], east[ny] */
  int64_t wet_count;        /* number of open cells (rain volume in the ledger)       */
  /* Stage and inflow ghosts (Ghost::Stage / Ghost::Inflow, terrain.rs:121-129, filled by
   * boundary.rs:43-50,66-71). Indexed like bc; read only at ITR_BC_STAGE / ITR_BC_INFLOW
   * cells, so all may be NULL when bc has neither. Zero-initialise the struct otherwise. */
  const double* bc_stage;   /* stage cells: water level above the terrain datum [m]   */
  const int32_t* bc_hydro;  /* inflow cells: index of the cell's hydrograph           */
  const double* bc_inv_len; /* inflow cells: 1 / length of the cell's segment [1/m]   */
  int32_t n_hydro;          /* inflow hydrographs (Boundaries::hydrographs)           */
  const int32_t* hydro_off; /* n_hydro+1 offsets into hydro_t / hydro_q               */
  const double* hydro_t;    /* hydrograph points: time [s] (a Hyetograph, scenario.rs:526) */
  const double* hydro_q;    /*                    discharge [m^3/s]                    */
} itr_grid;

/* Limits of the inflow tables: distinct (hydrograph, segment length) pairs over the inflow
 * cells, and hydrograph points summed over those pairs. */
#define ITR_MAX_INFLOW_GROUPS 8
#define ITR_MAX_INFLOW_POINTS 64

/* One candidate: the face jumps of its PreparedTerrain (lib.rs:177-194 packs the same
 * arrays). dzx[r*(nx+1) + f] is x-face f of row r (f = 0 and f = nx are the domain edges
 * and are 0); dzy[f*nx + c] is y-face f of column c (f = 0 and f = ny are 0). Crest mode
 * adds the second jump of every face in dzx2/dzy2. */
typedef struct itr_design {
  const float* dzx;         /* ny*(nx+1) */
  const float* dzy;         /* (ny+1)*nx */
  const float* dzx2;        /* crest mode only, else NULL */
  const float* dzy2;        /* crest mode only, else NULL */
  const float* h0;          /* nx*ny initial depth, or NULL for params.initial_depth on open cells;
                               infinite values or values above 1e4 m give ITR_INVALID_ARG (the first
                               dt would vanish), NaN or negative ones an unhealthy run */
  double cut_m3, fill_m3;   /* earthwork volumes of the edit (J's earthwork term)      */
  const double* z_edge;     /* 2*nx+2*ny, indexed like grid.bc: z level above the datum of the
                               interior cell behind each boundary cell (PreparedTerrain::z_level,
                               which the design's edit changes); required when grid.bc has
                               stage cells (a stage ghost's depth is stage - z_edge), else NULL */
} itr_design;

/* Objective and abort rules (objective.rs:8-150, GuardObserver evaluator.rs:88-108).
 * Positions index the monitor list. NULL means: no objective, no aborts, J not computed. */
typedef struct itr_objective {
  int32_t n_assets;
  const int32_t* asset_off;      /* n_assets+1 offsets into asset_pos */
  const int32_t* asset_pos;      /* monitor positions of each asset's cells */
  const double* asset_threshold; /* eta_k [m] */
  const double* asset_weight;    /* w_k */
  int32_t n_guard;
  const int32_t* guard_pos;      /* monitor positions, in guard-cell order */
  const double* baseline_max;    /* n_mon baseline maxima, or NULL (no guard test) */
  double guard_tolerance;        /* eps_G [m] */
  double tau;                    /* softplus scale [m] */
  double cut_cost, fill_cost, earth_weight;
  int32_t require_no_worsening;
  int32_t guard_abort;           /* 1: stop a design at its first breached sync point */
  int32_t has_incumbent;         /* 1: incumbent abort live (frozen for the batch)  */
  double incumbent;
} itr_objective;

/* Per-design results, caller-allocated. Array members may be NULL (not wanted). The
 * reference's BatchRun (evaluator.rs:118-125) is {monitor_max, steps, cell_updates, bad}. */
typedef struct itr_result {
  double* monitor_max;      /* n_mon: running max depth at monitored cells (f64) */
  float* peak;              /* nx*ny: running max depth of every cell, or NULL */
  float* depth;             /* nx*ny: final depth (GpuRun::depth), or NULL */
  double* ledger;           /* max_rows * 8: t, volume, rain, inflow, outflow, infil, fix, residual */
  int32_t max_rows;
  /* written by the library: */
  uint64_t steps;
  uint64_t cell_updates;    /* cells advanced: steps * nx * ny (gpubench.rs:28) less skipped dry rows */
  double t_end;
  uint32_t sync_count;
  int32_t status;           /* itr_run_status */
  uint32_t breach_cell;     /* guard abort: cell id of the worst guard cell */
  uint32_t breach_sync;     /* guard abort: sync index of the breach */
  double violation;         /* guard abort: exceedance [m]; else guard violation of the finished run */
  double lower_bound;       /* incumbent abort: running J lower bound */
  double j;                 /* objective J of the run (monitor maxima so far), if obj given */
  int32_t feasible;         /* 1 if no guard violation (objective.rs:126) */
  int32_t n_rows;           /* ledger rows written */
  double volume_m3;         /* stored volume at the end */
  double rel_residual;      /* |ledger residual| / gross input at the last sync */
  uint64_t warm_start_steps;/* steps taken over from the baseline record (RunSummary::warm_start_steps) */
  double dt_fallback_t;     /* locked dt: time of the sync snapshot the run fell back to, -1 if it
                               kept the schedule or ran adaptively (RunSummary::dt_fallback_t) */
  uint64_t rows_skipped;    /* dry rows skipped (params.skip_dry; RunSummary::rows_skipped): rows
                               that, with no rain in a step, lay between dry rows; their cells
                               are left out of cell_updates = steps * nx * ny - rows_skipped * nx */
} itr_result;

/* GpuSolver::new (lib.rs:85). device < 0 selects the current device. Returns NULL on
 * failure with the reason in err. */
itr_ctx* itr_gpu_create(int device, char* err, size_t errlen);

void itr_gpu_destroy(itr_ctx* ctx);

/* Text of the last failure on this context (never NULL). */
const char* itr_gpu_last_error(itr_ctx* ctx);

/* GpuSolver::adapter_info (lib.rs:126): device name, SM count, memory, build. */
int itr_gpu_info(itr_ctx* ctx, char* buf, size_t len);

/* GpuSolver::run_batch (lib.rs:149) / BatchBackend::run (evaluator.rs:134): run every design
 * to its end (or its abort), one result per design, all from host buffers. Designs run
 * concurrently in one persistent launch, one design per thread-block cluster. */
int itr_gpu_run_batch(itr_ctx* ctx, const itr_params* p, const itr_grid* g, int32_t n_designs,
                      const itr_design* designs, const uint32_t* monitors, int32_t n_mon,
                      const itr_objective* obj, itr_result* results);

/* Options (GpuSolver::steps_per_submit, lib.rs:70, is the reference's one knob):
 *   "impl"     0 = batched cluster kernel (default; grids too large for 8 CTAs' shared memory
 *              take the tiled path), 1 = plain one-design-per-launch kernel, 2 = tiled
 *              batched path: all designs per launch, state in HBM, a CUDA graph per
 *              steps_per_submit steps
 *   "threads"  threads per CTA of the batched kernel (0 = autotune)
 *   "cluster"  CTAs per design of the batched kernel (0 = autotune)
 *   "graph"    tiled path: 1 = replay each block of steps as one CUDA graph (default 1)
 *   "steps_per_submit"  plain and tiled paths: steps between host polls (default 64)
 *   "warm_start"  1 = start each design from the baseline record (itr_gpu_record_baseline) where
 *                 that is exact; 0 = always cold (default)
 *   "exact_special"     1 = the batched kernel computes every reciprocal and square root
 *                       with the IEEE-exact library routines instead of its own branch-free
 *                       ones (identical results; for checking, default 0)
 *   "band"     tiled path update kernel: 1 = row-band sweep (default), 0 = 16x16 tiles with a
 *              halo (identical results; for comparison)
 *   "adj_band" adjoint kernels on row-band sweeps instead of 16x16 tiles with a halo: bit 0
 *              the replay of each segment, bit 1 the backward step; -1 (default) = the replay
 *              on bands, the backward step on bands for grids of 2^18 cells or more
 *              (identical gradients for every value)
 *   "adj_trim" 1 = the backward sweep of a design stops at the latest state that set one of its
 *              assets' maxima (after it the adjoint is zero: identical gradients, fewer steps;
 *              default 1), 0 = every step of the run
 *   "wait_limit"        try_wait rounds of the batched kernel's barrier wait in single-CTA
 *                       designs before the run gives up with ITR_DEVICE_TIMEOUT (default 2^22)
 *   "stall_wait_test"   1 = that barrier expects one arrival more than the CTA makes, so every
 *                       such wait runs to its limit and the call returns ITR_DEVICE_TIMEOUT with
 *                       the context still usable (test of the timeout path; default 0)
 * Returns ITR_INVALID_ARG for an unknown key. */
int itr_gpu_set_option(itr_ctx* ctx, const char* key, int64_t value);

/* Baseline-locked dt (SolverParams::locked_dt and cfl_hard, solver.rs:42-46; the run loop at
 * solver.rs:436-483; Problem::build sets it from the baseline's record, problem.rs:196-198).
 * Later itr_gpu_run_batch / itr_gpu_run_primitives calls on this context step every design
 * with dt[step] while dt[step] * smax of the design's current state <= cfl_hard (the baseline's
 * own dts, e.g. from a run of the unedited terrain, keep a zero edit bit-identical to it). At
 * the first step where that fails, or when the schedule has run out, the design goes back to
 * its last sync snapshot (state, peaks, integrator, ledger) and continues with the adaptive dt;
 * itr_result.dt_fallback_t gets the snapshot's time. The clip to the next sync instant still
 * applies. The schedule is copied; n = 0 (or dt NULL) clears it. Both batched paths take it
 * (the cluster kernel, and the tiled path of impl 2 and of grids too large for a cluster);
 * with a schedule set the designs start cold (no warm start), and the paths that have no
 * locked dt return ITR_UNSUPPORTED: impl 1 (plain, one design per launch), the adjoint and
 * the ladder. itr_gpu_record_baseline runs adaptively, like the reference's baseline.
 * Device memory while a schedule is set: 28 B (cluster) or 16 B (tiled) per cell per design
 * for the snapshot. */
int itr_gpu_set_locked_dt(itr_ctx* ctx, const double* dt, uint64_t n, double cfl_hard);

/* Timing of the last run_batch on the device, CUDA events on the context stream:
 * kernel_ms = the forward kernel(s) alone, total_ms = copies + kernels. last_cell_updates
 * mirrors GpuSolver::last_cell_updates (lib.rs:72). */
int itr_gpu_last_timing(itr_ctx* ctx, double* kernel_ms, double* total_ms, uint64_t* last_cell_updates,
                        int32_t* launches);

/* Re-run the last batch with its inputs still resident on the device (no host copies),
 * results kept on the device; for timing the kernel over resident inputs. */
int itr_gpu_rerun_resident(itr_ctx* ctx);

/* Uneven batch (the fidelity ladder: coarse, native and half-cell grids of one scene,
 * evaluator.rs:218-266 runs one batch per level). Each group is one grid with its designs,
 * monitors and objective, exactly the arguments of itr_gpu_run_batch; every group's
 * persistent cluster kernel runs as one branch of a single CUDA graph launch, each with
 * the launch shape autotuned for its grid, per-design adaptive dt and per-design aborts.
 * results holds sum(n_designs) entries in group order. */
typedef struct itr_group {
  const itr_grid* grid;
  int32_t n_designs;
  const itr_design* designs;
  const uint32_t* monitors;
  int32_t n_mon;
  const itr_objective* obj;    /* may be NULL */
} itr_group;

int itr_gpu_run_ladder(itr_ctx* ctx, const itr_params* p, int32_t n_groups, const itr_group* groups, itr_result* results);

/* Vector-Jacobian product of the forward (an addition: the reference has no adjoint,
 * its optimisers are derivative-free, crates/itr-opt/src/cmaes.rs). For every design it gives
 * dJ/d(face jump) of the asset term J = sum_k w_k tau softplus((P_k - eta_k) / tau)
 * (objective.rs:95-128; the earthwork term does not depend on the jumps):
 *   dj_ddzx  n_designs * ny * (nx+1), same layout as itr_design.dzx
 *   dj_ddzy  n_designs * (ny+1) * nx, same layout as itr_design.dzy
 * The forward runs to completion on the tiled path (aborts off), keeping the state every
 * checkpoint_interval steps; the backward recomputes each segment and steps the discrete
 * adjoint back through it with the recorded dt sequence held fixed. results are the
 * forward's, as itr_gpu_run_batch gives them. Signed faces; a crest-mode grid (coarse
 * levels) needs itr_gpu_vjp_crest (ITR_UNSUPPORTED here); obj must have at least one asset.
 * With stage cells the stage ghosts' depths
 * (stage - z_edge) are held fixed: the result is the derivative with respect to the face
 * jumps alone. Device memory: checkpoints of 12 B per cell
 * per design per interval, a tape of checkpoint_interval states. */
int itr_gpu_vjp(itr_ctx* ctx, const itr_params* p, const itr_grid* g, int32_t n_designs, const itr_design* designs,
                const uint32_t* monitors, int32_t n_mon, const itr_objective* obj, int32_t checkpoint_interval,
                itr_result* results, double* dj_ddzx, double* dj_ddzy);

/* itr_gpu_vjp for a crest-mode grid (face_crest, numerics.rs:114-129: two non-negative jumps
 * per face, one for each side): dj_ddzx / dj_ddzy receive dJ/d(dzx) / dJ/d(dzy) (the first
 * jumps, itr_design.dzx/dzy) and dj_ddzx2 / dj_ddzy2 dJ/d(dzx2) / dJ/d(dzy2), same layouts. */
int itr_gpu_vjp_crest(itr_ctx* ctx, const itr_params* p, const itr_grid* g, int32_t n_designs, const itr_design* designs,
                      const uint32_t* monitors, int32_t n_mon, const itr_objective* obj, int32_t checkpoint_interval,
                      itr_result* results, double* dj_ddzx, double* dj_ddzy, double* dj_ddzx2, double* dj_ddzy2);

/* Device time of the last itr_gpu_vjp: taped forward (kernels and checkpoints) and backward. */
int itr_gpu_last_vjp_timing(itr_ctx* ctx, double* forward_ms, double* backward_ms);

/* ---- Warm starts from a recorded baseline (BaselineRecord, solver.rs:95-118; used by the
 * evaluator, evaluator.rs:423). ----
 * itr_gpu_record_baseline runs `base` (the unedited terrain) to its end on the device and
 * keeps, every checkpoint_interval steps, its state, running peaks, integrator and ledger,
 * and which rows had held water by then. With option "warm_start" = 1, later batches on the
 * same grid and params (itr_gpu_run_batch, itr_gpu_run_primitives; not the adjoint) start
 * each design from the latest checkpoint at which every row its edit can reach (the cells
 * on both sides of every face jump that differs from base's, and the cells behind stage
 * edges whose depth differs) had stayed dry; rows beside stage or inflow edges count as
 * wet from the start, as in the reference (solver.rs:404-423). Dry cells exchange exactly
 * zero flux, so up to that point the design's run is the baseline's bit for bit: results
 * equal a cold start (the ledger to f64 rounding on the cluster path). A design whose
 * initial depth differs from base's, or a batch with an incumbent abort (the reference's
 * warm start skips the bound at the syncs it jumps over), starts cold. The record lives in
 * the context until the next itr_gpu_record_baseline; result (may be NULL) gets base's run. */
int itr_gpu_record_baseline(itr_ctx* ctx, const itr_params* p, const itr_grid* g, const itr_design* base,
                            const uint32_t* monitors, int32_t n_mon, int32_t checkpoint_interval, itr_result* result);

/* ---- Designs as primitives, materialised on the device. ----
 * The reference builds each candidate's face jumps on the host (DesignSpace::materialize,
 * design.rs:316-385, then PreparedTerrain::apply_edit, terrain.rs:460-505) and uploads the
 * full per-design jump arrays (lib.rs:177-194). itr_gpu_run_primitives takes the designs as
 * primitives and builds dz, the edited cell levels, the face jumps and the earthwork
 * volumes on the device (bit-identical to the host path), then runs itr_gpu_run_batch's
 * forward. Fidelity level 1 (signed faces) only; the designs start from
 * params.initial_depth (no per-design h0). */
enum itr_prim_kind { ITR_PRIM_BERM = 0, ITR_PRIM_SWALE = 1, ITR_PRIM_CUT = 2, ITR_PRIM_MOUND = 3 };

typedef struct itr_primitive {   /* Primitive (design.rs:84-93), already quantised */
  int32_t kind;                  /* itr_prim_kind */
  double cx, cy;                 /* centre, world coordinates [m] */
  double length, width;          /* [m] */
  double angle_deg;
  double height;                 /* [m]; negative lowers the terrain */
} itr_primitive;

typedef struct itr_design_space {  /* DesignSpace (design.rs:189-200) over the grid's cells */
  double origin_x, origin_y;       /* GeoTransform: west edge of column 0, north edge of row 0 */
  const double* z;                 /* nx*ny re-based cell levels of the base terrain, walls at z_wall */
  const uint8_t* wall;             /* nx*ny, 1 = wall */
  const uint8_t* editable;         /* nx*ny, 1 = a design may change the cell */
  double z_wall;
  double max_abs_dz;               /* clamp of |dz| [m] */
} itr_design_space;

/* Designs d = 0..n_designs-1 are prims[prim_off[d] .. prim_off[d+1]). cut_m3 / fill_m3
 * (n_designs each, may be NULL) receive the earthwork volumes computed on the device. */
int itr_gpu_run_primitives(itr_ctx* ctx, const itr_params* p, const itr_grid* g, const itr_design_space* space,
                           int32_t n_designs, const int32_t* prim_off, const itr_primitive* prims,
                           const uint32_t* monitors, int32_t n_mon, const itr_objective* obj, itr_result* results,
                           double* cut_m3, double* fill_m3);

/* The adjoint of itr_gpu_run_primitives' designs, closed on the device: dJ/d(height, width,
 * length) of every primitive, dj_dprim[3 * (k - prim_off[0]) + {0, 1, 2}] for primitive
 * prims[k], at fixed quantised centre and angle. The device runs itr_gpu_vjp's forward and backward on
 * the materialised designs, forms dJ/d(dz) per cell from the face-jump gradients, and
 * contracts it with the derivative of the materialisation written out from the profile
 * (Primitive::profile, design.rs:107-134: the (1 - s^2)^2 ridge and the flat-bottomed cut,
 * differentiated through the distance to the segment and the half width, summed over the 4x4
 * quadrature; cells clamped to +-max_abs_dz contribute nothing), adding the earthwork term's
 * derivative earth_weight (cut_cost dV_cut + fill_cost dV_fill).
 * dj_ddzx / dj_ddzy (may be NULL) receive the face-jump gradients as itr_gpu_vjp gives them. */
int itr_gpu_vjp_primitives(itr_ctx* ctx, const itr_params* p, const itr_grid* g, const itr_design_space* space,
                           int32_t n_designs, const int32_t* prim_off, const itr_primitive* prims,
                           const uint32_t* monitors, int32_t n_mon, const itr_objective* obj, int32_t checkpoint_interval,
                           itr_result* results, double* dj_dprim, double* dj_ddzx, double* dj_ddzy);

/* ---- Headless map image (presentation, not on the hot path). ----
 * The reference's result viewer draws its map with a WebGL fragment shader (viewer/viewer.js:
 * 72-100): a hillshade of the terrain, a logarithmic depth ramp (mode 0) or a diverging ramp
 * of depth differences (mode 1), and hatching where worse_dz > 1 cm. itr_gpu_render_map
 * computes the same image on the device without a graphics stack: rgba receives
 * (scale*nx) x (scale*ny) pixels, 4 bytes each, row 0 the northern row. z: cell levels (NaN
 * = no data); value: depth or difference per cell; worse_dz may be NULL (no hatching). */
int itr_gpu_render_map(itr_ctx* ctx, int32_t nx, int32_t ny, double cell_size, const float* z, const float* value,
                       const float* worse_dz, int32_t mode, float vex, int32_t scale, uint8_t* rgba);

/* ---- Headless flood-scene render (presentation, not on the hot path). ----
 * The reference's video renders each recorded frame with an SkSL ray marcher through Skia on
 * Metal (video/src/shaders/terrain.sksl; uniforms from video/src/lib.rs:52-77; textures packed
 * by video/src/data.rs:89-96). itr_gpu_render_scene runs the same shader on the device without
 * a graphics stack: rgba receives width x height pixels, 4 bytes each, row 0 the top.
 * Textures, 4 bytes per texel, row 0 the northern edge:
 *   terrain  tw x th (the simulation grid refined by `up`): R, G = elevation code (16 bit,
 *            R high) over z_span, B = material code (0 ground, 1-120 fill, 121-200 cut,
 *            >= 250 building)
 *   depth    nx x ny: R, G = depth code (16 bit) over depth_span, B = 255 where wet
 *   vel      nx x ny: R, G = velocity u, v as 128 + 127 v / vel_max
 * A texture read takes the texel under the coordinate, clamped to the image. */
typedef struct itr_scene_view {   /* the shader's uniforms */
  float cam_pos[3], cam_fwd[3], cam_right[3], cam_up[3];   /* camera frame (m; unit vectors) */
  float focal;                /* focal length in image-height units */
  float domain[3];            /* width, height, cell size (m) */
  float z_lo, z_span;         /* elevation of code 0 (m, not used by the shader) and of the code span */
  float up;                   /* terrain texels per simulation cell */
  float depth_span;           /* depth of code 65535 (m) */
  float ve;                   /* vertical exaggeration */
  float time;                 /* simulated time (s) */
  float rain, wet, overcast;  /* rain rate / peak rate, surface wetness, cloud cover, 0..1 */
  float vel_max;              /* velocity of code 255 (m/s) */
  float base;                 /* depth of the cut-away block below the lowest ground (m) */
  int32_t ortho;              /* 1: top-down map over the whole domain */
  int32_t debug;              /* 0 normal, 1 pixel coordinates, 2 elevation texture, 3 water texture */
} itr_scene_view;

int itr_gpu_render_scene(itr_ctx* ctx, const uint8_t* terrain, int32_t tw, int32_t th, const uint8_t* depth,
                         const uint8_t* vel, int32_t nx, int32_t ny, const itr_scene_view* view, int32_t width,
                         int32_t height, uint8_t* rgba);

/* ---- Allocation-free plain forward. No reference counterpart. ----
 * For callers that cannot allocate device memory when they run a design: a process that
 * has committed the whole device to its own pool, a caller whose other streams must not be
 * stalled by the device-wide synchronisation of cudaMalloc/cudaFree, a search loop that
 * must not fail mid-way on an out-of-memory error. It runs the plain path's kernels (same
 * bits as itr_gpu_run_batch) for ONE design on scratch held in a static device array of
 * fixed size. CUDA reserves that array when it loads the library's module on the device;
 * under CUDA's default lazy loading that is the first call on the device, not the opening
 * of the library. After that the call allocates nothing, on the device or the host. Inputs and results are host buffers with run_batch's meaning;
 * there is no objective (j = 0, no aborts), and boundaries are walls or transmissive
 * (stage and inflow cells, or inflow_scale other than 1, give ITR_UNSUPPORTED). Runs on
 * the device's legacy default stream and returns when the results are in the host buffers.
 * Limits, rejected with ITR_INVALID_ARG and a message in err before any device work: */
#define ITR_STATIC_MAX_POINTS 263169      /* (nx+1)*(ny+1), e.g. 512 x 512 cells      */
#define ITR_STATIC_MAX_TILES 16384        /* ceil(nx/16) * ceil(ny/16)                 */
#define ITR_STATIC_MAX_MONITORS 65536     /* n_mon                                     */
#define ITR_STATIC_MAX_LEDGER_ROWS 4096   /* result->max_rows when result->ledger set  */
/* One static array per device, shared by every call, which finds it holding the previous
 * call's contents (the call clears what must start at zero). Calls on the same device that
 * overlap in time (several host threads or streams) race on it and corrupt each other's
 * results. The first call on a device does the set-up: with that device current it loads the
 * module and looks up the array's device address (cudaGetSymbolAddress) and keeps it; make
 * that first call before any stream capture and before committing the device's memory to
 * another pool. Boundaries: walls and transmissive edges only, inflow_scale 1. */
int itr_gpu_run_plain_static(int device, const itr_params* p, const itr_grid* g, const itr_design* design,
                             const uint32_t* monitors, int32_t n_mon, itr_result* result, char* err, size_t errlen);

#ifdef __cplusplus
}
#endif
#endif /* ITR_GPU_H */
