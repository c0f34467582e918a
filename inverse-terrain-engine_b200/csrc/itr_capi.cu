// itr_capi.cu — the C ABI (include/itr_gpu.h): context, input checks, packing, launch
// configuration and autotuning, result assembly.
//
// Mirrors crates/itr-gpu/src/lib.rs: GpuSolver::new (:85) -> itr_gpu_create,
// run_batch (:149) -> itr_gpu_run_batch, adapter_info (:126) -> itr_gpu_info, and the
// input checks (:154-176) -> ITR_INVALID_ARG / ITR_UNSUPPORTED. The reference's rejections
// of stage and inflow boundaries and of inflow_scale != 1 (:166-176, backend.rs:53-55) are
// gone: build_boundaries and stage_depths pack them for the kernels.
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <cstdarg>
#include <cmath>
#include <string>
#include <vector>
#include <map>
#include <tuple>
#include <algorithm>
#include <chrono>
#include <mutex>
#include "../../include/itr_gpu.h"
#include "itr_device.cuh"
#include "itr_batched.cuh"
#include "itr_batched_table.cuh"
#include "itr_plain.cuh"
#include "itr_band.cuh"
#include "itr_adjoint.cuh"
#include "itr_adjoint_band.cuh"
#include "itr_design.cuh"
#include "itr_render.cuh"
#include "itr_raymarch.cuh"

using namespace itr;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr; n = 0;
    size_t b = bytes < 256 ? 256 : bytes;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaSuccess) n = b;
    return e;
  }
  void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct HostBuf {
  void* p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n && p) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr; n = 0;
    size_t b = bytes < 256 ? 256 : bytes;
    cudaError_t e = cudaMallocHost(&p, b);
    if (e == cudaSuccess) n = b;
    return e;
  }
  void release() { if (p) cudaFreeHost(p); p = nullptr; n = 0; }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct LaunchCfg {
  int C = 1, T = 512, W = 1, S = 1;
  size_t smem = 0;
  bool ok = false;
  bool tiled = false;   // the measured choice was the tiled HBM path
  int band = 1;         // ... with the row-band kernel (1) or the 16x16 tiles (0)
  bool bnd = false;     // the grid has stage or inflow cells (k_batched<..., BND>)
};

}  // namespace

// What the results phase of a batch needs (kept by a deferred ladder group until its launch).
struct Collect {
  int n = 0, n_mon = 0, max_rows = 0;
  size_t N = 0;
  int nx = 0;                        // cells per row (a skipped row's cell count)
  const itr_design* ds = nullptr;
  itr_result* res = nullptr;
  const itr_objective* ob = nullptr;
  const uint32_t* mon = nullptr;     // host monitor list
  const unsigned* dmon = nullptr;    // its device copy
  int launches = 0;
};

// A batch given as primitives (itr_gpu_run_primitives): the device materialises each design's
// jumps, stage depths and earthwork volumes from these before the forward.
struct Mat {
  const itr_design_space* space = nullptr;
  std::vector<MatPrim> prims;
  std::vector<MatDesign> des;
  std::vector<itr_design> ds;   // placeholders; cut/fill filled in from the device
};

// Baseline record for warm starts (BaselineRecord, solver.rs:95-118): checkpoints of the
// base terrain's run every K steps (state, peaks, integrator), which rows had held water by
// each, the base's ledger, and what the record was made with (to match later batches).
struct Record {
  bool valid = false;
  RunParams P;                                   // params, grid scalars, rain and inflow tables
  int nx = 0, ny = 0, mode = 0;
  std::vector<float> wet, gn2, dzx, dzy, dzx2, dzy2, bh, h0;   // h0 empty: initial_depth on open cells
  std::vector<uint8_t> bc, open_rows;            // device codes; rows beside stage / inflow edges
  struct Ckpt { DevBuf state; WarmStart ws; std::vector<uint8_t> wet; };   // state: [4][N] floats, then ny row flags
  std::vector<Ckpt> ck;
  std::vector<PlainCtl> ctl;                     // control block at each checkpoint
  std::vector<double> ledger;                    // base's ledger rows, 8 doubles each
  int K = 64;
};

struct itr_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  int sm_count = 0;
  size_t smem_optin = 0;
  char name[256] = {0};
  std::string err;
  // options
  int impl = 0, threads = 0, cluster = 0, graph = 1, steps_per_submit = 64;
  int autotune = 1, autotune_top = 6, probe_steps = 200;
  int exact_special = 0;
  int band = 1;           // tiled path update kernel: 1 = row-band sweep (k_band), 0 = 16x16 tiles
  int adj_band = -1;      // adjoint kernels on row bands: bit 0 the replay, bit 1 the backward step (else 16x16 tiles);
                          // -1: the replay on bands, the backward step on bands for grids of 2^18 cells or more
  int adj_trim = 1;       // adjoint: skip the steps after a design's latest asset maximum (zero adjoint there)
  unsigned wait_limit = 1u << 22;   // bounded barrier wait of single-CTA designs (try_wait rounds)
  int stall_wait_test = 0;          // test of the timeout path: that wait never completes
  float tune_ms = 0.0f;
  // baseline-locked dt (itr_gpu_set_locked_dt): the schedule, its limit, the snapshot buffers
  // and, per design of the last batch, the fallback time (-1: none)
  std::vector<double> locked_dt;
  double cfl_hard = 0.5;
  bool locked_run = false;
  DevBuf lDt, lS4, lS2, lSk, lSs, lFb;
  std::vector<double> fallback;
  // device buffers (batched path)
  DevBuf wet, gn2, bc, dzx, dzy, dzx2, dzy2, h0, cut, fill, mon, obj_i, obj_d, peak, depth, ledger, out, mmax;
  // plain path scratch
  DevBuf pH, pQX, pQY, pPK, ppart, pctl;
  // tiled batched path: state planes, tile partials, control blocks of all designs
  DevBuf tH, tQX, tQY, tpart, tctl;
  DevBuf tRow, tGw, tSnapRow;   // row-band path: dry-row flags, ghost wetness, flags at the locked snapshot
  // adjoint: argmax states, (dt, rain) ring, checkpoints, tape, adjoint state, gradients
  DevBuf aTpk, aRing, aTape, aTape2, aLA, aLB, aGx, aGy, aGx2, aGy2, aSeg, aNst, aSeedC, aSeedS, aSeedW, aSeedN, aTmon;
  DevBuf aPlan[2];   // row-band replay: the control blocks of each tape's segment, [K][n]
  cudaStream_t stream2 = nullptr;   // adjoint: the replay of the next segment runs beside the backward steps
  cudaEvent_t ev_rep[2] = {nullptr, nullptr}, ev_adj[2] = {nullptr, nullptr}, ev_bwd = nullptr;
  HostBuf aRingH;
  std::vector<DevBuf> aCkpt;
  struct Vjp* vjp = nullptr;
  Mat* mat = nullptr;
  Record* rec = nullptr;         // the baseline record (itr_gpu_record_baseline)
  Record* recording = nullptr;   // set while the record is being made
  int warm_start = 0;
  std::vector<uint64_t> warm_steps;   // per design of the last batch
  DevBuf wsb;
  DevBuf mDz, mZe, mAux, mJp, mJob, mOut;
  DevBuf rIn, rOut;   // map and scene rendering
  HostBuf mVol;
  // ladder: one child context per grid group; a deferred run stops before its launch
  std::vector<itr_ctx*> children;
  bool defer = false;
  bool pending_ok = false;
  Collect pending;
  cudaEvent_t ev_fork = nullptr;
  double vjp_fwd_ms = 0, vjp_bwd_ms = 0;
  HostBuf stage, hout;
  // last run
  double kernel_ms = 0, total_ms = 0;
  uint64_t cell_updates = 0;
  int launches = 0;
  bool have_last = false;
  BatchArgs last_args;
  LaunchCfg last_cfg;
  // plain rerun
  std::vector<PlainArgs> last_plain;
  std::vector<int> last_plain_blocks;
  bool last_was_plain = false;
  bool last_was_tiled = false;
  PlainArgs last_tiled;
  dim3 last_tgrid;
  int last_band = 1;   // the tiled update kernel of the last tiled batch (option band)
  // autotune cache: (nx, ny, n_designs, mode) -> cfg
  std::map<std::tuple<int, int, int, int>, LaunchCfg> tuned;
  cudaGraphExec_t gexec = nullptr;
};

static int fail(itr_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CU(x)                                                                                    \
  do {                                                                                           \
    cudaError_t e_ = (x);                                                                        \
    if (e_ != cudaSuccess) return fail(ctx, ITR_DEVICE_ERROR, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

// Step limit of every run on the device (status 4 beyond it).
constexpr unsigned long long kMaxSteps = 2000000000ull;

// ------------------------------------------------------------------ kernels table ----
#ifdef ITR_CHECKED
namespace itr {
ITR_BATCHED_TABLE(batched_fn_00, false, false)
ITR_BATCHED_TABLE(batched_fn_01, false, true)
ITR_BATCHED_TABLE(batched_fn_10, true, false)
ITR_BATCHED_TABLE(batched_fn_11, true, true)
}  // namespace itr
#endif

// skip: the dry-row instantiation (RunParams::skip_dry, set only when a rain-free step can occur)
static BatchedFn batched_fn(bool crest, bool clustered, int maxt, bool bnd, bool locked = false, bool skip = false) {
  if (crest) return bnd ? batched_fn_11(clustered, maxt, locked, skip) : batched_fn_10(clustered, maxt, locked, skip);
  return bnd ? batched_fn_01(clustered, maxt, locked, skip) : batched_fn_00(clustered, maxt, locked, skip);
}

static int maxt_bucket(int T) { return T <= 256 ? 256 : T <= 512 ? 512 : T <= 768 ? 768 : 1024; }

// Geometry of the batched kernel for (nx, ny) with C CTAs per design and about T threads.
static LaunchCfg make_cfg(const itr_ctx* ctx, int nx, int ny, int C, int T_target, bool crest, bool bnd) {
  LaunchCfg c;
  c.C = C;
  c.bnd = bnd;
  c.W = (nx + 1 + 63) / 64;   // warps per strip row; each lane holds two columns
  if (C < 1 || ny < C) return c;
  const int nr_min = ny / C, nr_max = (ny + C - 1) / C;
  int S = T_target / (32 * c.W);
  if (c.W > 1 && S > 15) S = 15;   // one named barrier per strip (ids 1..15)
  if (S > nr_min) S = nr_min;
  if (S < 1) return c;
  c.S = S;
  c.T = S * 32 * c.W;
  if (c.T > 1024) return c;
  c.smem = batched_smem_bytes(nr_max, nx, S, c.W, c.T / 32, crest ? 1 : 0, bnd ? 1 : 0, ny);
  c.ok = c.smem <= ctx->smem_optin;
  return c;
}

static int launch_batched(itr_ctx* ctx, const BatchArgs& A, const LaunchCfg& cfg, int n_designs, bool set_attr = true) {
  const bool crest = A.mode == 1, clustered = cfg.C > 1;
  BatchedFn fn = batched_fn(crest, clustered, maxt_bucket(cfg.T), cfg.bnd, A.locked_dt != nullptr, A.P.skip_dry != 0);
  if (set_attr) CU(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
  cudaLaunchConfig_t lc;
  memset(&lc, 0, sizeof(lc));
  lc.gridDim = dim3((unsigned)(n_designs * cfg.C), 1, 1);
  lc.blockDim = dim3((unsigned)cfg.T, 1, 1);
  lc.dynamicSmemBytes = cfg.smem;
  lc.stream = ctx->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)cfg.C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  CU(cudaLaunchKernelEx(&lc, fn, A));
  return ITR_OK;
}

static int max_active_clusters(itr_ctx* ctx, const LaunchCfg& cfg, bool crest) {
  BatchedFn fn = batched_fn(crest, cfg.C > 1, maxt_bucket(cfg.T), cfg.bnd);
  if (cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem) != cudaSuccess) return 0;
  cudaLaunchConfig_t lc;
  memset(&lc, 0, sizeof(lc));
  lc.gridDim = dim3((unsigned)(cfg.C * 148), 1, 1);
  lc.blockDim = dim3((unsigned)cfg.T, 1, 1);
  lc.dynamicSmemBytes = cfg.smem;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)cfg.C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, fn, &lc) != cudaSuccess) { cudaGetLastError(); return 0; }
  return n;
}

// Candidate configurations, best-first by a simple model: time ~ waves * work per CTA.
static std::vector<LaunchCfg> candidates(itr_ctx* ctx, int nx, int ny, int n_designs, bool crest, bool bnd) {
  std::vector<std::pair<double, LaunchCfg>> v;
  for (int C : {1, 2, 4, 8}) {
    for (int T : {256, 384, 512, 640, 768, 896, 1024}) {
      LaunchCfg c = make_cfg(ctx, nx, ny, C, T, crest, bnd);
      if (!c.ok) continue;
      bool dup = false;
      for (auto& e : v) if (e.second.C == c.C && e.second.T == c.T) dup = true;
      if (dup) continue;
      int act = max_active_clusters(ctx, c, crest);
      if (act <= 0) continue;
      double waves = std::ceil((double)n_designs / act);
      double rows = std::ceil((double)ny / C);
      // per-CTA cost ~ cells per thread; small penalty per cluster barrier
      double per_step = rows * nx / (double)c.T * (1.0 + 0.02 * (C - 1)) + 0.5;
      double cost = waves * per_step;
      v.push_back({cost, c});
    }
  }
  std::sort(v.begin(), v.end(), [](const std::pair<double, LaunchCfg>& a, const std::pair<double, LaunchCfg>& b) { return a.first < b.first; });
  std::vector<LaunchCfg> out;
  for (auto& p : v) out.push_back(p.second);
  return out;
}

// Time `probe_steps` steps of the batch under each candidate shape (CUDA events on the
// context stream) and return the fastest. The probe runs write only scratch outputs.
static int autotune(itr_ctx* ctx, const BatchArgs& A0, const std::vector<LaunchCfg>& cands, int n, LaunchCfg* best) {
  BatchArgs A = A0;
  A.max_steps = (unsigned long long)ctx->probe_steps;
  A.warm = nullptr;   // probe the cold start: the shapes compare the same
  A.ledger_out = nullptr;
  A.max_rows = 0;
  A.obj.enabled = 0;
  float best_ms = 1e30f;
  const size_t k = cands.size() < (size_t)ctx->autotune_top ? cands.size() : (size_t)ctx->autotune_top;
  for (size_t i = 0; i < k; ++i) {
    LaunchCfg c = cands[i];
    A.C = c.C; A.W = c.W; A.S = c.S;
    float ms = 0.0f;
    for (int rep = 0; rep < 2; ++rep) {   // first launch warms the instruction cache
      CU(cudaEventRecord(ctx->ev[1], ctx->stream));
      int rc = launch_batched(ctx, A, c, n);
      if (rc != ITR_OK) return rc;
      CU(cudaEventRecord(ctx->ev[2], ctx->stream));
      CU(cudaEventSynchronize(ctx->ev[2]));
      CU(cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]));
    }
    if (ms < best_ms) { best_ms = ms; *best = c; }
  }
  ctx->tune_ms = best_ms;
  return ITR_OK;
}

// ------------------------------------------------------------------ input checks ------
constexpr float kMaxInitialDepth = 1e4f;   // m

static int check_inputs(itr_ctx* ctx, const itr_params* p, const itr_grid* g, int32_t n, const itr_design* ds,
                        const uint32_t* mon, int32_t n_mon, const itr_objective* ob) {
  if (!p || !g) return fail(ctx, ITR_INVALID_ARG, "params and grid are required");
  if (n < 0) return fail(ctx, ITR_INVALID_ARG, "negative design count");
  if (n > 0 && !ds) return fail(ctx, ITR_INVALID_ARG, "designs is NULL");
  if (g->nx < 1 || g->ny < 1) return fail(ctx, ITR_INVALID_ARG, "grid must have nx, ny >= 1");
  if ((int64_t)g->nx * g->ny > (1ll << 30)) return fail(ctx, ITR_INVALID_ARG, "grid too large");
  if (!(g->dx > 0.0) || !(g->dy > 0.0)) return fail(ctx, ITR_INVALID_ARG, "cell size must be positive");
  if (!g->wet || !g->gn2 || !g->bc) return fail(ctx, ITR_INVALID_ARG, "grid arrays wet, gn2, bc are required");
  if (g->mode != ITR_FACE_SIGNED && g->mode != ITR_FACE_CREST) return fail(ctx, ITR_INVALID_ARG, "unknown face mode %d", g->mode);
  bool has_stage = false, has_inflow = false;
  for (int64_t i = 0; i < 2ll * g->nx + 2ll * g->ny; ++i) {
    if (g->bc[i] > ITR_BC_INFLOW) return fail(ctx, ITR_INVALID_ARG, "unknown boundary code %d", (int)g->bc[i]);
    has_stage = has_stage || g->bc[i] == ITR_BC_STAGE;
    has_inflow = has_inflow || g->bc[i] == ITR_BC_INFLOW;
  }
  if (has_stage) {
    if (!g->bc_stage) return fail(ctx, ITR_INVALID_ARG, "grid has stage cells but bc_stage is NULL");
    for (int32_t d = 0; d < n && !ctx->mat; ++d)
      if (!ds[d].z_edge) return fail(ctx, ITR_INVALID_ARG, "grid has stage cells but design %d has no z_edge", d);
  }
  if (has_inflow) {
    if (!g->bc_hydro || !g->bc_inv_len || !g->hydro_off || g->n_hydro < 1)
      return fail(ctx, ITR_INVALID_ARG, "grid has inflow cells but no inflow tables (bc_hydro, bc_inv_len, hydro_off, n_hydro)");
    if (g->hydro_off[0] < 0) return fail(ctx, ITR_INVALID_ARG, "hydro_off[0] is negative");
    for (int h = 0; h < g->n_hydro; ++h)
      if (g->hydro_off[h + 1] < g->hydro_off[h]) return fail(ctx, ITR_INVALID_ARG, "hydro_off is not non-decreasing");
    if (g->hydro_off[g->n_hydro] > 0 && (!g->hydro_t || !g->hydro_q)) return fail(ctx, ITR_INVALID_ARG, "hydrograph arrays are NULL");
    for (int64_t i = 0; i < 2ll * g->nx + 2ll * g->ny; ++i) {
      if (g->bc[i] != ITR_BC_INFLOW) continue;
      if (g->bc_hydro[i] < 0 || g->bc_hydro[i] >= g->n_hydro) return fail(ctx, ITR_INVALID_ARG, "boundary cell %lld: hydrograph index %d out of range", (long long)i, g->bc_hydro[i]);
      if (!(g->bc_inv_len[i] >= 0.0) || !std::isfinite(g->bc_inv_len[i])) return fail(ctx, ITR_INVALID_ARG, "boundary cell %lld: bad 1/length", (long long)i);
    }
    if (!std::isfinite(p->inflow_scale)) return fail(ctx, ITR_INVALID_ARG, "inflow_scale is not finite");
  }
  if (!(p->duration_s >= 0.0) || !(p->sync_interval_s > 0.0) || !(p->cfl > 0.0) || !(p->dt_max_s > 0.0))
    return fail(ctx, ITR_INVALID_ARG, "duration, sync interval, cfl and dt_max must be positive");
  if (p->n_rain < 0 || p->n_rain > kMaxRain) return fail(ctx, ITR_INVALID_ARG, "hyetograph has %d points (max %d)", p->n_rain, kMaxRain);
  if (p->n_rain > 0 && (!p->rain_t || !p->rain_rate)) return fail(ctx, ITR_INVALID_ARG, "hyetograph arrays are NULL");
  if (n_mon < 0 || (n_mon > 0 && !mon)) return fail(ctx, ITR_INVALID_ARG, "monitor list is invalid");
  for (int32_t k = 0; k < n_mon; ++k)
    if ((int64_t)mon[k] >= (int64_t)g->nx * g->ny) return fail(ctx, ITR_INVALID_ARG, "monitor cell out of range");
  for (int32_t d = 0; d < n && !ctx->mat; ++d) {
    if (!ds[d].dzx || !ds[d].dzy) return fail(ctx, ITR_INVALID_ARG, "design %d has no face jumps", d);
    if (g->mode == ITR_FACE_CREST && (!ds[d].dzx2 || !ds[d].dzy2)) return fail(ctx, ITR_INVALID_ARG, "design %d: crest mode needs dzx2/dzy2", d);
    // An infinite or absurdly deep start makes the first CFL dt zero or vanishing, so the run
    // would crawl towards its step limit; NaN and negative depths are left to the solver's
    // health test (Unhealthy at the first step, numerics.rs:163, solver.rs:541-544).
    if (ds[d].h0)
      for (size_t i = 0; i < (size_t)g->nx * g->ny; ++i)
        if (std::isinf(ds[d].h0[i]) || ds[d].h0[i] > kMaxInitialDepth)
          return fail(ctx, ITR_INVALID_ARG, "design %d: initial depth %g at cell %zu is infinite or above %g m", d,
                      (double)ds[d].h0[i], i, (double)kMaxInitialDepth);
  }
  if (ob) {
    if (ob->n_assets < 0 || ob->n_guard < 0) return fail(ctx, ITR_INVALID_ARG, "objective counts are negative");
    if (ob->n_assets > 0 && (!ob->asset_off || !ob->asset_pos || !ob->asset_threshold || !ob->asset_weight))
      return fail(ctx, ITR_INVALID_ARG, "objective asset arrays are NULL");
    for (int a = 0; a < ob->n_assets; ++a)
      for (int m = ob->asset_off[a]; m < ob->asset_off[a + 1]; ++m)
        if (ob->asset_pos[m] < 0 || ob->asset_pos[m] >= n_mon) return fail(ctx, ITR_INVALID_ARG, "asset position out of range");
    if (ob->n_guard > 0 && !ob->guard_pos) return fail(ctx, ITR_INVALID_ARG, "guard positions are NULL");
    for (int k = 0; k < ob->n_guard; ++k)
      if (ob->guard_pos[k] < 0 || ob->guard_pos[k] >= n_mon) return fail(ctx, ITR_INVALID_ARG, "guard position out of range");
    if (!(ob->tau > 0.0)) return fail(ctx, ITR_INVALID_ARG, "tau must be positive");
  }
  return ITR_OK;
}

// The storm's rate (linear between breakpoints, constant before the first and after the last)
// is 0 over an interval of positive length inside [0, duration], so a step of the run can be
// rain-free. Unsorted breakpoints: conservatively true. (A step inside a storm that is positive
// almost everywhere has a mean rate > 0 unless it is shorter than about 1e-30 s.)
static bool rain_free_stretch(const RunParams& P) {
  const Rain& R = P.rain;
  const double T = P.duration;
  if (R.n == 0 || !P.rain_sorted) return true;
  if (R.r[0] <= 0.0 && R.t[0] > 0.0) return true;
  if (R.r[R.n - 1] <= 0.0 && R.t[R.n - 1] < T) return true;
  for (int k = 0; k + 1 < R.n; ++k) {
    const double a = R.t[k] > 0.0 ? R.t[k] : 0.0, b = R.t[k + 1] < T ? R.t[k + 1] : T;
    if (R.r[k] <= 0.0 && R.r[k + 1] <= 0.0 && a < b) return true;
  }
  return false;
}

static RunParams make_run_params(const itr_params* p, const itr_grid* g) {
  RunParams P;
  memset(&P, 0, sizeof(P));
  P.duration = p->duration_s; P.sync = p->sync_interval_s; P.cfl = p->cfl; P.dt_max = p->dt_max_s;
  P.h_dry = p->h_dry; P.h_eps = p->h_eps; P.infil = p->infil_capacity; P.initial_depth = p->initial_depth;
  P.dx = g->dx; P.dy = g->dy; P.g = g->g; P.area = g->dx * g->dy; P.wet_count = (double)g->wet_count;
  P.n_sync = (uint32_t)std::ceil(p->duration_s / p->sync_interval_s);
  P.skip_dry = p->skip_dry;
  P.rain.n = p->n_rain;
  for (int i = 0; i < p->n_rain; ++i) { P.rain.t[i] = p->rain_t[i]; P.rain.r[i] = p->rain_rate[i]; }
  P.rain_sorted = 1;
  for (int i = 1; i < p->n_rain; ++i) if (!(p->rain_t[i] >= p->rain_t[i - 1])) P.rain_sorted = 0;
  // Dry-row skipping can act only on a step without rain: keep it on only when the storm has
  // a rain-free stretch inside the run (no skipping is possible otherwise, and the kernels
  // then leave out its bookkeeping; the results are the same either way).
  if (P.skip_dry && !rain_free_stretch(P)) P.skip_dry = 0;
  P.g_f = (float)g->g; P.g_half_f = (float)(0.5 * g->g);
  P.inv_dx_f = (float)(1.0 / g->dx); P.inv_dy_f = (float)(1.0 / g->dy);
  P.h_dry_f = (float)p->h_dry; P.heps2_f = (float)(p->h_eps * p->h_eps); P.q_min_f = (float)1e-30;
  P.nz = -0.0f;
  P.inflow.n = 0;   // build_boundaries fills the groups
  P.inflow.scale = p->inflow_scale;
  return P;
}

// Device boundary codes and inflow groups of a grid (boundary.rs:12-87): an inflow cell's
// code becomes 3 + its group, a group being a distinct (hydrograph, 1 / segment length)
// pair in boundary-cell order; other codes are copied. Stage depths are per design
// (stage_depths).
static int build_boundaries(itr_ctx* ctx, const itr_grid* g, Inflow& F, uint8_t* dbc) {
  const int64_t nb = 2ll * g->nx + 2ll * g->ny;
  int hyd[kMaxInflow];
  int npts = 0;
  F.n = 0;
  F.off[0] = 0;
  for (int64_t i = 0; i < nb; ++i) {
    const uint8_t c = g->bc[i];
    if (c != ITR_BC_INFLOW) { dbc[i] = c; continue; }
    const int h = g->bc_hydro[i];
    const double il = g->bc_inv_len[i];
    int k = 0;
    while (k < F.n && !(hyd[k] == h && F.inv_len[k] == il)) ++k;
    if (k == F.n) {
      if (F.n == kMaxInflow) return fail(ctx, ITR_UNSUPPORTED, "more than %d inflow groups (hydrograph, segment length)", kMaxInflow);
      const int a = g->hydro_off[h], b = g->hydro_off[h + 1];
      if (npts + (b - a) > kMaxInflowPts) return fail(ctx, ITR_UNSUPPORTED, "inflow hydrographs have more than %d points in all", kMaxInflowPts);
      for (int j = a; j < b; ++j) { F.t[npts] = g->hydro_t[j]; F.q[npts] = g->hydro_q[j]; ++npts; }
      hyd[k] = h;
      F.inv_len[k] = il;
      F.n += 1;
      F.off[F.n] = npts;
    }
    dbc[i] = (uint8_t)(3 + k);
  }
  return ITR_OK;
}

// Stage-ghost depth of every boundary cell of one design, f32(max(stage - z, 0)) rounded
// once from f64 (boundary.rs:45,68); 0 at other cells.
static void stage_depths(const itr_grid* g, const double* z_edge, float* out) {
  const int64_t nb = 2ll * g->nx + 2ll * g->ny;
  for (int64_t i = 0; i < nb; ++i) {
    if (g->bc[i] != ITR_BC_STAGE) { out[i] = 0.0f; continue; }
    const double v = g->bc_stage[i] - z_edge[i];
    out[i] = (float)(v > 0.0 ? v : 0.0);   // max(NaN, 0) is 0, as f64::max
  }
}

// Host copy of the objective (objective.rs:94-128) for J and feasibility of a finished run.
static void host_objective(const itr_objective* ob, const double* mm, double cut, double fill, double& j, double& worst) {
  double jr = 0.0;
  for (int a = 0; a < ob->n_assets; ++a) {
    double pk = 0.0;
    for (int m = ob->asset_off[a]; m < ob->asset_off[a + 1]; ++m) { double x = mm[ob->asset_pos[m]]; pk = pk > x ? pk : x; }
    jr += ob->asset_weight[a] * ob->tau * itr_math::softplus((pk - ob->asset_threshold[a]) / ob->tau);
  }
  j = jr + ob->earth_weight * (ob->cut_cost * cut + ob->fill_cost * fill);
  worst = 0.0;
  if (ob->baseline_max)
    for (int k = 0; k < ob->n_guard; ++k) {
      int mp = ob->guard_pos[k];
      double w = mm[mp] - ob->baseline_max[mp];
      worst = worst > w ? worst : w;
    }
}

// Gather monitor maxima from the per-cell peak array on the device.
__global__ void k_gather_monitors(const float* peak, const unsigned* mon, int n_mon, size_t cells, int n_designs, float* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_mon * n_designs) return;
  int d = i / n_mon, k = i % n_mon;
  out[i] = peak[(size_t)d * cells + mon[k]];
}

extern "C" {

itr_ctx* itr_gpu_create(int device, char* err, size_t errlen) {
  auto bad = [&](const char* what, cudaError_t e) -> itr_ctx* {
    if (err && errlen) snprintf(err, errlen, "%s: %s", what, cudaGetErrorString(e));
    return nullptr;
  };
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) return bad("cudaGetDeviceCount", e);
  if (n == 0) { if (err && errlen) snprintf(err, errlen, "no CUDA device"); return nullptr; }
  int dev = device;
  if (dev < 0) { e = cudaGetDevice(&dev); if (e != cudaSuccess) return bad("cudaGetDevice", e); }
  if (dev >= n) { if (err && errlen) snprintf(err, errlen, "device %d out of range (%d devices)", dev, n); return nullptr; }
  e = cudaSetDevice(dev);
  if (e != cudaSuccess) return bad("cudaSetDevice", e);
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) return bad("cudaGetDeviceProperties", e);
  if (prop.major < 10) {
    if (err && errlen) snprintf(err, errlen, "device %d (%s, sm_%d%d) is not sm_100; this build targets B200 only", dev, prop.name, prop.major, prop.minor);
    return nullptr;
  }
  itr_ctx* c = new itr_ctx();
  c->device = dev;
  c->sm_count = prop.multiProcessorCount;
  c->smem_optin = prop.sharedMemPerBlockOptin;
  snprintf(c->name, sizeof(c->name), "%s", prop.name);
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return bad("cudaStreamCreate", e); }
  for (int i = 0; i < 4; ++i) cudaEventCreate(&c->ev[i]);
  return c;
}

void itr_gpu_destroy(itr_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  for (DevBuf* b : {&ctx->wet, &ctx->gn2, &ctx->bc, &ctx->dzx, &ctx->dzy, &ctx->dzx2, &ctx->dzy2, &ctx->h0, &ctx->cut, &ctx->fill,
                    &ctx->mon, &ctx->obj_i, &ctx->obj_d, &ctx->peak, &ctx->depth, &ctx->ledger, &ctx->out, &ctx->mmax,
                    &ctx->pH, &ctx->pQX, &ctx->pQY, &ctx->pPK, &ctx->ppart, &ctx->pctl, &ctx->tH, &ctx->tQX, &ctx->tQY,
                    &ctx->tpart, &ctx->tctl, &ctx->tRow, &ctx->tGw, &ctx->tSnapRow, &ctx->aTpk, &ctx->aRing, &ctx->aTape, &ctx->aTape2, &ctx->aLA, &ctx->aLB, &ctx->aGx, &ctx->aGy, &ctx->aGx2, &ctx->aGy2,
                    &ctx->aSeg, &ctx->aNst, &ctx->aSeedC, &ctx->aSeedS, &ctx->aSeedW, &ctx->aSeedN, &ctx->aTmon,
                    &ctx->mDz, &ctx->mZe, &ctx->mAux, &ctx->mJp, &ctx->mJob, &ctx->mOut, &ctx->wsb, &ctx->rIn, &ctx->rOut,
                    &ctx->lDt, &ctx->lS4, &ctx->lS2, &ctx->lSk, &ctx->lSs, &ctx->lFb})
    b->release();
  for (DevBuf& b : ctx->aCkpt) b.release();
  for (itr_ctx* c : ctx->children) itr_gpu_destroy(c);
  if (ctx->rec) {
    for (auto& c : ctx->rec->ck) c.state.release();
    delete ctx->rec;
  }
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  for (int i = 0; i < 2; ++i) {
    if (ctx->ev_rep[i]) cudaEventDestroy(ctx->ev_rep[i]);
    if (ctx->ev_adj[i]) cudaEventDestroy(ctx->ev_adj[i]);
  }
  if (ctx->ev_bwd) cudaEventDestroy(ctx->ev_bwd);
  if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
  ctx->aRingH.release();
  ctx->mVol.release();
  ctx->stage.release();
  ctx->hout.release();
  for (int i = 0; i < 4; ++i) if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* itr_gpu_last_error(itr_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int itr_gpu_info(itr_ctx* ctx, char* buf, size_t len) {
  if (!ctx || !buf || !len) return ITR_INVALID_ARG;
  size_t fr = 0, tot = 0;
  cudaSetDevice(ctx->device);
  cudaMemGetInfo(&fr, &tot);
  int k = snprintf(buf, len, "%s (device %d, %d SMs, %.1f GB, %zu B smem/CTA opt-in; itr_gpu ABI %d, sm_100a)", ctx->name,
                   ctx->device, ctx->sm_count, tot / 1e9, ctx->smem_optin, ITR_GPU_ABI_VERSION);
  if (k > 0 && (size_t)k < len && ctx->have_last && !ctx->last_was_plain && !ctx->last_was_tiled)
    snprintf(buf + k, len - (size_t)k, "; last batch: cluster kernel, %d CTAs x %d threads (%d strips of %d warps)",
             ctx->last_cfg.C, ctx->last_cfg.T, ctx->last_cfg.S, ctx->last_cfg.W);
  else if (k > 0 && (size_t)k < len && ctx->have_last && ctx->last_was_tiled)
    snprintf(buf + k, len - (size_t)k, "; last batch: tiled path (%s)", ctx->band ? "row bands" : "16x16 tiles");
  return ITR_OK;
}

int itr_gpu_set_option(itr_ctx* ctx, const char* key, int64_t value) {
  if (!ctx || !key) return ITR_INVALID_ARG;
  std::string k(key);
  if (k == "impl") { if (value < 0 || value > 2) return fail(ctx, ITR_INVALID_ARG, "impl must be 0, 1 or 2"); ctx->impl = (int)value; }
  else if (k == "threads") { if (value < 0 || value > 1024) return fail(ctx, ITR_INVALID_ARG, "threads out of range"); ctx->threads = (int)value; }
  else if (k == "cluster") { if (!(value == 0 || value == 1 || value == 2 || value == 4 || value == 8)) return fail(ctx, ITR_INVALID_ARG, "cluster must be 0,1,2,4,8"); ctx->cluster = (int)value; }
  else if (k == "graph") ctx->graph = value != 0;
  else if (k == "steps_per_submit") { if (value < 1) return fail(ctx, ITR_INVALID_ARG, "steps_per_submit must be >= 1"); ctx->steps_per_submit = (int)value; }
  else if (k == "autotune") { ctx->autotune = value != 0; ctx->tuned.clear(); }
  else if (k == "exact_special") ctx->exact_special = value != 0;
  else if (k == "warm_start") ctx->warm_start = value != 0;
  else if (k == "band") ctx->band = value != 0;
  else if (k == "adj_trim") ctx->adj_trim = value != 0;
  else if (k == "adj_band") { if (value < -1 || value > 3) return fail(ctx, ITR_INVALID_ARG, "adj_band is -1 .. 3"); ctx->adj_band = (int)value; }
  else if (k == "wait_limit") { if (value < 1 || value > 0x7fffffff) return fail(ctx, ITR_INVALID_ARG, "wait_limit out of range"); ctx->wait_limit = (unsigned)value; }
  else if (k == "stall_wait_test") ctx->stall_wait_test = value != 0;
  else if (k == "probe_steps") { if (value < 1) return fail(ctx, ITR_INVALID_ARG, "probe_steps must be >= 1"); ctx->probe_steps = (int)value; }
  else return fail(ctx, ITR_INVALID_ARG, "unknown option '%s'", key);
  if (k == "threads" || k == "cluster") ctx->tuned.clear();
  return ITR_OK;
}

int itr_gpu_set_locked_dt(itr_ctx* ctx, const double* dt, uint64_t n, double cfl_hard) {
  if (!ctx) return ITR_INVALID_ARG;
  if (n > 0 && !dt) return fail(ctx, ITR_INVALID_ARG, "locked dt schedule is NULL");
  if (n > 0 && !(cfl_hard > 0.0)) return fail(ctx, ITR_INVALID_ARG, "cfl_hard must be positive");
  for (uint64_t i = 0; i < n; ++i)
    if (!(dt[i] > 0.0) || !std::isfinite(dt[i])) return fail(ctx, ITR_INVALID_ARG, "locked dt %llu is not a positive number", (unsigned long long)i);
  ctx->locked_dt.assign(dt ? dt : nullptr, dt ? dt + n : nullptr);
  ctx->cfl_hard = cfl_hard;
  return ITR_OK;
}

int itr_gpu_last_timing(itr_ctx* ctx, double* kernel_ms, double* total_ms, uint64_t* cell_updates, int32_t* launches) {
  if (!ctx) return ITR_INVALID_ARG;
  if (kernel_ms) *kernel_ms = ctx->kernel_ms;
  if (total_ms) *total_ms = ctx->total_ms;
  if (cell_updates) *cell_updates = ctx->cell_updates;
  if (launches) *launches = ctx->launches;
  return ITR_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ plain path ------
// One step's update kernel of the tiled path: the ghost rule with stage and inflow cells
// only where the grid has them.
static void launch_update(const PlainArgs& A, dim3 grid, cudaStream_t st) {
  const bool bnd = A.bh != nullptr || A.P.inflow.n > 0;
  if (A.mode == 1) {
    if (bnd) k_plain_update<true, true><<<grid, kTileThreads, 0, st>>>(A);
    else k_plain_update<true, false><<<grid, kTileThreads, 0, st>>>(A);
  } else {
    if (bnd) k_plain_update<false, true><<<grid, kTileThreads, 0, st>>>(A);
    else k_plain_update<false, false><<<grid, kTileThreads, 0, st>>>(A);
  }
}

// One step's update of the tiled batched path: the row-band sweep (itr_band.cuh) over
// (segment groups, bands, designs), or with option band = 0 the 16x16-tile kernel.
static void launch_tiled_update(const itr_ctx* ctx, const PlainArgs& A, dim3 grid, cudaStream_t st) {
  if (!ctx->band) { launch_update(A, grid, st); return; }
  const bool bnd = A.bh != nullptr || A.P.inflow.n > 0;
  const BandGeom bg = band_geom(A.nx, A.ny, A.band_rows);
  const dim3 block((unsigned)(32 * bg.wpb));
  if (A.mode == 1) {
    if (bnd) k_band<true, true><<<grid, block, 0, st>>>(A);
    else k_band<true, false><<<grid, block, 0, st>>>(A);
  } else {
    if (bnd) k_band<false, true><<<grid, block, 0, st>>>(A);
    else k_band<false, false><<<grid, block, 0, st>>>(A);
  }
}

// Blocks per design of the tiled path's update (the finalize's partials).
static dim3 tiled_grid(const itr_ctx* ctx, int nx, int ny, int n) {
  if (!ctx->band) return dim3((nx + kTile - 1) / kTile, (ny + kTile - 1) / kTile);
  const BandGeom bg = band_geom(nx, ny, band_rows_for(nx, ny, n, ctx->sm_count));
  return dim3((unsigned)bg.gx, (unsigned)bg.gy);
}

static int run_plain_design(itr_ctx* ctx, PlainArgs& A, int n_blocks, dim3 grid, int* launches) {
  k_plain_init<<<1, 1024, 0, ctx->stream>>>(A);
  k_plain_finalize<<<1, 32, 0, ctx->stream>>>(A, n_blocks, 1);
  *launches += 2;
  int done = 0;
  PlainCtl* hctl = ctx->hout.as<PlainCtl>();
  for (uint64_t guard = 0;; ++guard) {
    for (int s = 0; s < ctx->steps_per_submit; ++s) {
      launch_update(A, grid, ctx->stream);
      k_plain_finalize<<<1, kFinThreads, 0, ctx->stream>>>(A, n_blocks, 0);
      *launches += 2;
    }
    CU(cudaMemcpyAsync(hctl, A.ctl, sizeof(PlainCtl), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    done = hctl->done;
    if (done) break;
    // the device stops a run at its step limit (status 4), so this bound never ends a run
    if (guard > kMaxSteps / (uint64_t)ctx->steps_per_submit + 2) return fail(ctx, ITR_DEVICE_TIMEOUT, "plain run did not terminate");
  }
  return ITR_OK;
}

// ------------------------------------------------------------------ tiled batch ------
// All designs per launch: one update (tiles x designs) and one finalize (a warp per design)
// per step, driven entirely by the control blocks on the device, so a block of
// steps_per_submit steps is captured once in a CUDA graph and replayed until every design
// is done (the host reads the control blocks between replays).
// Adjoint request: while set, run_batch takes the tiled path and records a tape.
struct Vjp {
  int K;                                  // checkpoint interval (steps)
  std::vector<std::vector<double>> dt;    // per design: (dt, rain, t) of every step taken
  uint64_t blocks = 0;                    // checkpoints written (one per block of K steps)
  double* gx;                             // host outputs
  double* gy;
  double* gx2 = nullptr;                  // crest mode: gradients of the second jumps
  double* gy2 = nullptr;
};

static int run_tiled_batch(itr_ctx* ctx, PlainArgs& A, int n, dim3 tgrid, int* launches) {
  const int nb = (int)(tgrid.x * tgrid.y);
  const dim3 grid(tgrid.x, tgrid.y, (unsigned)n);
  const cudaStream_t st = ctx->stream;
  Vjp* tape = ctx->vjp;
  const size_t N = (size_t)A.nx * A.ny;
  // baseline-locked dt: the LOCKED finalize, each followed by the snapshot copy it may ask for
  const bool locked = A.locked_dt != nullptr;
  const dim3 cgrid(64, (unsigned)n);
  k_plain_init<<<n, 1024, 0, st>>>(A);
  if (locked) {
    k_plain_finalize_locked<<<n, 32, 0, st>>>(A, nb, 1);
    k_plain_locked_copy<<<cgrid, 256, 0, st>>>(A);
    *launches += 1;
  } else {
    k_plain_finalize<<<n, 32, 0, st>>>(A, nb, 1);
  }
  *launches += 2;
  const int K = tape ? tape->K : ctx->steps_per_submit;
  if (tape) { tape->dt.assign(n, std::vector<double>()); tape->blocks = 0; }
  auto block = [&]() {
    for (int s = 0; s < K; ++s) {
      launch_tiled_update(ctx, A, grid, st);
      if (locked) {
        k_plain_finalize_locked<<<n, kFinThreads, 0, st>>>(A, nb, 0);
        k_plain_locked_copy<<<cgrid, 256, 0, st>>>(A);
      } else {
        k_plain_finalize<<<n, kFinThreads, 0, st>>>(A, nb, 0);
      }
    }
  };
  cudaGraphExec_t ge = nullptr;
  if (ctx->graph) {
    cudaGraph_t gr = nullptr;
    CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    block();
    CU(cudaStreamEndCapture(st, &gr));
    const cudaError_t e = cudaGraphInstantiate(&ge, gr, 0);
    cudaGraphDestroy(gr);
    CU(e);
  }
  PlainCtl* hc = ctx->hout.as<PlainCtl>();
  int rc = ITR_OK;
  Record* rec = ctx->recording;
  if (rec) {   // the control block after the first plan: checkpoint 0's integrator
    CU(cudaMemcpyAsync(hc, A.ctl, sizeof(PlainCtl), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
  }
  for (uint64_t polls = 0;; ++polls) {
    if (rec) {   // baseline record: state, peaks and integrator at the start of this block
      rec->ck.emplace_back();
      Record::Ckpt& ck = rec->ck.back();
      cudaError_t e = ck.state.ensure(4 * N * 4 + (size_t)A.ny);
      if (e != cudaSuccess) { rc = fail(ctx, ITR_DEVICE_ERROR, "baseline record: %s", cudaGetErrorString(e)); break; }
      k_rec_state<<<dim3(64), 256, 0, st>>>(A, ck.state.as<float>());
      k_rec_rows<<<dim3((unsigned)A.ny), 128, 0, st>>>(A, ck.state.as<float>(), ck.state.as<uint8_t>() + 4 * N * 4);
      *launches += 2;
      rec->ctl.push_back(hc[0]);
    }
    if (tape) {   // checkpoint: the state at the start of this block
      if (ctx->aCkpt.size() <= polls) ctx->aCkpt.emplace_back();
      cudaError_t e = ctx->aCkpt[polls].ensure((size_t)n * 3 * N * 4);
      if (e != cudaSuccess) { rc = fail(ctx, ITR_DEVICE_ERROR, "checkpoint %llu: %s", (unsigned long long)polls, cudaGetErrorString(e)); break; }
      k_adj_ckpt<<<dim3(64, (unsigned)n), 256, 0, st>>>(A, ctx->aCkpt[polls].as<float>());
      *launches += 1;
      tape->blocks = polls + 1;
    }
    if (ge) { const cudaError_t e = cudaGraphLaunch(ge, st); if (e != cudaSuccess) { rc = fail(ctx, ITR_DEVICE_ERROR, "cudaGraphLaunch: %s", cudaGetErrorString(e)); break; } }
    else block();
    *launches += (locked ? 3 : 2) * K;
    cudaError_t e = cudaMemcpyAsync(hc, A.ctl, (size_t)n * sizeof(PlainCtl), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { rc = fail(ctx, ITR_DEVICE_ERROR, "tiled run: %s", cudaGetErrorString(e)); break; }
    if (tape) {   // (dt, rain, t) of this block's steps, from the ring of 2K slots
      double* ring = ctx->aRingH.as<double>();
      e = cudaMemcpy(ring, A.dt_log, (size_t)n * 2 * K * 3 * 8, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) { rc = fail(ctx, ITR_DEVICE_ERROR, "tape: %s", cudaGetErrorString(e)); break; }
      const uint64_t s0 = polls * (uint64_t)K;
      for (int d = 0; d < n; ++d)
        for (uint64_t s = s0; s < s0 + K && s < hc[d].step; ++s) {
          const double* q = ring + ((size_t)d * 2 * K + (size_t)(s % (2 * K))) * 3;
          tape->dt[d].push_back(q[0]);
          tape->dt[d].push_back(q[1]);
          tape->dt[d].push_back(q[2]);
        }
    }
    bool all = true;
    for (int d = 0; d < n; ++d) all = all && hc[d].done;
    if (all) break;
    if (polls > kMaxSteps / (uint64_t)K + 2) { rc = fail(ctx, ITR_DEVICE_TIMEOUT, "tiled run did not terminate"); break; }
  }
  if (ge) cudaGraphExecDestroy(ge);
  return rc;
}

// ------------------------------------------------------------------ adjoint ----------
// Backward sweep after a taped tiled forward (itr_adjoint.cuh): seeds from the monitor
// maxima and their argmax states, then segment by segment (last first) replay K steps from
// the checkpoint and step the adjoint back through them.
static int vjp_backward(itr_ctx* ctx, const PlainArgs& F, const itr_objective* ob, int n, const uint32_t* mon, int n_mon,
                        const float* hmm, const DesignOut* hdo) {
  Vjp* V = ctx->vjp;
  const int nx = F.nx, ny = F.ny, K = V->K;
  int rc_ = ITR_OK;
  const size_t N = (size_t)nx * ny, SX = (size_t)ny * (nx + 1), SY = (size_t)(ny + 1) * nx;
  const cudaStream_t st = ctx->stream;
  // argmax states of the monitored cells
  CU(ctx->aTmon.ensure((size_t)n * (n_mon > 0 ? n_mon : 1) * 4));
  std::vector<unsigned> tmon((size_t)n * (n_mon > 0 ? n_mon : 1), 0u);
  if (n_mon > 0) {
    k_gather_u32<<<(n * n_mon + 255) / 256, 256, 0, st>>>(ctx->aTpk.as<unsigned>(), F.mon_cells, n_mon, N, n, ctx->aTmon.as<unsigned>());
    CU(cudaMemcpyAsync(tmon.data(), ctx->aTmon.p, (size_t)n * n_mon * 4, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
  }
  // seeds: for each asset, its argmax cell (first on ties) at the state that set the max,
  // weighted by dJ/dP_k = w_k sigmoid((P_k - eta_k) / tau)
  const int ms = ob->n_assets > 0 ? ob->n_assets : 1;
  std::vector<unsigned> sc((size_t)n * ms, 0u), ss((size_t)n * ms, 0u);
  std::vector<float> sw((size_t)n * ms, 0.0f);
  std::vector<int> sn(n, 0);
  for (int d = 0; d < n; ++d)
    for (int a = 0; a < ob->n_assets; ++a) {
      double best = 0.0;
      int bp = -1;
      for (int m = ob->asset_off[a]; m < ob->asset_off[a + 1]; ++m) {
        const double v = (double)hmm[(size_t)d * n_mon + ob->asset_pos[m]];
        if (bp < 0 || v > best) { best = v; bp = ob->asset_pos[m]; }
      }
      if (bp < 0) continue;
      const unsigned state = tmon[(size_t)d * n_mon + bp];
      if (state == 0u) continue;   // never raised above 0: no dependence
      const double x = (best - ob->asset_threshold[a]) / ob->tau;
      const size_t q = (size_t)d * ms + sn[d]++;
      sc[q] = mon[bp]; ss[q] = state; sw[q] = (float)(ob->asset_weight[a] / (1.0 + std::exp(-x)));
    }
  std::vector<unsigned long long> nst(n);
  unsigned long long nmax = 0;
  for (int d = 0; d < n; ++d) {
    nst[d] = hdo[d].steps;
    // Past the latest state that set one of its assets' maxima, a design's adjoint is zero
    // (no seed is left to add and the adjoint after the last step starts at zero), so those
    // steps change no gradient: its backward covers steps 0 .. S - 1 (S = that state index,
    // 0 without seeds) and the later steps pass the zero adjoint through.
    if (ctx->adj_trim) {
      unsigned long long S = 0;
      for (int q = 0; q < sn[d]; ++q) S = ss[(size_t)d * ms + q] > S ? ss[(size_t)d * ms + q] : S;
      nst[d] = S < nst[d] ? S : nst[d];
    }
    nmax = nst[d] > nmax ? nst[d] : nmax;
  }
  const uint64_t nblocks = (nmax + K - 1) / K;
  if (nblocks > V->blocks) return fail(ctx, ITR_DEVICE_ERROR, "adjoint: %llu segments but %llu checkpoints",
                                       (unsigned long long)nblocks, (unsigned long long)V->blocks);
  CU(ctx->aSeedC.ensure(sc.size() * 4)); CU(ctx->aSeedS.ensure(ss.size() * 4)); CU(ctx->aSeedW.ensure(sw.size() * 4));
  CU(ctx->aSeedN.ensure((size_t)n * 4)); CU(ctx->aNst.ensure((size_t)n * 8));
  CU(cudaMemcpyAsync(ctx->aSeedC.p, sc.data(), sc.size() * 4, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(ctx->aSeedS.p, ss.data(), ss.size() * 4, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(ctx->aSeedW.p, sw.data(), sw.size() * 4, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(ctx->aSeedN.p, sn.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(ctx->aNst.p, nst.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st));
  const size_t S3 = (size_t)n * 3 * N;
  CU(ctx->aTape.ensure((size_t)K * S3 * 4));
  CU(ctx->aLA.ensure(S3 * 4)); CU(ctx->aLB.ensure(S3 * 4));
  CU(ctx->aGx.ensure((size_t)n * SX * 8)); CU(ctx->aGy.ensure((size_t)n * SY * 8));
  // (dt, rain, t) of every segment, laid out [segment][design][K][3], uploaded once
  const size_t seg_elems = (size_t)n * K * 3;
  CU(ctx->aSeg.ensure(nblocks * seg_elems * 8));
  CU(ctx->aRingH.ensure(nblocks * seg_elems * 8));
  CU(cudaMemsetAsync(ctx->aLA.p, 0, S3 * 4, st));
  CU(cudaMemsetAsync(ctx->aGx.p, 0, (size_t)n * SX * 8, st));
  CU(cudaMemsetAsync(ctx->aGy.p, 0, (size_t)n * SY * 8, st));
  const bool crest = F.mode == ITR_FACE_CREST;
  if (crest) {
    CU(ctx->aGx2.ensure((size_t)n * SX * 8)); CU(ctx->aGy2.ensure((size_t)n * SY * 8));
    CU(cudaMemsetAsync(ctx->aGx2.p, 0, (size_t)n * SX * 8, st));
    CU(cudaMemsetAsync(ctx->aGy2.p, 0, (size_t)n * SY * 8, st));
  }
  AdjArgs A;
  memset(&A, 0, sizeof(A));
  A.P = F.P; A.nx = nx; A.ny = ny; A.n_designs = n;
  A.wet = F.wet; A.gn2 = F.gn2; A.bc = F.bc; A.bh = F.bh; A.dzx = F.dzx; A.dzy = F.dzy;
  A.n_steps = ctx->aNst.as<unsigned long long>();
  A.seg = ctx->aSeg.as<double>(); A.K = K;
  A.tape = ctx->aTape.as<float>();
  A.gdzx = ctx->aGx.as<double>(); A.gdzy = ctx->aGy.as<double>();
  if (crest) {
    A.dzx2 = F.dzx2; A.dzy2 = F.dzy2;
    A.gdzx2 = ctx->aGx2.as<double>(); A.gdzy2 = ctx->aGy2.as<double>();
  }
  A.seed_cell = ctx->aSeedC.as<unsigned>(); A.seed_state = ctx->aSeedS.as<unsigned>(); A.seed_w = ctx->aSeedW.as<float>();
  A.seed_n = ctx->aSeedN.as<int>(); A.max_seeds = ms;
  const dim3 grid((nx + kTile - 1) / kTile, (ny + kTile - 1) / kTile, (unsigned)n);
  const bool bnd = F.bh != nullptr || F.P.inflow.n > 0;   // stage or inflow ghosts
  float* lin = ctx->aLA.as<float>();
  float* lout = ctx->aLB.as<float>();
  double* segh = ctx->aRingH.as<double>();
  for (uint64_t b = 0; b < nblocks; ++b)
    for (int d = 0; d < n; ++d)
      for (int j = 0; j < K; ++j) {
        const uint64_t s = b * K + j;
        const bool have = s < nst[d];
        double* q = segh + b * seg_elems + ((size_t)d * K + j) * 3;
        q[0] = have ? V->dt[d][3 * s] : 0.0;
        q[1] = have ? V->dt[d][3 * s + 1] : 0.0;
        q[2] = have ? V->dt[d][3 * s + 2] : 0.0;
      }
  CU(cudaMemcpyAsync(ctx->aSeg.p, segh, nblocks * seg_elems * 8, cudaMemcpyHostToDevice, st));
  // Two tapes: segment b's replay fills tape b % 2 on the second stream while the backward
  // steps of segment b + 1 read the other tape on the context stream, so each launch's
  // last partial wave overlaps the other stream's blocks. Events keep the order: a
  // segment's backward waits for its replay, a replay for the backward that last read its
  // tape. Same kernels, same order per tape: the gradients are unchanged.
  if (!ctx->stream2) {
    CU(cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
      CU(cudaEventCreateWithFlags(&ctx->ev_rep[i], cudaEventDisableTiming));
      CU(cudaEventCreateWithFlags(&ctx->ev_adj[i], cudaEventDisableTiming));
    }
    CU(cudaEventCreateWithFlags(&ctx->ev_bwd, cudaEventDisableTiming));
  }
  CU(ctx->aTape2.ensure((size_t)K * S3 * 4));
  float* tapes[2] = {ctx->aTape.as<float>(), ctx->aTape2.as<float>()};
  const cudaStream_t s2 = ctx->stream2;
  CU(cudaEventRecord(ctx->ev_bwd, st));   // the set-up above, before the first replay
  CU(cudaStreamWaitEvent(s2, ctx->ev_bwd, 0));
  // Row-band replay: k_band<..., TAPE> over the tape, slot j to slot j + 1, with the control
  // blocks k_adj_plan writes for the segment (one buffer per tape).
  // (measured: the band backward step is faster than the tile's on 1024^2 grids, slower on
  //  240 x 192; the band replay is faster on both)
  const int ab = ctx->adj_band >= 0 ? ctx->adj_band : (N >= (size_t(1) << 18) ? 3 : 1);
  const bool adj_band = (ab & 1) != 0, adj_step_band = (ab & 2) != 0;
  PlainArgs T;
  memset(&T, 0, sizeof(T));
  T.P = F.P; T.nx = nx; T.ny = ny; T.mode = F.mode; T.n_designs = n;
  T.wet = F.wet; T.gn2 = F.gn2; T.bc = F.bc; T.bh = F.bh;
  T.dzx = F.dzx; T.dzy = F.dzy; T.dzx2 = F.dzx2; T.dzy2 = F.dzy2;
  T.state_stride = 3 * N; T.plane_stride = S3;
  T.band_rows = band_rows_for(nx, ny, n, ctx->sm_count);
  const BandGeom tg = band_geom(nx, ny, T.band_rows);
  const dim3 tgrid((unsigned)tg.gx, (unsigned)tg.gy, (unsigned)n), tblock((unsigned)(32 * tg.wpb));
  A.band_rows = adj_rows_for(nx, ny, n, ctx->sm_count);
  const AdjGeom ag = adj_geom(nx, ny, A.band_rows);
  const dim3 agrid((unsigned)ag.gx, (unsigned)ag.gy, (unsigned)n), ablock((unsigned)(32 * ag.wpb));
  if (adj_band)
    for (int i = 0; i < 2; ++i) CU(ctx->aPlan[i].ensure((size_t)K * n * sizeof(PlainCtl)));
  auto replay = [&](uint64_t b) -> int {
    const int slot = (int)(b & 1u);
    if (b + 2 < nblocks) CU(cudaStreamWaitEvent(s2, ctx->ev_adj[slot], 0));   // segment b + 2's backward is done with it
    CU(cudaMemcpyAsync(tapes[slot], ctx->aCkpt[b].p, S3 * 4, cudaMemcpyDeviceToDevice, s2));
    AdjArgs R = A;
    R.tape = tapes[slot];
    R.step0 = b * K;
    R.seg = ctx->aSeg.as<double>() + b * seg_elems;
    if (adj_band) {
      PlainCtl* plan = ctx->aPlan[slot].as<PlainCtl>();
      k_adj_plan<<<dim3((unsigned)K, (unsigned)n), 32, 0, s2>>>(R, plan);
      for (int j = 0; j + 1 < K; ++j) {
        PlainArgs Tj = T;
        Tj.H = tapes[slot] + (size_t)j * S3; Tj.QX = Tj.H + N; Tj.QY = Tj.H + 2 * N;
        Tj.ctl = plan + (size_t)j * n;
        if (crest) {
          if (bnd) k_band<true, true, true><<<tgrid, tblock, 0, s2>>>(Tj);
          else k_band<true, false, true><<<tgrid, tblock, 0, s2>>>(Tj);
        } else {
          if (bnd) k_band<false, true, true><<<tgrid, tblock, 0, s2>>>(Tj);
          else k_band<false, false, true><<<tgrid, tblock, 0, s2>>>(Tj);
        }
      }
      CU(cudaEventRecord(ctx->ev_rep[slot], s2));
      return ITR_OK;
    }
    for (int j = 0; j + 1 < K; ++j) {
      if (crest) {
        if (bnd) k_adj_replay<true, true><<<grid, kTileThreads, 0, s2>>>(R, j);
        else k_adj_replay<false, true><<<grid, kTileThreads, 0, s2>>>(R, j);
      } else {
        if (bnd) k_adj_replay<true, false><<<grid, kTileThreads, 0, s2>>>(R, j);
        else k_adj_replay<false, false><<<grid, kTileThreads, 0, s2>>>(R, j);
      }
    }
    CU(cudaEventRecord(ctx->ev_rep[slot], s2));
    return ITR_OK;
  };
  if (nblocks > 0) {   // (none: no design has a seed, every gradient is zero)
    rc_ = replay(nblocks - 1);
    if (rc_ != ITR_OK) return rc_;
  }
  for (uint64_t b = nblocks; b-- > 0;) {   // no host round trip between segments
    const int slot = (int)(b & 1u);
    CU(cudaStreamWaitEvent(st, ctx->ev_rep[slot], 0));
    A.tape = tapes[slot];
    A.step0 = b * K;
    A.seg = ctx->aSeg.as<double>() + b * seg_elems;
    for (int j = K - 1; j >= 0; --j) {
      A.lin = lin; A.lout = lout;
      if (adj_step_band) {
        if (crest) {
          if (bnd) k_adj_band<true, true><<<agrid, ablock, 0, st>>>(A, j);
          else k_adj_band<false, true><<<agrid, ablock, 0, st>>>(A, j);
        } else {
          if (bnd) k_adj_band<true, false><<<agrid, ablock, 0, st>>>(A, j);
          else k_adj_band<false, false><<<agrid, ablock, 0, st>>>(A, j);
        }
      } else if (crest) {
        if (bnd) k_adj_step<true, true><<<grid, kTileThreads, 0, st>>>(A, j);
        else k_adj_step<false, true><<<grid, kTileThreads, 0, st>>>(A, j);
      } else {
        if (bnd) k_adj_step<true, false><<<grid, kTileThreads, 0, st>>>(A, j);
        else k_adj_step<false, false><<<grid, kTileThreads, 0, st>>>(A, j);
      }
      std::swap(lin, lout);
    }
    CU(cudaEventRecord(ctx->ev_adj[slot], st));
    if (b > 0) { rc_ = replay(b - 1); if (rc_ != ITR_OK) return rc_; }
    CU(cudaGetLastError());
  }
  CU(cudaMemcpyAsync(V->gx, ctx->aGx.p, (size_t)n * SX * 8, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(V->gy, ctx->aGy.p, (size_t)n * SY * 8, cudaMemcpyDeviceToHost, st));
  if (crest && V->gx2) CU(cudaMemcpyAsync(V->gx2, ctx->aGx2.p, (size_t)n * SX * 8, cudaMemcpyDeviceToHost, st));
  if (crest && V->gy2) CU(cudaMemcpyAsync(V->gy2, ctx->aGy2.p, (size_t)n * SY * 8, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  return ITR_OK;
}

// Results of a finished batch: per-design outcomes, monitor maxima, ledgers, J (host), and
// for an adjoint request the backward sweep.
static int collect_results(itr_ctx* ctx, const Collect& c) {
  const int n = c.n, n_mon = c.n_mon, max_rows = c.max_rows;
  const size_t N = c.N;
  const itr_design* ds = c.ds;
  itr_result* res = c.res;
  const itr_objective* ob = c.ob;
  const uint32_t* mon = c.mon;
  int launches = c.launches;
  int rc = ITR_OK;
  // ---- results back ----
  unsigned char* ho = ctx->hout.as<unsigned char>();
  size_t hoff = 0;
  DesignOut* hdo = reinterpret_cast<DesignOut*>(ho);
  hoff = align_up((size_t)n * sizeof(DesignOut), 256);
  float* hmm = reinterpret_cast<float*>(ho + hoff);
  hoff = align_up(hoff + (size_t)n * (n_mon > 0 ? n_mon : 1) * 4, 256);
  double* hled = reinterpret_cast<double*>(ho + hoff);
  hoff = align_up(hoff + (size_t)n * (max_rows > 0 ? max_rows : 1) * 64, 256);
  CU(cudaMemcpyAsync(hdo, ctx->out.p, (size_t)n * sizeof(DesignOut), cudaMemcpyDeviceToHost, ctx->stream));
  if (n_mon > 0) {
    int tot = n_mon * n;
    k_gather_monitors<<<(tot + 255) / 256, 256, 0, ctx->stream>>>(ctx->peak.as<float>(), c.dmon, n_mon, N, n,
                                                                   ctx->mmax.as<float>());
    launches += 1;
    CU(cudaMemcpyAsync(hmm, ctx->mmax.p, (size_t)tot * 4, cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (max_rows > 0) CU(cudaMemcpyAsync(hled, ctx->ledger.p, (size_t)n * max_rows * 64, cudaMemcpyDeviceToHost, ctx->stream));
  ctx->fallback.assign((size_t)n, -1.0);
  if (ctx->locked_run) CU(cudaMemcpyAsync(ctx->fallback.data(), ctx->lFb.p, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  for (int d = 0; d < n; ++d) {
    if (res[d].peak) CU(cudaMemcpyAsync(res[d].peak, ctx->peak.as<float>() + d * N, N * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (res[d].depth) CU(cudaMemcpyAsync(res[d].depth, ctx->depth.as<float>() + d * N, N * 4, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CU(cudaEventRecord(ctx->ev[3], ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
#ifdef ITR_CHECKED
  {
    unsigned long long e[4];
    CU(cudaMemcpyFromSymbol(e, g_itr_err, sizeof(e)));
    if (e[0]) return fail(ctx, ITR_DEVICE_ERROR, "checked build: bounds violation code %llu index %lld block %llu thread %llu",
                          e[0], (long long)e[1], e[2], e[3]);
  }
#endif
  float k_ms = 0, t_ms = 0;
  cudaEventElapsedTime(&k_ms, ctx->ev[1], ctx->ev[2]);
  cudaEventElapsedTime(&t_ms, ctx->ev[0], ctx->ev[3]);
  ctx->kernel_ms = k_ms; ctx->total_ms = t_ms; ctx->launches = launches;
  uint64_t cu = 0;
  for (int d = 0; d < n; ++d) {
    const DesignOut& o = hdo[d];
    itr_result& r = res[d];
    if (o.status >= 4) return fail(ctx, ITR_DEVICE_TIMEOUT, "design %d: run exceeded its step or wait limit (status %d)", d, o.status);
    r.steps = o.steps;
    r.rows_skipped = o.rows_skipped;
    // cells actually advanced (RunSummary::cell_updates: steps x cells minus skipped dry rows)
    r.cell_updates = o.steps * (uint64_t)N - o.rows_skipped * (uint64_t)c.nx;
    cu += r.cell_updates;
    r.t_end = o.t_end;
    r.sync_count = o.sync_count;
    r.status = o.status;
    r.breach_cell = o.breach_cell;
    r.breach_sync = o.breach_sync;
    r.lower_bound = o.lower_bound;
    r.n_rows = o.n_rows < r.max_rows ? o.n_rows : r.max_rows;
    r.volume_m3 = o.volume;
    r.rel_residual = o.rel_residual;
    r.warm_start_steps = (size_t)d < ctx->warm_steps.size() ? ctx->warm_steps[d] : 0;
    r.dt_fallback_t = ctx->fallback[(size_t)d];
    if (r.monitor_max) for (int k = 0; k < n_mon; ++k) r.monitor_max[k] = (double)hmm[(size_t)d * n_mon + k];
    if (r.ledger && r.max_rows > 0) memcpy(r.ledger, hled + (size_t)d * max_rows * 8, (size_t)r.n_rows * 64);
    r.j = 0.0; r.feasible = 1; r.violation = 0.0;
    if (ob) {
      std::vector<double> mm(n_mon > 0 ? n_mon : 1);
      for (int k = 0; k < n_mon; ++k) mm[k] = (double)hmm[(size_t)d * n_mon + k];
      double j, worst;
      host_objective(ob, mm.data(), ds[d].cut_m3, ds[d].fill_m3, j, worst);
      r.j = j;
      if (ob->require_no_worsening && ob->baseline_max && worst > ob->guard_tolerance) r.violation = worst - ob->guard_tolerance;
      if (o.status == ITR_RUN_GUARD_ABORT) r.violation = o.violation;
      r.feasible = (r.violation == 0.0 && o.status != ITR_RUN_GUARD_ABORT && o.status != ITR_RUN_UNHEALTHY) ? 1 : 0;
    } else if (o.status == ITR_RUN_UNHEALTHY) {
      r.feasible = 0;
    }
  }
  ctx->cell_updates = cu;
  if (ctx->vjp) {
    CU(cudaEventRecord(ctx->ev[1], ctx->stream));
    rc = vjp_backward(ctx, ctx->last_tiled, ob, n, mon, n_mon, hmm, hdo);
    if (rc != ITR_OK) return rc;
    CU(cudaEventRecord(ctx->ev[2], ctx->stream));
    CU(cudaEventSynchronize(ctx->ev[2]));
    float b_ms = 0;
    cudaEventElapsedTime(&b_ms, ctx->ev[1], ctx->ev[2]);
    ctx->vjp_fwd_ms = ctx->kernel_ms;
    ctx->vjp_bwd_ms = b_ms;
  }
  return ITR_OK;
}

// ------------------------------------------------------------------ warm starts ------
// Whether a batch runs on the grid and params the baseline record was made with.
static bool record_matches(const Record& R, const RunParams& P, const itr_grid* g, const uint8_t* dbc) {
  const size_t N = (size_t)g->nx * g->ny, NB = 2 * (size_t)(g->nx + g->ny);
  if (!R.valid || R.nx != g->nx || R.ny != g->ny || R.mode != g->mode) return false;
  if (memcmp(&R.P, &P, sizeof(RunParams)) != 0) return false;
  return memcmp(R.wet.data(), g->wet, N * 4) == 0 && memcmp(R.gn2.data(), g->gn2, N * 4) == 0 &&
         memcmp(R.bc.data(), dbc, NB) == 0;
}

// Rows of a design whose cells sit beside a face jump (or behind a stage edge) that differs
// from the base's: until one of them holds water, the design's run is the base's.
static bool touched_rows(const Record& R, const itr_grid* g, const itr_design& ds, std::vector<uint8_t>& t) {
  const int nx = g->nx, ny = g->ny;
  const size_t N = (size_t)nx * ny, SX = (size_t)ny * (nx + 1), SY = (size_t)(ny + 1) * nx, NB = 2 * (size_t)(nx + ny);
  if (ds.h0 ? (R.h0.empty() || memcmp(ds.h0, R.h0.data(), N * 4) != 0) : !R.h0.empty()) return false;   // other start
  t.assign((size_t)ny, 0);
  auto differ = [](const float* a, const float* b, size_t i) { return memcmp(a + i, b + i, 4) != 0; };
  const bool crest = g->mode == ITR_FACE_CREST;
  for (size_t i = 0; i < SX; ++i)
    if (differ(ds.dzx, R.dzx.data(), i) || (crest && differ(ds.dzx2, R.dzx2.data(), i))) t[i / (nx + 1)] = 1;
  for (size_t i = 0; i < SY; ++i)
    if (differ(ds.dzy, R.dzy.data(), i) || (crest && differ(ds.dzy2, R.dzy2.data(), i))) {
      const int f = (int)(i / nx);
      if (f >= 1) t[f - 1] = 1;
      if (f < ny) t[f] = 1;
    }
  if (!R.bh.empty()) {
    std::vector<float> bh(NB);
    stage_depths(g, ds.z_edge, bh.data());
    for (size_t i = 0; i < NB; ++i)
      if (memcmp(&bh[i], &R.bh[i], 4) != 0) {
        const int row = i < (size_t)nx ? 0 : i < 2 * (size_t)nx ? ny - 1 : (int)((i - 2 * (size_t)nx) % ny);
        t[row] = 1;
      }
  }
  return true;
}

// The latest checkpoint at which every touched row had stayed dry and none is beside a
// stage or inflow edge (BaselineRecord::best_for, solver.rs:110-115); 0 means a cold start.
static size_t warm_pick(const Record& R, const std::vector<uint8_t>& t) {
  for (size_t c = R.ck.size(); c-- > 1;) {
    bool ok = true;
    for (int j = 0; j < R.ny && ok; ++j) ok = !(t[j] && (R.ck[c].wet[j] || R.open_rows[j]));
    if (ok) return c;
  }
  return 0;
}

// ------------------------------------------------------------------ run_batch -------
extern "C" int itr_gpu_run_batch(itr_ctx* ctx, const itr_params* p, const itr_grid* g, int32_t n, const itr_design* ds,
                                 const uint32_t* mon, int32_t n_mon, const itr_objective* ob, itr_result* res) {
  if (!ctx) return ITR_INVALID_ARG;
  int rc = check_inputs(ctx, p, g, n, ds, mon, n_mon, ob);
  if (rc != ITR_OK) return rc;
  if (n == 0) { ctx->kernel_ms = ctx->total_ms = 0; ctx->cell_updates = 0; ctx->launches = 0; return ITR_OK; }
  if (!res) return fail(ctx, ITR_INVALID_ARG, "results is NULL");
  CU(cudaSetDevice(ctx->device));
  const int nx = g->nx, ny = g->ny;
  const size_t N = (size_t)nx * ny, SX = (size_t)ny * (nx + 1), SY = (size_t)(ny + 1) * nx;
  const bool crest = g->mode == ITR_FACE_CREST;
  int max_rows = 0;
  for (int d = 0; d < n; ++d) if (res[d].ledger && res[d].max_rows > max_rows) max_rows = res[d].max_rows;
  const int n_assets = ob ? ob->n_assets : 0, n_guard = ob ? ob->n_guard : 0;
  const int n_apos = ob && n_assets > 0 ? ob->asset_off[n_assets] : 0;
  const size_t NB = 2 * (size_t)(nx + ny);   // boundary cells
  bool has_stage = false;
  for (size_t i = 0; i < NB; ++i) has_stage = has_stage || g->bc[i] == ITR_BC_STAGE;

  // ---- pack into pinned staging ----
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + bytes, 256); return o; };
  const size_t o_wet = take(N * 4), o_gn2 = take(N * 4), o_bc = take(NB);
  const size_t o_bh = has_stage ? take(n * NB * 4) : 0;
  const size_t o_dzx = take(n * SX * 4), o_dzy = take(n * SY * 4);
  const size_t o_dzx2 = crest ? take(n * SX * 4) : 0, o_dzy2 = crest ? take(n * SY * 4) : 0;
  const size_t o_h0 = take(n * N * 4), o_cut = take((size_t)n * 8), o_fill = take((size_t)n * 8);
  const size_t o_mon = take((size_t)(n_mon > 0 ? n_mon : 1) * 4);
  const size_t o_oi = take((size_t)(n_assets + 1 + n_apos + n_guard + 1) * 4);
  const size_t o_od = take((size_t)(2 * n_assets + (n_mon > 0 ? n_mon : 1)) * 8);
  Mat* M = ctx->mat;   // designs as primitives: the space, primitives and boxes go up instead of jumps
  const size_t o_mz = M ? take(N * 8) : 0, o_mw = M ? take(N) : 0, o_me = M ? take(N) : 0;
  const size_t o_mst = M && has_stage ? take(NB * 8) : 0;
  const size_t o_mp = M ? take((M->prims.size() > 0 ? M->prims.size() : 1) * sizeof(MatPrim)) : 0;
  const size_t o_md = M ? take((size_t)n * sizeof(MatDesign)) : 0;
  const size_t in_bytes = off;
  CU(ctx->stage.ensure(in_bytes));
  unsigned char* st = ctx->stage.as<unsigned char>();
  memcpy(st + o_wet, g->wet, N * 4);
  memcpy(st + o_gn2, g->gn2, N * 4);
  RunParams P = make_run_params(p, g);
  rc = build_boundaries(ctx, g, P.inflow, st + o_bc);
  if (rc != ITR_OK) return rc;
  const bool bnd = has_stage || P.inflow.n > 0;
  if (has_stage && !M)
    for (int d = 0; d < n; ++d) stage_depths(g, ds[d].z_edge, reinterpret_cast<float*>(st + o_bh) + d * NB);
  if (M) {
    memcpy(st + o_mz, M->space->z, N * 8);
    memcpy(st + o_mw, M->space->wall, N);
    memcpy(st + o_me, M->space->editable, N);
    if (has_stage) memcpy(st + o_mst, g->bc_stage, NB * 8);
    if (!M->prims.empty()) memcpy(st + o_mp, M->prims.data(), M->prims.size() * sizeof(MatPrim));
    memcpy(st + o_md, M->des.data(), (size_t)n * sizeof(MatDesign));
  }
  const float hinit = (float)(p->initial_depth > 0.0 ? p->initial_depth : 0.0);
  for (int d = 0; d < n; ++d) {
    if (!M) {
      memcpy(st + o_dzx + d * SX * 4, ds[d].dzx, SX * 4);
      memcpy(st + o_dzy + d * SY * 4, ds[d].dzy, SY * 4);
    }
    if (crest) { memcpy(st + o_dzx2 + d * SX * 4, ds[d].dzx2, SX * 4); memcpy(st + o_dzy2 + d * SY * 4, ds[d].dzy2, SY * 4); }
    float* h0 = reinterpret_cast<float*>(st + o_h0) + d * N;
    if (ds[d].h0) memcpy(h0, ds[d].h0, N * 4);
    else for (size_t i = 0; i < N; ++i) h0[i] = g->wet[i] != 0.0f ? (hinit == 0.0f ? 0.0f : hinit) : 0.0f;  // init_state
    reinterpret_cast<double*>(st + o_cut)[d] = ds[d].cut_m3;
    reinterpret_cast<double*>(st + o_fill)[d] = ds[d].fill_m3;
  }
  if (n_mon > 0) memcpy(st + o_mon, mon, (size_t)n_mon * 4);
  int* oi = reinterpret_cast<int*>(st + o_oi);
  double* od = reinterpret_cast<double*>(st + o_od);
  if (ob) {
    for (int a = 0; a <= n_assets; ++a) oi[a] = n_assets > 0 ? ob->asset_off[a] : 0;
    for (int m = 0; m < n_apos; ++m) oi[n_assets + 1 + m] = ob->asset_pos[m];
    for (int k = 0; k < n_guard; ++k) oi[n_assets + 1 + n_apos + k] = ob->guard_pos[k];
    for (int a = 0; a < n_assets; ++a) { od[a] = ob->asset_threshold[a]; od[n_assets + a] = ob->asset_weight[a]; }
    if (ob->baseline_max) for (int k = 0; k < n_mon; ++k) od[2 * n_assets + k] = ob->baseline_max[k];
  }

  // ---- device buffers ----
  CU(ctx->dzx.ensure(in_bytes));  // one slab for all inputs
  unsigned char* dv = ctx->dzx.as<unsigned char>();
  CU(ctx->peak.ensure(n * N * 4));
  CU(ctx->depth.ensure(n * N * 4));
  CU(ctx->ledger.ensure((size_t)n * (max_rows > 0 ? max_rows : 1) * 8 * 8));
  CU(ctx->out.ensure((size_t)n * sizeof(DesignOut)));
  CU(ctx->mmax.ensure((size_t)n * (n_mon > 0 ? n_mon : 1) * 4));
  const size_t out_bytes = (size_t)n * sizeof(DesignOut) + (size_t)n * (n_mon > 0 ? n_mon : 1) * 4 +
                           (size_t)n * (max_rows > 0 ? max_rows : 1) * 64 + 2 * n * N * 4 + 1024;
  const size_t ctl_bytes = (size_t)n * sizeof(PlainCtl);
  CU(ctx->hout.ensure(out_bytes > ctl_bytes ? out_bytes : ctl_bytes));

  DevObjective DO;
  memset(&DO, 0, sizeof(DO));
  if (ob) {
    DO.enabled = 1;
    DO.n_assets = n_assets;
    DO.asset_off = reinterpret_cast<const int*>(dv + o_oi);
    DO.asset_pos = DO.asset_off + n_assets + 1;
    DO.guard_pos = DO.asset_pos + n_apos;
    DO.n_guard = n_guard;
    DO.asset_thr = reinterpret_cast<const double*>(dv + o_od);
    DO.asset_w = DO.asset_thr + n_assets;
    DO.baseline = ob->baseline_max ? DO.asset_thr + 2 * n_assets : nullptr;
    DO.tol = ob->guard_tolerance; DO.tau = ob->tau; DO.cut_cost = ob->cut_cost; DO.fill_cost = ob->fill_cost;
    DO.earth_w = ob->earth_weight; DO.require = ob->require_no_worsening; DO.guard_abort = ob->guard_abort;
    DO.has_incumbent = ob->has_incumbent; DO.incumbent = ob->incumbent;
  }

  CU(cudaEventRecord(ctx->ev[0], ctx->stream));
#ifdef ITR_CHECKED
  {
    unsigned long long z[4] = {0, 0, 0, 0};
    CU(cudaMemcpyToSymbolAsync(g_itr_err, z, sizeof(z), 0, cudaMemcpyHostToDevice, ctx->stream));
  }
#endif
  CU(cudaMemcpyAsync(dv, st, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
  int launches = 0;
  if (M) {   // materialise every design on the device; the volumes come back for J
    CU(ctx->mDz.ensure((size_t)n * N * 8));
    CU(ctx->mZe.ensure((size_t)n * N * 8));
    CU(ctx->mVol.ensure((size_t)n * 2 * 8));
    MatArgs MA;
    memset(&MA, 0, sizeof(MA));
    MA.nx = nx; MA.ny = ny; MA.n = n;
    MA.ox = M->space->origin_x; MA.oy = M->space->origin_y; MA.dx = g->dx; MA.dy = g->dy;
    MA.z_wall = M->space->z_wall; MA.max_abs_dz = M->space->max_abs_dz;
    MA.z = reinterpret_cast<const double*>(dv + o_mz);
    MA.wall = dv + o_mw; MA.editable = dv + o_me;
    MA.prims = reinterpret_cast<const MatPrim*>(dv + o_mp);
    MA.des = reinterpret_cast<const MatDesign*>(dv + o_md);
    MA.dz = ctx->mDz.as<double>(); MA.ze = ctx->mZe.as<double>();
    MA.dzx = reinterpret_cast<float*>(dv + o_dzx); MA.dzy = reinterpret_cast<float*>(dv + o_dzy);
    MA.cut = reinterpret_cast<double*>(dv + o_cut); MA.fill = reinterpret_cast<double*>(dv + o_fill);
    if (has_stage) {
      MA.bc = g->bc ? dv + o_bc : nullptr;   // device codes: stage cells keep code 2
      MA.stage = reinterpret_cast<const double*>(dv + o_mst);
      MA.bh = reinterpret_cast<float*>(dv + o_bh);
    }
    const size_t faces = SX > SY ? SX : SY;
    const size_t items = faces > NB ? faces : NB;
    k_materialize<<<dim3((unsigned)((N + 255) / 256), (unsigned)n), 256, 0, ctx->stream>>>(MA);
    k_mat_jumps<<<dim3((unsigned)((items + 255) / 256), (unsigned)n), 256, 0, ctx->stream>>>(MA);
    k_mat_volumes<<<(n + 3) / 4, 128, 0, ctx->stream>>>(MA);   // a warp per design
    launches += 3;
    double* hv = ctx->mVol.as<double>();
    CU(cudaMemcpyAsync(hv, dv + o_cut, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(hv + n, dv + o_fill, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    for (int d = 0; d < n; ++d) { M->ds[d].cut_m3 = hv[d]; M->ds[d].fill_m3 = hv[n + d]; }
  }
  // ---- baseline-locked dt: the batched cluster kernel only; the baseline record runs adaptively ----
  const bool locked = !ctx->locked_dt.empty() && !ctx->recording;
  ctx->locked_run = false;
  if (locked && (ctx->impl == 1 || ctx->vjp || ctx->defer))
    return fail(ctx, ITR_UNSUPPORTED, "a baseline-locked dt schedule runs on the batched paths only (impl 0 and 2; "
                                      "no plain one-design path, adjoint or ladder)");
  // ---- warm starts from the baseline record (a locked run starts cold: its snapshot is the start) ----
  ctx->warm_steps.assign((size_t)n, 0);
  const WarmStart* warm_dev = nullptr;
  if (ctx->warm_start && ctx->rec && !ctx->vjp && !ctx->recording && !locked && !(ob && ob->has_incumbent) &&
      record_matches(*ctx->rec, P, g, st + o_bc)) {
    const Record& R = *ctx->rec;
    std::vector<WarmStart> ws((size_t)n);
    memset(ws.data(), 0, ws.size() * sizeof(WarmStart));
    bool any = false;
    for (int d = 0; d < n; ++d) {
      std::vector<uint8_t> t;
      if (M) {   // a box of primitives: its rows and the one on either side (the edit_rows of apply_edit)
        if (!R.h0.empty()) continue;
        t.assign((size_t)ny, 0);
        const MatDesign& B = M->des[d];
        if (B.c0 < B.c1 && B.r0 < B.r1)
          for (int r = B.r0 - 1; r <= B.r1; ++r) if (r >= 0 && r < ny) t[r] = 1;
      } else if (!touched_rows(R, g, ds[d], t)) {
        continue;
      }
      const size_t c = warm_pick(R, t);
      if (c == 0) continue;
      ws[d] = R.ck[c].ws;
      ctx->warm_steps[d] = ws[d].step;
      any = true;
      const int rows = ws[d].n_rows < max_rows ? ws[d].n_rows : max_rows;   // the base's ledger rows so far
      if (rows > 0)
        CU(cudaMemcpyAsync(ctx->ledger.as<double>() + (size_t)d * max_rows * 8, R.ledger.data(), (size_t)rows * 64,
                           cudaMemcpyHostToDevice, ctx->stream));
    }
    if (any) {
      CU(ctx->wsb.ensure((size_t)n * sizeof(WarmStart)));
      CU(cudaMemcpyAsync(ctx->wsb.p, ws.data(), (size_t)n * sizeof(WarmStart), cudaMemcpyHostToDevice, ctx->stream));
      CU(cudaStreamSynchronize(ctx->stream));   // ws is a local vector
      warm_dev = ctx->wsb.as<WarmStart>();
    }
  }
  const unsigned long long max_steps = kMaxSteps;

  // impl 2, or a grid no cluster shape can hold: the tiled batched path (state in HBM)
  bool tiled = ctx->impl == 2 || ctx->vjp != nullptr;
  dim3 tgrid = tiled_grid(ctx, nx, ny, n);   // blocks per design of the tiled path's update
  int n_tiles = (int)(tgrid.x * tgrid.y);
  const int band0 = ctx->band;
  const int max_tiles = std::max((nx + kTile - 1) / kTile * ((ny + kTile - 1) / kTile), n_tiles);
  const bool bnd_grid = has_stage || P.inflow.n > 0;   // stage or inflow ghosts
  auto tiled_args = [&](PlainArgs& A) -> cudaError_t {
    cudaError_t e = ctx->tH.ensure((size_t)n * 2 * N * 4);
    if (e == cudaSuccess) e = ctx->tQX.ensure((size_t)n * 2 * N * 4);
    if (e == cudaSuccess) e = ctx->tQY.ensure((size_t)n * 2 * N * 4);
    if (e == cudaSuccess) e = ctx->tpart.ensure((size_t)n * max_tiles * kPart * 8);
    if (e == cudaSuccess) e = ctx->tctl.ensure((size_t)n * sizeof(PlainCtl));
    memset(&A, 0, sizeof(A));
    A.P = P; A.nx = nx; A.ny = ny; A.mode = g->mode; A.n_designs = n;
    A.wet = reinterpret_cast<const float*>(dv + o_wet);
    A.gn2 = reinterpret_cast<const float*>(dv + o_gn2);
    A.bc = reinterpret_cast<const uint8_t*>(dv + o_bc);
    A.bh = has_stage ? reinterpret_cast<const float*>(dv + o_bh) : nullptr;
    A.dzx = reinterpret_cast<const float*>(dv + o_dzx);
    A.dzy = reinterpret_cast<const float*>(dv + o_dzy);
    A.dzx2 = crest ? reinterpret_cast<const float*>(dv + o_dzx2) : nullptr;
    A.dzy2 = crest ? reinterpret_cast<const float*>(dv + o_dzy2) : nullptr;
    A.h0 = reinterpret_cast<const float*>(dv + o_h0);
    A.cut_d = reinterpret_cast<const double*>(dv + o_cut);
    A.fill_d = reinterpret_cast<const double*>(dv + o_fill);
    A.n_mon = n_mon; A.mon_cells = reinterpret_cast<const unsigned*>(dv + o_mon);
    A.obj = DO;
    A.H = ctx->tH.as<float>(); A.QX = ctx->tQX.as<float>(); A.QY = ctx->tQY.as<float>();
    A.PK = ctx->peak.as<float>();
    A.part = ctx->tpart.as<double>(); A.ctl = ctx->tctl.as<PlainCtl>();
    A.ledger = max_rows > 0 ? ctx->ledger.as<double>() : nullptr;
    A.max_rows = max_rows;
    A.max_steps = max_steps;
    A.warm = warm_dev;
    if (locked && e == cudaSuccess) {
      const size_t nl = ctx->locked_dt.size();
      e = ctx->lDt.ensure(nl * 8);
      if (e == cudaSuccess) e = ctx->lS4.ensure((size_t)n * 4 * N * 4);
      if (e == cudaSuccess) e = ctx->lSs.ensure((size_t)n * sizeof(PlainCtl));
      if (e == cudaSuccess) e = ctx->lFb.ensure((size_t)n * 8);
      if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->lDt.p, ctx->locked_dt.data(), nl * 8, cudaMemcpyHostToDevice, ctx->stream);
      A.locked_dt = ctx->lDt.as<double>();
      A.n_locked = (unsigned long long)nl;
      A.cfl_hard = ctx->cfl_hard;
      A.snap = ctx->lS4.as<float>();
      A.snapctl = ctx->lSs.as<PlainCtl>();
      A.fallback_t = ctx->lFb.as<double>();
      ctx->locked_run = true;
    }
    A.band_rows = band_rows_for(nx, ny, n, ctx->sm_count);
    if (ctx->band && e == cudaSuccess) {   // dry-row skipping on the row-band path
      const size_t R = (size_t)ny + 2;
      e = ctx->tRow.ensure((size_t)n * 2 * R * 4);
      if (e == cudaSuccess && bnd_grid) e = ctx->tGw.ensure((size_t)n * R);
      if (e == cudaSuccess && locked) e = ctx->tSnapRow.ensure((size_t)n * R * 4);
      A.rowwet = ctx->tRow.as<unsigned>();
      A.gwet = bnd_grid ? ctx->tGw.as<uint8_t>() : nullptr;
      A.snaprow = locked ? ctx->tSnapRow.as<unsigned>() : nullptr;
    }
    return e;
  };
  int tiled_band = ctx->band;   // the tiled path's update kernel for this batch (the autotuner may pick)
  if (ctx->impl == 0 && !tiled) {
    BatchArgs A;
    memset(&A, 0, sizeof(A));
    A.P = P; A.nx = nx; A.ny = ny; A.mode = g->mode; A.n_designs = n;
    A.wet = reinterpret_cast<const float*>(dv + o_wet);
    A.gn2 = reinterpret_cast<const float*>(dv + o_gn2);
    A.bc = reinterpret_cast<const uint8_t*>(dv + o_bc);
    A.bh = has_stage ? reinterpret_cast<const float*>(dv + o_bh) : nullptr;
    A.dzx = reinterpret_cast<const float*>(dv + o_dzx);
    A.dzy = reinterpret_cast<const float*>(dv + o_dzy);
    A.dzx2 = crest ? reinterpret_cast<const float*>(dv + o_dzx2) : nullptr;
    A.dzy2 = crest ? reinterpret_cast<const float*>(dv + o_dzy2) : nullptr;
    A.h0 = reinterpret_cast<const float*>(dv + o_h0);
    A.cut = reinterpret_cast<const double*>(dv + o_cut);
    A.fill = reinterpret_cast<const double*>(dv + o_fill);
    A.n_mon = n_mon;
    A.mon_cells = reinterpret_cast<const unsigned*>(dv + o_mon);
    A.obj = DO;
    A.peak_out = ctx->peak.as<float>();
    A.depth_out = ctx->depth.as<float>();
    A.ledger_out = max_rows > 0 ? ctx->ledger.as<double>() : nullptr;
    A.max_rows = max_rows;
    A.out = ctx->out.as<DesignOut>();
    A.max_steps = max_steps;
    A.exact = ctx->exact_special ? 1u : 0u;
    A.wait_limit = ctx->wait_limit;
    A.stall_test = ctx->stall_wait_test ? 1u : 0u;
    A.warm = warm_dev;
    // launch configuration
    LaunchCfg cfg;
    // (the dry-row instantiation is tuned apart: its bookkeeping changes the best shape)
    auto key = std::make_tuple(nx, ny, n, (int)g->mode + (bnd ? 2 : 0) + (A.P.skip_dry ? 4 : 0));
    if (ctx->cluster > 0 || ctx->threads > 0) {
      cfg = make_cfg(ctx, nx, ny, ctx->cluster > 0 ? ctx->cluster : 1, ctx->threads > 0 ? ctx->threads : 512, crest, bnd);
      if (!cfg.ok) return fail(ctx, ITR_UNSUPPORTED, "cluster=%d threads=%d does not fit a %dx%d grid in shared memory", ctx->cluster, ctx->threads, nx, ny);
    } else if (ctx->tuned.count(key) && !(locked && ctx->tuned[key].tiled)) {
      cfg = ctx->tuned[key];
      tiled = cfg.tiled;
      if (tiled) tiled_band = cfg.band;
    } else {
      std::vector<LaunchCfg> cands = candidates(ctx, nx, ny, n, crest, bnd);
      if (cands.empty()) {
        tiled = true;   // a design needs more shared memory than 8 CTAs hold
      } else {
        // Measured autotuning: time a short probe (the first steps of this very batch) of
        // the best few shapes by the model and keep the fastest for this (grid, population).
        cfg = cands[0];
        if (ctx->autotune) {   // (a single candidate is timed too: the tiled path is compared with it)
          rc = autotune(ctx, A, cands, n, &cfg);
          if (rc != ITR_OK) return rc;
        }
        if (ctx->autotune && !locked && !ctx->defer) {
          // the tiled HBM path as one more candidate, timed over the same probe steps (not for
          // a ladder group: the ladder runs every group's cluster kernel in one graph launch)
          PlainArgs T;
          CU(tiled_args(T));   // (no locked schedule here: the tiled candidate is timed only unlocked)
          T.max_steps = (unsigned long long)ctx->probe_steps;
          T.warm = nullptr;
          T.obj.enabled = 0; T.ledger = nullptr; T.max_rows = 0;
          int dummy = 0;
          // both update kernels of the tiled path, row bands and 16x16 tiles; direct launches
          // and one poll: no graph build or host round trips in the timing
          const int g0 = ctx->graph, k0 = ctx->steps_per_submit;
          ctx->graph = 0; ctx->steps_per_submit = ctx->probe_steps;
          for (int bk = 1; bk >= 0 && rc == ITR_OK; --bk) {
            ctx->band = bk;
            const dim3 tg = tiled_grid(ctx, nx, ny, n);
            float t_ms = 0.0f;
            cudaError_t e = tiled_args(T);
            T.max_steps = (unsigned long long)ctx->probe_steps;
            T.warm = nullptr;
            T.obj.enabled = 0; T.ledger = nullptr; T.max_rows = 0;
            if (e == cudaSuccess) e = cudaEventRecord(ctx->ev[1], ctx->stream);
            if (e != cudaSuccess) { rc = fail(ctx, ITR_DEVICE_ERROR, "tiled probe: %s", cudaGetErrorString(e)); break; }
            rc = run_tiled_batch(ctx, T, n, tg, &dummy);
            if (rc != ITR_OK) break;
            e = cudaEventRecord(ctx->ev[2], ctx->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(ctx->ev[2]);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&t_ms, ctx->ev[1], ctx->ev[2]);
            if (e != cudaSuccess) { rc = fail(ctx, ITR_DEVICE_ERROR, "tiled probe: %s", cudaGetErrorString(e)); break; }
            if (t_ms < ctx->tune_ms) { cfg.tiled = true; cfg.band = bk; ctx->tune_ms = t_ms; }
          }
          ctx->graph = g0; ctx->steps_per_submit = k0;
          ctx->band = band0;
          if (rc != ITR_OK) return rc;
        }
        if (!(locked && ctx->tuned.count(key))) ctx->tuned[key] = cfg;   // a locked run keeps a cached tiled choice
        tiled = cfg.tiled;
        if (tiled) tiled_band = cfg.band;
      }
    }
    if (!tiled) {
      A.C = cfg.C; A.W = cfg.W; A.S = cfg.S;
      if (locked) {
        const size_t nl = ctx->locked_dt.size();
        CU(ctx->lDt.ensure(nl * 8));
        CU(ctx->lS4.ensure((size_t)n * N * 16));
        CU(ctx->lS2.ensure((size_t)n * N * 8));
        CU(ctx->lSk.ensure((size_t)n * N * 4));
        CU(ctx->lSs.ensure((size_t)n * cfg.C * sizeof(LockedSnap)));
        CU(ctx->lFb.ensure((size_t)n * 8));
        CU(cudaMemcpyAsync(ctx->lDt.p, ctx->locked_dt.data(), nl * 8, cudaMemcpyHostToDevice, ctx->stream));
        A.locked_dt = ctx->lDt.as<double>();
        A.n_locked = (unsigned long long)nl;
        A.cfl_hard = ctx->cfl_hard;
        A.snap4 = ctx->lS4.as<float4>(); A.snap2 = ctx->lS2.as<float2>(); A.snapk = ctx->lSk.as<float>();
        A.snap_s = ctx->lSs.as<LockedSnap>();
        A.fallback_t = ctx->lFb.as<double>();
        ctx->locked_run = true;
      }
      if (ctx->defer) {   // ladder group: the launch goes into the ladder's graph
        BatchedFn fn = batched_fn(crest, cfg.C > 1, maxt_bucket(cfg.T), cfg.bnd, A.locked_dt != nullptr, A.P.skip_dry != 0);
        CU(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
        ctx->last_args = A; ctx->last_cfg = cfg; ctx->have_last = true;
        ctx->last_was_plain = false; ctx->last_was_tiled = false;
        Collect& c = ctx->pending;
        c.n = n; c.nx = nx; c.n_mon = n_mon; c.max_rows = max_rows; c.N = N; c.ds = ds; c.res = res; c.ob = ob;
        c.mon = mon; c.dmon = reinterpret_cast<const unsigned*>(dv + o_mon); c.launches = launches;
        ctx->pending_ok = true;
        return ITR_OK;
      }
      CU(cudaEventRecord(ctx->ev[1], ctx->stream));
      rc = launch_batched(ctx, A, cfg, n);
      if (rc != ITR_OK) return rc;
      CU(cudaEventRecord(ctx->ev[2], ctx->stream));
      launches += 1;
      ctx->last_args = A;
      ctx->last_cfg = cfg;
      ctx->have_last = true;
      ctx->last_was_plain = false;
      ctx->last_was_tiled = false;
    }
  }
  if (tiled) {
    struct BandScope {   // the tuned kernel choice for this batch; the option stays the caller's
      itr_ctx* c; int v;
      ~BandScope() { c->band = v; }
    } band_scope{ctx, band0};
    ctx->band = tiled_band;
    tgrid = tiled_grid(ctx, nx, ny, n);
    n_tiles = (int)(tgrid.x * tgrid.y);
    const int nb = n_tiles;
    PlainArgs A;
    CU(tiled_args(A));
    if (ctx->vjp) {
      const int K = ctx->vjp->K;
      CU(ctx->aTpk.ensure((size_t)n * N * 4));
      CU(ctx->aRing.ensure((size_t)n * 2 * K * 3 * 8));
      CU(ctx->aRingH.ensure((size_t)n * 2 * K * 3 * 8));
      A.tpk = ctx->aTpk.as<unsigned>();
      A.dt_log = ctx->aRing.as<double>();
      A.max_log = 2 * K;
    }
    CU(cudaEventRecord(ctx->ev[1], ctx->stream));
    rc = run_tiled_batch(ctx, A, n, tgrid, &launches);
    ctx->last_band = ctx->band;
    if (rc != ITR_OK) return rc;
    k_plain_outputs<<<n, 256, 0, ctx->stream>>>(A, nb, ctx->out.as<DesignOut>(), ctx->depth.as<float>());
    launches += 1;
    CU(cudaEventRecord(ctx->ev[2], ctx->stream));
    ctx->last_tiled = A;
    ctx->last_tgrid = tgrid;
    ctx->have_last = true;
    ctx->last_was_plain = false;
    ctx->last_was_tiled = true;
  } else if (ctx->impl == 1) {
    // plain: one design after another
    CU(ctx->pH.ensure(2 * N * 4)); CU(ctx->pQX.ensure(2 * N * 4)); CU(ctx->pQY.ensure(2 * N * 4));
    CU(ctx->pPK.ensure(N * 4));
    dim3 grid((nx + kTile - 1) / kTile, (ny + kTile - 1) / kTile);
    int nb = grid.x * grid.y;
    CU(ctx->ppart.ensure((size_t)nb * kPart * 8));
    CU(ctx->pctl.ensure(sizeof(PlainCtl)));
    CU(cudaEventRecord(ctx->ev[1], ctx->stream));
    ctx->last_plain.clear();
    ctx->last_plain_blocks.clear();
    for (int d = 0; d < n; ++d) {
      PlainArgs A;
      memset(&A, 0, sizeof(A));
      A.P = P; A.nx = nx; A.ny = ny; A.mode = g->mode;
      A.wet = reinterpret_cast<const float*>(dv + o_wet);
      A.gn2 = reinterpret_cast<const float*>(dv + o_gn2);
      A.bc = reinterpret_cast<const uint8_t*>(dv + o_bc);
      A.bh = has_stage ? reinterpret_cast<const float*>(dv + o_bh) + d * NB : nullptr;
      A.dzx = reinterpret_cast<const float*>(dv + o_dzx) + d * SX;
      A.dzy = reinterpret_cast<const float*>(dv + o_dzy) + d * SY;
      A.dzx2 = crest ? reinterpret_cast<const float*>(dv + o_dzx2) + d * SX : nullptr;
      A.dzy2 = crest ? reinterpret_cast<const float*>(dv + o_dzy2) + d * SY : nullptr;
      A.h0 = reinterpret_cast<const float*>(dv + o_h0) + d * N;
      A.cut = ds[d].cut_m3; A.fill = ds[d].fill_m3;
      A.n_mon = n_mon; A.mon_cells = reinterpret_cast<const unsigned*>(dv + o_mon);
      A.obj = DO;
      A.H = ctx->pH.as<float>(); A.QX = ctx->pQX.as<float>(); A.QY = ctx->pQY.as<float>(); A.PK = ctx->pPK.as<float>();
      A.part = ctx->ppart.as<double>(); A.ctl = ctx->pctl.as<PlainCtl>();
      A.ledger = max_rows > 0 ? ctx->ledger.as<double>() + (size_t)d * max_rows * 8 : nullptr;
      A.max_rows = max_rows;
      A.max_steps = max_steps;
      A.warm = warm_dev ? warm_dev + d : nullptr;
      rc = run_plain_design(ctx, A, nb, grid, &launches);
      if (rc != ITR_OK) return rc;
      // copy this design's outputs into the batched output slots
      PlainCtl* hc = ctx->hout.as<PlainCtl>();
      DesignOut o;
      memset(&o, 0, sizeof(o));
      o.steps = hc->step; o.t_end = hc->t; o.sync_count = hc->sync_index; o.status = hc->status;
      o.breach_cell = hc->breach_cell; o.breach_sync = hc->breach_sync; o.violation = hc->violation;
      o.lower_bound = hc->lower_bound; o.v0 = hc->v0; o.volume = hc->volume; o.rel_residual = hc->rel_res; o.n_rows = hc->n_rows;
      CU(cudaMemcpyAsync(ctx->out.as<DesignOut>() + d, &o, sizeof(o), cudaMemcpyHostToDevice, ctx->stream));
      CU(cudaMemcpyAsync(ctx->peak.as<float>() + d * N, A.PK, N * 4, cudaMemcpyDeviceToDevice, ctx->stream));
      CU(cudaMemcpyAsync(ctx->depth.as<float>() + d * N, A.H + (size_t)hc->par * N, N * 4, cudaMemcpyDeviceToDevice, ctx->stream));
      CU(cudaStreamSynchronize(ctx->stream));
      ctx->last_plain.push_back(A);
      ctx->last_plain_blocks.push_back(nb);
    }
    CU(cudaEventRecord(ctx->ev[2], ctx->stream));
    ctx->last_was_plain = true;
    ctx->last_was_tiled = false;
    ctx->have_last = true;
  }
  CU(cudaGetLastError());

  Collect col;
  col.n = n; col.nx = nx; col.n_mon = n_mon; col.max_rows = max_rows; col.N = N; col.ds = ds; col.res = res; col.ob = ob;
  col.mon = mon; col.dmon = reinterpret_cast<const unsigned*>(dv + o_mon); col.launches = launches;
  return collect_results(ctx, col);
}

// Uneven batch: several grid groups (the fidelity ladder's coarse, native and half-cell
// grids) in one CUDA graph launch. Each group is prepared on its own child context (inputs
// uploaded, launch shape autotuned for its grid) and its persistent cluster kernel becomes
// one parallel branch of the graph; a group whose grid needs the tiled path runs on its own
// before the graph. Results come back per group, in group order.
extern "C" int itr_gpu_run_ladder(itr_ctx* ctx, const itr_params* p, int32_t n_groups, const itr_group* groups,
                                  itr_result* results) {
  if (!ctx) return ITR_INVALID_ARG;
  if (n_groups < 1 || !groups || !results || !p) return fail(ctx, ITR_INVALID_ARG, "ladder: groups, params and results are required");
  if (!ctx->locked_dt.empty())   // a schedule belongs to one grid (Problem::build records one per level, problem.rs:196-198)
    return fail(ctx, ITR_UNSUPPORTED, "ladder: a baseline-locked dt schedule belongs to one grid; run each level with itr_gpu_run_batch");
  CU(cudaSetDevice(ctx->device));
  while ((int)ctx->children.size() < n_groups) {
    char err[256] = {0};
    itr_ctx* c = itr_gpu_create(ctx->device, err, sizeof(err));
    if (!c) return fail(ctx, ITR_DEVICE_ERROR, "ladder group context: %s", err);
    ctx->children.push_back(c);
  }
  if (!ctx->ev_fork) CU(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
  size_t off = 0;
  for (int gi = 0; gi < n_groups; ++gi) {
    itr_ctx* c = ctx->children[gi];
    c->impl = ctx->impl; c->threads = ctx->threads; c->cluster = ctx->cluster; c->graph = ctx->graph;
    c->steps_per_submit = ctx->steps_per_submit; c->autotune = ctx->autotune; c->autotune_top = ctx->autotune_top;
    c->probe_steps = ctx->probe_steps; c->exact_special = ctx->exact_special;
    c->wait_limit = ctx->wait_limit; c->stall_wait_test = ctx->stall_wait_test;
    if (!c->ev_fork) CU(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    c->defer = true;
    c->pending_ok = false;
    const itr_group& G = groups[gi];
    const int rc = itr_gpu_run_batch(c, p, G.grid, G.n_designs, G.designs, G.monitors, G.n_mon, G.obj, results + off);
    c->defer = false;
    if (rc != ITR_OK) return fail(ctx, rc, "ladder group %d: %s", gi, c->err.c_str());
    CU(cudaStreamSynchronize(c->stream));   // its inputs are on the device before the graph runs
    off += (size_t)(G.n_designs > 0 ? G.n_designs : 0);
  }
  // Groups whose launch shapes use the same kernel instantiation share its maximum dynamic
  // shared-memory attribute: set it to the largest of their needs before the capture.
  {
    std::vector<std::pair<BatchedFn, size_t>> need;
    for (int gi = 0; gi < n_groups; ++gi) {
      itr_ctx* c = ctx->children[gi];
      if (!c->pending_ok) continue;
      const LaunchCfg& cf = c->last_cfg;
      BatchedFn fn = batched_fn(c->last_args.mode == 1, cf.C > 1, maxt_bucket(cf.T), cf.bnd, c->last_args.locked_dt != nullptr,
                                c->last_args.P.skip_dry != 0);
      bool found = false;
      for (auto& e : need) if (e.first == fn) { e.second = std::max(e.second, cf.smem); found = true; }
      if (!found) need.push_back({fn, cf.smem});
    }
    for (auto& e : need) CU(cudaFuncSetAttribute((const void*)e.first, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.second));
  }
  // one graph: fork from the context stream into every deferred group's stream, join back
  cudaGraph_t gr = nullptr;
  CU(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t ce = cudaEventRecord(ctx->ev_fork, ctx->stream);
  for (int gi = 0; gi < n_groups && ce == cudaSuccess; ++gi) {
    itr_ctx* c = ctx->children[gi];
    if (!c->pending_ok) continue;
    ce = cudaStreamWaitEvent(c->stream, ctx->ev_fork, 0);
    if (ce == cudaSuccess && launch_batched(c, c->last_args, c->last_cfg, c->pending.n, false) != ITR_OK) ce = cudaErrorLaunchFailure;
    if (ce == cudaSuccess) ce = cudaEventRecord(c->ev_fork, c->stream);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(ctx->stream, c->ev_fork, 0);
  }
  const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &gr);
  if (ce != cudaSuccess || ee != cudaSuccess) {
    if (gr) cudaGraphDestroy(gr);
    return fail(ctx, ITR_DEVICE_ERROR, "ladder graph capture: %s", cudaGetErrorString(ce != cudaSuccess ? ce : ee));
  }
  cudaGraphExec_t ge = nullptr;
  ce = cudaGraphInstantiate(&ge, gr, 0);
  cudaGraphDestroy(gr);
  CU(ce);
  CU(cudaEventRecord(ctx->ev[1], ctx->stream));
  ce = cudaGraphLaunch(ge, ctx->stream);
  if (ce == cudaSuccess) ce = cudaEventRecord(ctx->ev[2], ctx->stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
  cudaGraphExecDestroy(ge);
  CU(ce);
  float k_ms = 0.0f;
  CU(cudaEventElapsedTime(&k_ms, ctx->ev[1], ctx->ev[2]));
  uint64_t cu = 0;
  int launches = 1;
  for (int gi = 0; gi < n_groups; ++gi) {
    itr_ctx* c = ctx->children[gi];
    if (c->pending_ok) {
      c->pending_ok = false;
      const int rc = collect_results(c, c->pending);
      if (rc != ITR_OK) return fail(ctx, rc, "ladder group %d: %s", gi, c->err.c_str());
    }
    cu += c->cell_updates;
    launches += c->launches;
  }
  ctx->kernel_ms = k_ms;
  ctx->total_ms = k_ms;
  ctx->cell_updates = cu;
  ctx->launches = launches;
  ctx->have_last = false;
  return ITR_OK;
}

// ------------------------------------------------------------------ map image ---------
extern "C" int itr_gpu_render_map(itr_ctx* ctx, int32_t nx, int32_t ny, double cell_size, const float* z, const float* value,
                                  const float* worse_dz, int32_t mode, float vex, int32_t scale, uint8_t* rgba) {
  if (!ctx) return ITR_INVALID_ARG;
  if (nx < 1 || ny < 1 || (int64_t)nx * ny > (1ll << 28)) return fail(ctx, ITR_INVALID_ARG, "bad grid size");
  if (scale < 1 || (int64_t)nx * scale * (int64_t)ny * scale > (1ll << 30)) return fail(ctx, ITR_INVALID_ARG, "bad scale");
  if (!z || !value || !rgba) return fail(ctx, ITR_INVALID_ARG, "z, value and rgba are required");
  if (mode != 0 && mode != 1) return fail(ctx, ITR_INVALID_ARG, "mode must be 0 (depth) or 1 (difference)");
  if (!(cell_size > 0.0)) return fail(ctx, ITR_INVALID_ARG, "cell size must be positive");
  CU(cudaSetDevice(ctx->device));
  const size_t N = (size_t)nx * ny, P = N * (size_t)scale * scale;
  CU(ctx->rIn.ensure(3 * N * 4));
  CU(ctx->rOut.ensure(P * 4));
  float* din = ctx->rIn.as<float>();
  CU(cudaMemcpyAsync(din, z, N * 4, cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(din + N, value, N * 4, cudaMemcpyHostToDevice, ctx->stream));
  if (worse_dz) CU(cudaMemcpyAsync(din + 2 * N, worse_dz, N * 4, cudaMemcpyHostToDevice, ctx->stream));
  RenderArgs A;
  A.nx = nx; A.ny = ny; A.scale = scale; A.mode = mode; A.worse = worse_dz ? 1 : 0;
  A.vex = vex; A.cs = (float)cell_size;
  A.z = din; A.value = din + N; A.dz = worse_dz ? din + 2 * N : nullptr;
  A.out = ctx->rOut.as<uchar4>();
  const dim3 blk(16, 16), grd((unsigned)((nx * scale + 15) / 16), (unsigned)((ny * scale + 15) / 16));
  k_render_map<<<grd, blk, 0, ctx->stream>>>(A);
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(rgba, ctx->rOut.p, P * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return ITR_OK;
}

extern "C" int itr_gpu_render_scene(itr_ctx* ctx, const uint8_t* terrain, int32_t tw, int32_t th, const uint8_t* depth,
                                    const uint8_t* vel, int32_t nx, int32_t ny, const itr_scene_view* v, int32_t width,
                                    int32_t height, uint8_t* rgba) {
  if (!ctx) return ITR_INVALID_ARG;
  if (!terrain || !depth || !vel || !v || !rgba) return fail(ctx, ITR_INVALID_ARG, "terrain, depth, vel, view and rgba are required");
  if (tw < 1 || th < 1 || (int64_t)tw * th > (1ll << 28)) return fail(ctx, ITR_INVALID_ARG, "bad terrain texture size");
  if (nx < 1 || ny < 1 || (int64_t)nx * ny > (1ll << 28)) return fail(ctx, ITR_INVALID_ARG, "bad grid size");
  if (width < 1 || height < 1 || (int64_t)width * height > (1ll << 28)) return fail(ctx, ITR_INVALID_ARG, "bad image size");
  if (!(v->domain[0] > 0.0f) || !(v->domain[1] > 0.0f) || !(v->domain[2] > 0.0f) || !(v->up > 0.0f) || !(v->ve > 0.0f))
    return fail(ctx, ITR_INVALID_ARG, "domain, cell size, up and ve must be positive");
  if (v->debug < 0 || v->debug > 3) return fail(ctx, ITR_INVALID_ARG, "debug must be 0..3");
  CU(cudaSetDevice(ctx->device));
  const size_t T = (size_t)tw * th, N = (size_t)nx * ny, P = (size_t)width * height;
  CU(ctx->rIn.ensure((T + 2 * N) * 4));
  CU(ctx->rOut.ensure(P * 4));
  uchar4* din = ctx->rIn.as<uchar4>();
  CU(cudaMemcpyAsync(din, terrain, T * 4, cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(din + T, depth, N * 4, cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(din + T + N, vel, N * 4, cudaMemcpyHostToDevice, ctx->stream));
  SceneArgs A;
  memset(&A, 0, sizeof(A));
  A.terrain = din; A.depth = din + T; A.vel = din + T + N;
  A.tw = tw; A.th = th; A.nx = nx; A.ny = ny; A.width = width; A.height = height;
  for (int i = 0; i < 3; ++i) {
    A.cam_pos[i] = v->cam_pos[i]; A.cam_fwd[i] = v->cam_fwd[i]; A.cam_right[i] = v->cam_right[i]; A.cam_up[i] = v->cam_up[i];
  }
  A.focal = v->focal; A.dom_w = v->domain[0]; A.dom_h = v->domain[1]; A.cell = v->domain[2];
  A.z_span = v->z_span; A.up = v->up; A.depth_span = v->depth_span; A.ve = v->ve; A.time = v->time;
  A.rain = v->rain; A.wet = v->wet; A.overcast = v->overcast; A.vel_max = v->vel_max; A.base = v->base;
  A.ortho = v->ortho ? 1 : 0; A.debug = v->debug;
  A.out = ctx->rOut.as<uchar4>();
  const dim3 blk(16, 16), grd((unsigned)((width + 15) / 16), (unsigned)((height + 15) / 16));
  CU(cudaEventRecord(ctx->ev[1], ctx->stream));
  k_render_scene<<<grd, blk, 0, ctx->stream>>>(A);
  CU(cudaGetLastError());
  CU(cudaEventRecord(ctx->ev[2], ctx->stream));
  CU(cudaMemcpyAsync(rgba, ctx->rOut.p, P * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  float k_ms = 0;
  cudaEventElapsedTime(&k_ms, ctx->ev[1], ctx->ev[2]);
  ctx->kernel_ms = k_ms; ctx->total_ms = k_ms; ctx->launches = 1; ctx->cell_updates = 0;
  return ITR_OK;
}

// ------------------------------------------------------------------ baseline record ----
extern "C" int itr_gpu_record_baseline(itr_ctx* ctx, const itr_params* p, const itr_grid* g, const itr_design* base,
                                       const uint32_t* mon, int32_t n_mon, int32_t K, itr_result* result) {
  if (!ctx) return ITR_INVALID_ARG;
  if (!base) return fail(ctx, ITR_INVALID_ARG, "base design is NULL");
  if (K < 1 || K > 65536) return fail(ctx, ITR_INVALID_ARG, "checkpoint interval out of range");
  int rc = check_inputs(ctx, p, g, 1, base, mon, n_mon, nullptr);
  if (rc != ITR_OK) return rc;
  CU(cudaSetDevice(ctx->device));
  if (ctx->rec) {   // a new record replaces the old one
    for (auto& c : ctx->rec->ck) c.state.release();
    delete ctx->rec;
    ctx->rec = nullptr;
  }
  const int nx = g->nx, ny = g->ny;
  const size_t N = (size_t)nx * ny, SX = (size_t)ny * (nx + 1), SY = (size_t)(ny + 1) * nx, NB = 2 * (size_t)(nx + ny);
  Record* R = new Record();
  R->K = K; R->nx = nx; R->ny = ny; R->mode = g->mode;
  R->P = make_run_params(p, g);
  R->bc.resize(NB);
  rc = build_boundaries(ctx, g, R->P.inflow, R->bc.data());
  if (rc != ITR_OK) { delete R; return rc; }
  R->wet.assign(g->wet, g->wet + N); R->gn2.assign(g->gn2, g->gn2 + N);
  R->dzx.assign(base->dzx, base->dzx + SX); R->dzy.assign(base->dzy, base->dzy + SY);
  if (g->mode == ITR_FACE_CREST) { R->dzx2.assign(base->dzx2, base->dzx2 + SX); R->dzy2.assign(base->dzy2, base->dzy2 + SY); }
  if (base->h0) R->h0.assign(base->h0, base->h0 + N);
  bool has_stage = false;
  R->open_rows.assign((size_t)ny, 0);
  for (size_t i = 0; i < NB; ++i) {
    const bool open = g->bc[i] == ITR_BC_STAGE || g->bc[i] == ITR_BC_INFLOW;
    has_stage = has_stage || g->bc[i] == ITR_BC_STAGE;
    if (!open) continue;   // rows beside water-creating edges are wet from the start (solver.rs:404-423)
    const int row = i < (size_t)nx ? 0 : i < 2 * (size_t)nx ? ny - 1 : (int)((i - 2 * (size_t)nx) % ny);
    R->open_rows[row] = 1;
  }
  if (has_stage) { R->bh.resize(NB); stage_depths(g, base->z_edge, R->bh.data()); }
  // the base's run on the tiled path, checkpointed every K steps, with its whole ledger
  const int max_rows = (int)R->P.n_sync;
  std::vector<double> led((size_t)(max_rows > 0 ? max_rows : 1) * 8);
  itr_result local;
  memset(&local, 0, sizeof(local));
  if (result) { local.monitor_max = result->monitor_max; local.peak = result->peak; local.depth = result->depth; }
  local.ledger = led.data();
  local.max_rows = max_rows;
  const int impl0 = ctx->impl, k0 = ctx->steps_per_submit, w0 = ctx->warm_start;
  ctx->impl = 2; ctx->steps_per_submit = K; ctx->warm_start = 0;
  ctx->recording = R;
  rc = itr_gpu_run_batch(ctx, p, g, 1, base, mon, n_mon, nullptr, &local);
  ctx->recording = nullptr;
  ctx->impl = impl0; ctx->steps_per_submit = k0; ctx->warm_start = w0;
  auto drop = [&]() { for (auto& c : R->ck) c.state.release(); delete R; };
  if (rc != ITR_OK) { drop(); return rc; }
  for (size_t c = 0; c < R->ck.size(); ++c) {
    Record::Ckpt& ck = R->ck[c];
    ck.wet.resize((size_t)ny);
    const cudaError_t e = cudaMemcpy(ck.wet.data(), ck.state.as<uint8_t>() + 4 * N * 4, (size_t)ny, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { drop(); return fail(ctx, ITR_DEVICE_ERROR, "baseline record: %s", cudaGetErrorString(e)); }
    const PlainCtl& cl = R->ctl[c];
    WarmStart w;
    memset(&w, 0, sizeof(w));
    w.state = ck.state.as<float>();
    w.t = cl.t; w.dt_cfl = cl.dt_cfl; w.acc_rain = cl.acc_rain; w.v0 = cl.v0; w.volume = cl.volume; w.rel_res = cl.rel_res;
    w.tot_infil = cl.tot_infil; w.tot_fix = cl.tot_fix; w.tot_in = cl.tot_in; w.tot_out = cl.tot_out;
    w.step = cl.step; w.sync_index = cl.sync_index; w.n_rows = cl.n_rows;
    ck.ws = w;
  }
  R->ledger.assign(led.begin(), led.begin() + (size_t)local.n_rows * 8);
  if (result) {
    double* ul = result->ledger;
    const int um = result->max_rows;
    itr_result keep = local;
    keep.ledger = ul; keep.max_rows = um;
    keep.n_rows = local.n_rows < um ? local.n_rows : um;
    if (ul && keep.n_rows > 0) memcpy(ul, led.data(), (size_t)keep.n_rows * 64);
    if (!ul) keep.n_rows = 0;
    *result = keep;
  }
  R->valid = true;
  ctx->rec = R;
  return ITR_OK;
}

// ------------------------------------------------------------------ primitives -------
// Primitive::segment (design.rs:95-106) on the host, with libm sin and cos as the reference.
static MatPrim mat_prim(const itr_primitive& q) {
  MatPrim m;
  memset(&m, 0, sizeof(m));
  m.kind = q.kind; m.width = q.width; m.height = q.height; m.length = q.length;
  if (q.kind == ITR_PRIM_MOUND) {
    m.x0 = m.x1 = q.cx; m.y0 = m.y1 = q.cy;
  } else {
    const double a = q.angle_deg * (3.141592653589793 / 180.0);   // f64::to_radians
    const double sa = std::sin(a), ca = std::cos(a);
    const double hl = 0.5 * q.length;
    m.x0 = q.cx - ca * hl; m.y0 = q.cy - sa * hl; m.x1 = q.cx + ca * hl; m.y1 = q.cy + sa * hl;
  }
  return m;
}

static double nan_min(double a, double b) { if (a != a) return b; if (b != b) return a; return a < b ? a : b; }
static double nan_max(double a, double b) { if (a != a) return b; if (b != b) return a; return a > b ? a : b; }

// The union bounding box of a design's primitives in cells (materialize, design.rs:322-340).
static MatDesign mat_box(const MatPrim* ps, int p0, int p1, const itr_design_space* sp, const itr_grid* g) {
  const size_t nx = (size_t)g->nx, ny = (size_t)g->ny;
  size_t c0 = SIZE_MAX, r0 = SIZE_MAX, c1 = 0, r1 = 0;
  auto fl = [](double v) { v = std::floor(v); return v < 0 ? 0.0 : v; };
  auto ce = [](double v) { v = std::ceil(v); return v < 0 ? 0.0 : v; };
  for (int k = p0; k < p1; ++k) {
    const MatPrim& p = ps[k];
    if (p.height == 0.0) continue;
    const double r = 0.5 * p.width;
    const double bx0 = nan_min(p.x0, p.x1) - r, by0 = nan_min(p.y0, p.y1) - r;
    const double bx1 = nan_max(p.x0, p.x1) + r, by1 = nan_max(p.y0, p.y1) + r;
    const double fc0 = (bx0 - sp->origin_x) / g->dx, fr1 = (sp->origin_y - by0) / g->dy;
    const double fc1 = (bx1 - sp->origin_x) / g->dx, fr0 = (sp->origin_y - by1) / g->dy;
    const size_t a = std::min((size_t)fl(fc0), nx), b = std::min((size_t)fl(fr0), ny);
    const size_t c = std::min((size_t)ce(fc1), nx), d = std::min((size_t)ce(fr1), ny);
    if (a < c && b < d) { c0 = std::min(c0, a); r0 = std::min(r0, b); c1 = std::max(c1, c); r1 = std::max(r1, d); }
  }
  MatDesign m;
  m.p0 = p0; m.p1 = p1;
  if (c0 >= c1 || r0 >= r1) { m.c0 = m.r0 = m.c1 = m.r1 = 0; }
  else { m.c0 = (int)c0; m.r0 = (int)r0; m.c1 = (int)c1; m.r1 = (int)r1; }
  return m;
}

// Checks and host preparation of a batch of designs given as primitives.
static int build_mat(itr_ctx* ctx, const itr_grid* g, const itr_design_space* sp, int32_t n, const int32_t* prim_off,
                     const itr_primitive* prims, Mat& M) {
  if (!g || !sp) return fail(ctx, ITR_INVALID_ARG, "grid and design space are required");
  if (g->mode != ITR_FACE_SIGNED) return fail(ctx, ITR_UNSUPPORTED, "designs as primitives: signed faces (fidelity level 1) only");
  if (!sp->z || !sp->wall || !sp->editable) return fail(ctx, ITR_INVALID_ARG, "design space arrays z, wall, editable are required");
  if (!(sp->max_abs_dz >= 0.0)) return fail(ctx, ITR_INVALID_ARG, "max_abs_dz must be non-negative");
  if (n < 0) return fail(ctx, ITR_INVALID_ARG, "negative design count");
  M.space = sp;
  if (n == 0) return ITR_OK;
  if (!prim_off) return fail(ctx, ITR_INVALID_ARG, "prim_off is NULL");
  if (prim_off[0] < 0) return fail(ctx, ITR_INVALID_ARG, "prim_off[0] is negative");
  for (int d = 0; d < n; ++d)
    if (prim_off[d + 1] < prim_off[d]) return fail(ctx, ITR_INVALID_ARG, "prim_off is not non-decreasing");
  const int total = prim_off[n];
  if (total > 0 && !prims) return fail(ctx, ITR_INVALID_ARG, "prims is NULL");
  M.prims.resize((size_t)total);
  for (int k = prim_off[0]; k < total; ++k) {
    if (prims[k].kind < ITR_PRIM_BERM || prims[k].kind > ITR_PRIM_MOUND) return fail(ctx, ITR_INVALID_ARG, "primitive %d: unknown kind %d", k, prims[k].kind);
    if (!(prims[k].width > 0.0)) return fail(ctx, ITR_INVALID_ARG, "primitive %d: width must be positive", k);
    M.prims[k] = mat_prim(prims[k]);
  }
  M.des.resize((size_t)n);
  for (int d = 0; d < n; ++d) M.des[d] = mat_box(M.prims.data(), prim_off[d], prim_off[d + 1], sp, g);
  M.ds.assign((size_t)n, itr_design{});
  return ITR_OK;
}

extern "C" int itr_gpu_run_primitives(itr_ctx* ctx, const itr_params* p, const itr_grid* g, const itr_design_space* sp,
                                      int32_t n, const int32_t* prim_off, const itr_primitive* prims, const uint32_t* mon,
                                      int32_t n_mon, const itr_objective* ob, itr_result* res, double* cut_m3, double* fill_m3) {
  if (!ctx) return ITR_INVALID_ARG;
  Mat M;
  int rc = build_mat(ctx, g, sp, n, prim_off, prims, M);
  if (rc != ITR_OK) return rc;
  ctx->mat = &M;
  rc = itr_gpu_run_batch(ctx, p, g, n, M.ds.data(), mon, n_mon, ob, res);
  ctx->mat = nullptr;
  if (rc == ITR_OK)
    for (int d = 0; d < n; ++d) {
      if (cut_m3) cut_m3[d] = M.ds[d].cut_m3;
      if (fill_m3) fill_m3[d] = M.ds[d].fill_m3;
    }
  return rc;
}

static int vjp_impl(itr_ctx* ctx, const itr_params* p, const itr_grid* g, int32_t n, const itr_design* ds,
                    const uint32_t* mon, int32_t n_mon, const itr_objective* ob, int32_t checkpoint_interval,
                    itr_result* res, double* dj_ddzx, double* dj_ddzy, double* dj_ddzx2, double* dj_ddzy2) {
  if (!ctx) return ITR_INVALID_ARG;
  if (!ob || ob->n_assets < 1) return fail(ctx, ITR_INVALID_ARG, "the adjoint needs an objective with assets");
  if (!g) return fail(ctx, ITR_INVALID_ARG, "grid is NULL");
  if (g->mode == ITR_FACE_CREST && n > 0 && (!dj_ddzx2 || !dj_ddzy2))
    return fail(ctx, ITR_UNSUPPORTED, "crest faces: use itr_gpu_vjp_crest for the second jumps' gradients");
  if (checkpoint_interval < 1 || checkpoint_interval > 65536) return fail(ctx, ITR_INVALID_ARG, "checkpoint interval out of range");
  if (n > 0 && (!dj_ddzx || !dj_ddzy)) return fail(ctx, ITR_INVALID_ARG, "gradient outputs are NULL");
  itr_objective o = *ob;          // the taped forward runs every design to its end
  o.guard_abort = 0;
  o.has_incumbent = 0;
  Vjp V;
  V.K = checkpoint_interval; V.gx = dj_ddzx; V.gy = dj_ddzy; V.gx2 = dj_ddzx2; V.gy2 = dj_ddzy2;
  ctx->vjp = &V;
  const int rc = itr_gpu_run_batch(ctx, p, g, n, ds, mon, n_mon, &o, res);
  ctx->vjp = nullptr;
  return rc;
}

extern "C" int itr_gpu_vjp_primitives(itr_ctx* ctx, const itr_params* p, const itr_grid* g, const itr_design_space* sp,
                                      int32_t n, const int32_t* prim_off, const itr_primitive* prims, const uint32_t* mon,
                                      int32_t n_mon, const itr_objective* ob, int32_t checkpoint_interval, itr_result* res,
                                      double* dj_dprim, double* dj_ddzx, double* dj_ddzy) {
  if (!ctx) return ITR_INVALID_ARG;
  if (n > 0 && !dj_dprim) return fail(ctx, ITR_INVALID_ARG, "dj_dprim is NULL");
  Mat M;
  int rc = build_mat(ctx, g, sp, n, prim_off, prims, M);
  if (rc != ITR_OK) return rc;
  if (n == 0) return ITR_OK;
  const int nx = g->nx, ny = g->ny;
  const size_t N = (size_t)nx * ny, SX = (size_t)ny * (nx + 1), SY = (size_t)(ny + 1) * nx;
  std::vector<double> gxs, gys;
  if (!dj_ddzx) { gxs.resize((size_t)n * SX); dj_ddzx = gxs.data(); }
  if (!dj_ddzy) { gys.resize((size_t)n * SY); dj_ddzy = gys.data(); }
  ctx->mat = &M;
  rc = itr_gpu_vjp(ctx, p, g, n, M.ds.data(), mon, n_mon, ob, checkpoint_interval, res, dj_ddzx, dj_ddzy);
  ctx->mat = nullptr;
  if (rc != ITR_OK) return rc;
  // the written-out derivative of the materialisation, one job per primitive over its own box
  std::vector<MatPrim> jp;
  std::vector<MatJob> jobs;
  for (int d = 0; d < n; ++d)
    for (int k = prim_off[d]; k < prim_off[d + 1]; ++k) {
      MatJob J;
      memset(&J, 0, sizeof(J));
      J.design = d;
      J.prim = (int)jp.size();
      J.out = 3 * (k - prim_off[0]);
      MatPrim one = M.prims[k];
      one.height = 1.0;   // the box of this primitive alone, also when its height is 0
      jp.push_back(M.prims[k]);
      const MatDesign B = mat_box(&one, 0, 1, sp, g);
      J.c0 = B.c0; J.r0 = B.r0; J.c1 = B.c1; J.r1 = B.r1;
      jobs.push_back(J);
    }
  const cudaStream_t st = ctx->stream;
  CU(ctx->mAux.ensure(2 * N));
  CU(ctx->mJp.ensure((jp.size() > 0 ? jp.size() : 1) * sizeof(MatPrim)));
  CU(ctx->mJob.ensure((jobs.size() > 0 ? jobs.size() : 1) * sizeof(MatJob)));
  CU(ctx->mOut.ensure((size_t)(3 * (jobs.size() > 0 ? jobs.size() : 1)) * 8));
  CU(ctx->mZe.ensure((size_t)n * N * 8));
  CU(cudaMemcpyAsync(ctx->mAux.p, sp->editable, N, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(ctx->mAux.as<uint8_t>() + N, sp->wall, N, cudaMemcpyHostToDevice, st));
  if (!jp.empty()) CU(cudaMemcpyAsync(ctx->mJp.p, jp.data(), jp.size() * sizeof(MatPrim), cudaMemcpyHostToDevice, st));
  if (!jobs.empty()) CU(cudaMemcpyAsync(ctx->mJob.p, jobs.data(), jobs.size() * sizeof(MatJob), cudaMemcpyHostToDevice, st));
  // dz of the designs is still in mDz (the forward's materialisation); the edited levels in
  // mZe are no longer needed and take dJ/d(dz)
  double* gdz = ctx->mZe.as<double>();
  k_mat_gdz<<<dim3((unsigned)((N + 255) / 256), (unsigned)n), 256, 0, st>>>(nx, ny, ctx->aGx.as<double>(), ctx->aGy.as<double>(),
                                                                           ctx->mAux.as<uint8_t>() + N, gdz);
  if (!jobs.empty()) {
    MatArgs MA;
    memset(&MA, 0, sizeof(MA));
    MA.nx = nx; MA.ny = ny; MA.n = n;
    MA.ox = sp->origin_x; MA.oy = sp->origin_y; MA.dx = g->dx; MA.dy = g->dy;
    MA.z_wall = sp->z_wall; MA.max_abs_dz = sp->max_abs_dz;
    MA.editable = ctx->mAux.as<uint8_t>();
    k_mat_dgrad<<<(unsigned)jobs.size(), 256, 0, st>>>(MA, ctx->mJp.as<MatPrim>(), ctx->mJob.as<MatJob>(), ctx->mDz.as<double>(),
                                                       gdz, ob->earth_weight, ob->cut_cost, ob->fill_cost, ctx->mOut.as<double>());
    CU(cudaMemcpyAsync(dj_dprim, ctx->mOut.p, 3 * jobs.size() * 8, cudaMemcpyDeviceToHost, st));
  }
  CU(cudaStreamSynchronize(st));
  return ITR_OK;
}

extern "C" int itr_gpu_vjp(itr_ctx* ctx, const itr_params* p, const itr_grid* g, int32_t n, const itr_design* ds,
                           const uint32_t* mon, int32_t n_mon, const itr_objective* ob, int32_t checkpoint_interval,
                           itr_result* res, double* dj_ddzx, double* dj_ddzy) {
  return vjp_impl(ctx, p, g, n, ds, mon, n_mon, ob, checkpoint_interval, res, dj_ddzx, dj_ddzy, nullptr, nullptr);
}

extern "C" int itr_gpu_vjp_crest(itr_ctx* ctx, const itr_params* p, const itr_grid* g, int32_t n, const itr_design* ds,
                                 const uint32_t* mon, int32_t n_mon, const itr_objective* ob, int32_t checkpoint_interval,
                                 itr_result* res, double* dj_ddzx, double* dj_ddzy, double* dj_ddzx2, double* dj_ddzy2) {
  if (ctx && g && g->mode != ITR_FACE_CREST) return fail(ctx, ITR_INVALID_ARG, "itr_gpu_vjp_crest needs a crest-mode grid");
  if (ctx && n > 0 && (!dj_ddzx2 || !dj_ddzy2)) return fail(ctx, ITR_INVALID_ARG, "second-jump gradient outputs are NULL");
  return vjp_impl(ctx, p, g, n, ds, mon, n_mon, ob, checkpoint_interval, res, dj_ddzx, dj_ddzy, dj_ddzx2, dj_ddzy2);
}

extern "C" int itr_gpu_last_vjp_timing(itr_ctx* ctx, double* forward_ms, double* backward_ms) {
  if (!ctx) return ITR_INVALID_ARG;
  if (forward_ms) *forward_ms = ctx->vjp_fwd_ms;
  if (backward_ms) *backward_ms = ctx->vjp_bwd_ms;
  return ITR_OK;
}

extern "C" int itr_gpu_rerun_resident(itr_ctx* ctx) {
  if (!ctx) return ITR_INVALID_ARG;
  if (!ctx->have_last) return fail(ctx, ITR_INVALID_ARG, "no previous batch to rerun");
  CU(cudaSetDevice(ctx->device));
  int launches = 0;
  CU(cudaEventRecord(ctx->ev[1], ctx->stream));
  if (ctx->last_was_tiled) {
    PlainArgs A = ctx->last_tiled;
    const int band = ctx->band;
    ctx->band = ctx->last_band;   // the kernel its partials were laid out for
    int rc = run_tiled_batch(ctx, A, A.n_designs, ctx->last_tgrid, &launches);
    ctx->band = band;
    if (rc != ITR_OK) return rc;
  } else if (!ctx->last_was_plain) {
    int rc = launch_batched(ctx, ctx->last_args, ctx->last_cfg, ctx->last_args.n_designs);
    if (rc != ITR_OK) return rc;
    launches = 1;
  } else {
    for (size_t i = 0; i < ctx->last_plain.size(); ++i) {
      const PlainArgs& A0 = ctx->last_plain[i];
      PlainArgs A = A0;
      dim3 grid((A.nx + kTile - 1) / kTile, (A.ny + kTile - 1) / kTile);
      int rc = run_plain_design(ctx, A, ctx->last_plain_blocks[i], grid, &launches);
      if (rc != ITR_OK) return rc;
    }
  }
  CU(cudaEventRecord(ctx->ev[2], ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  CU(cudaGetLastError());
  float k_ms = 0;
  cudaEventElapsedTime(&k_ms, ctx->ev[1], ctx->ev[2]);
  ctx->kernel_ms = k_ms;
  ctx->total_ms = k_ms;
  ctx->launches = launches;
  return ITR_OK;
}

// Allocation-free variant of the plain path (static device scratch).
#include "itr_static.cuh"
