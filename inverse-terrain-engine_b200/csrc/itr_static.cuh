// itr_static.cuh — the plain forward of one design with no device allocation at all.
//
// itr_gpu_run_batch keeps its scratch in device buffers owned by a context and grown with
// cudaMalloc on demand. Some callers cannot allocate device memory at the point where they
// want a forward run:
//   * a process that commits the whole device to its own pool up front (a serving process
//     sized to HBM, an optimiser that reserves memory for its population) has no free
//     memory left for a library to take;
//   * cudaMalloc and cudaFree synchronise the device, so a caller that interleaves short
//     re-evaluations between launches of other streams would stall all of them;
//   * a search loop must not fail half-way through on an out-of-memory error that depends
//     on what else happens to be resident.
// For them, itr_gpu_run_plain_static runs the same kernels as the plain path (k_plain_init,
// k_plain_update, k_plain_finalize; bit-identical results) on scratch that lives in one
// file-scope static device array of fixed size. CUDA reserves that array on a device when it
// loads the library's module there; under CUDA's default lazy module loading that happens at
// the first use of the module on the device, i.e. inside the first itr_gpu_run_plain_static
// call (its cudaGetSymbolAddress), not when the library is opened. A caller that commits the
// device's memory to its own pool therefore makes one call first. After that the entry point
// calls no allocator (device or host): inputs are copied into the static array, results are
// copied out of it.
//
// Limits (rejected with ITR_INVALID_ARG and a message before any device work):
//   (nx+1)*(ny+1) <= ITR_STATIC_MAX_POINTS, ceil(nx/16)*ceil(ny/16) <= ITR_STATIC_MAX_TILES,
//   n_mon <= ITR_STATIC_MAX_MONITORS, ledger rows <= ITR_STATIC_MAX_LEDGER_ROWS, no objective.
// One static array per device, kept from call to call: each call clears what must start at
// zero. Calls on the same device that overlap in time (two host threads, or several
// streams) race on it and corrupt each other's results; callers serialise them. The first
// call on a device loads the module and looks up the array's address (see static_scratch):
// it should come before any stream capture and before the caller commits the device's memory.
#pragma once

namespace itr {

constexpr size_t kStaticPoints = ITR_STATIC_MAX_POINTS;
constexpr size_t kStaticTiles = ITR_STATIC_MAX_TILES;
constexpr size_t kStaticMon = ITR_STATIC_MAX_MONITORS;
constexpr size_t kStaticRows = ITR_STATIC_MAX_LEDGER_ROWS;
constexpr unsigned long long kStaticMaxSteps = 2000000000ull;   // device step limit (status 4 beyond it)

// Fixed layout of the static array (byte offsets, each 256-aligned). Planes are sized for
// kStaticPoints entries, which bounds nx*ny, ny*(nx+1) and (ny+1)*nx alike.
constexpr size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
struct StaticLayout {
  static constexpr size_t plane = al256(kStaticPoints * 4);
  static constexpr size_t H = 0;   // two planes at stride nx*ny (PlainArgs: plane par at par*nx*ny)
  static constexpr size_t QX = H + 2 * plane;
  static constexpr size_t QY = QX + 2 * plane;
  static constexpr size_t PK = QY + 2 * plane;
  static constexpr size_t WET = PK + plane;
  static constexpr size_t GN2 = WET + plane;
  static constexpr size_t DZX = GN2 + plane;
  static constexpr size_t DZY = DZX + plane;
  static constexpr size_t DZX2 = DZY + plane;
  static constexpr size_t DZY2 = DZX2 + plane;
  static constexpr size_t H0 = DZY2 + plane;
  static constexpr size_t BC = H0 + plane;             // 2*nx + 2*ny codes
  static constexpr size_t MON = BC + al256(2 * kStaticPoints);
  static constexpr size_t MMAX = MON + al256(kStaticMon * 4);
  static constexpr size_t PART = MMAX + al256(kStaticMon * 8);
  static constexpr size_t LEDGER = PART + al256(kStaticTiles * kPart * 8);
  static constexpr size_t CTL = LEDGER + al256(kStaticRows * 8 * 8);
  static constexpr size_t bytes = CTL + al256(sizeof(PlainCtl));
};

static __device__ __align__(256) unsigned char g_static_scratch[StaticLayout::bytes];

__global__ void k_gather_monitors_f64(const float* peak, const unsigned* mon, int n_mon, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_mon) out[i] = (double)peak[mon[i]];
}

// h0 of init_state (solver.rs:287-312) for a design without an explicit initial depth.
__global__ void k_static_h0(const float* wet, size_t n, float hinit, float* h0) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    h0[i] = wet[i] != 0.0f ? hinit : 0.0f;
}

}  // namespace itr

namespace {

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
void* g_static_addr[kStaticMaxDevices] = {};

int static_fail(char* err, size_t errlen, int code, const char* fmt, ...) {
  if (err && errlen > 0) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, errlen, fmt, ap);
    va_end(ap);
  }
  return code;
}

// Restores the caller's current device on every exit path.
struct DeviceGuard {
  int prev = -1;
  bool changed = false;
  cudaError_t enter(int device) {
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return e;
    if (prev != device) { changed = true; return cudaSetDevice(device); }
    return cudaSuccess;
  }
  ~DeviceGuard() { if (changed) cudaSetDevice(prev); }
};

// Device address of the static array on `device`, looked up once per device with that
// device current (the symbol has one instance per device). In host code the array's name
// is only a host-side stand-in, so kernels get this address, never the name. The lookup
// happens in the first call on a device; that first call belongs before any stream capture.
int static_scratch(int device, unsigned char** out, char* err, size_t errlen) {
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, itr::g_static_scratch);
    if (e != cudaSuccess || !p)
      return static_fail(err, errlen, ITR_DEVICE_ERROR, "cudaGetSymbolAddress(static scratch) on device %d: %s", device,
                         cudaGetErrorString(e));
    g_static_addr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_static_addr[device]);
  return ITR_OK;
}

}  // namespace

#define SCU(x)                                                                                            \
  do {                                                                                                    \
    cudaError_t e_ = (x);                                                                                 \
    if (e_ != cudaSuccess) return static_fail(err, errlen, ITR_DEVICE_ERROR, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

extern "C" int itr_gpu_run_plain_static(int device, const itr_params* p, const itr_grid* g, const itr_design* ds,
                                        const uint32_t* mon, int32_t n_mon, itr_result* res, char* err, size_t errlen) {
  using namespace itr;
  using L = StaticLayout;
  // ---- validation, before any device work ----
  if (!p || !g || !ds || !res) return static_fail(err, errlen, ITR_INVALID_ARG, "params, grid, design and result are required");
  if (device < 0 || device >= kStaticMaxDevices) return static_fail(err, errlen, ITR_INVALID_ARG, "device %d out of range", device);
  if (g->nx < 1 || g->ny < 1) return static_fail(err, errlen, ITR_INVALID_ARG, "grid must have nx, ny >= 1");
  const int nx = g->nx, ny = g->ny;
  const size_t points = ((size_t)nx + 1) * ((size_t)ny + 1);
  if (points > kStaticPoints)
    return static_fail(err, errlen, ITR_INVALID_ARG,
                       "grid %dx%d needs (nx+1)*(ny+1) = %zu points; the static scratch holds %zu (e.g. 512x512)", nx, ny,
                       points, kStaticPoints);
  const dim3 grid((nx + kTile - 1) / kTile, (ny + kTile - 1) / kTile);
  const int nb = (int)(grid.x * grid.y);
  if ((size_t)nb > kStaticTiles)
    return static_fail(err, errlen, ITR_INVALID_ARG, "grid %dx%d has %d tiles of 16x16; the static scratch holds %zu", nx, ny, nb,
                       kStaticTiles);
  if (n_mon < 0 || (size_t)n_mon > kStaticMon || (n_mon > 0 && !mon))
    return static_fail(err, errlen, ITR_INVALID_ARG, "monitor list invalid or longer than %zu", kStaticMon);
  if (res->ledger && (res->max_rows < 0 || (size_t)res->max_rows > kStaticRows))
    return static_fail(err, errlen, ITR_INVALID_ARG, "ledger rows %d exceed the static limit %zu", res->max_rows, kStaticRows);
  if (!(g->dx > 0.0) || !(g->dy > 0.0)) return static_fail(err, errlen, ITR_INVALID_ARG, "cell size must be positive");
  if (!g->wet || !g->gn2 || !g->bc) return static_fail(err, errlen, ITR_INVALID_ARG, "grid arrays wet, gn2, bc are required");
  if (g->mode != ITR_FACE_SIGNED && g->mode != ITR_FACE_CREST) return static_fail(err, errlen, ITR_INVALID_ARG, "unknown face mode %d", g->mode);
  for (int64_t i = 0; i < 2ll * nx + 2ll * ny; ++i) {
    if (g->bc[i] == ITR_BC_STAGE || g->bc[i] == ITR_BC_INFLOW)
      return static_fail(err, errlen, ITR_UNSUPPORTED,
                         "Stage and Inflow boundaries are not supported by itr_gpu_run_plain_static (use itr_gpu_run_batch)");
    if (g->bc[i] > ITR_BC_INFLOW) return static_fail(err, errlen, ITR_INVALID_ARG, "unknown boundary code %d", (int)g->bc[i]);
  }
  if (p->inflow_scale != 1.0)
    return static_fail(err, errlen, ITR_UNSUPPORTED,
                       "inflow_scale other than 1 is not supported by itr_gpu_run_plain_static (use itr_gpu_run_batch)");
  if (!(p->duration_s >= 0.0) || !(p->sync_interval_s > 0.0) || !(p->cfl > 0.0) || !(p->dt_max_s > 0.0))
    return static_fail(err, errlen, ITR_INVALID_ARG, "duration, sync interval, cfl and dt_max must be positive");
  if (p->n_rain < 0 || p->n_rain > kMaxRain) return static_fail(err, errlen, ITR_INVALID_ARG, "hyetograph has %d points (max %d)", p->n_rain, kMaxRain);
  if (p->n_rain > 0 && (!p->rain_t || !p->rain_rate)) return static_fail(err, errlen, ITR_INVALID_ARG, "hyetograph arrays are NULL");
  for (int32_t k = 0; k < n_mon; ++k)
    if ((int64_t)mon[k] >= (int64_t)nx * ny) return static_fail(err, errlen, ITR_INVALID_ARG, "monitor cell out of range");
  const bool crest = g->mode == ITR_FACE_CREST;
  if (!ds->dzx || !ds->dzy) return static_fail(err, errlen, ITR_INVALID_ARG, "design has no face jumps");
  if (crest && (!ds->dzx2 || !ds->dzy2)) return static_fail(err, errlen, ITR_INVALID_ARG, "crest mode needs dzx2/dzy2");
  // The same start check as itr_gpu_run_batch: an infinite or absurdly deep start makes the
  // first CFL dt zero or vanishing, so the run would crawl towards its step limit. NaN and
  // negative depths are left to the solver's health test (Unhealthy at the first step).
  if (ds->h0)
    for (size_t i = 0; i < (size_t)nx * ny; ++i)
      if (std::isinf(ds->h0[i]) || ds->h0[i] > kMaxInitialDepth)
        return static_fail(err, errlen, ITR_INVALID_ARG, "initial depth %g at cell %zu is infinite or above %g m",
                           (double)ds->h0[i], i, (double)kMaxInitialDepth);

  // ---- set-up: the static array of this device ----
  DeviceGuard dg;
  SCU(dg.enter(device));
  unsigned char* base = nullptr;
  int rc = static_scratch(device, &base, err, errlen);
  if (rc != ITR_OK) return rc;
  float* H = reinterpret_cast<float*>(base + L::H);
  float* QX = reinterpret_cast<float*>(base + L::QX);
  float* QY = reinterpret_cast<float*>(base + L::QY);
  float* PK = reinterpret_cast<float*>(base + L::PK);
  const size_t N = (size_t)nx * ny, SX = (size_t)ny * (nx + 1), SY = (size_t)(ny + 1) * nx;
  float* wet = reinterpret_cast<float*>(base + L::WET);
  float* gn2 = reinterpret_cast<float*>(base + L::GN2);
  float* dzx = reinterpret_cast<float*>(base + L::DZX);
  float* dzy = reinterpret_cast<float*>(base + L::DZY);
  float* dzx2 = reinterpret_cast<float*>(base + L::DZX2);
  float* dzy2 = reinterpret_cast<float*>(base + L::DZY2);
  float* h0 = reinterpret_cast<float*>(base + L::H0);
  uint8_t* bc = base + L::BC;
  unsigned* dmon = reinterpret_cast<unsigned*>(base + L::MON);
  double* mmax = reinterpret_cast<double*>(base + L::MMAX);
  double* part = reinterpret_cast<double*>(base + L::PART);
  double* ledger = reinterpret_cast<double*>(base + L::LEDGER);
  PlainCtl* ctl = reinterpret_cast<PlainCtl*>(base + L::CTL);
  const cudaStream_t st = 0;   // legacy default stream: ordered after the caller's blocking work

  // ---- inputs into the static array ----
  SCU(cudaMemcpyAsync(wet, g->wet, N * 4, cudaMemcpyHostToDevice, st));
  SCU(cudaMemcpyAsync(gn2, g->gn2, N * 4, cudaMemcpyHostToDevice, st));
  SCU(cudaMemcpyAsync(bc, g->bc, 2 * (size_t)nx + 2 * (size_t)ny, cudaMemcpyHostToDevice, st));
  SCU(cudaMemcpyAsync(dzx, ds->dzx, SX * 4, cudaMemcpyHostToDevice, st));
  SCU(cudaMemcpyAsync(dzy, ds->dzy, SY * 4, cudaMemcpyHostToDevice, st));
  if (crest) {
    SCU(cudaMemcpyAsync(dzx2, ds->dzx2, SX * 4, cudaMemcpyHostToDevice, st));
    SCU(cudaMemcpyAsync(dzy2, ds->dzy2, SY * 4, cudaMemcpyHostToDevice, st));
  }
  if (ds->h0) {
    SCU(cudaMemcpyAsync(h0, ds->h0, N * 4, cudaMemcpyHostToDevice, st));
  } else {
    const float hinit = (float)(p->initial_depth > 0.0 ? p->initial_depth : 0.0);
    k_static_h0<<<148, 256, 0, st>>>(wet, N, hinit, h0);
  }
  if (n_mon > 0) SCU(cudaMemcpyAsync(dmon, mon, (size_t)n_mon * 4, cudaMemcpyHostToDevice, st));
  // What must start at zero: the control block (its smax/bad words are accumulated with
  // atomics) and the per-tile partials. k_plain_init rewrites the control block and the
  // state and peak planes of plane 0 as well, so nothing survives from an earlier call.
  SCU(cudaMemsetAsync(ctl, 0, sizeof(PlainCtl), st));
  SCU(cudaMemsetAsync(part, 0, (size_t)nb * kPart * 8, st));

  // ---- the plain forward (the launch sequence of the context path) ----
  PlainArgs A;
  memset(&A, 0, sizeof(A));
  A.P = make_run_params(p, g);
  A.nx = nx; A.ny = ny; A.mode = g->mode;
  A.wet = wet; A.gn2 = gn2; A.bc = bc;
  A.dzx = dzx; A.dzy = dzy;
  A.dzx2 = crest ? dzx2 : nullptr; A.dzy2 = crest ? dzy2 : nullptr;
  A.h0 = h0;
  A.cut = ds->cut_m3; A.fill = ds->fill_m3;
  A.n_mon = n_mon; A.mon_cells = dmon;
  A.obj.enabled = 0;
  A.H = H; A.QX = QX; A.QY = QY; A.PK = PK;
  A.part = part; A.ctl = ctl;
  const int max_rows = res->ledger ? res->max_rows : 0;
  A.ledger = max_rows > 0 ? ledger : nullptr;
  A.max_rows = max_rows;
  A.max_steps = kStaticMaxSteps;
  k_plain_init<<<1, 1024, 0, st>>>(A);
  k_plain_finalize<<<1, 32, 0, st>>>(A, nb, 1);
  constexpr int kStepsPerPoll = 64;
  PlainCtl hc;
  for (uint64_t polls = 0;; ++polls) {
    for (int s = 0; s < kStepsPerPoll; ++s) {
      if (crest) k_plain_update<true><<<grid, kTileThreads, 0, st>>>(A);
      else k_plain_update<false><<<grid, kTileThreads, 0, st>>>(A);
      k_plain_finalize<<<1, kFinThreads, 0, st>>>(A, nb, 0);   // as run_plain_design: same summation order
    }
    SCU(cudaGetLastError());
    SCU(cudaMemcpyAsync(&hc, ctl, sizeof(PlainCtl), cudaMemcpyDeviceToHost, st));
    SCU(cudaStreamSynchronize(st));
    if (hc.done) break;
    // the device stops a run at max_steps (status 4), so this bound is never the one that ends it
    if (polls > kStaticMaxSteps / kStepsPerPoll + 2)
      return static_fail(err, errlen, ITR_DEVICE_TIMEOUT, "plain run did not terminate");
  }
  if (hc.status >= 4) return static_fail(err, errlen, ITR_DEVICE_TIMEOUT, "run exceeded its step limit (status %d)", hc.status);

  // ---- results out of the static array ----
  if (n_mon > 0 && res->monitor_max) {
    k_gather_monitors_f64<<<(n_mon + 255) / 256, 256, 0, st>>>(PK, dmon, n_mon, mmax);
    SCU(cudaMemcpyAsync(res->monitor_max, mmax, (size_t)n_mon * 8, cudaMemcpyDeviceToHost, st));
  }
  if (res->peak) SCU(cudaMemcpyAsync(res->peak, PK, N * 4, cudaMemcpyDeviceToHost, st));
  if (res->depth) SCU(cudaMemcpyAsync(res->depth, H + (size_t)hc.par * N, N * 4, cudaMemcpyDeviceToHost, st));
  const int rows = hc.n_rows < max_rows ? hc.n_rows : max_rows;
  if (rows > 0) SCU(cudaMemcpyAsync(res->ledger, ledger, (size_t)rows * 64, cudaMemcpyDeviceToHost, st));
  SCU(cudaStreamSynchronize(st));
  SCU(cudaGetLastError());
  res->steps = hc.step;
  res->cell_updates = hc.step * (uint64_t)N;
  res->t_end = hc.t;
  res->sync_count = hc.sync_index;
  res->status = hc.status;
  res->breach_cell = 0; res->breach_sync = 0;
  res->violation = 0.0; res->lower_bound = 0.0;
  res->j = 0.0;
  res->feasible = hc.status == ITR_RUN_UNHEALTHY ? 0 : 1;
  res->n_rows = rows;
  res->volume_m3 = hc.volume;
  res->rel_residual = hc.rel_res;
  res->warm_start_steps = 0;
  res->dt_fallback_t = -1.0;
  return ITR_OK;
}

#undef SCU
