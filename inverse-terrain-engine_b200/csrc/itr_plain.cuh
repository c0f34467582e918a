// itr_plain.cuh — tiled forward with the state in HBM (global-memory ping-pong).
//
// This is the straightforward CUDA form of the reference's GPU backend structure
// (crates/itr-gpu/src/shader.wgsl:135-365, lib.rs:302-328): per step one tiled `update`
// kernel (16x16 cells, 18x18 halo in shared memory, faces computed once per tile) and one
// single-warp `finalize` kernel that advances the f64 integrator on the device; the host
// polls a control word every `steps_per_submit` steps.
// Launched with one design (gridDim.z = 1, designs one after another) it is the plain
// forward, the baseline the batched cluster kernel is measured against. Launched with all
// designs at once (design = blockIdx.z of the update, blockIdx.x of finalize/init) it is the
// tiled batched forward for grids too large for a cluster's shared memory, and the forward
// recomputation of the adjoint (optional argmax-of-peak and dt/rain logs). Per-cell
// arithmetic is itr_device.cuh's, so results are bit-identical to the cluster kernel's and
// to the f32 CPU oracle's.
#pragma once
#include "itr_device.cuh"

namespace itr {

constexpr int kTile = 16;
// Threads of the tiled kernels: 9 warps, so the 272 x-faces and 272 y-faces of a 16x16 tile
// take one pass (with 256 threads a second pass would run 16 faces on a full block); the
// 256 cells of the tile use the first 8 warps.
constexpr int kTileThreads = 288;
static_assert(kTileThreads >= 17 * 16, "one x-face and one y-face per thread");
// Per-tile partial sums written by the update kernel: infiltration, positivity fix, x-edge
// inflow and outflow volumes, volume (sync steps), and the top and bottom edges' summed
// mass fluxes (signed: the reference nets a y-edge over its whole row before splitting it
// into inflow and outflow, kernel.rs:452-472).
constexpr int kPart = 7;
// The update kernels ask for 6 resident blocks per SM (32 registers a thread): with the
// 18x18 halo loads waiting on HBM, more resident warps beat fewer registers (measured +10%).

// Device-side integrator state of one design (the reference's Ctl words, in f64).
struct PlainCtl {
  double t, dt_cfl, acc_rain, v0, volume, rel_res;
  double tot_infil, tot_fix, tot_in, tot_out;
  double violation, lower_bound;
  unsigned long long step;
  unsigned sync_index, breach_cell, breach_sync;
  int status;   // 0 running, else itr_run_status (+10 once finished OK)
  int done;
  int par;
  int n_rows;
  unsigned smax_bits, bad;
  StepPlan pl;
  StepK k;
  float2 inf[kMaxInflow];   // inflow groups at the step's start time (inflow_values)
  // baseline-locked dt (k_plain_finalize_locked): smax of the current state, whether the
  // schedule still holds, and the state copy the finalize asks of k_plain_locked_copy
  // (1 save into the sync snapshot, 2 restore from it)
  double s_cur;
  int locked_live;
  int copy_req;
  unsigned long long rows_skipped;   // dry rows skipped so far (kernel.rs:605-612)
};

struct PlainArgs {
  RunParams P;
  int nx, ny, mode;
  const float* wet;
  const float* gn2;
  const uint8_t* bc;  // device codes (ghost_state): 0 wall, 1 transmissive, 2 stage, 3 + inflow group
  const float* bh;    // stage-ghost depths, per design [2 nx + 2 ny] indexed like bc; NULL without stage cells
  const float* dzx;   // design 0; design d at + d * ny * (nx + 1)
  const float* dzy;   //                         + d * (ny + 1) * nx
  const float* dzx2;
  const float* dzy2;
  const float* h0;    // + d * nx * ny
  double cut, fill;   // one design, or per design in cut_d / fill_d when those are set
  const double* cut_d;
  const double* fill_d;
  int n_designs;
  int n_mon;
  const unsigned* mon_cells;
  DevObjective obj;
  float* H;           // per design [2][nx*ny]
  float* QX;
  float* QY;
  float* PK;          // per design nx*ny
  double* part;       // per design, per tile: [kPart]
  PlainCtl* ctl;      // per design
  double* ledger;     // per design max_rows*8
  int max_rows;
  unsigned long long max_steps;
  unsigned* tpk;      // optional, per design nx*ny: index of the state that last raised PK
  double* dt_log;     // optional, per design a ring of max_log (dt, rain, t): slot step % max_log
  int max_log;
  const WarmStart* warm;   // optional, per design (state NULL: cold)
  // Baseline-locked dt (SolverParams::locked_dt / cfl_hard, solver.rs:42-46); read only by
  // k_plain_finalize_locked and k_plain_locked_copy
  const double* locked_dt;   // n_locked dts of the baseline, shared by every design
  unsigned long long n_locked;
  double cfl_hard;
  float* snap;               // per design [4][nx*ny]: h, qx, qy, peaks at the last sync snapshot
  PlainCtl* snapctl;         // per design: the control block at that snapshot
  double* fallback_t;        // per design: time the run fell back to adaptive dt, -1 for none
  // Dry-row skipping (kernel.rs:605-612), on the row-band path only (NULL elsewhere): per design
  // [2][ny + 2] flags, padded row j (0 and ny + 1 the ghost rows) held water in the state of
  // that parity (written by k_band, cleared by the finalize once read); the ghost wetness of
  // the current step per padded row (stage / inflow grids only, else NULL); the flags at the
  // locked-dt snapshot.
  unsigned* rowwet;
  uint8_t* gwet;
  unsigned* snaprow;
  int band_rows;             // row-band kernel: rows per band (1 .. 32)
  // State layout (0: the ping-pong default, design d's planes at H + d 2 N, plane p at + p N).
  // The adjoint's replay (k_band with TAPE) reads and writes its tape through these: design
  // stride 3 N, and plane 1 = the next step's slot.
  size_t state_stride;
  size_t plane_stride;
};

// Padded row j is dry for the step about to run: no water in its state nor in its stage or
// inflow ghosts (B.dry of step_fused, kernel.rs:590-612).
ITR_DEV bool plain_row_dry(const unsigned* rw, const uint8_t* gw, int j) { return rw[j] == 0u && !(gw && gw[j]); }

// Ghost wetness of every padded row for a step starting at the inflow values `inf`
// (ghost_row_wet); one warp.
ITR_DEV void plain_ghost_wet(const PlainArgs& A, const float* bh, const float2* inf, uint8_t* gw, int lane) {
  ghost_row_wet(A.bc, A.nx, A.ny, bh, inf, gw, lane);
}

// Pointers of design d inside a launch over n_designs designs.
struct PlainDesign {
  const float *dzx, *dzy, *dzx2, *dzy2, *h0, *bh;
  float *H, *QX, *QY, *PK;
  double* part;
  PlainCtl* ctl;
  double* ledger;
  unsigned* tpk;
  double* dt_log;
  double cut, fill;
  unsigned* rowwet;   // [2][ny + 2]
  uint8_t* gwet;      // [ny + 2]
  unsigned* snaprow;  // [ny + 2]
};

ITR_DEV PlainDesign plain_design(const PlainArgs& A, int d, int n_tiles) {
  const size_t N = (size_t)A.nx * A.ny, SX = (size_t)A.ny * (A.nx + 1), SY = (size_t)(A.ny + 1) * A.nx;
  PlainDesign v;
  v.dzx = A.dzx + d * SX; v.dzy = A.dzy + d * SY;
  v.dzx2 = A.dzx2 ? A.dzx2 + d * SX : nullptr; v.dzy2 = A.dzy2 ? A.dzy2 + d * SY : nullptr;
  v.h0 = A.h0 + d * N;
  v.bh = A.bh ? A.bh + (size_t)d * (2 * A.nx + 2 * A.ny) : nullptr;
  const size_t ss = A.state_stride ? A.state_stride : 2 * N;
  v.H = A.H + d * ss; v.QX = A.QX + d * ss; v.QY = A.QY + d * ss;
  v.PK = A.PK + d * N;
  v.part = A.part + (size_t)d * n_tiles * kPart;
  v.ctl = A.ctl + d;
  v.ledger = A.ledger ? A.ledger + (size_t)d * A.max_rows * 8 : nullptr;
  v.tpk = A.tpk ? A.tpk + d * N : nullptr;
  v.dt_log = A.dt_log ? A.dt_log + (size_t)d * A.max_log * 3 : nullptr;
  v.cut = A.cut_d ? A.cut_d[d] : A.cut;
  v.fill = A.fill_d ? A.fill_d[d] : A.fill;
  const size_t R = (size_t)A.ny + 2;
  v.rowwet = A.rowwet ? A.rowwet + (size_t)d * 2 * R : nullptr;
  v.gwet = A.gwet ? A.gwet + (size_t)d * R : nullptr;
  v.snaprow = A.snaprow ? A.snaprow + (size_t)d * R : nullptr;
  return v;
}

// Old state of padded cell (gx, gy) with ghost cells outside (boundary.rs:36-87). BND: the
// grid has stage or inflow cells (ghost_state); without, only walls flip a sign.
template <bool BND>
ITR_DEV void plain_load(const PlainArgs& A, const PlainDesign& D, int par, int gx, int gy, float& h, float& qx, float& qy) {
  const int nx = A.nx, ny = A.ny;
  const bool ox = gx < 0 || gx >= nx, oy = gy < 0 || gy >= ny;
  if (ox && oy) { h = 0.0f; qx = 0.0f; qy = 0.0f; return; }
  int sx = gx < 0 ? 0 : (gx >= nx ? nx - 1 : gx);
  int sy = gy < 0 ? 0 : (gy >= ny ? ny - 1 : gy);
  size_t i = (size_t)par * nx * ny + (size_t)sy * nx + sx;
  h = D.H[i]; qx = D.QX[i]; qy = D.QY[i];
  if (!BND) {
    if (ox) { int code = gx < 0 ? A.bc[2 * nx + sy] : A.bc[2 * nx + ny + sy]; if (code == 0) qx = -qx; }
    else if (oy) { int code = gy < 0 ? A.bc[sx] : A.bc[nx + sx]; if (code == 0) qy = -qy; }
  } else if (ox || oy) {
    const int p = ox ? (gx < 0 ? 2 * nx + sy : 2 * nx + ny + sy) : (gy < 0 ? sx : nx + sx);
    const int code = A.bc[p];
    const float hs = code == 2 ? D.bh[p] : 0.0f;
    const float2 fi = code >= 3 ? D.ctl->inf[code - 3] : make_float2(0.0f, 0.0f);
    if (ox) ghost_state<true>(code, h, qx, qy, hs, fi, gx < 0);
    else ghost_state<false>(code, h, qx, qy, hs, fi, gy < 0);
  }
}

template <bool CREST, bool BND = false>
__global__ void __launch_bounds__(kTileThreads, 6) k_plain_update(const PlainArgs A) {
  __shared__ float sh[18 * 18], su[18 * 18], sv[18 * 18], sc[18 * 18], sqx[18 * 18], sqy[18 * 18];
  __shared__ FaceF fx[16 * 17], fy[17 * 16];
  __shared__ float wmax[kTileThreads / 32];
  __shared__ unsigned wbad[kTileThreads / 32];
  __shared__ double wsum[kTileThreads / 32][5];
  __shared__ double yedge[2][kTile];   // mass flux of the tile's top-edge / bottom-edge faces per column
  const PlainDesign D = plain_design(A, blockIdx.z, gridDim.x * gridDim.y);
  const PlainCtl& cl = *D.ctl;
  if (cl.done) return;
  const int par = cl.par;
  const StepK k = cl.k;
  const bool hits = cl.pl.hits;
  const double dt_dy = cl.pl.dt * A.P.dy;
  const int nx = A.nx, ny = A.ny;
  const int gx0 = blockIdx.x * kTile, gy0 = blockIdx.y * kTile;
  const int li = threadIdx.x;
  // Every global load of this thread is issued first, so their latencies overlap: the
  // jumps of its x- and y-face (thread e computes x-face e and y-face e), its cell's wet,
  // g n^2 and running peak, then its halo cells.
  const int fxr = li / 17, fxcol = li % 17, fyr_ = li / 16, fycol = li % 16;
  const bool xv = li < 272 && gy0 + fxr < ny && gx0 + fxcol <= nx;
  const bool yv = li < 272 && gx0 + fycol < nx && gy0 + fyr_ <= ny;
  const size_t xo = (size_t)(gy0 + fxr) * (nx + 1) + gx0 + fxcol;
  const size_t yo = (size_t)(gy0 + fyr_) * nx + gx0 + fycol;
  const float xd0 = xv ? D.dzx[xo] : 0.0f, xd1 = (CREST && xv) ? D.dzx2[xo] : 0.0f;
  const float yd0 = yv ? D.dzy[yo] : 0.0f, yd1 = (CREST && yv) ? D.dzy2[yo] : 0.0f;
  const int lx = li % 16, ly = li / 16;
  const int gx = gx0 + lx, gy = gy0 + ly;
  const bool cv = li < 256 && gx < nx && gy < ny;
  const size_t gi = (size_t)gy * nx + gx;
  const float wet_c = cv ? A.wet[gi] : 0.0f, gn2_c = cv ? A.gn2[gi] : 0.0f, pk_c = cv ? D.PK[gi] : 0.0f;
  if (li < 2 * kTile) yedge[li / kTile][li % kTile] = 0.0;
  for (int e = li; e < 324; e += kTileThreads) {
    int hx = e % 18, hy = e / 18;
    float h, qx, qy;
    plain_load<BND>(A, D, par, gx0 - 1 + hx, gy0 - 1 + hy, h, qx, qy);
    float u, v, c;
    cell_vel(h, qx, qy, k.g, k.heps2, u, v, c);
    sh[e] = h; sqx[e] = qx; sqy[e] = qy; su[e] = u; sv[e] = v; sc[e] = c;
  }
  __syncthreads();
  if (xv) {  // x-faces: 16 rows x 17
    const int a = (fxr + 1) * 18 + fxcol;
    fx[li] = face<true, CREST>(sh[a], su[a], sv[a], sc[a], sh[a + 1], su[a + 1], sv[a + 1], sc[a + 1], xd0, xd1, k);
  }
  if (yv) {  // y-faces: 17 rows x 16
    const int a = fyr_ * 18 + fycol + 1, b = a + 18;
    fy[li] = face<false, CREST>(sh[a], su[a], sv[a], sc[a], sh[b], su[b], sv[b], sc[b], yd0, yd1, k);
  }
  __syncthreads();
  float smax = 0.0f;
  bool bad = false;
  double acc[5] = {0, 0, 0, 0, 0};
  if (cv) {
    const FaceF w = fx[ly * 17 + lx], e = fx[ly * 17 + lx + 1];
    const FaceF n = fy[ly * 16 + lx], s = fy[(ly + 1) * 16 + lx];
    const int a = (ly + 1) * 18 + lx + 1;
    CellNew o = update_cell(sh[a], sqx[a], sqy[a], w, e, n, s, wet_c, gn2_c, k);
    const size_t wo = (size_t)(par ^ 1) * nx * ny + gi;
    D.H[wo] = o.h; D.QX[wo] = o.qx; D.QY[wo] = o.qy;
    if (o.h > pk_c) {
      D.PK[gi] = o.h;
      if (D.tpk) D.tpk[gi] = (unsigned)(cl.step + 1);   // this step makes state step+1
    }
    smax = o.s;
    bad = o.bad;
    acc[0] = (double)o.infil; acc[1] = (double)o.fix;
    if (hits) acc[4] = (double)o.h;
    // boundary faces: x-edges split per face (kernel.rs:435-450), y-edges summed first
    if (gx == 0) { double v = (double)w.m * dt_dy; if (v > 0.0) acc[2] += v; else acc[3] -= v; }
    if (gx == nx - 1) { double v = (double)e.m * dt_dy; if (v > 0.0) acc[3] += v; else acc[2] -= v; }
    if (gy == 0) yedge[0][lx] = (double)n.m;
    if (gy == ny - 1) yedge[1][lx] = (double)s.m;
  }
  // block reductions, fixed order
  float m = smax;
  for (int o = 16; o > 0; o >>= 1) m = rmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  unsigned b = __any_sync(0xffffffffu, bad) ? 1u : 0u;
  for (int j = 0; j < 5; ++j)
    for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
  const int wid = li >> 5;
  if ((li & 31) == 0) { wmax[wid] = m; wbad[wid] = b; for (int j = 0; j < 5; ++j) wsum[wid][j] = acc[j]; }
  __syncthreads();
  double yt = 0.0, yb = 0.0;   // the tile's top / bottom edge fluxes, summed by warp 0
  if (li < 32) {
    yt = li < kTile ? yedge[0][li] : 0.0;
    yb = li < kTile ? yedge[1][li] : 0.0;
    for (int o = kTile / 2; o > 0; o >>= 1) {
      yt += __shfl_xor_sync(0xffffffffu, yt, o);
      yb += __shfl_xor_sync(0xffffffffu, yb, o);
    }
  }
  if (li == 0) {
    float mm = 0.0f; unsigned bb = 0u; double ss[5] = {0, 0, 0, 0, 0};
    for (int w = 0; w < kTileThreads / 32; ++w) { mm = rmax(mm, wmax[w]); bb |= wbad[w]; for (int j = 0; j < 5; ++j) ss[j] += wsum[w][j]; }
    if (mm > 0.0f) atomicMax(&D.ctl->smax_bits, __float_as_uint(mm));
    if (bb) atomicOr(&D.ctl->bad, 1u);
    double* p = D.part + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * kPart;
    for (int j = 0; j < 5; ++j) p[j] = ss[j];
    p[5] = yt; p[6] = yb;
  }
}

// Threads per design of the step finalize (any multiple of 32 up to 1024 works).
constexpr int kFinThreads = 256;

// Advance the integrator after a step (or plan the first step when `first`). Launched with
// a block of warps per design: all of them sum the tile partials (one warp alone waits on
// hundreds of dependent rounds of loads for a large grid), warp 0 does the rest.
// LOCKED: the baseline-locked dt (solver.rs:436-483): each step takes the schedule's dt while
// dt * smax of the current state stays within cfl_hard; at the first step where it would not
// (or the schedule has run out) the control block goes back to the last sync snapshot, which
// the next k_plain_locked_copy completes with the state planes, and the run continues with the
// adaptive dt. Snapshots: at the start and after every sync's abort tests.
template <bool LOCKED>
ITR_DEV void plain_finalize_body(const PlainArgs& A, int n_blocks, int first) {
  __shared__ double red[32][kPart];
  const PlainDesign D = plain_design(A, blockIdx.x, n_blocks);
  PlainCtl& c = *D.ctl;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const RunParams& P = A.P;
  if constexpr (LOCKED) { if (threadIdx.x == 0) c.copy_req = 0; }   // the last request has been served
  if (c.done) return;
  if (!first && D.rowwet) {
    // dry rows the step just skipped (k_band's predicate on the flags it read: the state of
    // parity c.par, not yet flipped), then clear those flags: the next step writes them
    __shared__ unsigned s_skip;
    if (threadIdx.x == 0) s_skip = 0u;
    __syncthreads();
    const int R = A.ny + 2;
    unsigned* rw = D.rowwet + (size_t)c.par * R;
    if (P.skip_dry && !(c.k.rain > 0.0f)) {
      unsigned cnt = 0u;
      for (int j = 1 + threadIdx.x; j <= A.ny; j += blockDim.x)
        cnt += (plain_row_dry(rw, D.gwet, j - 1) && plain_row_dry(rw, D.gwet, j) && plain_row_dry(rw, D.gwet, j + 1)) ? 1u : 0u;
      if (cnt) atomicAdd(&s_skip, cnt);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < R; j += blockDim.x) rw[j] = 0u;
    if (threadIdx.x == 0) c.rows_skipped += s_skip;
  }
  double tot[kPart] = {0, 0, 0, 0, 0, 0, 0};
  if (!first) {
    for (int b = threadIdx.x; b < n_blocks; b += blockDim.x)
      for (int j = 0; j < kPart; ++j) tot[j] += D.part[(size_t)b * kPart + j];
    for (int j = 0; j < kPart; ++j)
      for (int o = 16; o > 0; o >>= 1) tot[j] += __shfl_xor_sync(0xffffffffu, tot[j], o);
    if (nw > 1) {
      if (lane == 0)
        for (int j = 0; j < kPart; ++j) red[wid][j] = tot[j];
      __syncthreads();
      for (int j = 0; j < kPart; ++j) {
        tot[j] = lane < nw ? red[lane][j] : 0.0;
        for (int o = 16; o > 0; o >>= 1) tot[j] += __shfl_xor_sync(0xffffffffu, tot[j], o);
      }
    }
  }
  if (wid != 0) return;
  if (!first) {
    {   // y_boundary (kernel.rs:452-472): the top edge is inflow when its net flux is > 0,
        // the bottom edge outflow
      const double dt_dx = c.pl.dt * P.dx;
      const double vt = tot[5] * dt_dx, vb = tot[6] * dt_dx;
      if (vt > 0.0) tot[2] += vt; else tot[3] -= vt;
      if (vb > 0.0) tot[3] += vb; else tot[2] -= vb;
    }
    const double smax = (double)__uint_as_float(c.smax_bits);
    const unsigned badv = c.bad;
    __syncwarp();
    if (lane == 0) {
      c.tot_infil += tot[0]; c.tot_fix += tot[1]; c.tot_in += tot[2]; c.tot_out += tot[3];
      c.smax_bits = 0u;
      c.step += 1;
      c.t = c.pl.t_new;
      c.acc_rain += c.pl.rain * P.area * P.wet_count;
      c.par ^= 1;
    }
    __syncwarp();
    if (badv) { if (lane == 0) { c.status = 3; c.done = 1; } return; }
    if (lane == 0) c.dt_cfl = smax > 0.0 ? P.cfl / smax : P.dt_max;
    if constexpr (LOCKED) { if (lane == 0) c.s_cur = smax; }
    __syncwarp();
    if (c.pl.hits) {
      int decision = 0;
      if (lane == 0) {
        c.sync_index += 1;
        const double v = tot[4] * P.area, infil = c.tot_infil * P.area, fix = c.tot_fix * P.area;
        const double expected = c.v0 + c.acc_rain + c.tot_in - c.tot_out - infil + fix;
        c.volume = v;
        const double gross = c.v0 + c.acc_rain + c.tot_in;
        c.rel_res = fabs(v - expected) / (gross > 1e-300 ? gross : 1e-300);
        if (c.n_rows < A.max_rows && D.ledger) {
          double* o = D.ledger + (size_t)c.n_rows * 8;
          o[0] = c.t; o[1] = v; o[2] = c.acc_rain; o[3] = c.tot_in; o[4] = c.tot_out; o[5] = infil; o[6] = fix; o[7] = v - expected;
        }
        c.n_rows += 1;
        const DevObjective& ob = A.obj;
        if (ob.enabled) {
          if (ob.guard_abort && ob.require && ob.baseline) {
            double best = 0.0; int bk = -1;
            for (int g = 0; g < ob.n_guard; ++g) {
              int mp = ob.guard_pos[g];
              double w = (double)D.PK[A.mon_cells[mp]] - ob.baseline[mp] - ob.tol;
              if (w > 0.0 && (bk < 0 || w > best)) { best = w; bk = g; }
            }
            if (bk >= 0) {
              decision = 1;
              c.breach_cell = A.mon_cells[ob.guard_pos[bk]]; c.breach_sync = c.sync_index; c.violation = best;
            }
          }
          if (decision == 0 && ob.has_incumbent) {
            double jr = 0.0;
            for (int a = 0; a < ob.n_assets; ++a) {
              double pk = 0.0;
              for (int m = ob.asset_off[a]; m < ob.asset_off[a + 1]; ++m) {
                double x = (double)D.PK[A.mon_cells[ob.asset_pos[m]]];
                pk = pk > x ? pk : x;
              }
              jr += ob.asset_w[a] * ob.tau * itr_math::softplus((pk - ob.asset_thr[a]) / ob.tau);
            }
            const double lb = jr + ob.earth_w * (ob.cut_cost * D.cut + ob.fill_cost * D.fill);
            if (lb >= ob.incumbent) { decision = 2; c.lower_bound = lb; }
          }
        }
        if (decision) { c.status = decision; c.done = 1; }
      }
      __syncwarp();
      if (c.done) return;
      if constexpr (LOCKED) {   // sync snapshot (solver.rs:611-614)
        if (lane == 0 && c.locked_live) { A.snapctl[blockIdx.x] = c; c.copy_req = 1; }
        __syncwarp();
      }
    }
  }
  if constexpr (LOCKED) {
    if (lane == 0) {
      if (first) {   // the snapshot at the start (solver.rs:444-447)
        c.locked_live = 1;
        A.fallback_t[blockIdx.x] = -1.0;
        A.snapctl[blockIdx.x] = c;
        c.copy_req = 1;
      }
      if (!(c.t < P.duration && c.sync_index < P.n_sync)) {
        c.done = 1;
      } else if (c.step >= A.max_steps) {
        c.status = 4; c.done = 1;
      } else if (c.locked_live && !(c.step < A.n_locked && A.locked_dt[c.step] * c.s_cur <= A.cfl_hard)) {
        // back to the last sync snapshot, adaptive from here on. A snapshot taken by this very
        // finalize (save still pending) is the current state: nothing to copy back.
        const int pending_save = c.copy_req;
        c = A.snapctl[blockIdx.x];
        c.locked_live = 0;
        c.copy_req = pending_save == 1 ? 0 : 2;
        A.fallback_t[blockIdx.x] = c.t;
      }
    }
    __syncwarp();
    if (c.done) return;
    if (lane < P.inflow.n) c.inf[lane] = inflow_values(P.inflow, lane, c.t, P.g);
    __syncwarp();
    if (D.gwet) plain_ghost_wet(A, D.bh, c.inf, D.gwet, lane);
    if (lane == 0) {
      const double dt = c.locked_live ? A.locked_dt[c.step] : dmin_num(c.dt_cfl, P.dt_max);
      c.pl = plan_step_dt(P, c.t, c.sync_index, dt);
      c.k = step_consts(P, c.pl.dt, c.pl.rain);
    }
    return;
  }
  // inflow ghosts of the next step, at its start time c.t (fill_ghosts(t), solver.rs), and
  // the ghost wetness the row-band kernel's dry-row test reads
  if (lane < P.inflow.n) c.inf[lane] = inflow_values(P.inflow, lane, c.t, P.g);
  __syncwarp();
  if (D.gwet) plain_ghost_wet(A, D.bh, c.inf, D.gwet, lane);
  if (lane == 0) {
    if (!(c.t < P.duration && c.sync_index < P.n_sync)) { c.done = 1; return; }
    if (c.step >= A.max_steps) { c.status = 4; c.done = 1; return; }
    c.pl = plan_step(P, c.t, c.sync_index, c.dt_cfl);
    if (D.dt_log) {   // ring of max_log entries, slot step mod max_log
      const size_t slot = (size_t)(c.step % (unsigned long long)A.max_log);
      D.dt_log[3 * slot] = c.pl.dt; D.dt_log[3 * slot + 1] = c.pl.rain; D.dt_log[3 * slot + 2] = c.t;
    }
    c.k = step_consts(P, c.pl.dt, c.pl.rain);
  }
}

__global__ void k_plain_finalize(const PlainArgs A, int n_blocks, int first) { plain_finalize_body<false>(A, n_blocks, first); }
__global__ void k_plain_finalize_locked(const PlainArgs A, int n_blocks, int first) {
  plain_finalize_body<true>(A, n_blocks, first);
}

// Baseline-locked dt: after a finalize that asked for it, copy each design's current state
// plane and peaks into its sync snapshot (copy_req 1) or back from it (copy_req 2). A grid of
// (blocks, designs); the control block is read only, so every block sees the same request.
__global__ void k_plain_locked_copy(const PlainArgs A) {
  const int d = blockIdx.y;
  const PlainDesign D = plain_design(A, d, 0);
  const PlainCtl& c = *D.ctl;
  const int req = c.copy_req;
  if (c.done || req == 0) return;
  const size_t N = (size_t)A.nx * A.ny, pl = (size_t)c.par * N;
  float* s = A.snap + (size_t)d * 4 * N;
  if (D.rowwet && blockIdx.x == 0) {   // the dry-row flags of the state (k_band's skipping)
    const int R = A.ny + 2;
    for (int j = threadIdx.x; j < R; j += blockDim.x) {
      if (req == 1) {
        D.snaprow[j] = D.rowwet[(size_t)c.par * R + j];
      } else {
        D.rowwet[(size_t)c.par * R + j] = D.snaprow[j];
        D.rowwet[(size_t)(c.par ^ 1) * R + j] = 0u;
      }
    }
  }
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
    if (req == 1) {
      s[i] = D.H[pl + i]; s[N + i] = D.QX[pl + i]; s[2 * N + i] = D.QY[pl + i]; s[3 * N + i] = D.PK[i];
    } else {
      D.H[pl + i] = s[i]; D.QX[pl + i] = s[N + i]; D.QY[pl + i] = s[2 * N + i]; D.PK[i] = s[3 * N + i];
    }
  }
}

// Initial state and the first dt (solver.rs:381-390), or a warm start's checkpoint.
__global__ void k_plain_init(const PlainArgs A) {
  const PlainDesign D = plain_design(A, blockIdx.x, 0);
  const int nx = A.nx, ny = A.ny, n = nx * ny;
  const RunParams& P = A.P;
  const WarmStart* W = (A.warm && A.warm[blockIdx.x].state) ? &A.warm[blockIdx.x] : nullptr;
  // dry-row flags of the initial state (init_state: a row is dry when all its depths are 0)
  if (D.rowwet) {
    for (int j = threadIdx.x; j < 2 * (ny + 2); j += blockDim.x) D.rowwet[j] = 0u;
    __syncthreads();
  }
  if (W) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      D.H[i] = W->state[i]; D.QX[i] = W->state[n + i]; D.QY[i] = W->state[2 * n + i]; D.PK[i] = W->state[3 * n + i];
      if (D.tpk) D.tpk[i] = 0u;
      if (D.rowwet && W->state[i] != 0.0f) D.rowwet[1 + i / nx] = 1u;
    }
    if (threadIdx.x == 0) {
      PlainCtl c;
      memset(&c, 0, sizeof(c));
      c.t = W->t; c.dt_cfl = W->dt_cfl; c.acc_rain = W->acc_rain; c.v0 = W->v0; c.volume = W->volume; c.rel_res = W->rel_res;
      c.tot_infil = W->tot_infil; c.tot_fix = W->tot_fix; c.tot_in = W->tot_in; c.tot_out = W->tot_out;
      c.step = W->step; c.sync_index = W->sync_index; c.n_rows = W->n_rows;
      *D.ctl = c;
    }
    return;
  }
  __shared__ double ss[32], sv[32];
  double s0 = 0.0, v0 = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    float h = D.h0[i];
    D.H[i] = h; D.QX[i] = 0.0f; D.QY[i] = 0.0f; D.PK[i] = 0.0f;
    if (D.tpk) D.tpk[i] = 0u;
    if (D.rowwet && h != 0.0f) D.rowwet[1 + i / nx] = 1u;
    double hd = (double)h;
    v0 += hd;
    if (hd > P.h_dry) {
      double cd = sqrt(P.g * hd);
      double r = (0.0 / hd + cd) / P.dx + (0.0 / hd + cd) / P.dy;
      s0 = s0 > r ? s0 : r;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    double a = __shfl_xor_sync(0xffffffffu, s0, o); s0 = s0 > a ? s0 : a;
    v0 += __shfl_xor_sync(0xffffffffu, v0, o);
  }
  if ((threadIdx.x & 31) == 0) { ss[threadIdx.x >> 5] = s0; sv[threadIdx.x >> 5] = v0; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0, v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { s = s > ss[w] ? s : ss[w]; v += sv[w]; }
    PlainCtl c;
    memset(&c, 0, sizeof(c));
    c.v0 = v * P.area; c.volume = c.v0;
    c.dt_cfl = s > 0.0 ? dmin_num(P.cfl / s, P.dt_max) : P.dt_max;
    c.s_cur = s;
    *D.ctl = c;
  }
}

// Baseline record (one design): the current state plane and running peaks into dst [4][N].
__global__ void k_rec_state(const PlainArgs A, float* dst) {
  const PlainDesign D = plain_design(A, 0, 0);
  const size_t N = (size_t)A.nx * A.ny;
  const int par = D.ctl->par;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
    dst[i] = D.H[par * N + i]; dst[N + i] = D.QX[par * N + i]; dst[2 * N + i] = D.QY[par * N + i]; dst[3 * N + i] = D.PK[i];
  }
}

// Whether row blockIdx.x has held water in any state so far: initial depth or running peak
// above 0 in any of its cells (the peak plane is state [3] of a record checkpoint).
__global__ void k_rec_rows(const PlainArgs A, const float* state, uint8_t* wet) {
  const int r = blockIdx.x, nx = A.nx;
  const size_t N = (size_t)A.nx * A.ny;
  const PlainDesign D = plain_design(A, 0, 0);
  int any = 0;
  for (int c = threadIdx.x; c < nx; c += blockDim.x) {
    const size_t i = (size_t)r * nx + c;
    any |= (D.h0[i] > 0.0f || state[3 * N + i] > 0.0f) ? 1 : 0;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) wet[r] = any ? 1 : 0;
}

// Per-design results of a tiled batched run: the scalar outcome from the control block and
// the final depth (the plane the last step wrote).
__global__ void k_plain_outputs(const PlainArgs A, int n_tiles, DesignOut* out, float* depth) {
  const PlainDesign D = plain_design(A, blockIdx.x, n_tiles);
  const PlainCtl& c = *D.ctl;
  const size_t N = (size_t)A.nx * A.ny;
  const float* H = D.H + (size_t)c.par * N;
  for (size_t i = threadIdx.x; i < N; i += blockDim.x) depth[blockIdx.x * N + i] = H[i];
  if (threadIdx.x == 0) {
    DesignOut o;
    memset(&o, 0, sizeof(o));
    o.steps = c.step; o.t_end = c.t; o.sync_count = c.sync_index; o.status = c.status;
    o.breach_cell = c.breach_cell; o.breach_sync = c.breach_sync; o.violation = c.violation;
    o.lower_bound = c.lower_bound; o.v0 = c.v0; o.volume = c.volume; o.rel_residual = c.rel_res; o.n_rows = c.n_rows;
    o.rows_skipped = c.rows_skipped;
    out[blockIdx.x] = o;
  }
}

}  // namespace itr
