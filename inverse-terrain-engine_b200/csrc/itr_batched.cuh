// itr_batched.cuh — the batched forward operator: one design per thread-block cluster.
//
// Replaces the reference's per-step `update` + `finalize` dispatch pair and its 64-step host
// polling (crates/itr-gpu/src/shader.wgsl:135-365, crates/itr-gpu/src/lib.rs:302-328) with a
// single persistent launch over the whole population: every cluster owns one design for the
// whole simulated storm and never leaves the SM between steps.
//
// Layout on chip. The design's rows are split into bands, one per CTA of the cluster; a band
// lives in shared memory, 28 B/cell: float4 (h, qx, qy, u), float2 (v, c) and the running
// peak depth, so the state never goes back to HBM until the run ends. Inside a CTA the band
// is cut into S strips; each strip is swept row by row by W warps, every lane holding two
// columns, c and c + 32W (W = ceil((nx+1)/64)), whose faces and cell updates run as paired
// FP32 instructions (itr_device.cuh, face2 / update_cell2). It is the in-place row sweep of
// the reference's fused kernel (crates/itr-hydro/src/kernel.rs:637-697):
//   * the north y-face of a row is carried in registers from the row above,
//   * the west x-face of the next row is computed one row early; the east face is the
//     west face of lane+1 (shuffle; lane 31 reads lane 0 of the next warp, or the second
//     column of warp 0, through shared memory),
//   * velocities (u, v) and celerity c are stored with the state when a cell is updated, so
//     each is computed once per cell-step (c is the sources' sqrt(g*h)),
//   * the y-face between two strips (and between two CTAs) is computed at the start of the
//     step from the old state, the reference's strip pre-phase (kernel.rs:614-622).
// Synchronisation per step: one named barrier per strip per row, one split cluster barrier
// (arrive after the strip pre-phase, wait before a strip's last row), one full cluster
// barrier for the CFL reduction. The CFL max and the health flag are reduced by warp
// shuffles, a shared-memory atomic per warp, and a DSMEM read of every CTA's slot. The f64
// time integrator (dt rule, sync clipping, exact rain integral, solver.rs:449-489) runs in
// every thread redundantly on identical inputs, so no broadcast is needed.
//
// Ledgers: per-step f32 warp partials of infiltration and positivity fix and the per-face
// boundary mass fluxes go to shared memory; one warp folds them into f64 running totals in a
// fixed order. At sync points the volume, the ledger row, the guard test (objective.rs:
// 130-145) and the incumbent lower bound (objective.rs:146-149) are evaluated on the device,
// so an aborted design stops at once.
#pragma once
#include <cooperative_groups.h>
#include "itr_device.cuh"

namespace itr {
namespace cg = cooperative_groups;


// Scalars of one CTA at a sync snapshot of a baseline-locked run (the Checkpoint of
// solver.rs:78-92 that the fallback restores): the integrator, which is the same in every
// CTA of a design, and this CTA's f64 ledger totals.
struct LockedSnap {
  double t, dt_cfl, s_cur, acc_rain, volume, rel_res;
  double led[4];
  unsigned long long step;
  unsigned sync_index;
  int n_rows;
};

struct BatchArgs {
  RunParams P;
  int nx, ny, mode;
  int C;          // CTAs per design (cluster size)
  int W, S;       // warps per strip row, strips per CTA
  int n_designs;
  const float* wet;   // nx*ny
  const float* gn2;   // nx*ny
  const uint8_t* bc;  // north[nx], south[nx], west[ny], east[ny]; device codes (ghost_state)
  const float* bh;    // stage-ghost depths, n_designs * [2 nx + 2 ny] indexed like bc, or NULL
  const float* dzx;   // n_designs * ny*(nx+1)
  const float* dzy;   // n_designs * (ny+1)*nx
  const float* dzx2;  // crest only
  const float* dzy2;
  const float* h0;    // n_designs * nx*ny
  const double* cut;  // n_designs
  const double* fill; // n_designs
  int n_mon;
  const unsigned* mon_cells;
  DevObjective obj;
  float* peak_out;    // n_designs * nx*ny
  float* depth_out;   // n_designs * nx*ny
  double* ledger_out; // n_designs * max_rows * 8
  int max_rows;
  DesignOut* out;     // n_designs
  unsigned long long max_steps;
  unsigned exact;     // 1: every paired reciprocal through the IEEE routine (checking)
  unsigned wait_limit;   // try_wait rounds of a single-CTA design's barrier wait before status 5
  unsigned stall_test;   // 1: that barrier expects one arrival more than the CTA makes (timeout test)
  const WarmStart* warm;   // optional, per design (state NULL: cold start)
  // Baseline-locked dt (SolverParams::locked_dt / cfl_hard, solver.rs:42-46); read only by the
  // LOCKED instantiation, which is launched when locked_dt is set.
  const double* locked_dt;   // n_locked dts of the baseline, shared by every design
  unsigned long long n_locked;
  double cfl_hard;
  float4* snap4;             // sync snapshot of the state, n_designs * nx*ny (h, qx, qy, u)
  float2* snap2;             //                                              (v, c)
  float* snapk;              //                              running peaks
  LockedSnap* snap_s;        // n_designs * C records
  double* fallback_t;        // n_designs: time the run fell back to adaptive dt, -1 for none
};

__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

ITR_DEV unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Shared-memory plan of one CTA. Every CTA of a cluster uses the plan of the largest band,
// so an offset names the same array in every CTA (DSMEM maps local pointers to peers).
struct SmemPlan {
  size_t s4, s2, pk, bf, xb, bx, by, wsum, led, slot, red, mbar, inf, pf, wf, gwf, nsk, total;
};

// Values staged per thread and row by the prefetch ring: south y-face jump, next row's
// x-face jump, wet, g n^2 (+ the second jumps in crest mode).
__host__ __device__ inline int prefetch_k(int crest) { return crest ? 6 : 4; }

__host__ __device__ inline SmemPlan smem_plan(int nr_max, int nx, int S, int W, int nwarps, int crest = 0, int bnd = 0,
                                               int ny = 0) {
  SmemPlan p;
  size_t n = (size_t)nr_max * nx, o = 0;
  p.s4 = o;   o += n * 16;                         // float4 h, qx, qy, u
  p.s2 = o;   o += n * 8;                          // float2 v, c
  p.pk = o;   o += n * 4;                          // peak depth
  o = align_up(o, 16);
  p.bf = o;   o += (size_t)(S + 1) * nx * 16;      // float4 strip-top y-faces
  p.xb = o;   o += (size_t)2 * S * W * 2 * 16;     // float4 lane-0 x-face exchange [2][S][W][2]
  p.bx = o;   o += (size_t)2 * 2 * nr_max * 4;     // west/east boundary mass flux [2][2][nr]
  p.by = o;   o += (size_t)2 * 2 * nx * 4;         // top/bottom boundary mass flux [2][2][nx]
  o = align_up(o, 16);
  p.wsum = o; o += (size_t)2 * nwarps * 2 * 4;     // per-warp f32 step sums [2][nwarps][2]
  o = align_up(o, 16);
  p.led = o;  o += 8 * 8;                          // f64 running totals: infil, fix, in, out
  p.slot = o; o += 8 * 4;                          // smax bits [2], bad [2]
  o = align_up(o, 16);
  p.red = o;  o += (size_t)nwarps * 8 * 8;         // f64 reductions at sync points
  p.mbar = o; o += 16;
  p.inf = o;  o += bnd ? (size_t)2 * kMaxInflow * 8 : 0;   // float2 inflow values [2 parity][groups]
  o = align_up(o, 16);
  p.pf = o;   o += (size_t)2 * S * prefetch_k(crest) * 64 * W * 4;   // [2 slot][S][K][64W] floats
  p.wf = o;   o += (size_t)2 * nr_max * W;           // row wetness bytes [2 parity][nr_max][W]
  p.gwf = o;  o += bnd ? (size_t)2 * (ny + 2) : 0;    // ghost wetness [2 parity][ny + 2 padded rows]
  o = align_up(o, 8);
  p.nsk = o;  o += 8;                                 // rows skipped by this CTA
  p.total = align_up(o, 16);
  return p;
}

__host__ __device__ inline size_t batched_smem_bytes(int nr_max, int nx, int S, int W, int nwarps, int crest = 0, int bnd = 0,
                                                     int ny = 0) {
  return smem_plan(nr_max, nx, S, W, nwarps, crest, bnd, ny).total;
}

// 4-byte asynchronous global->shared copy (cp.async, cached in L1), commit and wait.
ITR_DEV void cp_async4(float* smem_dst, const float* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(smem_dst)), "l"(gsrc) : "memory");
}
ITR_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> ITR_DEV void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

ITR_DEV void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

ITR_DEV void cluster_arrive() { asm volatile("barrier.cluster.arrive.release;" ::: "memory"); }
ITR_DEV void cluster_wait() { asm volatile("barrier.cluster.wait.acquire;" ::: "memory"); }

ITR_DEV void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
ITR_DEV void mbar_arrive(unsigned long long* bar) {
  asm volatile("{ .reg .b64 st; mbarrier.arrive.release.cta.shared::cta.b64 st, [%0]; }" ::"r"(smem_u32(bar)) : "memory");
}
// Bounded wait on phase `parity`: at most `limit` try_wait rounds; returns false if the
// bound ran out.
ITR_DEV bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned limit) {
  for (unsigned it = 0; it < limit; ++it) {
    unsigned ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Self-checking build (-DITR_CHECKED): every shared, distributed-shared and global index
// is checked against its array; the first violation is recorded in g_itr_err (code, index,
// block, thread) and the access is redirected to element 0 instead of faulting.
#ifdef ITR_CHECKED
__device__ unsigned long long g_itr_err[4];
ITR_DEV long long chk(long long i, long long lim, int code) {
  if (i < 0 || i >= lim) {
    if (atomicCAS(&g_itr_err[0], 0ull, (unsigned long long)code) == 0ull) {
      g_itr_err[1] = (unsigned long long)i; g_itr_err[2] = blockIdx.x; g_itr_err[3] = threadIdx.x;
    }
    return 0;
  }
  return i;
}
#define CK(i, lim, code) ((int)chk((long long)(i), (long long)(lim), (code)))
#else
#define CK(i, lim, code) (i)
#endif

// A cell's stored state (old values during a step).
struct Cell { float h, qx, qy, u, v, c; };

struct Smem {
  float4* S4;      // (h, qx, qy, u)
  float2* S2;      // (v, c)
  float* PK;
  float4* BF;      // strip boundary y-faces (m, nl, nr, t)
  float4* XB;
  float* BX;       // [2 parity][2 side][nr_max]
  float* BY;       // [2 parity][2 side][nx]
  float* WS;       // [2 parity][nwarps][2]
  double* LED;     // [4]
  unsigned* slot;  // [2] smax bits, [2] bad
  double* red;     // [nwarps][8]
  unsigned long long* mbar;
  float2* INF;     // inflow group values [2 parity][kMaxInflow] (stage/inflow grids only)
  float* PF;       // prefetch ring, [2 slot][S][K][64W]
  uint8_t* WF;     // [2 parity][nr_max][W]: the warp's columns of the row held water (state of that parity)
  uint8_t* GWF;    // [2 parity][ny + 2]: a stage / inflow ghost of padded row j holds water (BND)
  unsigned long long* NSK;
  int ncell, nbf, nxb;
};

ITR_DEV Cell load_cell(const Smem& s, int idx) {
  idx = CK(idx, s.ncell, 1);
  const float4 a = s.S4[idx];
  const float2 b = s.S2[idx];
  Cell c;
  c.h = a.x; c.qx = a.y; c.qy = a.z; c.u = a.w; c.v = b.x; c.c = b.y;
  return c;
}

// Ghost cells (boundary.rs:36-87) from the interior cell c behind them: a wall mirrors the
// normal momentum (so the normal velocity flips sign exactly), a transmissive edge copies
// the cell. BND (the grid has stage or inflow cells): a stage or inflow ghost takes its
// state from ghost_state and its velocities and celerity from cell_vel, as every padded
// cell's do in the reference's velocity pass. NX: across an x-normal face; pos: index in
// bc / bh; inward_pos: west or north side.
template <bool BND, bool NX>
ITR_DEV Cell ghost_cell(Cell c, int code, const float* bh, int pos, const float2* inf, bool inward_pos, float g,
                        float heps2) {
  if (!BND || code < 2) {
    if (code == 0) {
      if (NX) { c.qx = -c.qx; c.u = -c.u; } else { c.qy = -c.qy; c.v = -c.v; }
    }
    return c;
  }
  const float hs = code == 2 ? bh[pos] : 0.0f;
  const float2 fi = code >= 3 ? inf[code - 3] : make_float2(0.0f, 0.0f);
  ghost_state<NX>(code, c.h, c.qx, c.qy, hs, fi, inward_pos);
  cell_vel(c.h, c.qx, c.qy, g, heps2, c.u, c.v, c.c);
  return c;
}

ITR_DEV Cell shfl_up_cell(Cell c) {
  Cell o;
  o.h = __shfl_up_sync(0xffffffffu, c.h, 1);
  o.qx = 0.0f; o.qy = 0.0f;
  o.u = __shfl_up_sync(0xffffffffu, c.u, 1);
  o.v = __shfl_up_sync(0xffffffffu, c.v, 1);
  o.c = __shfl_up_sync(0xffffffffu, c.c, 1);
  return o;
}
ITR_DEV FaceF shfl_down_face(FaceF f) {
  FaceF o;
  o.m = __shfl_down_sync(0xffffffffu, f.m, 1);
  o.nl = __shfl_down_sync(0xffffffffu, f.nl, 1);
  o.nr = __shfl_down_sync(0xffffffffu, f.nr, 1);
  o.t = __shfl_down_sync(0xffffffffu, f.t, 1);
  return o;
}
ITR_DEV float4 f4(const FaceF& f) { return make_float4(f.m, f.nl, f.nr, f.t); }
ITR_DEV FaceF ff(const float4& v) { FaceF f; f.m = v.x; f.nl = v.y; f.nr = v.z; f.t = v.w; return f; }

// Per-thread views of the inputs at this thread's column: row r of x-face jumps is
// dzx[r * (nx + 1)], y-face f is dzy[f * nx], cell (r, col) of wet/gn2 is wet[r * nx].
struct Col {
  const float* dzx;
  const float* dzy;
  const float* dzx2;
  const float* dzy2;
  const float* wet;
  const float* gn2;
  long long off_x, off_y, lim_x, lim_y;   // bounds (checked build)
};

template <bool CREST>
ITR_DEV FaceF xface(const Cell& l, const Cell& r, const Col& cp, int row, int nxp1, const StepK& k) {
  const int o = CK(row * nxp1, cp.lim_x - cp.off_x, 2);
  const float d0 = __ldg(cp.dzx + o);
  const float d1 = CREST ? __ldg(cp.dzx2 + o) : 0.0f;
  return face<true, CREST>(l.h, l.u, l.v, l.c, r.h, r.u, r.v, r.c, d0, d1, k);
}
template <bool CREST>
ITR_DEV FaceF yface(const Cell& t, const Cell& b, const Col& cp, int f, int nx, const StepK& k) {
  const int o = CK(f * nx, cp.lim_y - cp.off_y, 3);
  const float d0 = __ldg(cp.dzy + o);
  const float d1 = CREST ? __ldg(cp.dzy2 + o) : 0.0f;
  return face<false, CREST>(t.h, t.u, t.v, t.c, b.h, b.u, b.v, b.c, d0, d1, k);
}

ITR_DEV double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
ITR_DEV float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
ITR_DEV float warp_max_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = rmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <bool CLUSTERED>
struct GroupSync {
  unsigned long long* mbar;
  unsigned phase;
  unsigned limit;
  bool timed_out;
  ITR_DEV void b1_arrive() {
    if (CLUSTERED) cluster_arrive(); else mbar_arrive(mbar);
  }
  ITR_DEV void b1_wait() {
    if (CLUSTERED) cluster_wait();
    else { if (!mbar_wait(mbar, phase & 1u, limit)) timed_out = true; }
  }
  ITR_DEV void b1_done() { phase += 1; }
  ITR_DEV void full() {
    if (CLUSTERED) { cluster_arrive(); cluster_wait(); } else __syncthreads();
  }
};

// Map a pointer into shared memory to the same offset in CTA `rank` of the cluster.
template <class T> ITR_DEV T* remote(T* p, int rank) {
  return cg::this_cluster().map_shared_rank(p, (unsigned)rank);
}

// Two cells of a lane: column c (component x) and column c + 32W (component y).
struct Cell2 { float2 h, qx, qy, u, v, c; };

ITR_DEV Cell2 cell2_of(const Cell& a, const Cell& b) {
  Cell2 r;
  r.h = make_float2(a.h, b.h); r.qx = make_float2(a.qx, b.qx); r.qy = make_float2(a.qy, b.qy);
  r.u = make_float2(a.u, b.u); r.v = make_float2(a.v, b.v); r.c = make_float2(a.c, b.c);
  return r;
}
ITR_DEV Cell cx(const Cell2& a) { Cell c; c.h = a.h.x; c.qx = a.qx.x; c.qy = a.qy.x; c.u = a.u.x; c.v = a.v.x; c.c = a.c.x; return c; }
ITR_DEV Cell cy(const Cell2& a) { Cell c; c.h = a.h.y; c.qx = a.qx.y; c.qy = a.qy.y; c.u = a.u.y; c.v = a.v.y; c.c = a.c.y; return c; }
ITR_DEV FaceF fx_(const Face2& f) { FaceF r; r.m = f.m.x; r.nl = f.nl.x; r.nr = f.nr.x; r.t = f.t.x; return r; }
ITR_DEV FaceF fy_(const Face2& f) { FaceF r; r.m = f.m.y; r.nl = f.nl.y; r.nr = f.nr.y; r.t = f.t.y; return r; }
ITR_DEV Face2 face2_of(const FaceF& a, const FaceF& b) {
  Face2 f;
  f.m = make_float2(a.m, b.m); f.nl = make_float2(a.nl, b.nl); f.nr = make_float2(a.nr, b.nr); f.t = make_float2(a.t, b.t);
  return f;
}
ITR_DEV Cell2 shfl_up_cell2(const Cell2& c) {
  Cell2 o;
  o.h = make_float2(__shfl_up_sync(0xffffffffu, c.h.x, 1), __shfl_up_sync(0xffffffffu, c.h.y, 1));
  o.qx = f2(0.0f); o.qy = f2(0.0f);
  o.u = make_float2(__shfl_up_sync(0xffffffffu, c.u.x, 1), __shfl_up_sync(0xffffffffu, c.u.y, 1));
  o.v = make_float2(__shfl_up_sync(0xffffffffu, c.v.x, 1), __shfl_up_sync(0xffffffffu, c.v.y, 1));
  o.c = make_float2(__shfl_up_sync(0xffffffffu, c.c.x, 1), __shfl_up_sync(0xffffffffu, c.c.y, 1));
  return o;
}
ITR_DEV Face2 shfl_down_face2(const Face2& f) {
  Face2 o;
  o.m = make_float2(__shfl_down_sync(0xffffffffu, f.m.x, 1), __shfl_down_sync(0xffffffffu, f.m.y, 1));
  o.nl = make_float2(__shfl_down_sync(0xffffffffu, f.nl.x, 1), __shfl_down_sync(0xffffffffu, f.nl.y, 1));
  o.nr = make_float2(__shfl_down_sync(0xffffffffu, f.nr.x, 1), __shfl_down_sync(0xffffffffu, f.nr.y, 1));
  o.t = make_float2(__shfl_down_sync(0xffffffffu, f.t.x, 1), __shfl_down_sync(0xffffffffu, f.t.y, 1));
  return o;
}

// Sync snapshot of one CTA of a baseline-locked run: its rows of the state and peaks (cells
// [0, ncell) of shared memory, global offset base) and, by thread 0, the integrator scalars and
// the CTA's ledger totals into record `rec`. Ends with a CTA barrier, so no thread writes the
// state of the next step before all of it is saved.
ITR_DEV void locked_save(const BatchArgs& A, const Smem& sm, size_t base, int ncell, size_t rec, double t, double dt_cfl,
                         double s_cur, double acc_rain, double volume, double rel_res, unsigned long long step,
                         unsigned sync_index, int n_rows) {
  for (int idx = threadIdx.x; idx < ncell; idx += blockDim.x) {
    A.snap4[base + idx] = sm.S4[idx]; A.snap2[base + idx] = sm.S2[idx]; A.snapk[base + idx] = sm.PK[idx];
  }
  if (threadIdx.x == 0) {
    LockedSnap& o = A.snap_s[rec];
    o.t = t; o.dt_cfl = dt_cfl; o.s_cur = s_cur; o.acc_rain = acc_rain; o.volume = volume; o.rel_res = rel_res;
    for (int j = 0; j < 4; ++j) o.led[j] = sm.LED[j];
    o.step = step; o.sync_index = sync_index; o.n_rows = n_rows;
  }
  __syncthreads();
}

// Row wetness flags of the CTA's rows from the state in shared memory (init_state's rule: a
// row is dry when every depth is 0), into parity slot `par`: warp-strided rows, entry 0 of a
// row holds the flag, the other W - 1 entries are cleared.
ITR_DEV void row_flags(const Smem& sm, int par, int nr, int nr_max, int nx, int W, int wid, int nwarps, int lane) {
  for (int lr = wid; lr < nr; lr += nwarps) {
    bool w = false;
    for (int c = lane; c < nx; c += 32) w = w || sm.S4[lr * nx + c].x != 0.0f;
    w = __any_sync(0xffffffffu, w);
    uint8_t* e = sm.WF + ((size_t)par * nr_max + lr) * W;
    for (int k = lane; k < W; k += 32) e[k] = (k == 0 && w) ? 1 : 0;
  }
}

// SKIP: the dry-row test of rain-free steps (kernel.rs:605-612) and the row wetness flags it
// reads. The host launches the SKIP instantiation when params.skip_dry is set and the storm
// has a rain-free interval inside the run; every other run has no rain-free step, where the
// test never skips, and takes the instantiation without the bookkeeping (same results).
template <bool CREST, bool CLUSTERED, int MAXT, bool BND, bool LOCKED = false, bool SKIP = false>
__global__ void __launch_bounds__(MAXT, 1) k_batched(const BatchArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int C = A.C;
  const int q = CLUSTERED ? (int)cg::this_cluster().block_rank() : 0;
  const int d = blockIdx.x / C;
  if (d >= A.n_designs) return;   // whole clusters only (grid is a multiple of C)
  const int nx = A.nx, ny = A.ny;
  const int ra = (int)((long long)q * ny / C), rb = (int)((long long)(q + 1) * ny / C);
  const int nr = rb - ra;
  const int nr_max = (ny + C - 1) / C;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarps = blockDim.x >> 5;
  const int W = A.W, S = A.S;        // W warps per strip row, 64W columns per row
  const int s = wid / W, wis = wid % W;
  const int col0 = wis * 32 + lane, col1 = col0 + 32 * W;
  const bool in_strip = s < S;
  const bool cell0 = in_strip && col0 < nx, cell1 = in_strip && col1 < nx;
  const bool face0 = in_strip && col0 <= nx, face1 = in_strip && col1 <= nx;
  const bool any_face = face0 || face1;
  // strip rows (global row indices)
  const int r0 = in_strip ? ra + (int)((long long)s * nr / S) : rb;
  const int r1 = in_strip ? ra + (int)((long long)(s + 1) * nr / S) : rb;
  const int L = r1 - r0;

  Smem sm;
  {
    const SmemPlan pl = smem_plan(nr_max, nx, S, W, nwarps, CREST ? 1 : 0, BND ? 1 : 0, ny);
    sm.S4 = reinterpret_cast<float4*>(smem_raw + pl.s4);
    sm.S2 = reinterpret_cast<float2*>(smem_raw + pl.s2);
    sm.PK = reinterpret_cast<float*>(smem_raw + pl.pk);
    sm.BF = reinterpret_cast<float4*>(smem_raw + pl.bf);
    sm.XB = reinterpret_cast<float4*>(smem_raw + pl.xb);
    sm.BX = reinterpret_cast<float*>(smem_raw + pl.bx);
    sm.BY = reinterpret_cast<float*>(smem_raw + pl.by);
    sm.WS = reinterpret_cast<float*>(smem_raw + pl.wsum);
    sm.LED = reinterpret_cast<double*>(smem_raw + pl.led);
    sm.slot = reinterpret_cast<unsigned*>(smem_raw + pl.slot);
    sm.red = reinterpret_cast<double*>(smem_raw + pl.red);
    sm.mbar = reinterpret_cast<unsigned long long*>(smem_raw + pl.mbar);
    sm.INF = reinterpret_cast<float2*>(smem_raw + pl.inf);
    sm.PF = reinterpret_cast<float*>(smem_raw + pl.pf);
    sm.WF = reinterpret_cast<uint8_t*>(smem_raw + pl.wf);
    sm.GWF = reinterpret_cast<uint8_t*>(smem_raw + pl.gwf);
    sm.NSK = reinterpret_cast<unsigned long long*>(smem_raw + pl.nsk);
    sm.ncell = nr_max * nx; sm.nbf = (S + 1) * nx; sm.nxb = 2 * S * W * 2;
  }
  const RunParams& P = A.P;
  const size_t cell0_off = (size_t)d * nx * ny;
  const int nxp1 = nx + 1;
  // Per-thread input offsets of both columns (idle lanes point at a valid column, never
  // read): x-face jumps of (row r, col) at dzx[ox + r (nx+1)], y-face f at dzy[oy + f nx],
  // wet / g n^2 of (r, col) at wet[oc + r nx]. Offsets, not pointers, to save registers.
  const int cc0 = col0 <= nx ? col0 : nx, cc1 = col1 <= nx ? col1 : nx;
  const int oc0 = cc0 < nx ? cc0 : nx - 1, oc1 = cc1 < nx ? cc1 : nx - 1;
  const size_t ox0 = (size_t)d * ny * nxp1 + cc0, ox1 = (size_t)d * ny * nxp1 + cc1;
  const size_t oy0 = (size_t)d * (ny + 1) * nx + oc0, oy1 = (size_t)d * (ny + 1) * nx + oc1;
  const int bc_w = 2 * nx, bc_e = 2 * nx + ny, bc_n = 0, bc_s = nx, nbc = 2 * nx + 2 * ny;
  (void)nbc;   // used by the checked build's index checks
  const float* const bh = BND ? A.bh + (size_t)d * nbc : nullptr;   // this design's stage depths

  // Prefetch ring: row r's operands for this thread's two columns are copied one row ahead.
  constexpr int K = CREST ? 6 : 4;
  const int vlanes = 64 * W;
  float* const pf_base = sm.PF + (size_t)(s < S ? s : 0) * K * vlanes + col0;   // slot 0, column col0
  const size_t pf_slot = (size_t)S * K * vlanes;
  auto prefetch_row = [&](int r, int slot) {
    // dzy[r+1] (south face), dzx[r+1] (next row's west face; clamped in range for the last
    // row, where it is not used), wet and g n^2 of row r, for columns col0 and col1
    float* dst = pf_base + slot * pf_slot;
    const int rn = r + 1 < ny ? r + 1 : ny - 1;
    const size_t fy = (size_t)(r + 1) * nx, fx = (size_t)rn * nxp1, fc = (size_t)r * nx;
    if (face0) {
      cp_async4(dst + 0 * vlanes, A.dzy + oy0 + fy);
      cp_async4(dst + 1 * vlanes, A.dzx + ox0 + fx);
      cp_async4(dst + 2 * vlanes, A.wet + oc0 + fc);
      cp_async4(dst + 3 * vlanes, A.gn2 + oc0 + fc);
      if (CREST) {
        cp_async4(dst + 4 * vlanes, A.dzy2 + oy0 + fy);
        cp_async4(dst + 5 * vlanes, A.dzx2 + ox0 + fx);
      }
    }
    if (face1) {
      float* d1 = dst + 32 * W;
      cp_async4(d1 + 0 * vlanes, A.dzy + oy1 + fy);
      cp_async4(d1 + 1 * vlanes, A.dzx + ox1 + fx);
      cp_async4(d1 + 2 * vlanes, A.wet + oc1 + fc);
      cp_async4(d1 + 3 * vlanes, A.gn2 + oc1 + fc);
      if (CREST) {
        cp_async4(d1 + 4 * vlanes, A.dzy2 + oy1 + fy);
        cp_async4(d1 + 5 * vlanes, A.dzx2 + ox1 + fx);
      }
    }
  };

  // ---------------------------------------------------------------- initial state ----
  // (or a warm start: the baseline's state, peaks and integrator at a checkpoint)
  const WarmStart* WS = (A.warm && A.warm[d].state) ? &A.warm[d] : nullptr;
  const double t_start = WS ? WS->t : 0.0;
  double s0_l = 0.0, v0_l = 0.0;
  for (int idx = tid; idx < nr * nx; idx += blockDim.x) {
    const int r = ra + idx / nx, c = idx % nx;
    if (WS) {
      const size_t i = (size_t)r * nx + c, NN = (size_t)nx * ny;
      const float h = WS->state[i], qx = WS->state[NN + i], qy = WS->state[2 * NN + i];
      float u, v, cc;
      cell_vel(h, qx, qy, P.g_f, P.heps2_f, u, v, cc);
      sm.S4[idx] = make_float4(h, qx, qy, u);
      sm.S2[idx] = make_float2(v, cc);
      sm.PK[idx] = WS->state[3 * NN + i];
      continue;
    }
    const float h = A.h0[cell0_off + (size_t)r * nx + c];
    float u, v, cc;
    cell_vel(h, 0.0f, 0.0f, P.g_f, P.heps2_f, u, v, cc);
    sm.S4[idx] = make_float4(h, 0.0f, 0.0f, u);
    sm.S2[idx] = make_float2(v, cc);
    sm.PK[idx] = 0.0f;
    const double hd = (double)h;
    v0_l += hd;
    if (hd > P.h_dry) {  // initial_smax (solver.rs:314-332) with q = 0
      const double cd = sqrt(P.g * hd);
      const double rr = (0.0 / hd + cd) / P.dx + (0.0 / hd + cd) / P.dy;
      s0_l = s0_l > rr ? s0_l : rr;
    }
  }
  // prefetch slots of columns past the grid are never written: zero them once, so the lanes
  // that carry no cell compute on zeros (finite operands, no needless reciprocal fallbacks)
  for (int i = tid; i < 2 * S * K * vlanes; i += blockDim.x) sm.PF[i] = 0.0f;
  if (tid < 8) { sm.slot[tid] = 0u; sm.LED[tid] = 0.0; }
  if (tid == 0) *sm.NSK = 0ull;
  if (WS && q == 0 && tid == 0) { sm.LED[0] = WS->tot_infil; sm.LED[1] = WS->tot_fix; sm.LED[2] = WS->tot_in; sm.LED[3] = WS->tot_out; }
  if (tid == 0) mbar_init(sm.mbar, blockDim.x + (A.stall_test ? 1u : 0u));
  // inflow ghosts of step 0 (at t = 0), and the ghost wetness the dry-row test reads; each
  // later step's are written one step ahead
  if (BND && wid == nwarps - 1) {
    if (lane < P.inflow.n) sm.INF[lane] = inflow_values(P.inflow, lane, t_start, P.g);
    __syncwarp();
    if (SKIP) ghost_row_wet(A.bc, nx, ny, bh, sm.INF, sm.GWF, lane);
  }
  {
    double sw = s0_l;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) { double t = __shfl_xor_sync(0xffffffffu, sw, o); sw = sw > t ? sw : t; }
    const double vw = warp_sum_d(v0_l);
    if (lane == 0) { sm.red[wid * 8 + 0] = sw; sm.red[wid * 8 + 1] = vw; }
  }
  if (CLUSTERED) { cluster_arrive(); cluster_wait(); } else __syncthreads();
  if (SKIP) row_flags(sm, 0, nr, nr_max, nx, W, wid, nwarps, lane);   // wetness of the initial state (parity 0)
  double s0 = 0.0, v0 = 0.0;
  for (int qq = 0; qq < C; ++qq) {
    const double* rr = CLUSTERED ? remote(sm.red, qq) : sm.red;
    for (int w = 0; w < nwarps; ++w) { const double a = rr[w * 8 + 0]; s0 = s0 > a ? s0 : a; v0 += rr[w * 8 + 1]; }
  }
  v0 *= P.area;
  if (WS) v0 = WS->v0;
  if (CLUSTERED) { cluster_arrive(); cluster_wait(); } else __syncthreads();   // red reused below

  // ------------------------------------------------------------------ integrator ----
  double t = t_start;
  unsigned long long step = WS ? WS->step : 0ull;
  unsigned sync_index = WS ? WS->sync_index : 0u;
  double dt_cfl = WS ? WS->dt_cfl : (s0 > 0.0 ? dmin_num(P.cfl / s0, P.dt_max) : P.dt_max);
  double acc_rain = WS ? WS->acc_rain : 0.0;
  int status = 0;
  unsigned breach_cell = 0, breach_sync = 0;
  double violation = 0.0, lower_bound = 0.0, volume = WS ? WS->volume : v0, rel_res = WS ? WS->rel_res : 0.0;
  int n_rows = WS ? WS->n_rows : 0;
  GroupSync<CLUSTERED> gs;
  gs.mbar = sm.mbar; gs.phase = 0; gs.limit = A.wait_limit; gs.timed_out = false;
  const float heps2 = P.heps2_f;
  RainCursor rcur;
  rcur.seg = 0; rcur.brk = 0;
  const int lr0 = r0 - ra;
  const bool top_dom = (r0 == 0);
  const int xb_next = wis + 1 < W ? wis + 1 : 0;          // warp whose lane 0 holds col0 + 1 of lane 31
  const int xb_next_comp = wis + 1 < W ? 0 : 1;

  const float2* inf_cur = sm.INF;   // this step's inflow group values (parity slot)
  auto ghost_x = [&](const Cell& c, int pos, bool west) -> Cell {
    return ghost_cell<BND, true>(c, A.bc[CK(pos, nbc, 13)], bh, pos, inf_cur, west, P.g_f, P.heps2_f);
  };
  auto ghost_y = [&](const Cell& c, int pos, bool north) -> Cell {
    return ghost_cell<BND, false>(c, A.bc[CK(pos, nbc, 15)], bh, pos, inf_cur, north, P.g_f, P.heps2_f);
  };
  // Loads the two cells of row lr (local) for this lane: interior cells, or the east ghost
  // for a lane whose column is nx (built from cell nx-1 and the east code of global row r).
  auto load_pair = [&](int lr, int r) -> Cell2 {
    Cell a{}, b{};
    if (cell0) a = load_cell(sm, lr * nx + col0);
    else if (face0) a = ghost_x(load_cell(sm, lr * nx + nx - 1), bc_e + r, false);
    if (cell1) b = load_cell(sm, lr * nx + col1);
    else if (face1) b = ghost_x(load_cell(sm, lr * nx + nx - 1), bc_e + r, false);
    return cell2_of(a, b);
  };
  // West neighbours of the lane's two cells in row lr: lane-1 by shuffle; lane 0 reads the
  // cell at column-1 from shared memory (another warp's column), or the west ghost at col 0.
  auto left_pair = [&](const Cell2& cur, int lr, int r) -> Cell2 {
    Cell2 left = shfl_up_cell2(cur);
    if (lane == 0) {
      Cell a = cx(left), b = cy(left);
      if (face0) a = col0 == 0 ? ghost_x(cx(cur), bc_w + r, true) : load_cell(sm, lr * nx + col0 - 1);
      if (face1) b = load_cell(sm, lr * nx + col1 - 1);
      left = cell2_of(a, b);
    }
    return left;
  };

  // ---- baseline-locked dt (solver.rs:436-483, 611-614) ----
  // Each step takes the baseline's dt while dt * smax of the current state stays within
  // cfl_hard. At the first step where it would not (or the schedule has run out), every CTA
  // restores its rows and scalars from the last sync snapshot and the run continues with the
  // adaptive dt. smax, the step and the schedule are the same in every thread of the cluster,
  // so the decision is uniform.
  bool locked_live = LOCKED;
  double s_cur = s0;
  if constexpr (LOCKED) {
    if (q == 0 && tid == 0) A.fallback_t[d] = -1.0;
    locked_save(A, sm, cell0_off + (size_t)ra * nx, nr * nx, (size_t)d * C + q, t, dt_cfl, s_cur, acc_rain, volume, rel_res,
                step, sync_index, n_rows);
  }

  while (t < P.duration && sync_index < P.n_sync) {
    if (step >= A.max_steps) { status = 4; break; }
    double dt_pick = 0.0;
    if constexpr (LOCKED) {
      dt_pick = dmin_num(dt_cfl, P.dt_max);
      if (locked_live) {
        if (step < A.n_locked && A.locked_dt[step] * s_cur <= A.cfl_hard) {
          dt_pick = A.locked_dt[step];
        } else {
          gs.full();   // every CTA has finished reading this CTA's shared memory
          for (int idx = tid; idx < nr * nx; idx += blockDim.x) {
            const size_t g = cell0_off + (size_t)ra * nx + idx;
            sm.S4[idx] = A.snap4[g]; sm.S2[idx] = A.snap2[g]; sm.PK[idx] = A.snapk[g];
          }
          const LockedSnap& o = A.snap_s[(size_t)d * C + q];
          t = o.t; dt_cfl = o.dt_cfl; s_cur = o.s_cur; acc_rain = o.acc_rain; volume = o.volume; rel_res = o.rel_res;
          step = o.step; sync_index = o.sync_index; n_rows = o.n_rows;
          if (tid < 4) { sm.LED[tid] = o.led[tid]; sm.slot[tid] = 0u; }
          rcur.seg = 0; rcur.brk = 0;
          if (BND && wid == nwarps - 1) {
            if (lane < P.inflow.n) sm.INF[(int)(step & 1ull) * kMaxInflow + lane] = inflow_values(P.inflow, lane, t, P.g);
            __syncwarp();
            if (SKIP)
              ghost_row_wet(A.bc, nx, ny, bh, sm.INF + (int)(step & 1ull) * kMaxInflow, sm.GWF + (int)(step & 1ull) * (ny + 2), lane);
          }
          if (SKIP) {
            __syncthreads();   // the restored rows complete before their flags are taken
            row_flags(sm, (int)(step & 1ull), nr, nr_max, nx, W, wid, nwarps, lane);
          }
          if (q == 0 && tid == 0) A.fallback_t[d] = t;
          locked_live = false;
          gs.full();   // the restored state of every CTA visible before the next step
          continue;
        }
      }
    }
    const StepPlan pl = LOCKED ? plan_step_dt_c(P, t, sync_index, dt_pick, rcur) : plan_step_c(P, t, sync_index, dt_cfl, rcur);
    StepK k = step_consts(P, pl.dt, pl.rain);
    k.exact = A.exact;
    const int sp = (int)(step & 1ull);
    if (BND) {
      inf_cur = sm.INF + sp * kMaxInflow;
      // the next step's inflow ghosts, at its start time (slot read after this step's
      // closing barrier; the other slot's readers finished before the previous one)
      if (wid == nwarps - 1) {
        if (lane < P.inflow.n) sm.INF[(sp ^ 1) * kMaxInflow + lane] = inflow_values(P.inflow, lane, pl.t_new, P.g);
        if (SKIP) {
          __syncwarp();
          ghost_row_wet(A.bc, nx, ny, bh, sm.INF + (sp ^ 1) * kMaxInflow, sm.GWF + (sp ^ 1) * (ny + 2), lane);
        }
      }
    }
    float smax_l = 0.0f, infil_l = 0.0f, fix_l = 0.0f;
    bool bad_l = false;
    int par = 0;

    // ---- strip pre-phase: first row, its west faces, the strip's top y-faces ----
    // Control flow is uniform per warp here (L is per strip); lane predicates only guard
    // loads and arithmetic, never the shuffles.
    Cell2 cur{};
    Face2 fW{}, fN{};
    if (L > 0) prefetch_row(r0, 0);
    cp_async_commit();
    if (L > 0) {
      cur = load_pair(lr0, r0);
      const Cell2 left = left_pair(cur, lr0, r0);
      const size_t fx = (size_t)r0 * nxp1, fy = (size_t)r0 * nx;
      const float2 dx0 = make_float2(__ldg(A.dzx + ox0 + fx), __ldg(A.dzx + ox1 + fx));
      const float2 dx1 = CREST ? make_float2(__ldg(A.dzx2 + ox0 + fx), __ldg(A.dzx2 + ox1 + fx)) : f2(0.0f);
      // the cells above the strip's first row: ghost, same CTA, or the CTA above
      Cell a0{}, a1{};
      if (top_dom) {
        if (cell0) a0 = ghost_y(cx(cur), bc_n + col0, true);
        if (cell1) a1 = ghost_y(cy(cur), bc_n + col1, true);
      } else if (r0 - 1 >= ra) {
        if (cell0) a0 = load_cell(sm, (lr0 - 1) * nx + col0);
        if (cell1) a1 = load_cell(sm, (lr0 - 1) * nx + col1);
      } else {
        // last row of the CTA above (old state; that CTA updates it only after B1)
        const int rap = (int)((long long)(q - 1) * ny / C);
        Smem rs = sm;
        rs.S4 = remote(sm.S4, q - 1);
        rs.S2 = remote(sm.S2, q - 1);
        if (cell0) a0 = load_cell(rs, (ra - 1 - rap) * nx + col0);
        if (cell1) a1 = load_cell(rs, (ra - 1 - rap) * nx + col1);
      }
      const Cell2 above = cell2_of(a0, a1);
      const float2 dy0 = make_float2(__ldg(A.dzy + oy0 + fy), __ldg(A.dzy + oy1 + fy));
      const float2 dy1 = CREST ? make_float2(__ldg(A.dzy2 + oy0 + fy), __ldg(A.dzy2 + oy1 + fy)) : f2(0.0f);
      fW = face2<true, CREST>(left.h, left.u, left.v, left.c, cur.h, cur.u, cur.v, cur.c, dx0, dx1, k);
      fN = face2<false, CREST>(above.h, above.u, above.v, above.c, cur.h, cur.u, cur.v, cur.c, dy0, dy1, k);
      if (lane == 0) {
        sm.XB[CK(((par * S + s) * W + wis) * 2 + 0, sm.nxb, 7)] = f4(fx_(fW));
        sm.XB[CK(((par * S + s) * W + wis) * 2 + 1, sm.nxb, 7)] = f4(fy_(fW));
      }
      if (cell0) sm.BF[CK(s * nx + col0, sm.nbf, 4)] = f4(fx_(fN));
      if (cell1) sm.BF[CK(s * nx + col1, sm.nbf, 4)] = f4(fy_(fN));
      if (top_dom) {   // y_boundary top (kernel.rs:452-472)
        if (cell0) sm.BY[(sp * 2 + 0) * nx + col0] = fN.m.x;
        if (cell1) sm.BY[(sp * 2 + 0) * nx + col1] = fN.m.y;
      }
    }
    if (in_strip) { if (W > 1) named_bar(1 + s, 32 * W); else __syncwarp(); }
    gs.b1_arrive();

    // ---- dry-row skipping (kernel.rs:605-612) ----
    // With no rain this step, grid row r is skipped when rows r - 1, r, r + 1 held no water in
    // the old state (flags of parity sp, written during the previous step; the rows beside the
    // CTA's band through DSMEM) and no stage or inflow ghost of theirs holds water. Its faces
    // are exactly 0 and its cells keep their zero state: skipping changes no result. The
    // decision depends only on shared flags, so every warp of a strip takes it alike.
    const bool try_skip = SKIP && !(k.rain > 0.0f);
    auto row_dry = [&](int j) -> bool {   // grid row j in [-1, ny]
      bool dr = !BND || sm.GWF[sp * (ny + 2) + j + 1] == 0;
      if (j < 0 || j >= ny) return dr;
      const uint8_t* wf = sm.WF;
      int lj = j - ra;
      if (CLUSTERED && (j < ra || j >= rb)) {
        const int qq = j < ra ? q - 1 : q + 1;
        wf = remote(sm.WF, qq);
        lj = j - (int)((long long)qq * ny / C);
      }
      const uint8_t* e = wf + ((size_t)sp * nr_max + lj) * W;
      for (int w = 0; w < W; ++w) dr = dr && e[w] == 0;
      return dr;
    };
    // Bit i of dmask: grid row r0 - 1 + mbase + i is dry, for the rows up to r0 + L, one row
    // per lane and ballot (64 rows per fill; a strip longer than 61 rows refills as it goes).
    unsigned long long dmask = 0ull;
    int mbase = 0;
    auto fill_mask = [&](int from) {
      const int ja = r0 - 1 + from + lane, jb = ja + 32, jmax = r0 + L;
      const bool da = ja <= jmax && row_dry(ja);
      const bool db = jb <= jmax && row_dry(jb);
      dmask = (unsigned long long)__ballot_sync(0xffffffffu, da) | ((unsigned long long)__ballot_sync(0xffffffffu, db) << 32);
      mbase = from;
    };
    if (try_skip && L > 0) fill_mask(0);

    // ---- row sweep ----
#pragma unroll 1
    for (int p = 0; p < L; ++p) {
      const int r = r0 + p;
      const int lr = lr0 + p;
      const bool last = (p == L - 1);
      bool skip = false, skip_next = false;
      if (try_skip) {
        if (p - mbase > 60) fill_mask(p);
        const int i = p - mbase;   // bits i, i + 1, i + 2: rows r - 1, r, r + 1
        skip = ((dmask >> i) & 7ull) == 7ull;
        skip_next = !last && ((dmask >> (i + 1)) & 7ull) == 7ull;
      }
      if (last) gs.b1_wait();
      if (!last) prefetch_row(r + 1, (p + 1) & 1);
      cp_async_commit();
      cp_async_wait<1>();
      const float* pfv = pf_base + (p & 1) * pf_slot;
      const float* pfv1 = pfv + 32 * W;
      const float2 d_s = make_float2(pfv[0 * vlanes], pfv1[0 * vlanes]);
      const float2 d_xn = make_float2(pfv[1 * vlanes], pfv1[1 * vlanes]);
      const float2 wet_r = make_float2(pfv[2 * vlanes], pfv1[2 * vlanes]);
      const float2 gn2_r = make_float2(pfv[3 * vlanes], pfv1[3 * vlanes]);
      const float2 d_s2 = CREST ? make_float2(pfv[4 * vlanes], pfv1[4 * vlanes]) : f2(0.0f);
      const float2 d_xn2 = CREST ? make_float2(pfv[5 * vlanes], pfv1[5 * vlanes]) : f2(0.0f);
      const bool bottom = last && s + 1 >= S && q + 1 >= C;
      Cell2 nxt{};
      Face2 fS{}, fWn{};
      if (SKIP && skip) {   // a dry row between dry rows: zero faces, nothing to update
        if (!last && !skip_next) {   // the next row's west faces
          nxt = load_pair(lr + 1, r + 1);
          const Cell2 left = left_pair(nxt, lr + 1, r + 1);
          fWn = face2<true, CREST>(left.h, left.u, left.v, left.c, nxt.h, nxt.u, nxt.v, nxt.c, d_xn, d_xn2, k);
          if (lane == 0) {
            sm.XB[CK((((par ^ 1) * S + s) * W + wis) * 2 + 0, sm.nxb, 9)] = f4(fx_(fWn));
            sm.XB[CK((((par ^ 1) * S + s) * W + wis) * 2 + 1, sm.nxb, 9)] = f4(fy_(fWn));
          }
        }
        if (bottom) {
          if (cell0) sm.BY[(sp * 2 + 1) * nx + col0] = 0.0f;
          if (cell1) sm.BY[(sp * 2 + 1) * nx + col1] = 0.0f;
        }
        if (in_strip && col0 == 0) sm.BX[(sp * 2 + 0) * nr_max + lr] = 0.0f;
        if (in_strip && (col0 == nx || col1 == nx)) sm.BX[(sp * 2 + 1) * nr_max + lr] = 0.0f;
        if (lane == 0) sm.WF[((size_t)(sp ^ 1) * nr_max + lr) * W + wis] = 0;
        if (lane == 0 && wis == 0) atomicAdd(sm.NSK, 1ull);   // once per skipped row (rain-free steps only)
        cur = nxt; fN = Face2{}; fW = fWn; par ^= 1;
        if (in_strip) { if (W > 1) named_bar(1 + s, 32 * W); else __syncwarp(); }
        continue;
      }
      // east faces: west faces of lane+1; lane 31 reads the published face of the lane
      // holding the next column
      Face2 fE = shfl_down_face2(fW);
      if (lane == 31) {
        FaceF ex = fx_(fE), ey = fy_(fE);
        if (cell0) ex = ff(sm.XB[CK(((par * S + s) * W + xb_next) * 2 + xb_next_comp, sm.nxb, 8)]);
        if (cell1 && wis + 1 < W) ey = ff(sm.XB[CK(((par * S + s) * W + wis + 1) * 2 + 1, sm.nxb, 8)]);
        fE = face2_of(ex, ey);
      }
      // operands of this row's new faces: the next row (and its west neighbours), or for a
      // strip's last row the next strip's / next CTA's top faces, or the south ghost row
      Cell2 left{}, below{};
      Face2 fS_in{};
      if (!last) {
        nxt = load_pair(lr + 1, r + 1);
        left = left_pair(nxt, lr + 1, r + 1);
      } else if (s + 1 < S) {
        FaceF sx{}, sy{};
        if (cell0) sx = ff(sm.BF[CK((s + 1) * nx + col0, sm.nbf, 5)]);
        if (cell1) sy = ff(sm.BF[CK((s + 1) * nx + col1, sm.nbf, 5)]);
        fS_in = face2_of(sx, sy);
      } else if (q + 1 < C) {
        const float4* rbf = remote(sm.BF, q + 1);
        FaceF sx{}, sy{};
        if (cell0) sx = ff(rbf[CK(col0, sm.nbf, 6)]);
        if (cell1) sy = ff(rbf[CK(col1, sm.nbf, 6)]);
        fS_in = face2_of(sx, sy);
      } else {
        Cell b0{}, b1{};
        if (cell0) b0 = ghost_y(cx(cur), bc_s + col0, false);
        if (cell1) b1 = ghost_y(cy(cur), bc_s + col1, false);
        below = cell2_of(b0, b1);
      }
      // new faces and the cell update; every lane of the strip computes (lanes past the grid
      // on zeros or ghost values), so the warp-uniform reciprocal fallback sees all 32 lanes
      CellNew2 o;
      float2 uu, vv;
      if (!last) {
        // (the next row's west faces are computed even when that row will be skipped: one
        // straight-line body keeps both faces' instructions interleaved)
        fS = face2<false, CREST>(cur.h, cur.u, cur.v, cur.c, nxt.h, nxt.u, nxt.v, nxt.c, d_s, d_s2, k);
        fWn = face2<true, CREST>(left.h, left.u, left.v, left.c, nxt.h, nxt.u, nxt.v, nxt.c, d_xn, d_xn2, k);
      } else if (bottom) {
        fS = face2<false, CREST>(cur.h, cur.u, cur.v, cur.c, below.h, below.u, below.v, below.c, d_s, d_s2, k);
      } else {
        fS = fS_in;
      }
      o = update_cell2(cur.h, cur.qx, cur.qy, fW, fE, fN, fS, wet_r, gn2_r, k);
      {
        const float2 h2 = mul2(o.h, o.h, k.nz);
        const float2 inv = rcp2f(add2(h2, max2(h2, f2(heps2))), k.exact);
        const float2 tt = mul2(add2(o.h, o.h), inv, k.nz);
        uu = mul2(o.qx, tt, k.nz);
        vv = mul2(o.qy, tt, k.nz);
      }
      if (!last && lane == 0) {
        sm.XB[CK((((par ^ 1) * S + s) * W + wis) * 2 + 0, sm.nxb, 9)] = f4(fx_(fWn));
        sm.XB[CK((((par ^ 1) * S + s) * W + wis) * 2 + 1, sm.nxb, 9)] = f4(fy_(fWn));
      }
      if (bottom) {   // y_boundary bottom (kernel.rs:452-472)
        if (cell0) sm.BY[(sp * 2 + 1) * nx + col0] = fS.m.x;
        if (cell1) sm.BY[(sp * 2 + 1) * nx + col1] = fS.m.y;
      }
      // x_boundary (kernel.rs:435-450): mass flux of the west and east domain faces
      if (in_strip && col0 == 0) sm.BX[(sp * 2 + 0) * nr_max + lr] = fW.m.x;
      if (in_strip && col0 == nx) sm.BX[(sp * 2 + 1) * nr_max + lr] = fW.m.x;
      if (in_strip && col1 == nx) sm.BX[(sp * 2 + 1) * nr_max + lr] = fW.m.y;
      if (cell0) {
        const int li = CK(lr * nx + col0, sm.ncell, 10);
        sm.S4[li] = make_float4(o.h.x, o.qx.x, o.qy.x, uu.x);
        sm.S2[li] = make_float2(vv.x, o.c.x);
        const float pk = sm.PK[li];
        if (o.h.x > pk) sm.PK[li] = o.h.x;
        smax_l = rmax(smax_l, o.s.x);
        bad_l = bad_l || o.bad.x;
        infil_l += o.infil.x;
        fix_l += o.fix.x;
      }
      if (cell1) {
        const int li = CK(lr * nx + col1, sm.ncell, 10);
        sm.S4[li] = make_float4(o.h.y, o.qx.y, o.qy.y, uu.y);
        sm.S2[li] = make_float2(vv.y, o.c.y);
        const float pk = sm.PK[li];
        if (o.h.y > pk) sm.PK[li] = o.h.y;
        smax_l = rmax(smax_l, o.s.y);
        bad_l = bad_l || o.bad.y;
        infil_l += o.infil.y;
        fix_l += o.fix.y;
      }
      if (SKIP) {   // the warp's columns of this row hold water in the new state (read next step)
        const bool wet_any = __any_sync(0xffffffffu, (cell0 && o.h.x > 0.0f) || (cell1 && o.h.y > 0.0f));
        if (lane == 0) sm.WF[((size_t)(sp ^ 1) * nr_max + lr) * W + wis] = wet_any ? 1 : 0;
      }
      cur = nxt; fN = fS; fW = fWn; par ^= 1;
      if (in_strip) { if (W > 1) named_bar(1 + s, 32 * W); else __syncwarp(); }
    }
    if (L == 0) gs.b1_wait();
    gs.b1_done();
    (void)any_face;
    // ---- end of step: CFL max, health, per-warp ledger partials ----
    {
      const float m = warp_max_f(smax_l);
      const unsigned b = __any_sync(0xffffffffu, bad_l) ? 1u : 0u;
      const float wi = warp_sum_f(infil_l), wf = warp_sum_f(fix_l);
      if (lane == 0) {
        if (m > 0.0f) atomicMax(&sm.slot[sp], __float_as_uint(m));
        if (b) atomicOr(&sm.slot[2 + sp], 1u);
        sm.WS[(sp * nwarps + wid) * 2 + 0] = wi;
        sm.WS[(sp * nwarps + wid) * 2 + 1] = wf;
      }
    }
    if (CLUSTERED) {
      gs.full();
    } else if (__syncthreads_or(gs.timed_out ? 1 : 0)) {
      // a barrier wait of this step ran out (bounded wait): the whole CTA leaves together
      status = 5;
      break;
    }
    unsigned smax_bits = 0u, badv = 0u;
    for (int qq = 0; qq < C; ++qq) {
      const unsigned* sl = CLUSTERED ? remote(sm.slot, qq) : sm.slot;
      const unsigned a = sl[sp];
      smax_bits = smax_bits > a ? smax_bits : a;
      badv |= sl[2 + sp];
    }
    if (wid == 0) {
      // fold this CTA's step partials into its f64 running totals, in a fixed order
      double di = 0.0, df = 0.0, din = 0.0, dout = 0.0;
      for (int w = lane; w < nwarps; w += 32) {
        di += (double)sm.WS[(sp * nwarps + w) * 2 + 0];
        df += (double)sm.WS[(sp * nwarps + w) * 2 + 1];
      }
      const double dt_dy = pl.dt * P.dy, dt_dx = pl.dt * P.dx;
      for (int j = lane; j < nr; j += 32) {
        const double vw = (double)sm.BX[(sp * 2 + 0) * nr_max + j] * dt_dy;   // west: inflow when m > 0
        if (vw > 0.0) din += vw; else dout -= vw;
        const double ve = (double)sm.BX[(sp * 2 + 1) * nr_max + j] * dt_dy;   // east: outflow when m > 0
        if (ve > 0.0) dout += ve; else din -= ve;
      }
      // y_boundary (kernel.rs:452-472): a y-edge's mass fluxes are summed over the row first
      // (FixedSum<f64>: lane (col + 1) & 15 in column order, then the pairwise tree, which
      // the butterfly over lanes 0-15 reproduces), then split: the top edge is inflow when
      // the net flux is > 0, the bottom edge outflow
      for (int side = 0; side < 2; ++side) {
        if (side == 0 ? q != 0 : q != C - 1) continue;
        double acc16 = 0.0;
        if (lane < 16)
          for (int j = (lane + 15) & 15; j < nx; j += 16) acc16 += (double)sm.BY[(sp * 2 + side) * nx + j];
#pragma unroll
        for (int o = 1; o < 16; o <<= 1) acc16 += __shfl_xor_sync(0xffffffffu, acc16, o);
        const double v = acc16 * dt_dx;
        if (lane == 0) {
          if (side == 0) { if (v > 0.0) din += v; else dout -= v; }
          else { if (v > 0.0) dout += v; else din -= v; }
        }
      }
      di = warp_sum_d(di); df = warp_sum_d(df); din = warp_sum_d(din); dout = warp_sum_d(dout);
      if (lane == 0) { sm.LED[0] += di; sm.LED[1] += df; sm.LED[2] += din; sm.LED[3] += dout; }
    }
    if (tid == 0) { sm.slot[sp ^ 1] = 0u; sm.slot[2 + (sp ^ 1)] = 0u; }
    const double smax = (double)__uint_as_float(smax_bits);
    step += 1;
    t = pl.t_new;
    acc_rain += pl.rain * P.area * P.wet_count;
    if (badv) { status = 3; break; }
    dt_cfl = smax > 0.0 ? P.cfl / smax : P.dt_max;
    if constexpr (LOCKED) s_cur = smax;
    if (pl.hits) {
      // ---- sync point: volume, ledger row, guard and incumbent tests ----
      sync_index += 1;
      double vol_l = 0.0;
      for (int idx = tid; idx < nr * nx; idx += blockDim.x) vol_l += (double)sm.S4[idx].x;
      vol_l = warp_sum_d(vol_l);
      if (lane == 0) sm.red[wid * 8 + 0] = vol_l;
      gs.full();   // volume partials and ledger totals of every CTA visible
      double tot[5] = {0, 0, 0, 0, 0};
      for (int qq = 0; qq < C; ++qq) {
        const double* rr = CLUSTERED ? remote(sm.red, qq) : sm.red;
        const double* lg = CLUSTERED ? remote(sm.LED, qq) : sm.LED;
        for (int w = 0; w < nwarps; ++w) tot[0] += rr[w * 8 + 0];
        for (int j = 0; j < 4; ++j) tot[1 + j] += lg[j];
      }
      const double v = tot[0] * P.area;
      const double infil = tot[1] * P.area, fix = tot[2] * P.area;
      const double expected = v0 + acc_rain + tot[3] - tot[4] - infil + fix;
      volume = v;
      const double gross = v0 + acc_rain + tot[3];
      rel_res = fabs(v - expected) / (gross > 1e-300 ? gross : 1e-300);
      if (q == 0 && tid == 0 && n_rows < A.max_rows && A.ledger_out) {
        double* o = A.ledger_out + ((size_t)d * A.max_rows + n_rows) * 8;
        o[0] = t; o[1] = v; o[2] = acc_rain; o[3] = tot[3]; o[4] = tot[4]; o[5] = infil; o[6] = fix; o[7] = v - expected;
      }
      n_rows += 1;
      // guard breach (objective.rs:132-145) and incumbent bound (objective.rs:147-149).
      // Every warp decides from the same peaks; the barrier below comes before any thread
      // acts, so no warp writes next-step peaks (or red, LED) while another still reads them.
      const DevObjective& ob = A.obj;
      int decision = 0;
      if (ob.enabled) {
        auto peak_of = [&](int mpos) -> double {
          const unsigned cell = A.mon_cells[mpos];
          const int rr_ = (int)(cell / (unsigned)nx), cc_ = (int)(cell % (unsigned)nx);
          int owner = 0;
          while (owner + 1 < C && rr_ >= (int)((long long)(owner + 1) * ny / C)) ++owner;
          const int ra_o = (int)((long long)owner * ny / C);
          const float* pk = CLUSTERED ? remote(sm.PK, owner) : sm.PK;
          return (double)pk[CK((rr_ - ra_o) * nx + cc_, sm.ncell, 21)];
        };
        if (ob.guard_abort && ob.require && ob.baseline) {
          double best = 0.0; int bk = -1;
          for (int g0 = 0; g0 < ob.n_guard; g0 += 32) {
            const int gk = g0 + lane;
            double w = 0.0; int kk = -1;
            if (gk < ob.n_guard) {
              const int mp = ob.guard_pos[gk];
              w = peak_of(mp) - ob.baseline[mp] - ob.tol;
              if (w > 0.0) kk = gk;
            }
            // warp argmax, first index on ties
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
              const double w2 = __shfl_xor_sync(0xffffffffu, w, o);
              const int k2 = __shfl_xor_sync(0xffffffffu, kk, o);
              const bool take = (k2 >= 0) && (kk < 0 || w2 > w || (w2 == w && k2 < kk));
              if (take) { w = w2; kk = k2; }
            }
            if (kk >= 0 && (bk < 0 || w > best)) { best = w; bk = kk; }
          }
          if (bk >= 0) {
            decision = 1;
            breach_cell = A.mon_cells[ob.guard_pos[bk]];
            breach_sync = sync_index;
            violation = best;
          }
        }
        if (decision == 0 && ob.has_incumbent) {
          double jr = 0.0;
          for (int a = 0; a < ob.n_assets; ++a) {
            double pkv = 0.0;
            for (int m = ob.asset_off[a] + lane; m < ob.asset_off[a + 1]; m += 32) {
              const double x = peak_of(ob.asset_pos[m]);
              pkv = pkv > x ? pkv : x;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) { const double x = __shfl_xor_sync(0xffffffffu, pkv, o); pkv = pkv > x ? pkv : x; }
            jr += ob.asset_w[a] * ob.tau * itr_math::softplus((pkv - ob.asset_thr[a]) / ob.tau);
          }
          const double je = ob.cut_cost * A.cut[d] + ob.fill_cost * A.fill[d];
          const double lb = jr + ob.earth_w * je;
          if (lb >= ob.incumbent) { decision = 2; lower_bound = lb; }
        }
      }
      gs.full();
      if (decision != 0) { status = decision; break; }
      if constexpr (LOCKED) {
        if (locked_live)
          locked_save(A, sm, cell0_off + (size_t)ra * nx, nr * nx, (size_t)d * C + q, t, dt_cfl, s_cur, acc_rain, volume,
                      rel_res, step, sync_index, n_rows);
      }
    }
  }
  if (gs.timed_out) status = 5;

  // ---------------------------------------------------------------- outputs ----------
  // All CTAs of the cluster leave the loop at the same step (identical decisions).
  if (CLUSTERED) { cluster_arrive(); cluster_wait(); } else __syncthreads();
  for (int idx = tid; idx < nr * nx; idx += blockDim.x) {
    const size_t g = cell0_off + (size_t)ra * nx + idx;
    A.depth_out[g] = sm.S4[idx].x;
    A.peak_out[g] = sm.PK[idx];
  }
  if (q == 0 && tid == 0) {
    DesignOut o;
    o.steps = step; o.t_end = t; o.sync_count = sync_index; o.status = status;
    o.breach_cell = breach_cell; o.breach_sync = breach_sync; o.violation = violation;
    o.lower_bound = lower_bound; o.v0 = v0; o.volume = volume; o.rel_residual = rel_res;
    o.n_rows = n_rows; o.pad = 0;
    unsigned long long tot_skip = 0ull;
    if (SKIP)
      for (int qq = 0; qq < C; ++qq) tot_skip += CLUSTERED ? *remote(sm.NSK, qq) : *sm.NSK;
    o.rows_skipped = tot_skip;
    A.out[d] = o;
  }
  // keep every CTA's shared memory alive until all remote reads are done
  if (CLUSTERED) { cluster_arrive(); cluster_wait(); }
}

}  // namespace itr
