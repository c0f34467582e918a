// itr_batched.cuh — the batched forward operator: one design per thread-block cluster.
//
// Replaces the reference's per-step `update` + `finalize` dispatch pair and its 64-step host
// polling (crates/itr-gpu/src/shader.wgsl:135-365, crates/itr-gpu/src/lib.rs:302-328) with a
// single persistent launch over the whole population: every cluster owns one design for the
// whole simulated storm and never leaves the SM between steps.
//
// Layout on chip. The design's rows are split into bands, one per CTA of the cluster; a band
// lives in shared memory as structure-of-arrays (h, qx, qy, u, v, c, peak), 28 B/cell, so the
// state never goes back to HBM until the run ends. Inside a CTA the band is cut into S strips;
// each strip is swept row by row by W warps (one lane per column, W = ceil((nx+1)/32)), the
// in-place row sweep of the reference's fused kernel (crates/itr-hydro/src/kernel.rs:637-697):
//   * the north y-face of a row is carried in registers from the row above,
//   * the west x-face of the next row is computed one phase early; the east face is the
//     west face of lane+1 (shuffle; lane 31 reads lane 0 of the next warp via shared memory),
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
// Ledgers are f64 per-thread accumulators reduced in a fixed order at sync points; the guard
// test (objective.rs:130-145) and the incumbent lower bound (objective.rs:146-149) run on
// the device at sync points, so an aborted design stops immediately.
#pragma once
#include <cooperative_groups.h>
#include "itr_device.cuh"

namespace itr {
namespace cg = cooperative_groups;

struct BatchArgs {
  RunParams P;
  int nx, ny, mode;
  int C;          // CTAs per design (cluster size)
  int W, S;       // warps per strip row, strips per CTA
  int n_designs;
  const float* wet;   // nx*ny
  const float* gn2;   // nx*ny
  const uint8_t* bc;  // north[nx], south[nx], west[ny], east[ny]
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
};

// Shared-memory carve-up of one CTA (sizes in floats unless noted).
struct Smem {
  float *H, *QX, *QY, *U, *V, *Cc, *PK;        // nr*nx each
  float *BM, *BNL, *BNR, *BT;                 // (S+1)*nx strip-boundary y-faces
  float* XB;                                  // [2][S][W][4] lane-0 x-face exchange
  unsigned* slot;                             // [2] smax bits, [2] bad, [2] pad
  double* red;                                // [NW][8] sync reductions
  unsigned long long* mbar;                   // CTA split barrier
  int ncell, nbface, nxb;                     // array lengths (bounds checks)
};

__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

__host__ __device__ inline size_t batched_smem_bytes(int nr, int nx, int S, int W, int nwarps) {
  size_t b = 0;
  b += (size_t)7 * nr * nx * 4;
  b += (size_t)4 * (S + 1) * nx * 4;
  b += (size_t)2 * S * W * 4 * 4;
  b = align_up(b, 16);
  b += 8 * 4;                       // slots
  b = align_up(b, 16);
  b += (size_t)nwarps * 8 * 8;      // reductions
  b = align_up(b, 16);
  b += 16;                          // mbarrier
  return b;
}

ITR_DEV void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

ITR_DEV void cluster_arrive() { asm volatile("barrier.cluster.arrive.release;" ::: "memory"); }
ITR_DEV void cluster_wait() { asm volatile("barrier.cluster.wait.acquire;" ::: "memory"); }

ITR_DEV unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

ITR_DEV void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
ITR_DEV void mbar_arrive(unsigned long long* bar) {
  asm volatile("{ .reg .b64 st; mbarrier.arrive.release.cta.shared::cta.b64 st, [%0]; }" ::"r"(smem_u32(bar)) : "memory");
}
// Bounded wait on phase `parity`; returns false if the bound ran out.
ITR_DEV bool mbar_wait(unsigned long long* bar, unsigned parity) {
  for (unsigned it = 0; it < (1u << 28); ++it) {
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
#define CKZ(i, lim, code) ((size_t)chk((long long)(i), (long long)(lim), (code)))
#else
#define CK(i, lim, code) (i)
#define CKZ(i, lim, code) (i)
#endif

// A cell's stored state (old values during a step).
struct Cell { float h, qx, qy, u, v, c; };

ITR_DEV Cell load_cell(const Smem& s, int idx) {
  idx = CK(idx, s.ncell, 1);
  Cell c;
  c.h = s.H[idx]; c.qx = s.QX[idx]; c.qy = s.QY[idx];
  c.u = s.U[idx]; c.v = s.V[idx]; c.c = s.Cc[idx];
  return c;
}

// Ghost cells (boundary.rs:36-57): a wall mirrors the normal momentum (so the normal
// velocity flips sign exactly), a transmissive edge copies the interior cell.
ITR_DEV Cell ghost_x(Cell c, int code) { if (code == 0) { c.qx = -c.qx; c.u = -c.u; } return c; }
ITR_DEV Cell ghost_y(Cell c, int code) { if (code == 0) { c.qy = -c.qy; c.v = -c.v; } return c; }

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

template <bool CREST>
ITR_DEV FaceF xface(const Cell& l, const Cell& r, const BatchArgs& A, int d, int row, int f, const StepK& k) {
  size_t o = (size_t)d * A.ny * (A.nx + 1) + (size_t)row * (A.nx + 1) + f;
  o = CKZ(o, (long long)A.n_designs * A.ny * (A.nx + 1), 2);
  float d0 = __ldg(A.dzx + o);
  float d1 = CREST ? __ldg(A.dzx2 + o) : 0.0f;
  return face<true, CREST>(l.h, l.u, l.v, l.c, r.h, r.u, r.v, r.c, d0, d1, k);
}
template <bool CREST>
ITR_DEV FaceF yface(const Cell& t, const Cell& b, const BatchArgs& A, int d, int f, int col, const StepK& k) {
  size_t o = (size_t)d * (A.ny + 1) * A.nx + (size_t)f * A.nx + col;
  o = CKZ(o, (long long)A.n_designs * (A.ny + 1) * A.nx, 3);
  float d0 = __ldg(A.dzy + o);
  float d1 = CREST ? __ldg(A.dzy2 + o) : 0.0f;
  return face<false, CREST>(t.h, t.u, t.v, t.c, b.h, b.u, b.v, b.c, d0, d1, k);
}

ITR_DEV void store_face(float* M, float* NL, float* NR, float* Tt, int idx, const FaceF& f) {
  M[idx] = f.m; NL[idx] = f.nl; NR[idx] = f.nr; Tt[idx] = f.t;
}
ITR_DEV FaceF load_face(const float* M, const float* NL, const float* NR, const float* Tt, int idx) {
  FaceF f; f.m = M[idx]; f.nl = NL[idx]; f.nr = NR[idx]; f.t = Tt[idx]; return f;
}

ITR_DEV double warp_sum_d(double v) {
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
  bool timed_out;
  ITR_DEV void b1_arrive() {
    if (CLUSTERED) cluster_arrive(); else mbar_arrive(mbar);
  }
  ITR_DEV void b1_wait() {
    if (CLUSTERED) cluster_wait();
    else { if (!mbar_wait(mbar, phase & 1u)) timed_out = true; }
  }
  ITR_DEV void b1_done() { phase += 1; }
  ITR_DEV void b2() {
    if (CLUSTERED) { cluster_arrive(); cluster_wait(); } else __syncthreads();
  }
};

// Map a pointer into shared memory to the same offset in CTA `rank` of the cluster.
template <class T> ITR_DEV T* remote(T* p, int rank) {
  return cg::this_cluster().map_shared_rank(p, (unsigned)rank);
}

template <bool CREST, bool CLUSTERED, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) k_batched(const BatchArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int C = A.C;
  const int q = CLUSTERED ? (int)cg::this_cluster().block_rank() : 0;
  const int d = blockIdx.x / C;
  if (d >= A.n_designs) return;   // whole clusters only (grid is a multiple of C)
  const int nx = A.nx, ny = A.ny;
  const int ra = (int)((long long)q * ny / C), rb = (int)((long long)(q + 1) * ny / C);
  const int nr = rb - ra;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarps = blockDim.x >> 5;
  const int W = A.W, S = A.S;
  const int s = wid / W, wis = wid % W;
  const int col = wis * 32 + lane;
  const bool in_strip = s < S;
  const bool cell_lane = in_strip && col < nx;
  const bool face_lane = in_strip && col <= nx;
  // strip rows (global row indices)
  const int r0 = in_strip ? ra + (int)((long long)s * nr / S) : rb;
  const int r1 = in_strip ? ra + (int)((long long)(s + 1) * nr / S) : rb;
  const int L = r1 - r0;

  // Every CTA of a cluster carves shared memory for the largest band, so an offset means
  // the same array in every CTA (DSMEM reads map a local pointer to a peer CTA).
  const int nr_max = (ny + C - 1) / C;
  Smem sm;
  {
    float* f = reinterpret_cast<float*>(smem_raw);
    size_t n = (size_t)nr_max * nx;
    sm.H = f; sm.QX = f + n; sm.QY = f + 2 * n; sm.U = f + 3 * n; sm.V = f + 4 * n; sm.Cc = f + 5 * n; sm.PK = f + 6 * n;
    float* b = f + 7 * n;
    size_t nb = (size_t)(S + 1) * nx;
    sm.BM = b; sm.BNL = b + nb; sm.BNR = b + 2 * nb; sm.BT = b + 3 * nb;
    sm.XB = b + 4 * nb;
    size_t off = align_up((size_t)((unsigned char*)(sm.XB + 2 * S * W * 4) - smem_raw), 16);
    sm.slot = reinterpret_cast<unsigned*>(smem_raw + off);
    off = align_up(off + 8 * 4, 16);
    sm.red = reinterpret_cast<double*>(smem_raw + off);
    off = align_up(off + (size_t)nwarps * 8 * 8, 16);
    sm.mbar = reinterpret_cast<unsigned long long*>(smem_raw + off);
    sm.ncell = (int)n; sm.nbface = (int)nb; sm.nxb = 2 * S * W * 4;
  }
  const RunParams& P = A.P;
  const size_t cell0 = (size_t)d * nx * ny;

  // ---------------------------------------------------------------- initial state ----
  double s0_l = 0.0, v0_l = 0.0;
  for (int idx = tid; idx < nr * nx; idx += blockDim.x) {
    int r = ra + idx / nx, c = idx % nx;
    float h = A.h0[CKZ(cell0 + (size_t)r * nx + c, (long long)A.n_designs * nx * ny, 12)];
    sm.H[idx] = h; sm.QX[idx] = 0.0f; sm.QY[idx] = 0.0f;
    float u, v, cc;
    cell_vel(h, 0.0f, 0.0f, (float)P.g, (float)(P.h_eps * P.h_eps), u, v, cc);
    sm.U[idx] = u; sm.V[idx] = v; sm.Cc[idx] = cc; sm.PK[idx] = 0.0f;
    double hd = (double)h;
    v0_l += hd;
    if (hd > P.h_dry) {  // initial_smax (solver.rs:314-332) with q = 0
      double cd = sqrt(P.g * hd);
      double rr = (0.0 / hd + cd) / P.dx + (0.0 / hd + cd) / P.dy;
      s0_l = s0_l > rr ? s0_l : rr;
    }
  }
  if (tid < 8) sm.slot[tid] = 0u;
  if (tid == 0) mbar_init(sm.mbar, blockDim.x);
  {
    // reduce s0 (max) and v0 (sum, fixed order) across the cluster
    double sw = s0_l;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) { double t = __shfl_xor_sync(0xffffffffu, sw, o); sw = sw > t ? sw : t; }
    double vw = warp_sum_d(v0_l);
    if (lane == 0) { sm.red[wid * 8 + 0] = sw; sm.red[wid * 8 + 1] = vw; }
  }
  if (CLUSTERED) { cluster_arrive(); cluster_wait(); } else __syncthreads();
  double s0 = 0.0, v0 = 0.0;
  for (int qq = 0; qq < C; ++qq) {
    const double* rr = CLUSTERED ? remote(sm.red, qq) : sm.red;
    for (int w = 0; w < nwarps; ++w) { double a = rr[w * 8 + 0]; s0 = s0 > a ? s0 : a; v0 += rr[w * 8 + 1]; }
  }
  v0 *= P.area;
  if (CLUSTERED) { cluster_arrive(); cluster_wait(); } else __syncthreads();   // red reused below

  // ------------------------------------------------------------------ integrator ----
  double t = 0.0;
  unsigned long long step = 0;
  unsigned sync_index = 0;
  double dt_cfl = s0 > 0.0 ? dmin_num(P.cfl / s0, P.dt_max) : P.dt_max;
  double acc_rain = 0.0;
  // per-thread f64 ledgers (cumulative)
  double l_infil = 0.0, l_fix = 0.0, l_in = 0.0, l_out = 0.0;
  int status = 0;
  unsigned breach_cell = 0, breach_sync = 0;
  double violation = 0.0, lower_bound = 0.0, volume = v0, rel_res = 0.0;
  int n_rows = 0;
  GroupSync<CLUSTERED> gs;
  gs.mbar = sm.mbar; gs.phase = 0; gs.timed_out = false;

  const float heps2 = (float)(P.h_eps * P.h_eps);

  while (t < P.duration && sync_index < P.n_sync) {
    if (step >= A.max_steps) { status = 4; break; }
    const StepPlan pl = plan_step(P, t, sync_index, dt_cfl);
    const StepK k = make_consts(P, pl.dt, pl.rain);
    const double dt_dy = pl.dt * P.dy, dt_dx = pl.dt * P.dx;
    float smax_l = 0.0f;
    bool bad_l = false;
    double vol_l = 0.0;
    int par = 0;

    // ---- strip pre-phase: first row, its west face, the strip's top y-face ----
    // Control flow is uniform per warp here (L is per strip); lane predicates only guard
    // loads and arithmetic, never the shuffles.
    Cell cur{};
    FaceF fW{}, fN{};
    if (L > 0) {
      const int lr = r0 - ra;
      if (cell_lane) cur = load_cell(sm, lr * nx + col);
      else if (face_lane) cur = ghost_x(load_cell(sm, lr * nx + nx - 1), A.bc[CK(2 * nx + ny + r0, 2 * nx + 2 * ny, 13)]);  // east ghost lane
      Cell left = shfl_up_cell(cur);
      if (lane == 0 && face_lane) {
        if (col == 0) left = ghost_x(cur, A.bc[CK(2 * nx + r0, 2 * nx + 2 * ny, 14)]);
        else left = load_cell(sm, lr * nx + col - 1);
      }
      if (face_lane) fW = xface<CREST>(left, cur, A, d, r0, col, k);
      if (lane == 0 && face_lane && wis > 0) {
        float* xb = sm.XB + CK(((par * S + s) * W + wis) * 4, sm.nxb - 3, 7);
        xb[0] = fW.m; xb[1] = fW.nl; xb[2] = fW.nr; xb[3] = fW.t;
      }
      if (cell_lane) {
        Cell above;
        if (r0 == 0) above = ghost_y(cur, A.bc[CK(col, 2 * nx + 2 * ny, 15)]);
        else if (r0 - 1 >= ra) above = load_cell(sm, (r0 - 1 - ra) * nx + col);
        else {
          // last row of the CTA above (old state; that CTA updates it only after B1)
          const int rap = (int)((long long)(q - 1) * ny / C);
          Smem rs = sm;
          rs.H = remote(sm.H, q - 1); rs.QX = remote(sm.QX, q - 1); rs.QY = remote(sm.QY, q - 1);
          rs.U = remote(sm.U, q - 1); rs.V = remote(sm.V, q - 1); rs.Cc = remote(sm.Cc, q - 1);
          above = load_cell(rs, CK((ra - 1 - rap) * nx + col, (rb - ra > 0 ? nr_max : 0) * nx, 19));
        }
        fN = yface<CREST>(above, cur, A, d, r0, col, k);
        store_face(sm.BM, sm.BNL, sm.BNR, sm.BT, CK(s * nx + col, sm.nbface, 4), fN);
        if (r0 == 0) {  // y_boundary top (kernel.rs:452-472), per face
          double v = (double)fN.m * dt_dx;
          if (v > 0.0) l_in += v; else l_out -= v;
        }
      }
    }
    if (in_strip) { if (W > 1) named_bar(1 + s, 32 * W); else __syncwarp(); }
    gs.b1_arrive();

    // ---- row sweep ----
    for (int p = 0; p < L; ++p) {
      const int r = r0 + p;
      const int lr = r - ra;
      const bool last = (p == L - 1);
      if (last) gs.b1_wait();
      Cell nxt{};
      FaceF fS{}, fWn{};
      FaceF fE = shfl_down_face(fW);
      if (lane == 31 && cell_lane) {
        const float* xb = sm.XB + CK(((par * S + s) * W + wis + 1) * 4, sm.nxb - 3, 8);
        fE.m = xb[0]; fE.nl = xb[1]; fE.nr = xb[2]; fE.t = xb[3];
      }
      if (!last) {
        const int lr1 = lr + 1;
        if (cell_lane) nxt = load_cell(sm, lr1 * nx + col);
        else if (face_lane) nxt = ghost_x(load_cell(sm, lr1 * nx + nx - 1), A.bc[CK(2 * nx + ny + r + 1, 2 * nx + 2 * ny, 16)]);
        if (cell_lane) fS = yface<CREST>(cur, nxt, A, d, r + 1, col, k);
        Cell left = shfl_up_cell(nxt);
        if (lane == 0 && face_lane) {
          if (col == 0) left = ghost_x(nxt, A.bc[CK(2 * nx + r + 1, 2 * nx + 2 * ny, 17)]);
          else left = load_cell(sm, lr1 * nx + col - 1);
        }
        if (face_lane) fWn = xface<CREST>(left, nxt, A, d, r + 1, col, k);
        if (lane == 0 && face_lane && wis > 0) {
          float* xb = sm.XB + CK((((par ^ 1) * S + s) * W + wis) * 4, sm.nxb - 3, 9);
          xb[0] = fWn.m; xb[1] = fWn.nl; xb[2] = fWn.nr; xb[3] = fWn.t;
        }
      } else if (cell_lane) {
        if (s + 1 < S) fS = load_face(sm.BM, sm.BNL, sm.BNR, sm.BT, CK((s + 1) * nx + col, sm.nbface, 5));
        else if (q + 1 < C) {
          fS = load_face(remote(sm.BM, q + 1), remote(sm.BNL, q + 1), remote(sm.BNR, q + 1), remote(sm.BT, q + 1), CK(col, sm.nbface, 6));
        } else {
          Cell below = ghost_y(cur, A.bc[CK(nx + col, 2 * nx + 2 * ny, 18)]);
          fS = yface<CREST>(cur, below, A, d, ny, col, k);
          double v = (double)fS.m * dt_dx;  // y_boundary bottom
          if (v > 0.0) l_out += v; else l_in -= v;
        }
      }
      // x_boundary (kernel.rs:435-450), per face
      if (in_strip && col == 0) { double v = (double)fW.m * dt_dy; if (v > 0.0) l_in += v; else l_out -= v; }
      if (in_strip && col == nx) { double v = (double)fW.m * dt_dy; if (v > 0.0) l_out += v; else l_in -= v; }
      if (cell_lane) {
        const size_t gi = CKZ((size_t)r * nx + col, (long long)nx * ny, 11);
        CellNew o = update_cell(cur.h, cur.qx, cur.qy, fW, fE, fN, fS, __ldg(A.wet + gi), __ldg(A.gn2 + gi), k);
        float u, v;
        {
          float h2 = o.h * o.h;
          float inv = 1.0f / (h2 + rmax(h2, heps2));
          float tt = (o.h + o.h) * inv;
          u = o.qx * tt; v = o.qy * tt;
        }
        const int li = CK(lr * nx + col, nr * nx, 10);
        sm.H[li] = o.h; sm.QX[li] = o.qx; sm.QY[li] = o.qy; sm.U[li] = u; sm.V[li] = v; sm.Cc[li] = o.c;
        float pk = sm.PK[li];
        if (o.h > pk) sm.PK[li] = o.h;
        smax_l = rmax(smax_l, o.s);
        bad_l = bad_l || o.bad;
        l_infil += (double)o.infil;
        l_fix += (double)o.fix;
        if (pl.hits) vol_l += (double)o.h;
      }
      cur = nxt; fN = fS; fW = fWn; par ^= 1;
      if (in_strip) { if (W > 1) named_bar(1 + s, 32 * W); else __syncwarp(); }
    }
    if (L == 0) gs.b1_wait();
    gs.b1_done();

    // ---- end of step: CFL max, health, sync-point reductions ----
    const int sp = (int)(step & 1ull);
    {
      float m = warp_max_f(smax_l);
      unsigned b = __any_sync(0xffffffffu, bad_l) ? 1u : 0u;
      if (lane == 0) {
        if (m > 0.0f) atomicMax(&sm.slot[sp], __float_as_uint(m));
        if (b) atomicOr(&sm.slot[2 + sp], 1u);
      }
      if (pl.hits) {
        double a0 = warp_sum_d(vol_l), a1 = warp_sum_d(l_infil), a2 = warp_sum_d(l_fix);
        double a3 = warp_sum_d(l_in), a4 = warp_sum_d(l_out);
        if (lane == 0) {
          double* rr = sm.red + wid * 8;
          rr[0] = a0; rr[1] = a1; rr[2] = a2; rr[3] = a3; rr[4] = a4;
        }
      }
    }
    gs.b2();
    unsigned smax_bits = 0u, badv = 0u;
    double tot[5] = {0, 0, 0, 0, 0};
    for (int qq = 0; qq < C; ++qq) {
      const unsigned* sl = CLUSTERED ? remote(sm.slot, qq) : sm.slot;
      unsigned a = sl[sp];
      smax_bits = smax_bits > a ? smax_bits : a;
      badv |= sl[2 + sp];
      if (pl.hits) {
        const double* rr = CLUSTERED ? remote(sm.red, qq) : sm.red;
        for (int w = 0; w < nwarps; ++w)
          for (int j = 0; j < 5; ++j) tot[j] += rr[w * 8 + j];
      }
    }
    if (tid == 0) { sm.slot[sp ^ 1] = 0u; sm.slot[2 + (sp ^ 1)] = 0u; }
    const double smax = (double)__uint_as_float(smax_bits);
    step += 1;
    t = pl.t_new;
    acc_rain += pl.rain * P.area * P.wet_count;
    if (badv) { status = 3; break; }
    dt_cfl = smax > 0.0 ? P.cfl / smax : P.dt_max;
    if (pl.hits) {
      sync_index += 1;
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
      // Every warp decides from the same peaks; a barrier follows before any thread acts, so
      // no warp can start writing next-step peaks while another is still reading them.
      const DevObjective& ob = A.obj;
      int decision = 0;
      if (ob.enabled) {
        auto peak_of = [&](int mpos) -> double {
          unsigned cell = A.mon_cells[mpos];
          int rr_ = (int)(cell / (unsigned)nx), cc_ = (int)(cell % (unsigned)nx);
          int owner = 0;
          while (owner + 1 < C && rr_ >= (int)((long long)(owner + 1) * ny / C)) ++owner;
          int ra_o = (int)((long long)owner * ny / C);
          const float* pk = CLUSTERED ? remote(sm.PK, owner) : sm.PK;
          return (double)pk[CK((rr_ - ra_o) * nx + cc_, sm.ncell, 21)];
        };
        if (ob.guard_abort && ob.require && ob.baseline) {
          double best = 0.0; int bk = -1;
          for (int g0 = 0; g0 < ob.n_guard; g0 += 32) {
            int gk = g0 + lane;
            double w = 0.0; int kk = -1;
            if (gk < ob.n_guard) {
              int mp = ob.guard_pos[gk];
              w = peak_of(mp) - ob.baseline[mp] - ob.tol;
              if (w > 0.0) kk = gk;
            }
            // warp argmax, first index on ties
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
              double w2 = __shfl_xor_sync(0xffffffffu, w, o);
              int k2 = __shfl_xor_sync(0xffffffffu, kk, o);
              bool take = (k2 >= 0) && (kk < 0 || w2 > w || (w2 == w && k2 < kk));
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
              double x = peak_of(ob.asset_pos[m]);
              pkv = pkv > x ? pkv : x;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) { double x = __shfl_xor_sync(0xffffffffu, pkv, o); pkv = pkv > x ? pkv : x; }
            jr += ob.asset_w[a] * ob.tau * itr_math::softplus((pkv - ob.asset_thr[a]) / ob.tau);
          }
          const double je = ob.cut_cost * A.cut[d] + ob.fill_cost * A.fill[d];
          const double lb = jr + ob.earth_w * je;
          if (lb >= ob.incumbent) { decision = 2; lower_bound = lb; }
        }
        gs.b2();
      }
      if (decision != 0) { status = decision; break; }
    }
  }
  if (gs.timed_out) status = 5;

  // ---------------------------------------------------------------- outputs ----------
  // All CTAs of the cluster leave the loop at the same step (identical decisions).
  if (CLUSTERED) { cluster_arrive(); cluster_wait(); } else __syncthreads();
  for (int idx = tid; idx < nr * nx; idx += blockDim.x) {
    size_t g = CKZ(cell0 + (size_t)ra * nx + idx, (long long)A.n_designs * nx * ny, 20);
    A.depth_out[g] = sm.H[idx];
    A.peak_out[g] = sm.PK[idx];
  }
  if (q == 0 && tid == 0) {
    DesignOut o;
    o.steps = step; o.t_end = t; o.sync_count = sync_index; o.status = status;
    o.breach_cell = breach_cell; o.breach_sync = breach_sync; o.violation = violation;
    o.lower_bound = lower_bound; o.v0 = v0; o.volume = volume; o.rel_residual = rel_res;
    o.n_rows = n_rows; o.pad = 0;
    A.out[d] = o;
  }
  // keep every CTA's shared memory alive until all remote reads are done
  if (CLUSTERED) { cluster_arrive(); cluster_wait(); }
}

}  // namespace itr
