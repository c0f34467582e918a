// itr_adjoint_band.cuh — the adjoint's replay and backward step as row-band sweeps.
//
// Replay: k_band<CREST, BND, TAPE = true> (itr_band.cuh) advances tape slot j to slot j + 1 with
// the recorded (dt, rain); k_adj_plan writes the control blocks it reads (the step's constants
// and inflow values, done past a design's last step). The update is the forward's own kernel,
// so the replayed states are the forward's bit for bit.
//
// Backward step (k_adj_band): the arithmetic of k_adj_step (itr_adjoint.cuh) in the same
// operation order, so its outputs are k_adj_step's bit for bit, on a row sweep instead of a
// 16x16 tile with a two-cell halo:
//   * a warp sweeps one band of rows of a segment of columns, one column per lane, with no
//     barrier inside the step; lanes 1 .. 29 own 29 columns, lane 0 (the column to the west)
//     and lanes 30, 31 (the two to the east) carry the halo the owned cells' faces need: the
//     source adjoint of lanes 0 and 30, the forward x-face of lane 31;
//   * per row, each lane computes the forward y-face below it and the forward x-face west of it
//     of the row ahead, the source adjoint of that row, and the adjoints of the y-face below
//     the current row and of its west x-face; the face adjoints reach their neighbours by
//     shuffles and the rolling window (states of three rows, the north face's adjoint) stays in
//     registers. Work per owned cell: 32/29 of one forward face pair, one source adjoint and
//     one face-adjoint pair, against 1.27 of each for the tile;
//   * lane 0's west x-face needs the cell two columns west: computed for every row of the band
//     before the sweep (one face per lane) and kept in shared memory.
#pragma once
#include <cmath>
#include "itr_adjoint.cuh"
#include "itr_band.cuh"

namespace itr {

constexpr int kAdjOwn = 29;     // columns a warp owns (lanes 1 .. 29)
constexpr int kAdjWarps = 4;    // most warps (segments) per block
constexpr int kAdjRows = 32;    // most rows per band
#ifndef ITR_ADJ_MIN_BLOCKS
#define ITR_ADJ_MIN_BLOCKS 6    // resident blocks per SM the register budget is cut for (85
                                // registers, a few spilled: measured faster than 4 and 8)
#endif

struct AdjGeom {
  int ns;      // segments of kAdjOwn columns
  int wpb;     // warps per block: the divisor-friendliest of 4, 3, 2 (fewest idle segments)
  int rows;    // rows per band
  int gx, gy;  // blocks per design
};

__host__ __device__ inline AdjGeom adj_geom(int nx, int ny, int rows) {
  AdjGeom g;
  g.ns = (nx + kAdjOwn - 1) / kAdjOwn;
  g.wpb = 1;
  int waste = 1 << 30;
  for (int w = kAdjWarps; w >= 1; --w) {
    const int e = (g.ns + w - 1) / w * w - g.ns;
    if (e < waste) { waste = e; g.wpb = w; }
  }
  g.rows = rows;
  g.gx = (g.ns + g.wpb - 1) / g.wpb;
  g.gy = (ny + rows - 1) / rows;
  return g;
}

// Rows per band: the busy fraction of the launch's rounds of resident warps (4 per block,
// ITR_ADJ_MIN_BLOCKS blocks per SM) times R / (R + 2), the share of rows a band does not
// recompute.
inline int adj_rows_for(int nx, int ny, int n_designs, int sm_count) {
  const double resident = 4.0 * ITR_ADJ_MIN_BLOCKS * (sm_count > 0 ? sm_count : 148);
  int best = kAdjRows;
  double best_score = -1.0;
  for (int rows = kAdjRows; rows >= 6; --rows) {
    const AdjGeom g = adj_geom(nx, ny, rows);
    const double warps = (double)n_designs * g.gx * g.wpb * g.gy;
    const double rounds = std::ceil(warps / resident);
    const double score = warps / (rounds * resident) * rows / (rows + 2.0);
    if (score > best_score + 1e-9) { best_score = score; best = rows; }
  }
  return best;
}

// Control blocks of a segment's replay: step j of design d at ctl[j * n_designs + d].
__global__ void k_adj_plan(const AdjArgs A, PlainCtl* ctl) {
  const int j = blockIdx.x, d = blockIdx.y;
  PlainCtl* c = ctl + (size_t)j * A.n_designs + d;
  const double* sg = A.seg + ((size_t)d * A.K + j) * 3;
  const bool live = A.step0 + j < A.n_steps[d];
  if ((int)threadIdx.x < A.P.inflow.n)
    c->inf[threadIdx.x] = live ? inflow_values(A.P.inflow, threadIdx.x, sg[2], A.P.g) : make_float2(0.0f, 0.0f);
  if (threadIdx.x == 0) {
    c->done = live ? 0 : 1;
    c->par = 0;
    c->step = A.step0 + j;
    c->k = step_consts(A.P, sg[0], sg[1]);
    c->pl.dt = sg[0]; c->pl.rain = sg[1]; c->pl.t_new = sg[2] + sg[0]; c->pl.hits = false;
  }
}

// One lane's cell: old state and its velocities.
struct ACell { float h, qx, qy, u, v, c; };

ITR_DEV ACell acell_shfl_up(const ACell& a) {
  ACell r;
  r.h = __shfl_up_sync(0xffffffffu, a.h, 1); r.qx = __shfl_up_sync(0xffffffffu, a.qx, 1);
  r.qy = __shfl_up_sync(0xffffffffu, a.qy, 1); r.u = __shfl_up_sync(0xffffffffu, a.u, 1);
  r.v = __shfl_up_sync(0xffffffffu, a.v, 1); r.c = __shfl_up_sync(0xffffffffu, a.c, 1);
  return r;
}
ITR_DEV ACell acell_shfl_down(const ACell& a) {
  ACell r;
  r.h = __shfl_down_sync(0xffffffffu, a.h, 1); r.qx = __shfl_down_sync(0xffffffffu, a.qx, 1);
  r.qy = __shfl_down_sync(0xffffffffu, a.qy, 1); r.u = __shfl_down_sync(0xffffffffu, a.u, 1);
  r.v = __shfl_down_sync(0xffffffffu, a.v, 1); r.c = __shfl_down_sync(0xffffffffu, a.c, 1);
  return r;
}
ITR_DEV FaceF facef_shfl_down(const FaceF& f) {
  FaceF r;
  r.m = __shfl_down_sync(0xffffffffu, f.m, 1); r.nl = __shfl_down_sync(0xffffffffu, f.nl, 1);
  r.nr = __shfl_down_sync(0xffffffffu, f.nr, 1); r.t = __shfl_down_sync(0xffffffffu, f.t, 1);
  return r;
}
ITR_DEV FaceBwd facebwd_shfl_down(const FaceBwd& b) {
  FaceBwd r;
  r.hl = __shfl_down_sync(0xffffffffu, b.hl, 1); r.ul = __shfl_down_sync(0xffffffffu, b.ul, 1);
  r.vl = __shfl_down_sync(0xffffffffu, b.vl, 1); r.cl = __shfl_down_sync(0xffffffffu, b.cl, 1);
  r.hr = __shfl_down_sync(0xffffffffu, b.hr, 1); r.ur = __shfl_down_sync(0xffffffffu, b.ur, 1);
  r.vr = __shfl_down_sync(0xffffffffu, b.vr, 1); r.cr = __shfl_down_sync(0xffffffffu, b.cr, 1);
  r.dz = 0.0f; r.dz2 = 0.0f;
  return r;
}

template <bool BND, bool CREST>
__global__ void __launch_bounds__(kAdjWarps * 32, ITR_ADJ_MIN_BLOCKS) k_adj_band(const AdjArgs A, int j) {
  __shared__ FaceF edge[kAdjWarps][2 * 32];   // lane 0's west x-face, rows r0 - 1 .. r1
  __shared__ float2 sinf[kMaxInflow];
  const int d = blockIdx.z;
  const int nx = A.nx, ny = A.ny, nxp1 = nx + 1;
  const size_t N = (size_t)nx * ny, SX = (size_t)ny * (nx + 1), SY = (size_t)(ny + 1) * nx;
  const unsigned long long n = A.step0 + j;
  const float* LI = A.lin + (size_t)d * 3 * N;
  float* LO = A.lout + (size_t)d * 3 * N;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  const int s = blockIdx.x * wpb + wid;            // this warp's segment
  const int cs = s * kAdjOwn;                      // its first owned column
  const int col = cs - 1 + lane;                   // this lane's column
  const int R = A.band_rows;
  const int r0 = blockIdx.y * R;
  const int r1 = r0 + R < ny ? r0 + R : ny;
  const bool own = lane >= 1 && lane <= kAdjOwn && col < nx;   // an owned cell column
  if (n >= A.n_steps[d]) {   // the design stopped before this step: the adjoint passes through
    const int c_lo = blockIdx.x * wpb * kAdjOwn;   // the block's cells, all threads at once
    const int w = (c_lo + wpb * kAdjOwn < nx ? c_lo + wpb * kAdjOwn : nx) - c_lo;
    if (w > 0)
      for (int e = threadIdx.x; e < w * (r1 - r0); e += blockDim.x) {
        const size_t gi = (size_t)(r0 + e / w) * nx + c_lo + e % w;
        const float a = LI[gi], b = LI[N + gi], c = LI[2 * N + gi];
        LO[gi] = a; LO[N + gi] = b; LO[2 * N + gi] = c;
      }
    return;
  }
  const float* X = A.tape + ((size_t)j * A.n_designs + d) * 3 * N;
  const double* sg = A.seg + ((size_t)d * A.K + j) * 3;
  const StepK k = step_consts(A.P, sg[0], sg[1]);
  const float* dzx = A.dzx + d * SX;
  const float* dzy = A.dzy + d * SY;
  const float* dzx2 = CREST ? A.dzx2 + d * SX : nullptr;
  const float* dzy2 = CREST ? A.dzy2 + d * SY : nullptr;
  const float* bh = BND && A.bh ? A.bh + (size_t)d * (2 * nx + 2 * ny) : nullptr;
  adj_inflow<BND>(A, sg[2], sinf);
  if (cs >= nx) return;   // no owned column (no block barrier after this point)

  auto raw = [&](int gx, int gy) -> ACell {   // old state of padded cell (gx, gy), no velocities yet
    ACell a;
    adj_load<BND>(A, X, gx, gy, a.h, a.qx, a.qy, bh, sinf);
    a.u = a.v = a.c = 0.0f;
    return a;
  };
  auto vel = [&](ACell a) -> ACell { cell_vel(a.h, a.qx, a.qy, k.g, k.heps2, a.u, a.v, a.c); return a; };
  auto cell = [&](int gx, int gy) -> ACell { return vel(raw(gx, gy)); };
  const bool xcol = col >= 0 && col <= nx;    // x-face `col` exists
  const bool ycol = col >= 0 && col < nx;     // y-faces of column `col` exist
  // forward x-face between (r, col - 1) and (r, col); L: the west cell
  // (computed on every lane, then zeroed where the face does not exist: one straight-line body
  //  lets the compiler interleave a row's independent chains)
  auto xfwd = [&](const ACell& L, const ACell& C, int r, float dz, float dz2) -> FaceF {
    FaceF o = face<true, CREST>(L.h, L.u, L.v, L.c, C.h, C.u, C.v, C.c, dz, dz2, k);
    if (!(xcol && r >= 0 && r < ny)) o = FaceF{};
    return o;
  };
  // forward y-face f between (f - 1, col) and (f, col)
  auto yfwd = [&](const ACell& T, const ACell& B, int f, float dz, float dz2) -> FaceF {
    FaceF o = face<false, CREST>(T.h, T.u, T.v, T.c, B.h, B.u, B.v, B.c, dz, dz2, k);
    if (!(ycol && f >= 0 && f <= ny)) o = FaceF{};
    return o;
  };
  auto jx = [&](const float* a, int r) -> float { return (xcol && r >= 0 && r < ny) ? a[(size_t)r * nxp1 + col] : 0.0f; };
  auto jy = [&](const float* a, int f) -> float { return (ycol && f >= 0 && f <= ny) ? a[(size_t)f * nx + col] : 0.0f; };

  // ---- pre-pass: lane 0's west x-face (columns cs - 2 | cs - 1) of rows r0 - 1 .. r1 ----
  for (int e = lane; e < r1 - r0 + 2; e += 32) {
    const int r = r0 - 1 + e, f = cs - 1;
    FaceF o{};
    if (f >= 0 && f <= nx && r >= 0 && r < ny) {
      const ACell a = cell(f - 1, r), b = cell(f, r);
      const size_t xo = (size_t)r * nxp1 + f;
      o = face<true, CREST>(a.h, a.u, a.v, a.c, b.h, b.u, b.v, b.c, dzx[xo], CREST ? dzx2[xo] : 0.0f, k);
    }
    edge[wid][e] = o;
  }
  __syncwarp();

  // seeds (peak terms) of this step inside the warp's cells, halo included: usually none
  const int* sn = A.seed_n;
  bool seeded = false;
  for (int q = lane; q < sn[d]; q += 32) {
    const size_t si = (size_t)d * A.max_seeds + q;
    if (A.seed_state[si] == n + 1) {
      const int sr = (int)(A.seed_cell[si] / (unsigned)nx), sc = (int)(A.seed_cell[si] % (unsigned)nx);
      seeded = seeded || (sr >= r0 - 1 && sr <= r1 && sc >= cs - 1 && sc <= cs + kAdjOwn);
    }
  }
  seeded = __any_sync(0xffffffffu, seeded);

  // adjoint of the sources of (r, col) (zero outside the grid), as phase 3 of k_adj_step
  struct L1 { float h, qx, qy; };
  auto l1_of = [&](const ACell& C, const FaceF& W, const FaceF& E, const FaceF& Nf, const FaceF& Sf, int r, float wet,
                   float gn2, float lh, float lqx, float lqy) -> L1 {
    L1 o{0.0f, 0.0f, 0.0f};
    const bool in = ycol && r >= 0 && r < ny;
    if (seeded && in) {
      const size_t gi = (size_t)r * nx + col;
      for (int q = 0; q < sn[d]; ++q) {
        const size_t si = (size_t)d * A.max_seeds + q;
        if (A.seed_cell[si] == gi && A.seed_state[si] == n + 1) lh += A.seed_w[si];
      }
    }
    sources_bwd(C.h, C.qx, C.qy, W, E, Nf, Sf, wet, gn2, k, lh, lqx, lqy, o.h, o.qx, o.qy);
    if (!in) o = L1{0.0f, 0.0f, 0.0f};
    return o;
  };
  // inputs of row r for this lane's column (zero outside)
  struct RowIn { float lh, lqx, lqy, wet, gn2; };
  auto load_in = [&](int r) -> RowIn {
    RowIn q{0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    if (ycol && r >= 0 && r < ny) {
      const size_t gi = (size_t)r * nx + col;
      q.lh = LI[gi]; q.lqx = LI[N + gi]; q.lqy = LI[2 * N + gi];
      q.wet = A.wet[gi]; q.gn2 = A.gn2[gi];
    }
    return q;
  };
  const bool xown = (own && col <= nx) || (lane == kAdjOwn + 1 && col == nx);   // owns x-face `col`

  // ---- prologue: rows r0 - 2 .. r0 + 1, the source adjoints of rows r0 - 1 and r0, and the
  //      adjoint of the band's top y-face (r0 - 1 | r0), whose gradient this band owns ----
  const ACell Sa = cell(col, r0 - 2), Sb = cell(col, r0 - 1);
  ACell Sc = cell(col, r0), Sd = cell(col, r0 + 1);
  const FaceF ya = yfwd(Sa, Sb, r0 - 1, jy(dzy, r0 - 1), CREST ? jy(dzy2, r0 - 1) : 0.0f);
  const float jyb = jy(dzy, r0), jyb2 = CREST ? jy(dzy2, r0) : 0.0f;
  const FaceF yb = yfwd(Sb, Sc, r0, jyb, jyb2);
  float jyc = jy(dzy, r0 + 1), jyc2 = CREST ? jy(dzy2, r0 + 1) : 0.0f;
  FaceF yc = yfwd(Sc, Sd, r0 + 1, jyc, jyc2);
  L1 lb, lc;
  {
    FaceF xb = xfwd(acell_shfl_up(Sb), Sb, r0 - 1, jx(dzx, r0 - 1), CREST ? jx(dzx2, r0 - 1) : 0.0f);
    if (lane == 0) xb = edge[wid][0];
    const FaceF xbe = facef_shfl_down(xb);
    const RowIn ib = load_in(r0 - 1);
    lb = l1_of(Sb, xb, xbe, ya, yb, r0 - 1, ib.wet, ib.gn2, ib.lh, ib.lqx, ib.lqy);
  }
  float jxc = jx(dzx, r0), jxc2 = CREST ? jx(dzx2, r0) : 0.0f;
  {
    FaceF xc = xfwd(acell_shfl_up(Sc), Sc, r0, jxc, jxc2);
    if (lane == 0) xc = edge[wid][1];
    const FaceF xce = facef_shfl_down(xc);
    const RowIn ic = load_in(r0);
    lc = l1_of(Sc, xc, xce, yb, yc, r0, ic.wet, ic.gn2, ic.lh, ic.lqx, ic.lqy);
  }
  FaceBwd nb{};   // adjoint of the north y-face of the current row
  {
    const float lm = -k.dtdy * lb.h + k.dtdy * lc.h;
    const float lt = -k.dtdy * lb.qx + k.dtdy * lc.qx;
    const float lnl = -k.dtdy * lb.qy, lnr = k.dtdy * lc.qy;
    nb = face_bwd<false, CREST>(Sb.h, Sb.u, Sb.v, Sb.c, Sc.h, Sc.u, Sc.v, Sc.c, jyb, jyb2, k, lm, lnl, lnr, lt);
    if (own) {
      double* gp = A.gdzy + d * SY + (size_t)r0 * nx + col;
      *gp = *gp + (double)nb.dz;
      if (CREST) { double* gp2 = A.gdzy2 + d * SY + (size_t)r0 * nx + col; *gp2 = *gp2 + (double)nb.dz2; }
    }
  }

  // ---- row sweep ----
  RowIn inn = load_in(r0 + 1);
  ACell Se = raw(col, r0 + 2);
#pragma unroll 1
  for (int r = r0; r < r1; ++r) {
    const RowIn in1 = inn;             // inputs of row r + 1
    const ACell Snext = vel(Se);       // state of row r + 2
    if (r + 1 < r1) {                  // the next row's operands, in flight while this row runs
      inn = load_in(r + 2);
      Se = raw(col, r + 3);
    }
    // this row's gradient sums, read before the arithmetic so the loads are in flight
    const bool yown_r = own && (r + 1 < r1 || r + 1 == ny);
    double* gyp = A.gdzy + d * SY + (size_t)(r + 1) * nx + col;
    double* gxp = A.gdzx + d * SX + (size_t)r * nxp1 + col;
    const double gy_old = yown_r ? *gyp : 0.0, gx_old = xown ? *gxp : 0.0;
    double gy2_old = 0.0, gx2_old = 0.0;
    if (CREST) {
      gy2_old = yown_r ? A.gdzy2[d * SY + (size_t)(r + 1) * nx + col] : 0.0;
      gx2_old = xown ? A.gdzx2[d * SX + (size_t)r * nxp1 + col] : 0.0;
    }
    // forward faces around row r + 1 and its source adjoint
    const float jyd = jy(dzy, r + 2), jyd2 = CREST ? jy(dzy2, r + 2) : 0.0f;
    const FaceF yd = yfwd(Sd, Snext, r + 2, jyd, jyd2);
    const float jxd = jx(dzx, r + 1), jxd2 = CREST ? jx(dzx2, r + 1) : 0.0f;
    FaceF xd = xfwd(acell_shfl_up(Sd), Sd, r + 1, jxd, jxd2);
    if (lane == 0) xd = edge[wid][r + 2 - r0];
    const FaceF xde = facef_shfl_down(xd);
    const L1 ld = l1_of(Sd, xd, xde, yc, yd, r + 1, in1.wet, in1.gn2, in1.lh, in1.lqx, in1.lqy);
    // adjoint of the y-face (r | r + 1)
    FaceBwd sb;
    {
      const float lm = -k.dtdy * lc.h + k.dtdy * ld.h;
      const float lt = -k.dtdy * lc.qx + k.dtdy * ld.qx;
      const float lnl = -k.dtdy * lc.qy, lnr = k.dtdy * ld.qy;
      sb = face_bwd<false, CREST>(Sc.h, Sc.u, Sc.v, Sc.c, Sd.h, Sd.u, Sd.v, Sd.c, jyc, jyc2, k, lm, lnl, lnr, lt);
    }
    // adjoint of the west x-face of (r, col), lanes 1 .. 30 (lane 30's is the east face of 29)
    const ACell Wc = acell_shfl_up(Sc);
    const float lwh = __shfl_up_sync(0xffffffffu, lc.h, 1), lwqx = __shfl_up_sync(0xffffffffu, lc.qx, 1),
                lwqy = __shfl_up_sync(0xffffffffu, lc.qy, 1);
    FaceBwd xb;
    {
      const float lm = -k.dtdx * lwh + k.dtdx * lc.h;
      const float lnl = -k.dtdx * lwqx, lnr = k.dtdx * lc.qx;
      const float lt = -k.dtdx * lwqy + k.dtdx * lc.qy;
      xb = face_bwd<true, CREST>(Wc.h, Wc.u, Wc.v, Wc.c, Sc.h, Sc.u, Sc.v, Sc.c, jxc, jxc2, k, lm, lnl, lnr, lt);
    }
    if (!(xcol && lane >= 1)) xb = FaceBwd{};   // (lane 0 and columns past the east face)
    if (yown_r) {
      *gyp = gy_old + (double)sb.dz;
      if (CREST) A.gdzy2[d * SY + (size_t)(r + 1) * nx + col] = gy2_old + (double)sb.dz2;
    }
    if (xown) {
      *gxp = gx_old + (double)xb.dz;
      if (CREST) A.gdzx2[d * SX + (size_t)r * nxp1 + col] = gx2_old + (double)xb.dz2;
    }
    const FaceBwd xe = facebwd_shfl_down(xb);
    const ACell Ec = acell_shfl_down(Sc);
    // ---- each owned cell: its four faces' input adjoints (+ its ghosts'), the velocity map
    //      and the identity part of the flux update (phase 5 of k_adj_step) ----
    if (own) {
      const float W[8] = {xb.hl, xb.ul, xb.vl, xb.cl, xb.hr, xb.ur, xb.vr, xb.cr};
      const float E[8] = {xe.hl, xe.ul, xe.vl, xe.cl, xe.hr, xe.ur, xe.vr, xe.cr};
      const float Nf[8] = {nb.hl, nb.ul, nb.vl, nb.cl, nb.hr, nb.ur, nb.vr, nb.cr};
      const float Sf[8] = {sb.hl, sb.ul, sb.vl, sb.cl, sb.hr, sb.ur, sb.vr, sb.cr};
      float lh = W[4] + E[0] + Nf[4] + Sf[0];
      float lu = W[5] + E[1] + Nf[5] + Sf[1];
      float lv = W[6] + E[2] + Nf[6] + Sf[2];
      float lcc = W[7] + E[3] + Nf[7] + Sf[3];
      float gh = 0.0f, gqx = 0.0f, gqy = 0.0f;
      auto fold = [&](int code, const float* L, const ACell& G) {   // L: the ghost's (h, u, v, c) adjoints
        const float crit = code >= 3 ? sinf[code - 3].y : 0.0f;
        ghost_bwd(code, L[0], L[1], L[2], L[3], G.h, G.qx, G.qy, G.c, Sc.h, crit, k.g, k.heps2, gh, gqx, gqy);
      };
      if (col == 0) {
        const int code = A.bc[2 * nx + r];
        if (BND && code >= 2) fold(code, W, Wc);
        else { const float sg_ = code == 0 ? -1.0f : 1.0f; lh += W[0]; lu += sg_ * W[1]; lv += W[2]; lcc += W[3]; }
      }
      if (col == nx - 1) {
        const int code = A.bc[2 * nx + ny + r];
        if (BND && code >= 2) fold(code, E + 4, Ec);
        else { const float sg_ = code == 0 ? -1.0f : 1.0f; lh += E[4]; lu += sg_ * E[5]; lv += E[6]; lcc += E[7]; }
      }
      if (r == 0) {
        const int code = A.bc[col];
        if (BND && code >= 2) fold(code, Nf, Sb);
        else { const float sg_ = code == 0 ? -1.0f : 1.0f; lh += Nf[0]; lu += Nf[1]; lv += sg_ * Nf[2]; lcc += Nf[3]; }
      }
      if (r == ny - 1) {
        const int code = A.bc[nx + col];
        if (BND && code >= 2) fold(code, Sf + 4, Sd);
        else { const float sg_ = code == 0 ? -1.0f : 1.0f; lh += Sf[4]; lu += Sf[5]; lv += sg_ * Sf[6]; lcc += Sf[7]; }
      }
      // velocity map (numerics.rs:38-45): u = qx t(h), v = qy t(h), c = sqrt(g h)
      const float h = Sc.h, qx = Sc.qx, qy = Sc.qy, c = Sc.c;
      const float h2 = h * h, den = h2 + rmax(h2, k.heps2);
      const float t = (h + h) * rcp(den);
      const float dtdh = h2 > k.heps2 ? -1.0f / h2 : 2.0f * (k.heps2 - h2) / (den * den);
      const size_t gi = (size_t)r * nx + col;
      float oh = lh + (lu * qx + lv * qy) * dtdh + (c > 0.0f ? lcc * k.g * 0.5f / c : 0.0f) + lc.h;
      float oqx = lu * t + lc.qx, oqy = lv * t + lc.qy;
      if (BND) { oh += gh; oqx += gqx; oqy += gqy; }
      LO[gi] = oh;
      LO[N + gi] = oqx;
      LO[2 * N + gi] = oqy;
    }
    // shift the window one row down
    Sc = Sd; Sd = Snext;
    yc = yd; jyc = jyd; jyc2 = jyd2;
    jxc = jxd; jxc2 = jxd2;
    lc = ld;
    nb = sb;
  }
}

}  // namespace itr
