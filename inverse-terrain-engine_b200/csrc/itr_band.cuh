// itr_band.cuh — forward step for grids whose state lives in HBM: a row-band sweep.
//
// The design's state stays in the ping-pong planes of the tiled path (PlainArgs: H, QX, QY
// [2][nx*ny], running peaks PK), the integrator in its control block (PlainCtl, advanced by
// k_plain_finalize); only the per-step update differs from k_plain_update. It is the row
// sweep of the cluster kernel (itr_batched.cuh) and of the reference's fused CPU kernel
// (crates/itr-hydro/src/kernel.rs:637-697), laid out for a state that is read from HBM:
//   * a warp owns a segment of 64 columns of a band of kBandRows rows; lane l holds the two
//     adjacent columns 64 s + 2 l and 64 s + 2 l + 1, whose faces and cell updates run as
//     paired FP32 instructions (face2 / update_cell2), every value bit-identical to the
//     scalar arithmetic;
//   * each face is computed once: the west x-face of each column and the south y-face of
//     each row of the band, the north y-face of a row carried in registers from the row
//     above. The east face of a column is the next column's west face (own register or a
//     shuffle from lane + 1). The two x-faces on the segment's edges (columns 64 s and
//     64 s + 64) are computed by the warp for all rows of the band at once before the sweep
//     (one paired face per lane) and kept in shared memory, so no warp waits on another;
//     the only faces computed twice are those edges and the band's top y-face row:
//     (1 + 1/32) x (1 + 1/64) of the faces, against 1.27 for a 16x16 tile with an 18x18 halo;
//   * velocities and celerity of a cell are computed once per step, when its row is loaded;
//   * the old state is read-only during a step (ping-pong), so warps never synchronise with
//     each other inside a step: row r + 1 is loaded while row r is updated, and the only
//     block barrier is the final reduction of the per-block partials.
// Outputs are k_plain_update's: the new plane, PK (and the argmax state index tpk), the
// per-block partials [kPart] in the finalize's layout, and the atomic smax / bad words.
// TAPE: the adjoint's replay of a recorded step (itr_adjoint_band.cuh): the same update, writing
// only the new plane (no peaks, partials, CFL maximum, health word or row flags).
#pragma once
#include <cmath>
#include "itr_plain.cuh"
#include "itr_batched.cuh"

namespace itr {

constexpr int kBandRows = 32;    // most rows per band (= lanes: one pre-pass edge face per lane)
constexpr int kBandWarps = 4;    // warps (64-column segments) per block

struct BandGeom {
  int ns;      // 64-column segments per row
  int wpb;     // warps per block
  int rows;    // rows per band
  int gx, gy;  // blocks per design: segment groups x bands
};

__host__ __device__ inline BandGeom band_geom(int nx, int ny, int rows) {
  BandGeom b;
  b.ns = (nx + 63) / 64;
  b.wpb = b.ns < kBandWarps ? b.ns : kBandWarps;
  b.rows = rows;
  b.gx = (b.ns + b.wpb - 1) / b.wpb;
  b.gy = (ny + rows - 1) / rows;
  return b;
}

// Rows per band. Every warp sweeps one band segment, all warps about equally long, so a launch
// takes ceil(warps / resident) rounds of the SMs (12 warps resident per SM: 3 blocks of 4
// warps, the register budget at which nothing spills, measured 7-8 % faster than 4 blocks
// with spills). The chosen height maximises the busy fraction of those rounds times
// R / (R + 1), the share of y-faces computed once (each band recomputes its top y-face row).
inline int band_rows_for(int nx, int ny, int n_designs, int sm_count) {
  const double resident = 12.0 * (sm_count > 0 ? sm_count : 148);
  int best = kBandRows;
  double best_score = -1.0;
  for (int rows = kBandRows; rows >= 6; --rows) {
    const BandGeom b = band_geom(nx, ny, rows);
    const double warps = (double)n_designs * b.ns * b.gy;
    const double rounds = std::ceil(warps / resident);
    const double score = warps / (rounds * resident) * rows / (rows + 1.0);
    if (score > best_score + 1e-9) { best_score = score; best = rows; }
  }
  return best;
}

// Paired desingularised velocity and celerity (cell_vel on two cells).
ITR_DEV void vel2(float2 h, float2 qx, float2 qy, const StepK& k, float2& u, float2& v, float2& c) {
  const float NZ = k.nz;
  const float2 h2 = mul2(h, h, NZ);
  const float2 inv = rcp2f(add2(h2, max2(h2, f2(k.heps2))), k.exact);
  const float2 t = mul2(add2(h, h), inv, NZ);
  u = mul2(qx, t, NZ);
  v = mul2(qy, t, NZ);
  c = sqrt2(mul2(f2(k.g), h, NZ));
}

ITR_DEV Cell2 cells_of(float2 h, float2 qx, float2 qy, const StepK& k) {
  Cell2 r;
  r.h = h; r.qx = qx; r.qy = qy;
  vel2(h, qx, qy, k, r.u, r.v, r.c);
  return r;
}

// Old state of cell (r, c) of the design; c == nx gives the east ghost of (r, nx - 1), c == -1
// the west ghost of (r, 0), r == -1 / ny the north / south ghost of (0, c) / (ny - 1, c)
// (boundary.rs:36-87; BND: stage and inflow ghosts through ghost_state). Anything else
// outside the grid (lanes past the last column) is still water on a flat bed.
template <bool BND>
ITR_DEV void band_cell(const PlainArgs& A, const PlainDesign& D, const float2* inf, size_t plane, int r, int c, float& h,
                       float& qx, float& qy) {
  const int nx = A.nx, ny = A.ny;
  h = 0.0f; qx = 0.0f; qy = 0.0f;
  const bool gxw = c == -1, gxe = c == nx, gyn = r == -1, gys = r == ny;
  if (c < -1 || c > nx || r < -1 || r > ny || ((gxw || gxe) && (gyn || gys))) return;
  const int sr = gyn ? 0 : (gys ? ny - 1 : r), sc = gxw ? 0 : (gxe ? nx - 1 : c);
  const size_t i = plane + (size_t)sr * nx + sc;
  h = D.H[i]; qx = D.QX[i]; qy = D.QY[i];
  if (!(gxw || gxe || gyn || gys)) return;
  const int p = gxw ? 2 * nx + sr : gxe ? 2 * nx + ny + sr : gyn ? sc : nx + sc;
  const int code = A.bc[p];
  if (!BND) {
    if (code == 0) { if (gxw || gxe) qx = -qx; else qy = -qy; }
    return;
  }
  const float hs = code == 2 ? D.bh[p] : 0.0f;
  const float2 fi = code >= 3 ? inf[code - 3] : make_float2(0.0f, 0.0f);
  if (gxw || gxe) ghost_state<true>(code, h, qx, qy, hs, fi, gxw);
  else ghost_state<false>(code, h, qx, qy, hs, fi, gyn);
}

// Raw (not yet velocity-complemented) state of the lane's two cells of row r.
struct Raw2 { float2 h, qx, qy; };

template <bool BND>
ITR_DEV Raw2 band_row(const PlainArgs& A, const PlainDesign& D, const float2* inf, size_t plane, int r, int c0, bool interior) {
  Raw2 o;
  if (interior) {   // both columns inside the grid and r a grid row: plain loads
    const size_t i = plane + (size_t)r * A.nx + c0;
    if ((A.nx & 1) == 0) {   // even rows: the pair is 8-byte aligned (c0 and the plane size are even)
      o.h = *reinterpret_cast<const float2*>(D.H + i);
      o.qx = *reinterpret_cast<const float2*>(D.QX + i);
      o.qy = *reinterpret_cast<const float2*>(D.QY + i);
    } else {
      o.h = make_float2(D.H[i], D.H[i + 1]);
      o.qx = make_float2(D.QX[i], D.QX[i + 1]);
      o.qy = make_float2(D.QY[i], D.QY[i + 1]);
    }
    return o;
  }
  band_cell<BND>(A, D, inf, plane, r, c0, o.h.x, o.qx.x, o.qy.x);
  band_cell<BND>(A, D, inf, plane, r, c0 + 1, o.h.y, o.qx.y, o.qy.y);
  return o;
}

// Inputs of one row for the lane's two columns: south y-face jumps (face row r + 1), x-face
// jumps of row r + 1, wet and g n^2 of row r.
struct RowIn { float2 dys, dys2, dxn, dxn2, wet, gn2, pk; };

template <bool CREST, bool BND, bool TAPE = false>
__global__ void __launch_bounds__(kBandWarps * 32, 3) k_band(const PlainArgs A) {
  __shared__ float4 edge_w[kBandWarps][kBandRows], edge_e[kBandWarps][kBandRows];
  __shared__ float wmax[kBandWarps];
  __shared__ unsigned wbad[kBandWarps];
  __shared__ double wsum[kBandWarps][kPart];
  const int nblk = gridDim.x * gridDim.y;
  const PlainDesign D = plain_design(A, blockIdx.z, nblk);
  const PlainCtl& cl = *D.ctl;
  if (cl.done) return;
  const int par = cl.par;
  const StepK k = cl.k;
  const bool hits = cl.pl.hits;
  const double dt_dy = cl.pl.dt * A.P.dy;
  const int nx = A.nx, ny = A.ny, nxp1 = nx + 1;
  const size_t N = (size_t)nx * ny, plane = A.plane_stride ? A.plane_stride : N;
  const size_t pin = (size_t)par * plane, pout = (size_t)(par ^ 1) * plane;
  const float2* inf = cl.inf;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int ns = (nx + 63) / 64;
  const int s = blockIdx.x * wpb + wid;             // this warp's segment
  const int R = A.band_rows;                          // rows per band, <= kBandRows
  const int r0 = blockIdx.y * R;
  const int r1 = r0 + R < ny ? r0 + R : ny;
  const int L = r1 - r0;
  const int cw = 64 * s, ce = cw + 64;              // the segment's edge x-faces
  const int c0 = cw + 2 * lane, c1 = c0 + 1;
  const bool v0 = c0 < nx, v1 = c1 < nx;            // cells of the lane
  const bool interior = c1 < nx;                    // both columns are grid cells
  const bool vec = interior && (nx & 1) == 0;       // their pairs are 8-byte aligned in every plane
  const bool seg = s < ns;
  const bool last_seg = ce > nx;                    // the east domain edge lies inside this segment

  float smax_l = 0.0f;
  double infil_l = 0.0, fix_l = 0.0, acc_in = 0.0, acc_out = 0.0, vol = 0.0, ytop = 0.0, ybot = 0.0;
  bool bad_l = false;

  if (seg) {
    // Dry-row skipping (kernel.rs:605-612): with no rain this step, grid row r is skipped when
    // padded rows r, r + 1, r + 2 (grid rows r - 1, r, r + 1 and their ghosts) held no water
    // in the old state. Its faces are then exactly 0 and its cells keep their (zero) state, so
    // skipping changes no result. Bit p of skipm: grid row r0 + p; bit i of m: padded row r0 + i.
    unsigned long long skipm = 0ull;
    const unsigned* rw_old = D.rowwet ? D.rowwet + (size_t)par * (ny + 2) : nullptr;
    unsigned* rw_new = D.rowwet ? D.rowwet + (size_t)(par ^ 1) * (ny + 2) : nullptr;
    if (!TAPE && rw_old && A.P.skip_dry && !(k.rain > 0.0f)) {
      const int ja = r0 + lane, jb = r0 + 32 + lane;
      const bool da = ja <= ny + 1 && plain_row_dry(rw_old, D.gwet, ja);
      const bool db = lane < 2 && jb <= ny + 1 && plain_row_dry(rw_old, D.gwet, jb);
      const unsigned long long m =
          (unsigned long long)__ballot_sync(0xffffffffu, da) | ((unsigned long long)__ballot_sync(0xffffffffu, db) << 32);
      skipm = m & (m >> 1) & (m >> 2);
    }
    // Rows the sweep needs: row p is updated unless skipped, and its state and inputs are also
    // read for the next row's west faces; need(p) is false when rows p and p + 1 (or the band's
    // end) are both skipped, and then nothing of row p is loaded.
    auto skipped = [&](int p) -> bool { return p >= L || ((skipm >> p) & 1ull); };
    auto need = [&](int p) -> bool { return !(skipped(p) && skipped(p + 1)); };
    // ---- pre-pass: the segment's two edge x-faces of every row of the band (skipped rows:
    //      zero faces, which they are) ----
    {
      const int r = r0 + lane;
      Raw2 lf, rt;
      float2 d0 = f2(0.0f), d1 = f2(0.0f);
      if (r < r1 && !skipped(lane)) {
        band_cell<BND>(A, D, inf, pin, r, cw - 1, lf.h.x, lf.qx.x, lf.qy.x);
        band_cell<BND>(A, D, inf, pin, r, cw, rt.h.x, rt.qx.x, rt.qy.x);
        if (ce <= nx) {
          band_cell<BND>(A, D, inf, pin, r, ce - 1, lf.h.y, lf.qx.y, lf.qy.y);
          band_cell<BND>(A, D, inf, pin, r, ce, rt.h.y, rt.qx.y, rt.qy.y);
        } else {
          lf.h.y = lf.qx.y = lf.qy.y = rt.h.y = rt.qx.y = rt.qy.y = 0.0f;
        }
        const size_t xo = (size_t)r * nxp1;
        d0.x = D.dzx[xo + cw];
        d0.y = ce <= nx ? D.dzx[xo + ce] : 0.0f;
        if (CREST) { d1.x = D.dzx2[xo + cw]; d1.y = ce <= nx ? D.dzx2[xo + ce] : 0.0f; }
      } else {
        lf.h = lf.qx = lf.qy = rt.h = rt.qx = rt.qy = f2(0.0f);
      }
      const Cell2 a = cells_of(lf.h, lf.qx, lf.qy, k), b = cells_of(rt.h, rt.qx, rt.qy, k);
      const Face2 f = face2<true, CREST>(a.h, a.u, a.v, a.c, b.h, b.u, b.v, b.c, d0, d1, k);
      edge_w[wid][lane] = f4(fx_(f));
      edge_e[wid][lane] = f4(fy_(f));
      // x_boundary (kernel.rs:435-450): the west domain face of every row, per face
      if (!TAPE && s == 0 && r < r1) {
        const double vw = (double)f.m.x * dt_dy;
        if (vw > 0.0) acc_in += vw; else acc_out -= vw;
      }
      if (!TAPE && ce == nx && r < r1) {   // the east domain face is this segment's edge
        const double ve = (double)f.m.y * dt_dy;
        if (ve > 0.0) acc_out += ve; else acc_in -= ve;
      }
    }
    __syncwarp();

    // ---- row sweep ----
    const float* dzx = D.dzx + c0;
    const float* dzy = D.dzy + c0;
    auto load_in = [&](int r) -> RowIn {   // inputs of row r (r < r1)
      RowIn q;
      const int rn = r + 1 < ny ? r + 1 : ny - 1;   // next row's x-faces (unused for the last row)
      const size_t fy = (size_t)(r + 1) * nx, fx = (size_t)rn * nxp1, fc = (size_t)r * nx;
      q.dxn = make_float2(c0 <= nx ? dzx[fx] : 0.0f, c1 <= nx ? dzx[fx + 1] : 0.0f);
      q.dys2 = q.dxn2 = f2(0.0f);
      if (CREST) {
        q.dys2 = make_float2(v0 ? D.dzy2[c0 + fy] : 0.0f, v1 ? D.dzy2[c0 + fy + 1] : 0.0f);
        q.dxn2 = make_float2(c0 <= nx ? D.dzx2[c0 + fx] : 0.0f, c1 <= nx ? D.dzx2[c0 + fx + 1] : 0.0f);
      }
      const size_t ci = fc + c0;
      if (vec) {   // 8-byte aligned pairs (even nx, both columns in the grid)
        q.wet = *reinterpret_cast<const float2*>(A.wet + ci);
        q.gn2 = *reinterpret_cast<const float2*>(A.gn2 + ci);
        q.pk = TAPE ? f2(0.0f) : *reinterpret_cast<const float2*>(D.PK + ci);
        q.dys = *reinterpret_cast<const float2*>(dzy + fy);
      } else {
        q.dys = make_float2(v0 ? dzy[fy] : 0.0f, v1 ? dzy[fy + 1] : 0.0f);
        q.wet = make_float2(v0 ? A.wet[ci] : 0.0f, v1 ? A.wet[ci + 1] : 0.0f);
        q.gn2 = make_float2(v0 ? A.gn2[ci] : 0.0f, v1 ? A.gn2[ci + 1] : 0.0f);
        q.pk = TAPE ? f2(0.0f) : make_float2(v0 ? D.PK[ci] : 0.0f, v1 ? D.PK[ci + 1] : 0.0f);
      }
      return q;
    };
    auto xfaces = [&](const Cell2& c, float2 d, float2 d2, int p) -> Face2 {
      // west faces of the lane's two columns: (c0 - 1 | c0) and (c0 | c1); lane 0's first
      // one is the segment's west edge face from the pre-pass
      Cell2 left;
      left.h = make_float2(__shfl_up_sync(0xffffffffu, c.h.y, 1), c.h.x);
      left.u = make_float2(__shfl_up_sync(0xffffffffu, c.u.y, 1), c.u.x);
      left.v = make_float2(__shfl_up_sync(0xffffffffu, c.v.y, 1), c.v.x);
      left.c = make_float2(__shfl_up_sync(0xffffffffu, c.c.y, 1), c.c.x);
      left.qx = left.qy = f2(0.0f);
      Face2 f = face2<true, CREST>(left.h, left.u, left.v, left.c, c.h, c.u, c.v, c.c, d, d2, k);
      if (lane == 0) {
        const FaceF w = ff(edge_w[wid][p]);
        f.m.x = w.m; f.nl.x = w.nl; f.nr.x = w.nr; f.t.x = w.t;
      }
      return f;
    };
    // the row above the band (old state; the north ghost row at the domain edge) and row r0
    const bool int_lane = interior;
    Cell2 cur{}, nxt{};
    Face2 fN{}, fW{};
    if (!skipped(0)) {
      const Raw2 ta = band_row<BND>(A, D, inf, pin, r0 - 1, c0, int_lane && r0 > 0);
      const Raw2 ca = band_row<BND>(A, D, inf, pin, r0, c0, int_lane);
      const Cell2 top = cells_of(ta.h, ta.qx, ta.qy, k);
      cur = cells_of(ca.h, ca.qx, ca.qy, k);
      const size_t fy = (size_t)r0 * nx, fx = (size_t)r0 * nxp1;
      const float2 dy0 = make_float2(v0 ? dzy[fy] : 0.0f, v1 ? dzy[fy + 1] : 0.0f);
      const float2 dy1 = CREST ? make_float2(v0 ? D.dzy2[c0 + fy] : 0.0f, v1 ? D.dzy2[c0 + fy + 1] : 0.0f) : f2(0.0f);
      const float2 dx0 = make_float2(c0 <= nx ? dzx[fx] : 0.0f, c1 <= nx ? dzx[fx + 1] : 0.0f);
      const float2 dx1 = CREST ? make_float2(c0 <= nx ? D.dzx2[c0 + fx] : 0.0f, c1 <= nx ? D.dzx2[c0 + fx + 1] : 0.0f) : f2(0.0f);
      fN = face2<false, CREST>(top.h, top.u, top.v, top.c, cur.h, cur.u, cur.v, cur.c, dy0, dy1, k);
      fW = xfaces(cur, dx0, dx1, 0);
      if (!TAPE && r0 == 0) {   // y_boundary top (kernel.rs:452-472): summed over the row first
        ytop += (v0 ? (double)fN.m.x : 0.0) + (v1 ? (double)fN.m.y : 0.0);
      }
    }
    RowIn in{};
    Raw2 raw{};
    if (need(0)) {
      in = load_in(r0);
      raw = band_row<BND>(A, D, inf, pin, r0 + 1, c0, int_lane && r0 + 1 < ny);
    }
#pragma unroll 1
    for (int p = 0; p < L; ++p) {
      const int r = r0 + p;
      const RowIn q = in;
      const bool skip = skipped(p);
      if (need(p)) nxt = cells_of(raw.h, raw.qx, raw.qy, k);
      if (p + 1 < L && need(p + 1)) {   // next row's operands, in flight while this row is updated
        in = load_in(r + 1);
        raw = band_row<BND>(A, D, inf, pin, r + 2, c0, int_lane && r + 2 < ny);
      }
      Face2 fWn{};
      if (!skipped(p + 1)) fWn = xfaces(nxt, q.dxn, q.dxn2, p + 1);
      if (skip) {   // a dry row between dry rows: zero faces, the (zero) state carried over
        const size_t ci = (size_t)r * nx + c0;
        if (vec) {
          *reinterpret_cast<float2*>(D.H + pout + ci) = f2(0.0f);
          *reinterpret_cast<float2*>(D.QX + pout + ci) = f2(0.0f);
          *reinterpret_cast<float2*>(D.QY + pout + ci) = f2(0.0f);
        } else {
          if (v0) { D.H[pout + ci] = 0.0f; D.QX[pout + ci] = 0.0f; D.QY[pout + ci] = 0.0f; }
          if (v1) { D.H[pout + ci + 1] = 0.0f; D.QX[pout + ci + 1] = 0.0f; D.QY[pout + ci + 1] = 0.0f; }
        }
        cur = nxt; fN = Face2{}; fW = fWn;
        continue;
      }
      const Face2 fS = face2<false, CREST>(cur.h, cur.u, cur.v, cur.c, nxt.h, nxt.u, nxt.v, nxt.c, q.dys, q.dys2, k);
      // east faces: the second column's west face, and lane + 1's first (lane 31: the edge)
      Face2 fE;
      fE.m.x = fW.m.y; fE.nl.x = fW.nl.y; fE.nr.x = fW.nr.y; fE.t.x = fW.t.y;
      fE.m.y = __shfl_down_sync(0xffffffffu, fW.m.x, 1);
      fE.nl.y = __shfl_down_sync(0xffffffffu, fW.nl.x, 1);
      fE.nr.y = __shfl_down_sync(0xffffffffu, fW.nr.x, 1);
      fE.t.y = __shfl_down_sync(0xffffffffu, fW.t.x, 1);
      if (lane == 31) {
        const FaceF e = ff(edge_e[wid][p]);
        fE.m.y = e.m; fE.nl.y = e.nl; fE.nr.y = e.nr; fE.t.y = e.t;
      }
      const CellNew2 o = update_cell2(cur.h, cur.qx, cur.qy, fW, fE, fN, fS, q.wet, q.gn2, k);
      const size_t ci = (size_t)r * nx + c0;
      if (vec) {
        *reinterpret_cast<float2*>(D.H + pout + ci) = o.h;
        *reinterpret_cast<float2*>(D.QX + pout + ci) = o.qx;
        *reinterpret_cast<float2*>(D.QY + pout + ci) = o.qy;
      } else {
        if (v0) { D.H[pout + ci] = o.h.x; D.QX[pout + ci] = o.qx.x; D.QY[pout + ci] = o.qy.x; }
        if (v1) { D.H[pout + ci + 1] = o.h.y; D.QX[pout + ci + 1] = o.qx.y; D.QY[pout + ci + 1] = o.qy.y; }
      }
      if constexpr (!TAPE) {
        if (v0) {
          if (o.h.x > q.pk.x) { D.PK[ci] = o.h.x; if (D.tpk) D.tpk[ci] = (unsigned)(cl.step + 1); }
          smax_l = rmax(smax_l, o.s.x);
          bad_l = bad_l || o.bad.x;
        }
        if (v1) {
          if (o.h.y > q.pk.y) { D.PK[ci + 1] = o.h.y; if (D.tpk) D.tpk[ci + 1] = (unsigned)(cl.step + 1); }
          smax_l = rmax(smax_l, o.s.y);
          bad_l = bad_l || o.bad.y;
        }
        // row partials: f32 over the lane's pair, f64 across rows
        infil_l += (double)((v0 ? o.infil.x : 0.0f) + (v1 ? o.infil.y : 0.0f));
        fix_l += (double)((v0 ? o.fix.x : 0.0f) + (v1 ? o.fix.y : 0.0f));
        if (hits) vol += (v0 ? (double)o.h.x : 0.0) + (v1 ? (double)o.h.y : 0.0);
        if (last_seg) {   // x_boundary: the east domain face inside this segment (kernel.rs:435-450)
          if (c0 == nx - 1) { const double ve = (double)fE.m.x * dt_dy; if (ve > 0.0) acc_out += ve; else acc_in -= ve; }
          if (c1 == nx - 1) { const double ve = (double)fE.m.y * dt_dy; if (ve > 0.0) acc_out += ve; else acc_in -= ve; }
        }
        if (r == ny - 1) ybot += (v0 ? (double)fS.m.x : 0.0) + (v1 ? (double)fS.m.y : 0.0);
        if (rw_new && __any_sync(0xffffffffu, (v0 && o.h.x > 0.0f) || (v1 && o.h.y > 0.0f)) && lane == 0)
          rw_new[r + 1] = 1u;   // the row holds water in the new state (every writer stores 1)
      }
      cur = nxt; fN = fS; fW = fWn;
    }
  }
  if constexpr (TAPE) return;
  // ---- block reduction into the finalize's partials (fixed order) ----
  const float m = warp_max_f(smax_l);
  const unsigned b = __any_sync(0xffffffffu, bad_l) ? 1u : 0u;
  double acc[kPart] = {infil_l, fix_l, acc_in, acc_out, vol, ytop, ybot};
#pragma unroll
  for (int j = 0; j < kPart; ++j) acc[j] = warp_sum_d(acc[j]);
  if (lane == 0) {
    wmax[wid] = m; wbad[wid] = b;
    for (int j = 0; j < kPart; ++j) wsum[wid][j] = acc[j];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float mm = 0.0f; unsigned bb = 0u; double ss[kPart] = {0, 0, 0, 0, 0, 0, 0};
    for (int w = 0; w < wpb; ++w) { mm = rmax(mm, wmax[w]); bb |= wbad[w]; for (int j = 0; j < kPart; ++j) ss[j] += wsum[w][j]; }
    if (mm > 0.0f) atomicMax(&D.ctl->smax_bits, __float_as_uint(mm));
    if (bb) atomicOr(&D.ctl->bad, 1u);
    double* pp = D.part + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * kPart;
    for (int j = 0; j < kPart; ++j) pp[j] = ss[j];
  }
}

}  // namespace itr
