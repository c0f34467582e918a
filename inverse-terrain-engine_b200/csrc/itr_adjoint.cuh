// itr_adjoint.cuh — reverse-mode derivative (vector-Jacobian product) of the forward step.
//
// The reference has no adjoint (its optimisers are derivative-free). For J = sum_k w_k tau
// softplus((P_k - eta_k)/tau) (objective.rs:95-128), with P_k the largest running-max depth
// over asset k's monitored cells, it gives dJ/d(face jump) for every x- and y-face of every
// design: dJ/ddzx[r][f] and dJ/ddzy[f][c] (the arrays the forward takes, shader.wgsl:25-26).
//
// Method (discrete adjoint of the f32 step, f32 adjoint state, f64 gradient sums):
//   * the forward runs on the tiled path and records, per design, (dt, rain) of every step,
//     the state every K steps (checkpoints) and, per cell, which state last raised the
//     running max (the argmax of the max-over-time term);
//   * per segment of K steps, last segment first, the states are recomputed from the
//     segment's checkpoint (k_adj_replay, bit-identical to the forward step) into a tape,
//     then stepped backwards (k_adj_step): lambda_n = (dF/dx_n)^T lambda_{n+1}, and
//     g_dz += (dF/ddz)^T lambda_{n+1}; the peak term adds w_k sigmoid((P_k - eta_k)/tau) to
//     lambda_h of the argmax cell at the argmax state;
//   * the time step sequence is held fixed (dt_n, rain_n as recorded): the derivative of the
//     discrete map with frozen dt, the usual treatment of an adaptive step;
//   * every branch (wet/dry, HLL upwinding, min/max of wave speeds, reconstruction clamps,
//     infiltration cap, drying, q_min flush) takes the derivative of the side the forward
//     took; sqrt(g h) has derivative 0 at h = 0; rcbrt(h) is differentiated as h^(-1/3).
// Stage and inflow ghosts: the replay rebuilds them as the forward did (the step's start
// time is on the tape); their adjoint folds back onto the interior cell through what the
// ghost copies (a stage ghost's momentum, an inflow ghost's depth where it exceeds the
// critical depth). The stage depths themselves (stage - z behind the edge) are held fixed:
// the gradient is the one with respect to the face jumps alone.
// Crest faces (coarse fidelity levels): two jumps per face, d_l and d_r, each side reduced by
// its own jump; the gradient comes in both jump arrays.
#pragma once
#include "itr_plain.cuh"

namespace itr {

struct AdjArgs {
  RunParams P;
  int nx, ny, n_designs;
  const float* wet;
  const float* gn2;
  const uint8_t* bc;                  // device codes (ghost_state)
  const float* bh;                    // stage-ghost depths per design [2 nx + 2 ny], or NULL
  const float* dzx;                   // all designs, as the forward
  const float* dzy;
  const float* dzx2;                  // crest mode: the second jumps, else NULL
  const float* dzy2;
  const unsigned long long* n_steps;  // per design: steps of the forward run
  const double* seg;                  // per design [K][3]: (dt, rain, t) of this segment's steps
  int K;
  unsigned long long step0;           // global index of the segment's first step
  const float* tape;                  // [K][n_designs][3][N]: state at step step0 + j
  const float* lin;                   // per design [3][N]: adjoint of the state after the step
  float* lout;                        // per design [3][N]: adjoint of the state before it
  double* gdzx;                       // per design ny*(nx+1)
  double* gdzy;                       // per design (ny+1)*nx
  double* gdzx2;                      // crest mode: gradients of the second jumps
  double* gdzy2;
  const unsigned* seed_cell;          // per design max_seeds: argmax cell of an asset
  const unsigned* seed_state;         //   the state index at which it peaked
  const float* seed_w;                //   w_k sigmoid((P_k - eta_k) / tau)
  const int* seed_n;                  // per design
  int max_seeds;
  int band_rows;                      // k_adj_band: rows per band (1 .. 32)
};

// Padded cell (gx, gy) of a state [3][N] with ghost cells (boundary.rs:36-87), as plain_load:
// bh = this design's stage depths, inf = the step's inflow group values (BND only).
template <bool BND>
ITR_DEV void adj_load(const AdjArgs& A, const float* X, int gx, int gy, float& h, float& qx, float& qy, const float* bh,
                      const float2* inf) {
  const int nx = A.nx, ny = A.ny;
  const size_t N = (size_t)nx * ny;
  const bool ox = gx < 0 || gx >= nx, oy = gy < 0 || gy >= ny;
  if (ox && oy) { h = 0.0f; qx = 0.0f; qy = 0.0f; return; }
  const int sx = gx < 0 ? 0 : (gx >= nx ? nx - 1 : gx);
  const int sy = gy < 0 ? 0 : (gy >= ny ? ny - 1 : gy);
  const size_t i = (size_t)sy * nx + sx;
  h = X[i]; qx = X[N + i]; qy = X[2 * N + i];
  if (!BND) {
    if (ox) { const int code = gx < 0 ? A.bc[2 * nx + sy] : A.bc[2 * nx + ny + sy]; if (code == 0) qx = -qx; }
    else if (oy) { const int code = gy < 0 ? A.bc[sx] : A.bc[nx + sx]; if (code == 0) qy = -qy; }
  } else if (ox || oy) {
    const int p = ox ? (gx < 0 ? 2 * nx + sy : 2 * nx + ny + sy) : (gy < 0 ? sx : nx + sx);
    const int code = A.bc[p];
    const float hs = code == 2 ? bh[p] : 0.0f;
    const float2 fi = code >= 3 ? inf[code - 3] : make_float2(0.0f, 0.0f);
    if (ox) ghost_state<true>(code, h, qx, qy, hs, fi, gx < 0);
    else ghost_state<false>(code, h, qx, qy, hs, fi, gy < 0);
  }
}

// Inflow group values of a step at its start time t, into shared memory (BND only).
template <bool BND>
ITR_DEV void adj_inflow(const AdjArgs& A, double t, float2* inf) {
  if (BND) {
    if ((int)threadIdx.x < A.P.inflow.n) inf[threadIdx.x] = inflow_values(A.P.inflow, threadIdx.x, t, A.P.g);
    __syncthreads();
  }
}

// Adjoint of a stage or inflow ghost folded onto the interior cell behind it. (lh, lu, lv,
// lc): adjoints of the ghost's (h, u, v, c) from its face; (hg, qxg, qyg, cg): the ghost's
// state; hi: the interior depth; crit: the group's critical depth (inflow). A stage ghost
// copies the momentum (u = qx t(hg), v = qy t(hg) with hg fixed); an inflow ghost's depth
// max(hi, crit) follows hi where hi > crit, its discharge is fixed. Adds to the interior
// cell's (h, qx, qy) adjoints.
ITR_DEV void ghost_bwd(int code, float lh, float lu, float lv, float lc, float hg, float qxg, float qyg, float cg, float hi,
                       float crit, float g, float heps2, float& ah, float& aqx, float& aqy) {
  const float h2 = hg * hg, den = h2 + rmax(h2, heps2);
  if (code == 2) {
    const float t = (hg + hg) * rcp(den);
    aqx += lu * t;
    aqy += lv * t;
  } else if (hi > crit) {
    const float dtdh = h2 > heps2 ? -1.0f / h2 : 2.0f * (heps2 - h2) / (den * den);
    ah += lh + (lu * qxg + lv * qyg) * dtdh + (cg > 0.0f ? lc * g * 0.5f / cg : 0.0f);
  }
}

// ---- forward replay: x_{n+1} = F(x_n) with the recorded (dt, rain) ----
template <bool BND, bool CREST>
__global__ void __launch_bounds__(kTileThreads, 6) k_adj_replay(const AdjArgs A, int j) {
  __shared__ float sh[18 * 18], su[18 * 18], sv[18 * 18], sc[18 * 18], sqx[18 * 18], sqy[18 * 18];
  __shared__ FaceF fx[16 * 17], fy[17 * 16];
  __shared__ float2 sinf[kMaxInflow];
  const int d = blockIdx.z;
  if (A.step0 + j >= A.n_steps[d]) return;
  const int nx = A.nx, ny = A.ny;
  const size_t N = (size_t)nx * ny, SX = (size_t)ny * (nx + 1), SY = (size_t)(ny + 1) * nx;
  const float* X = A.tape + ((size_t)j * A.n_designs + d) * 3 * N;
  float* Y = const_cast<float*>(A.tape) + ((size_t)(j + 1) * A.n_designs + d) * 3 * N;
  const double* sg = A.seg + ((size_t)d * A.K + j) * 3;
  const StepK k = step_consts(A.P, sg[0], sg[1]);
  const float* dzx = A.dzx + d * SX;
  const float* dzy = A.dzy + d * SY;
  const float* dzx2 = CREST ? A.dzx2 + d * SX : nullptr;
  const float* dzy2 = CREST ? A.dzy2 + d * SY : nullptr;
  const float* bh = BND && A.bh ? A.bh + (size_t)d * (2 * nx + 2 * ny) : nullptr;
  adj_inflow<BND>(A, sg[2], sinf);
  const int gx0 = blockIdx.x * kTile, gy0 = blockIdx.y * kTile;
  const int li = threadIdx.x;
  // global loads first (face jumps, wet / g n^2, halo), as k_plain_update
  const int fxr = li / 17, fxcol = li % 17, fyr_ = li / 16, fycol = li % 16;
  const bool xv = li < 272 && gy0 + fxr < ny && gx0 + fxcol <= nx;
  const bool yv = li < 272 && gx0 + fycol < nx && gy0 + fyr_ <= ny;
  const size_t xo = (size_t)(gy0 + fxr) * (nx + 1) + gx0 + fxcol;
  const size_t yo = (size_t)(gy0 + fyr_) * nx + gx0 + fycol;
  const float xd = xv ? dzx[xo] : 0.0f, yd = yv ? dzy[yo] : 0.0f;
  const float xd2 = (CREST && xv) ? dzx2[xo] : 0.0f, yd2 = (CREST && yv) ? dzy2[yo] : 0.0f;
  const int lx = li % 16, ly = li / 16, gx = gx0 + lx, gy = gy0 + ly;
  const bool cv = li < 256 && gx < nx && gy < ny;
  const size_t gi = (size_t)gy * nx + gx;
  const float wet_c = cv ? A.wet[gi] : 0.0f, gn2_c = cv ? A.gn2[gi] : 0.0f;
  for (int e = li; e < 324; e += kTileThreads) {
    const int hx = e % 18, hy = e / 18;
    float h, qx, qy, u, v, c;
    adj_load<BND>(A, X, gx0 - 1 + hx, gy0 - 1 + hy, h, qx, qy, bh, sinf);
    cell_vel(h, qx, qy, k.g, k.heps2, u, v, c);
    sh[e] = h; sqx[e] = qx; sqy[e] = qy; su[e] = u; sv[e] = v; sc[e] = c;
  }
  __syncthreads();
  if (xv) {
    const int a = (fxr + 1) * 18 + fxcol;
    fx[li] = face<true, CREST>(sh[a], su[a], sv[a], sc[a], sh[a + 1], su[a + 1], sv[a + 1], sc[a + 1], xd, xd2, k);
  }
  if (yv) {
    const int a = fyr_ * 18 + fycol + 1, b = a + 18;
    fy[li] = face<false, CREST>(sh[a], su[a], sv[a], sc[a], sh[b], su[b], sv[b], sc[b], yd, yd2, k);
  }
  __syncthreads();
  if (cv) {
    const int a = (ly + 1) * 18 + lx + 1;
    const CellNew o = update_cell(sh[a], sqx[a], sqy[a], fx[ly * 17 + lx], fx[ly * 17 + lx + 1], fy[ly * 16 + lx],
                                  fy[(ly + 1) * 16 + lx], wet_c, gn2_c, k);
    Y[gi] = o.h; Y[N + gi] = o.qx; Y[2 * N + gi] = o.qy;
  }
}

// ---- adjoints of the pieces of one step ----

// Input adjoints of face_signed / face_crest + hll (numerics.rs:60-129) given the output
// adjoints. dz: the (first) jump's adjoint; dz2: the crest face's second jump's.
struct FaceBwd { float hl, ul, vl, cl, hr, ur, vr, cr, dz, dz2; };

template <bool NORMAL_X, bool CREST>
ITR_DEV FaceBwd face_bwd(float hl, float ul, float vl, float cl, float hr, float ur, float vr, float cr, float dz,
                         float dz2, const StepK& k, float lm, float lnl, float lnr, float lt) {
  // forward, as face_signed / face_crest and hll compute it
  const bool pos = dz > 0.0f;
  const float a_l = CREST ? hl - dz : hl - rmax(dz, 0.0f), a_r = CREST ? hr - dz2 : hr - rmax(-dz, 0.0f);
  const float hsl = rmax(a_l, 0.0f), hsr = rmax(a_r, 0.0f);
  const float hred = pos ? hsl : hsr;
  const float cred = CREST ? 0.0f : sqrt_rn(k.g * hred);
  const float csl_c = (CREST && dz > 0.0f) ? sqrt_rn(k.g * hsl) : cl;
  const float csr_c = (CREST && dz2 > 0.0f) ? sqrt_rn(k.g * hsr) : cr;
  const float csl = CREST ? csl_c : (pos ? cred : cl), csr = CREST ? csr_c : (pos ? cr : cred);
  const float unl = NORMAL_X ? ul : vl, utl = NORMAL_X ? vl : ul;
  const float unr = NORMAL_X ? ur : vr, utr = NORMAL_X ? vr : ur;
  const bool dry_l = !(hsl > 0.0f), dry_r = !(hsr > 0.0f);
  const float ustar = 0.5f * (unl + unr) + csl - csr;
  const float cstar = 0.5f * (csl + csr) + 0.25f * (unl - unr);
  const float A1 = unl - csl, A2 = ustar - cstar, B1 = unr + csr, B2 = ustar + cstar;
  const float slw = rmin(A1, A2), srw = rmax(B1, B2);
  const float sl = dry_l ? unr - 2.0f * csr : (dry_r ? unl - csl : slw);
  const float sr = dry_l ? unr + csr : (dry_r ? unl + 2.0f * csl : srw);
  const float ml = hsl * unl, mr = hsr * unr;
  const float pl_ = k.g_half * hsl * hsl, pr_ = k.g_half * hsr * hsr;
  const float pl = ml * unl + pl_, pr = mr * unr + pr_;
  const bool both = dry_l && dry_r, use_l = sl >= 0.0f, use_r = sr <= 0.0f;
  const float den = (both || use_l || use_r) ? 1.0f : sr - sl;
  const float inv = rcp(den);
  const float F1 = sr * ml - sl * mr + sl * sr * (hsr - hsl);
  const float F2 = sr * pl - sl * pr + sl * sr * (mr - ml);
  const float fm = both ? 0.0f : (use_l ? ml : (use_r ? mr : F1 * inv));
  // reverse
  float lunl = 0, lutl = 0, lunr = 0, lutr = 0, lcsl = 0, lcsr = 0, lhsl = 0, lhsr = 0;
  float lml = 0, lmr = 0, lpl = 0, lpr = 0, lsl = 0, lsr = 0;
  const bool tpos = fm > 0.0f;
  const float lfm = lm + lt * (tpos ? utl : utr);
  if (tpos) lutl += lt * fm; else lutr += lt * fm;
  const float lfn = lnl + lnr;
  float lpl_ = -lnl, lpr_ = -lnr;
  if (!both) {
    if (use_l) { lml += lfm; lpl += lfn; }
    else if (use_r) { lmr += lfm; lpr += lfn; }
    else {
      const float lF1 = lfm * inv, lF2 = lfn * inv;
      const float linv = lfm * F1 + lfn * F2;
      const float lden = -linv * inv * inv;
      lsr += lden; lsl -= lden;
      lsr += lF1 * (ml + sl * (hsr - hsl)); lml += lF1 * sr; lsl += lF1 * (-mr + sr * (hsr - hsl)); lmr -= lF1 * sl;
      lhsr += lF1 * sl * sr; lhsl -= lF1 * sl * sr;
      lsr += lF2 * (pl + sl * (mr - ml)); lpl += lF2 * sr; lsl += lF2 * (-pr + sr * (mr - ml)); lpr -= lF2 * sl;
      lmr += lF2 * sl * sr; lml -= lF2 * sl * sr;
    }
  }
  lml += lpl * unl; lunl += lpl * ml; lpl_ += lpl;
  lmr += lpr * unr; lunr += lpr * mr; lpr_ += lpr;
  lhsl += lpl_ * 2.0f * k.g_half * hsl; lhsr += lpr_ * 2.0f * k.g_half * hsr;
  lhsl += lml * unl; lunl += lml * hsl;
  lhsr += lmr * unr; lunr += lmr * hsr;
  if (dry_l) { lunr += lsl; lcsr -= 2.0f * lsl; lunr += lsr; lcsr += lsr; }
  else if (dry_r) { lunl += lsl; lcsl -= lsl; lunl += lsr; lcsl += 2.0f * lsr; }
  else {
    float lA1 = 0, lA2 = 0, lB1 = 0, lB2 = 0;
    if (A1 < A2) lA1 = lsl; else lA2 = lsl;
    if (B1 > B2) lB1 = lsr; else lB2 = lsr;
    lunl += lA1; lcsl -= lA1;
    lunr += lB1; lcsr += lB1;
    const float lus = lA2 + lB2, lcs = lB2 - lA2;
    lunl += 0.5f * lus; lunr += 0.5f * lus; lcsl += lus; lcsr -= lus;
    lcsl += 0.5f * lcs; lcsr += 0.5f * lcs; lunl += 0.25f * lcs; lunr -= 0.25f * lcs;
  }
  FaceBwd b;
  b.cl = 0.0f; b.cr = 0.0f;
  if (CREST) {   // each side's celerity is its reduced depth's where its jump is positive
    if (dz > 0.0f) { if (csl > 0.0f) lhsl += lcsl * k.g * 0.5f / csl; } else b.cl = lcsl;
    if (dz2 > 0.0f) { if (csr > 0.0f) lhsr += lcsr * k.g * 0.5f / csr; } else b.cr = lcsr;
  } else {
    float lcred = 0.0f;
    if (pos) { lcred += lcsl; b.cr = lcsr; } else { b.cl = lcsl; lcred += lcsr; }
    const float lhred = cred > 0.0f ? lcred * k.g * 0.5f / cred : 0.0f;
    if (pos) lhsl += lhred; else lhsr += lhred;
  }
  const float la_l = a_l > 0.0f ? lhsl : 0.0f, la_r = a_r > 0.0f ? lhsr : 0.0f;
  b.hl = la_l; b.hr = la_r;
  if (CREST) { b.dz = -la_l; b.dz2 = -la_r; }
  else { b.dz = (dz > 0.0f ? -la_l : 0.0f) + (dz < 0.0f ? la_r : 0.0f); b.dz2 = 0.0f; }
  b.ul = NORMAL_X ? lunl : lutl; b.vl = NORMAL_X ? lutl : lunl;
  b.ur = NORMAL_X ? lunr : lutr; b.vr = NORMAL_X ? lutr : lunr;
  return b;
}

// Adjoint of the sources (numerics.rs:158-194): from the adjoint of the new (h, qx, qy) to
// that of (h1, qx1, qy1) after the flux update, recomputing the forward as update_cell does.
ITR_DEV void sources_bwd(float h, float qx, float qy, const FaceF& w, const FaceF& e, const FaceF& n, const FaceF& s,
                         float wet, float gn2, const StepK& k, float lh, float lqx, float lqy,
                         float& l1h, float& l1qx, float& l1qy) {
  const float h1 = h - k.dtdx * (e.m - w.m) - k.dtdy * (s.m - n.m);
  const float qx1 = qx - k.dtdx * (e.nl - w.nr) - k.dtdy * (s.t - n.t);
  const float qy1 = qy - k.dtdx * (e.t - w.t) - k.dtdy * (s.nl - n.nr);
  const float h1c = h1 < 0.0f ? 0.0f : h1;
  const float h2 = h1c + k.rain * wet;
  const float capw = k.cap * wet;
  const float h3 = h2 - rmin(capw, h2);
  const bool dry = h3 < k.h_dry;
  const float r = rcbrt(dry ? 1.0f : h3);
  const float r3 = r * r * r;
  const float r7 = r3 * r3 * r;
  const float qm = sqrt_rn(qx1 * qx1 + qy1 * qy1);
  const float a = k.dt * gn2;
  const float inv = rcp(1.0f + a * qm * r7);
  float lh3 = lh;
  l1qx = 0.0f; l1qy = 0.0f;
  if (!dry) {
    const float qx2 = qx1 * inv, qy2 = qy1 * inv;
    const float lqxe = rabs(qx2) < k.q_min ? 0.0f : lqx;   // q_min flush: constant 0
    const float lqye = rabs(qy2) < k.q_min ? 0.0f : lqy;
    l1qx = lqxe * inv; l1qy = lqye * inv;
    const float linv = lqxe * qx1 + lqye * qy1;
    const float lD = -linv * inv * inv;
    const float lqm = lD * a * r7;
    const float lr7 = lD * a * qm;
    lh3 += lr7 * (-7.0f / 3.0f) * r7 * r3;                  // d h^(-7/3) / dh
    if (qm > 0.0f) { l1qx += lqm * qx1 / qm; l1qy += lqm * qy1 / qm; }
  }
  const float lh2 = capw < h2 ? lh3 : 0.0f;                // infiltration capped at h2 -> h3 = 0
  l1h = h1 < 0.0f ? 0.0f : lh2;                            // positivity fix
}

// ---- the backward step ----
// One 16x16 tile of one design per block. The state is loaded with a 2-cell halo (20x20),
// forward faces are computed for the 18x18 cells around the tile, their source adjoints
// give the face adjoints of every face touching a tile cell, and each tile cell gathers its
// four faces' input adjoints (ghost sides folded back onto the interior cell).
constexpr int kR = 20, kQ = 18;

template <bool BND, bool CREST>
__global__ void __launch_bounds__(kTileThreads) k_adj_step(const AdjArgs A, int j) {
  __shared__ float sh[kR * kR], sqx[kR * kR], sqy[kR * kR], su[kR * kR], sv[kR * kR], sc[kR * kR];
  __shared__ FaceF fx[kQ * 19], fy[19 * kQ];           // forward faces of the 18x18 cells
  __shared__ float jx[kQ * 19], jy[19 * kQ];            // their jumps
  __shared__ float jx2[CREST ? kQ * 19 : 1], jy2[CREST ? 19 * kQ : 1];   // crest: second jumps
  __shared__ float l1[3][kQ * kQ];                      // adjoint of (h1, qx1, qy1)
  __shared__ float bx[16 * 17][8], by[17 * 16][8];      // face input adjoints: L (h,u,v,c), R (h,u,v,c)
  __shared__ float2 sinf[kMaxInflow];                   // the step's inflow group values
  const int d = blockIdx.z;
  const int nx = A.nx, ny = A.ny;
  const size_t N = (size_t)nx * ny, SX = (size_t)ny * (nx + 1), SY = (size_t)(ny + 1) * nx;
  const unsigned long long n = A.step0 + j;
  const float* LI = A.lin + (size_t)d * 3 * N;
  float* LO = A.lout + (size_t)d * 3 * N;
  const int gx0 = blockIdx.x * kTile, gy0 = blockIdx.y * kTile;
  const int li = threadIdx.x;
  if (n >= A.n_steps[d]) {   // the design stopped before this step: the adjoint passes through
    const int gx = gx0 + li % 16, gy = gy0 + li / 16;
    if (li < 256 && gx < nx && gy < ny) {
      const size_t gi = (size_t)gy * nx + gx;
      LO[gi] = LI[gi]; LO[N + gi] = LI[N + gi]; LO[2 * N + gi] = LI[2 * N + gi];
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
  // 1. state and velocities of the 20x20 region; the face jumps and this thread's old
  //    gradient sums are loaded first, so all these loads are in flight together
  float jxa = 0.0f, jxb = 0.0f, jya = 0.0f, jyb = 0.0f;
  const int e2 = li + kTileThreads;
  auto xjump = [&](const float* a, int e) -> float {
    const int jr = e / 19, fi = e % 19, row = gy0 - 1 + jr, f = gx0 - 1 + fi;
    return (row >= 0 && row < ny && f >= 0 && f <= nx) ? a[(size_t)row * (nx + 1) + f] : 0.0f;
  };
  auto yjump = [&](const float* a, int e) -> float {
    const int fr = e / kQ, ic = e % kQ, col = gx0 - 1 + ic, f = gy0 - 1 + fr;
    return (col >= 0 && col < nx && f >= 0 && f <= ny) ? a[(size_t)f * nx + col] : 0.0f;
  };
  jxa = xjump(dzx, li); jya = yjump(dzy, li);
  if (e2 < kQ * 19) { jxb = xjump(dzx, e2); jyb = yjump(dzy, e2); }
  float jx2a = 0.0f, jx2b = 0.0f, jy2a = 0.0f, jy2b = 0.0f;
  if (CREST) {
    jx2a = xjump(dzx2, li); jy2a = yjump(dzy2, li);
    if (e2 < kQ * 19) { jx2b = xjump(dzx2, e2); jy2b = yjump(dzy2, e2); }
  }
  // the faces this thread differentiates in step 4 and whether its tile owns them
  const int yr4 = li / 17 + 1, xl4 = li % 17 + 1, yt4 = li / 16 + 1, xc4 = li % 16 + 1;
  const int row4 = gy0 - 1 + yr4, fx4 = gx0 - 1 + xl4, col4 = gx0 - 1 + xc4, fy4 = gy0 - 1 + yt4;
  const bool xown = li < 272 && row4 < ny && fx4 <= nx && (fx4 < gx0 + kTile || fx4 == nx);
  const bool yown = li < 272 && col4 < nx && fy4 <= ny && (fy4 < gy0 + kTile || fy4 == ny);
  double* gxp = A.gdzx + d * SX + (size_t)row4 * (nx + 1) + fx4;
  double* gyp = A.gdzy + d * SY + (size_t)fy4 * nx + col4;
  const double gx_old = xown ? *gxp : 0.0, gy_old = yown ? *gyp : 0.0;
  double* gxp2 = CREST ? A.gdzx2 + d * SX + (size_t)row4 * (nx + 1) + fx4 : nullptr;
  double* gyp2 = CREST ? A.gdzy2 + d * SY + (size_t)fy4 * nx + col4 : nullptr;
  const double gx2_old = (CREST && xown) ? *gxp2 : 0.0, gy2_old = (CREST && yown) ? *gyp2 : 0.0;
  for (int e = li; e < kR * kR; e += kTileThreads) {
    const int ix = e % kR, iy = e / kR;
    float h, qx, qy, u, v, c;
    adj_load<BND>(A, X, gx0 - 2 + ix, gy0 - 2 + iy, h, qx, qy, bh, sinf);
    cell_vel(h, qx, qy, k.g, k.heps2, u, v, c);
    sh[e] = h; sqx[e] = qx; sqy[e] = qy; su[e] = u; sv[e] = v; sc[e] = c;
  }
  jx[li] = jxa; jy[li] = jya;
  if (e2 < kQ * 19) { jx[e2] = jxb; jy[e2] = jyb; }
  if (CREST) {
    jx2[li] = jx2a; jy2[li] = jy2a;
    if (e2 < kQ * 19) { jx2[e2] = jx2b; jy2[e2] = jy2b; }
  }
  __syncthreads();
  // 2. forward faces of the 18x18 cells: x-face (jr, fi) joins region cells (fi, jr+1) and
  //    (fi+1, jr+1); y-face (fr, ic) joins (ic+1, fr) and (ic+1, fr+1)
  for (int e = li; e < kQ * 19; e += kTileThreads) {
    {
      const int jr = e / 19, fi = e % 19;
      const int row = gy0 - 1 + jr, f = gx0 - 1 + fi;
      FaceF o{};
      if (row >= 0 && row < ny && f >= 0 && f <= nx) {
        const int a = (jr + 1) * kR + fi;
        o = face<true, CREST>(sh[a], su[a], sv[a], sc[a], sh[a + 1], su[a + 1], sv[a + 1], sc[a + 1], jx[e],
                              CREST ? jx2[e] : 0.0f, k);
      }
      fx[e] = o;
    }
    {
      const int fr = e / kQ, ic = e % kQ;
      const int col = gx0 - 1 + ic, f = gy0 - 1 + fr;
      FaceF o{};
      if (col >= 0 && col < nx && f >= 0 && f <= ny) {
        const int a = fr * kR + ic + 1, b = a + kR;
        o = face<false, CREST>(sh[a], su[a], sv[a], sc[a], sh[b], su[b], sv[b], sc[b], jy[e], CREST ? jy2[e] : 0.0f, k);
      }
      fy[e] = o;
    }
  }
  __syncthreads();
  // 3. adjoint through the sources of every in-domain cell of the 18x18 region
  const int* sn = A.seed_n;
  for (int e = li; e < kQ * kQ; e += kTileThreads) {
    const int ic = e % kQ, jr = e / kQ;
    const int gx = gx0 - 1 + ic, gy = gy0 - 1 + jr;
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
    if (gx >= 0 && gx < nx && gy >= 0 && gy < ny) {
      const size_t gi = (size_t)gy * nx + gx;
      float lh = LI[gi];
      const float lqx = LI[N + gi], lqy = LI[2 * N + gi];
      for (int q = 0; q < sn[d]; ++q) {   // peak term of the state this step makes
        const size_t si = (size_t)d * A.max_seeds + q;
        if (A.seed_cell[si] == gi && A.seed_state[si] == n + 1) lh += A.seed_w[si];
      }
      const int a = (jr + 1) * kR + ic + 1;
      sources_bwd(sh[a], sqx[a], sqy[a], fx[jr * 19 + ic], fx[jr * 19 + ic + 1], fy[jr * kQ + ic], fy[(jr + 1) * kQ + ic],
                  A.wet[gi], A.gn2[gi], k, lh, lqx, lqy, a0, a1, a2);
    }
    l1[0][e] = a0; l1[1][e] = a1; l1[2][e] = a2;
  }
  __syncthreads();
  // 4. face adjoints and their input adjoints, for every face touching a tile cell
  for (int e = li; e < 16 * 17; e += kTileThreads) {
    {  // x-face between tile-row cells (xl-1, yr) and (xl, yr) of the 18x18 region, xl = 1..17
      const int yr = e / 17 + 1, xl = e % 17 + 1;
      const int row = gy0 - 1 + yr, f = gx0 - 1 + xl;
      float* o = bx[e];
      for (int q = 0; q < 8; ++q) o[q] = 0.0f;
      if (row < ny && f <= nx) {
        const int L = yr * kQ + xl - 1, R = L + 1;
        const float lm = -k.dtdx * l1[0][L] + k.dtdx * l1[0][R];
        const float lnl = -k.dtdx * l1[1][L], lnr = k.dtdx * l1[1][R];
        const float lt = -k.dtdx * l1[2][L] + k.dtdx * l1[2][R];
        const int a = (yr + 1) * kR + xl;   // region cell of L
        const float dz = jx[yr * 19 + xl], dz2 = CREST ? jx2[yr * 19 + xl] : 0.0f;
        const FaceBwd b = face_bwd<true, CREST>(sh[a], su[a], sv[a], sc[a], sh[a + 1], su[a + 1], sv[a + 1], sc[a + 1], dz, dz2, k,
                                         lm, lnl, lnr, lt);
        o[0] = b.hl; o[1] = b.ul; o[2] = b.vl; o[3] = b.cl; o[4] = b.hr; o[5] = b.ur; o[6] = b.vr; o[7] = b.cr;
        if (xown) *gxp = gx_old + (double)b.dz;
        if (CREST && xown) *gxp2 = gx2_old + (double)b.dz2;
      }
    }
    {  // y-face between (xc, yt-1) and (xc, yt) of the 18x18 region, yt = 1..17
      const int yt = e / 16 + 1, xc = e % 16 + 1;
      const int col = gx0 - 1 + xc, f = gy0 - 1 + yt;
      float* o = by[e];
      for (int q = 0; q < 8; ++q) o[q] = 0.0f;
      if (col < nx && f <= ny) {
        const int T = (yt - 1) * kQ + xc, B = T + kQ;
        const float lm = -k.dtdy * l1[0][T] + k.dtdy * l1[0][B];
        const float lt = -k.dtdy * l1[1][T] + k.dtdy * l1[1][B];
        const float lnl = -k.dtdy * l1[2][T], lnr = k.dtdy * l1[2][B];
        const int a = yt * kR + xc + 1;      // region cell of T
        const float dz = jy[yt * kQ + xc], dz2 = CREST ? jy2[yt * kQ + xc] : 0.0f;
        const FaceBwd b = face_bwd<false, CREST>(sh[a], su[a], sv[a], sc[a], sh[a + kR], su[a + kR], sv[a + kR], sc[a + kR], dz, dz2,
                                          k, lm, lnl, lnr, lt);
        o[0] = b.hl; o[1] = b.ul; o[2] = b.vl; o[3] = b.cl; o[4] = b.hr; o[5] = b.ur; o[6] = b.vr; o[7] = b.cr;
        if (yown) *gyp = gy_old + (double)b.dz;
        if (CREST && yown) *gyp2 = gy2_old + (double)b.dz2;
      }
    }
  }
  __syncthreads();
  // 5. each tile cell: its four faces' input adjoints (+ its ghosts'), the velocity map, and
  //    the identity part of the flux update
  {
    const int lx = li % 16, ly = li / 16, gx = gx0 + lx, gy = gy0 + ly;
    if (li < 256 && gx < nx && gy < ny) {
      const float* W = bx[ly * 17 + lx];        // west face: this cell is its R side
      const float* E = bx[ly * 17 + lx + 1];    // east face: L side
      const float* Nf = by[ly * 16 + lx];       // north face: B side
      const float* Sf = by[(ly + 1) * 16 + lx]; // south face: T side
      float lh = W[4] + E[0] + Nf[4] + Sf[0];
      float lu = W[5] + E[1] + Nf[5] + Sf[1];
      float lv = W[6] + E[2] + Nf[6] + Sf[2];
      float lc = W[7] + E[3] + Nf[7] + Sf[3];
      // ghosts: a wall mirrors the normal velocity, a transmissive edge copies the cell; a
      // stage or inflow ghost (BND) adds straight to the cell's (h, qx, qy) adjoints
      const int a = (ly + 2) * kR + lx + 2;
      float gh = 0.0f, gqx = 0.0f, gqy = 0.0f;
      auto fold = [&](int code, const float* L, int ga) {   // L: the ghost's (h, u, v, c) adjoints
        const float crit = code >= 3 ? sinf[code - 3].y : 0.0f;
        ghost_bwd(code, L[0], L[1], L[2], L[3], sh[ga], sqx[ga], sqy[ga], sc[ga], sh[a], crit, k.g, k.heps2, gh, gqx, gqy);
      };
      if (gx == 0) {
        const int code = A.bc[2 * nx + gy];
        if (BND && code >= 2) fold(code, W, a - 1);
        else { const float s = code == 0 ? -1.0f : 1.0f; lh += W[0]; lu += s * W[1]; lv += W[2]; lc += W[3]; }
      }
      if (gx == nx - 1) {
        const int code = A.bc[2 * nx + ny + gy];
        if (BND && code >= 2) fold(code, E + 4, a + 1);
        else { const float s = code == 0 ? -1.0f : 1.0f; lh += E[4]; lu += s * E[5]; lv += E[6]; lc += E[7]; }
      }
      if (gy == 0) {
        const int code = A.bc[gx];
        if (BND && code >= 2) fold(code, Nf, a - kR);
        else { const float s = code == 0 ? -1.0f : 1.0f; lh += Nf[0]; lu += Nf[1]; lv += s * Nf[2]; lc += Nf[3]; }
      }
      if (gy == ny - 1) {
        const int code = A.bc[nx + gx];
        if (BND && code >= 2) fold(code, Sf + 4, a + kR);
        else { const float s = code == 0 ? -1.0f : 1.0f; lh += Sf[4]; lu += Sf[5]; lv += s * Sf[6]; lc += Sf[7]; }
      }
      // velocity map (numerics.rs:38-45): u = qx t(h), v = qy t(h), c = sqrt(g h)
      const float h = sh[a], qx = sqx[a], qy = sqy[a], c = sc[a];
      const float h2 = h * h, den = h2 + rmax(h2, k.heps2);
      const float t = (h + h) * rcp(den);
      const float dtdh = h2 > k.heps2 ? -1.0f / h2 : 2.0f * (k.heps2 - h2) / (den * den);
      const int q = (ly + 1) * kQ + lx + 1;
      const size_t gi = (size_t)gy * nx + gx;
      float oh = lh + (lu * qx + lv * qy) * dtdh + (c > 0.0f ? lc * k.g * 0.5f / c : 0.0f) + l1[0][q];
      float oqx = lu * t + l1[1][q], oqy = lv * t + l1[2][q];
      if (BND) { oh += gh; oqx += gqx; oqy += gqy; }
      LO[gi] = oh;
      LO[N + gi] = oqx;
      LO[2 * N + gi] = oqy;
    }
  }
}

// Checkpoint: the current state plane of every design into dst (per design [3][N]).
__global__ void k_adj_ckpt(const PlainArgs A, float* dst) {
  const PlainDesign D = plain_design(A, blockIdx.y, 0);
  const size_t N = (size_t)A.nx * A.ny;
  const int par = D.ctl->par;
  float* o = dst + (size_t)blockIdx.y * 3 * N;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
    o[i] = D.H[par * N + i]; o[N + i] = D.QX[par * N + i]; o[2 * N + i] = D.QY[par * N + i];
  }
}

__global__ void k_gather_u32(const unsigned* a, const unsigned* mon, int n_mon, size_t cells, int n_designs, unsigned* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_mon * n_designs) return;
  const int d = i / n_mon, m = i % n_mon;
  out[i] = a[(size_t)d * cells + mon[m]];
}

}  // namespace itr
