// itr_device.cuh — per-face and per-cell arithmetic of the first-order FV step, on sm_100a.
//
// Operation order follows crates/itr-hydro/src/numerics.rs exactly (every product and sum
// in the same association), and the library is compiled with -fmad=false, IEEE division
// and square root and no flush-to-zero, so each value here has the same bits as the
// reference's f32 kernel (the reference's rule: IEEE + - * / sqrt only, spec.md:618).
//   rcbrt        crates/itr-core/src/real.rs:116-130
//   cell_vel     numerics.rs:36-43
//   hll          numerics.rs:56-93
//   face_signed  numerics.rs:95-112
//   face_crest   numerics.rs:114-129
//   update_cell  numerics.rs:144-213 (flux_update + sources)
// NaN semantics of max/min/abs are the reference's (real.rs:38-58), not fmaxf/fabsf.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "itr_math.h"

namespace itr {

#define ITR_DEV __device__ __forceinline__

ITR_DEV float rmax(float a, float b) { return a > b ? a : b; }
ITR_DEV float rmin(float a, float b) { return a < b ? a : b; }
ITR_DEV float rabs(float a) { return a < 0.0f ? -a : a; }
ITR_DEV float canon(float a) { return a == 0.0f ? 0.0f : a; }

// x^(-1/3): bit seed 0x54A23280 - bits/3 and three short-chain Newton steps.
ITR_DEV float rcbrt(float x) {
  uint32_t bits = __float_as_uint(x);
  float r = __uint_as_float(0x54A23280u - bits / 3u);
  const float x3 = x * (float)(1.0 / 3.0);
  const float c43 = (float)(4.0 * (1.0 / 3.0));
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float r2 = r * r;
    r = r * c43 - x3 * (r2 * r2);
  }
  return r;
}

// Step constants, all rounded once from f64 (solver.rs:269-285).
struct StepK {
  float g, g_half, dt, dtdx, dtdy, inv_dx, inv_dy, h_dry, heps2, q_min, rain, cap;
  float nz;   // -0.0f read from the kernel parameters at run time (see mul2)
  unsigned exact;   // 1: paired reciprocals always through the IEEE routine (checking)
};

// A face flux tuple: mass, normal momentum seen from the low-index (n_l) and high-index
// (n_r) cell with the hydrostatic pressure correction folded in, tangential momentum.
struct FaceF { float m, nl, nr, t; };

// Desingularised velocity and celerity of a cell.
// 1/x rounded to nearest (IEEE): the same value as 1.0f / x compiled with IEEE division,
// through the reciprocal instruction path.
ITR_DEV float rcp(float x) { return __frcp_rn(x); }

// IEEE square root with zero kept off the instruction's special-case path: sqrt(+-0) is
// +-0 exactly, so returning x for x == 0 gives the same bits as sqrtf(x) for every input,
// while dry faces and cells (reduced depth 0) stay on the fast path.
ITR_DEV float sqrt_rn(float x) {
  const bool z = x == 0.0f;
  const float r = sqrtf(z ? 1.0f : x);
  return z ? x : r;
}

ITR_DEV void cell_vel(float h, float qx, float qy, float g, float heps2, float& u, float& v, float& c) {
  float h2 = h * h;
  float inv = rcp(h2 + rmax(h2, heps2));
  float t = (h + h) * inv;
  u = qx * t;
  v = qy * t;
  c = sqrt_rn(g * h);
}

// HLL flux with two-rarefaction wave speeds; dry-dry faces give exactly zero.
ITR_DEV FaceF hll(float hl, float ul, float tl, float cl, float hr, float ur, float tr, float cr, float g_half) {
  const bool dry_l = !(hl > 0.0f);
  const bool dry_r = !(hr > 0.0f);
  float ustar = 0.5f * (ul + ur) + cl - cr;
  float cstar = 0.5f * (cl + cr) + 0.25f * (ul - ur);
  float slw = rmin(ul - cl, ustar - cstar);
  float srw = rmax(ur + cr, ustar + cstar);
  float sl = dry_l ? ur - 2.0f * cr : (dry_r ? ul - cl : slw);
  float sr = dry_l ? ur + cr : (dry_r ? ul + 2.0f * cl : srw);
  float ml = hl * ul;
  float mr = hr * ur;
  float pl_ = g_half * hl * hl;
  float pr_ = g_half * hr * hr;
  float pl = ml * ul + pl_;
  float pr = mr * ur + pr_;
  const bool both_dry = dry_l && dry_r;
  const bool use_l = sl >= 0.0f;
  const bool use_r = sr <= 0.0f;
  float den = (both_dry || use_l || use_r) ? 1.0f : sr - sl;
  float inv = rcp(den);
  float slsr = sl * sr;
  float fm_star = (sr * ml - sl * mr + slsr * (hr - hl)) * inv;
  float fn_star = (sr * pl - sl * pr + slsr * (mr - ml)) * inv;
  float fm = both_dry ? 0.0f : (use_l ? ml : (use_r ? mr : fm_star));
  float fn = both_dry ? 0.0f : (use_l ? pl : (use_r ? pr : fn_star));
  float ft = fm * (fm > 0.0f ? tl : tr);
  FaceF f;
  f.m = fm; f.nl = fn - pl_; f.nr = fn - pr_; f.t = ft;
  return f;
}

// Signed-jump face (dz = z_R - z_L): one reduced side, one square root. `normal_x` picks
// which velocity component is normal. (ul,vl,cl) are the left/top cell's velocity.
template <bool NORMAL_X>
ITR_DEV FaceF face_signed(float hl, float ul, float vl, float cl, float hr, float ur, float vr, float cr,
                          float dz, float g, float g_half) {
  const bool pos = dz > 0.0f;
  float hsl = rmax(hl - rmax(dz, 0.0f), 0.0f);
  float hsr = rmax(hr - rmax(-dz, 0.0f), 0.0f);
  float hred = pos ? hsl : hsr;
  float cred = sqrt_rn(g * hred);
  float csl = pos ? cred : cl;
  float csr = pos ? cr : cred;
  if (NORMAL_X) return hll(hsl, ul, vl, csl, hsr, ur, vr, csr, g_half);
  return hll(hsl, vl, ul, csl, hsr, vr, ur, csr, g_half);
}

// Crest face: two non-negative jumps d_l = z_f - z_L, d_r = z_f - z_R.
template <bool NORMAL_X>
ITR_DEV FaceF face_crest(float hl, float ul, float vl, float cl, float hr, float ur, float vr, float cr,
                         float d_l, float d_r, float g, float g_half) {
  float hsl = rmax(hl - d_l, 0.0f);
  float hsr = rmax(hr - d_r, 0.0f);
  float csl = d_l > 0.0f ? sqrt_rn(g * hsl) : cl;
  float csr = d_r > 0.0f ? sqrt_rn(g * hsr) : cr;
  if (NORMAL_X) return hll(hsl, ul, vl, csl, hsr, ur, vr, csr, g_half);
  return hll(hsl, vl, ul, csl, hsr, vr, ur, csr, g_half);
}

template <bool NORMAL_X, bool CREST>
ITR_DEV FaceF face(float hl, float ul, float vl, float cl, float hr, float ur, float vr, float cr,
                   float d0, float d1, const StepK& k) {
  if (CREST) return face_crest<NORMAL_X>(hl, ul, vl, cl, hr, ur, vr, cr, d0, d1, k.g, k.g_half);
  return face_signed<NORMAL_X>(hl, ul, vl, cl, hr, ur, vr, cr, d0, k.g, k.g_half);
}

// Result of one cell update. c is sqrt(g*h) of the new depth, which is also the next
// step's celerity (h is never -0 here, so sqrt(g*h) of the stored value is the same bits).
struct CellNew {
  float h, qx, qy, s, infil, fix, c;
  bool bad;
};

// flux_update then sources (numerics.rs:144-195).
ITR_DEV CellNew update_cell(float h, float qx, float qy, const FaceF& w, const FaceF& e, const FaceF& n,
                            const FaceF& s, float wet, float gn2, const StepK& k) {
  float h1 = h - k.dtdx * (e.m - w.m) - k.dtdy * (s.m - n.m);
  float qx1 = qx - k.dtdx * (e.nl - w.nr) - k.dtdy * (s.t - n.t);
  float qy1 = qy - k.dtdx * (e.t - w.t) - k.dtdy * (s.nl - n.nr);
  CellNew o;
  bool bad = !(h1 >= -k.h_dry);
  o.fix = h1 < 0.0f ? -h1 : 0.0f;
  if (h1 < 0.0f) h1 = 0.0f;
  float h2 = h1 + k.rain * wet;
  o.infil = rmin(k.cap * wet, h2);
  float h3 = h2 - o.infil;
  const bool dry = h3 < k.h_dry;
  float r = rcbrt(dry ? 1.0f : h3);
  float r3 = r * r * r;
  float r7 = r3 * r3 * r;
  float qm = sqrt_rn(qx1 * qx1 + qy1 * qy1);
  float inv = rcp(1.0f + k.dt * gn2 * qm * r7);
  float keep = dry ? 0.0f : 1.0f;
  float qx2 = qx1 * inv * keep;
  float qy2 = qy1 * inv * keep;
  if (rabs(qx2) < k.q_min) qx2 = 0.0f;
  if (rabs(qy2) < k.q_min) qy2 = 0.0f;
  float c = sqrt_rn(k.g * h3);
  o.s = (rabs(qx2) * r3 + c) * k.inv_dx + (rabs(qy2) * r3 + c) * k.inv_dy;
  o.bad = bad || !(qm == qm);
  o.h = canon(h3);
  o.qx = canon(qx2);
  o.qy = canon(qy2);
  o.c = c;
  return o;
}

// ------------------------------------------------------------------ time integrator ----
// Hyetograph (scenario.rs:526-586) and the f64 step rule of solver.rs:449-489, evaluated by
// every thread of a design redundantly (identical inputs, identical bits).
constexpr int kMaxRain = 32;

struct Rain {
  int n;
  double t[kMaxRain];
  double r[kMaxRain];
};

ITR_DEV double rain_rate(const Rain& R, double x) {
  if (R.n == 0) return 0.0;
  if (x <= R.t[0]) return R.r[0];
  for (int k = 0; k + 1 < R.n; ++k) {
    if (x <= R.t[k + 1]) {
      double t0 = R.t[k], r0 = R.r[k], t1 = R.t[k + 1], r1 = R.r[k + 1];
      if (t1 == t0) return r1;
      return r0 + (r1 - r0) * (x - t0) / (t1 - t0);
    }
  }
  return R.r[R.n - 1];
}

ITR_DEV double rain_integral(const Rain& R, double a, double b) {
  if (b <= a) return 0.0;
  if (R.n == 0) return 0.0;
  double total = 0.0, tt = a, rr = rain_rate(R, a);
  for (int k = 0; k < R.n; ++k) {
    double tk = R.t[k];
    if (tk > a && tk < b) {
      double rk = rain_rate(R, tk);
      total += 0.5 * (rr + rk) * (tk - tt);
      tt = tk;
      rr = rk;
    }
  }
  double rb = rain_rate(R, b);
  total += 0.5 * (rr + rb) * (b - tt);
  return total;
}

// The same rate and integral, for sorted breakpoints, with a cursor that only moves
// forward (simulated time is monotone): identical arithmetic on identical operands, so
// identical bits, without rescanning the table every step.
struct RainCursor {
  int seg;   // first k with t[k+1] >= last query (rate) ...
  int brk;   // first breakpoint index with t[k] > last lower limit
};

ITR_DEV double rain_rate_c(const Rain& R, double x, int& seg) {
  if (R.n == 0) return 0.0;
  if (x <= R.t[0]) return R.r[0];
  while (seg + 1 < R.n && R.t[seg + 1] < x) ++seg;
  if (seg + 1 < R.n) {
    double t0 = R.t[seg], r0 = R.r[seg], t1 = R.t[seg + 1], r1 = R.r[seg + 1];
    if (t1 == t0) return r1;
    return r0 + (r1 - r0) * (x - t0) / (t1 - t0);
  }
  return R.r[R.n - 1];
}

ITR_DEV double rain_integral_c(const Rain& R, double a, double b, RainCursor& cu) {
  if (b <= a) return 0.0;
  if (R.n == 0) return 0.0;
  int seg = cu.seg;
  double total = 0.0, tt = a, rr = rain_rate_c(R, a, seg);
  cu.seg = seg;
  while (cu.brk < R.n && !(R.t[cu.brk] > a)) ++cu.brk;
  for (int k = cu.brk; k < R.n && R.t[k] < b; ++k) {
    double tk = R.t[k];
    int s2 = seg;
    double rk = rain_rate_c(R, tk, s2);
    total += 0.5 * (rr + rk) * (tk - tt);
    tt = tk;
    rr = rk;
    seg = s2;
  }
  double rb = rain_rate_c(R, b, seg);
  total += 0.5 * (rr + rb) * (b - tt);
  return total;
}

// Inflow boundaries (Ghost::Inflow, boundary.rs:26-31,45-50,66-71). The inflow cells of a
// grid fall into groups, one per distinct (hydrograph, 1 / segment length) pair; a group's
// discharge per unit width q = rate(t) * inv_len * inflow_scale and its critical depth
// (q^2/g)^(1/3) are the same for all its cells, so they are evaluated once per design and
// step and the cells read them.
constexpr int kMaxInflow = 8;       // groups
constexpr int kMaxInflowPts = 64;   // hydrograph points over all groups

struct Inflow {
  int n;                        // groups (0: no inflow cells)
  int off[kMaxInflow + 1];      // group g's hydrograph points are [off[g], off[g+1])
  double inv_len[kMaxInflow];   // 1 / segment length [1/m]
  double scale;                 // SolverParams::inflow_scale
  double t[kMaxInflowPts];      // time [s]
  double q[kMaxInflowPts];      // discharge [m^3/s]
};

// Real::rcbrt for f64 (crates/itr-core/src/real.rs:81-95): the f32 seed constant moved to
// the f64 exponent and mantissa, then four short-chain Newton steps.
ITR_DEV double rcbrt_d(double x) {
  const unsigned long long K = 0x5540000000000000ull - (0x8782Bull << 29);
  double r = __longlong_as_double((long long)(K - (unsigned long long)__double_as_longlong(x) / 3ull));
  const double third = 1.0 / 3.0;
  const double x3 = x * third;
  const double c43 = 4.0 * third;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    double r2 = r * r;
    r = r * c43 - x3 * (r2 * r2);
  }
  return r;
}

// Hyetograph::rate (scenario.rs:561-570) over points [a, b) of the inflow table; the same
// arithmetic as rain_rate.
ITR_DEV double inflow_rate(const Inflow& F, int a, int b, double x) {
  if (b <= a) return 0.0;
  if (x <= F.t[a]) return F.q[a];
  for (int k = a; k + 1 < b; ++k) {
    if (x <= F.t[k + 1]) {
      double t0 = F.t[k], r0 = F.q[k], t1 = F.t[k + 1], r1 = F.q[k + 1];
      if (t1 == t0) return r1;
      return r0 + (r1 - r0) * (x - t0) / (t1 - t0);
    }
  }
  return F.q[b - 1];
}

// Group g at time t (the start of a step): x = f32 of the discharge per unit width q, and
// y = f32 of the critical depth x * rcbrt(x) * rcbrt(x), x = q^2 / g, in f64 (boundary.rs:
// 27-31). A ghost's depth is f32(max(h, crit)) = max(h, f32(crit)) since rounding is
// monotone and h is already an f32; its normal discharge f32(+-q) = +-f32(q).
ITR_DEV float2 inflow_values(const Inflow& F, int g, double t, double gacc) {
  const double q = inflow_rate(F, F.off[g], F.off[g + 1], t) * F.inv_len[g] * F.scale;
  const double x = q * q / gacc;
  double crit = 0.0;
  if (x > 0.0) {
    const double r = rcbrt_d(x);
    crit = x * r * r;
  }
  return make_float2((float)q, (float)crit);
}

// Ghost state from the interior cell (h, qx, qy) behind it (boundary.rs:36-87), for device
// boundary codes: 0 wall (normal momentum mirrored), 1 transmissive (copy), 2 stage (the
// design's stage depth hstage, momentum copied), 3 + g inflow group g (depth max(h, crit),
// inward normal discharge, zero tangential discharge; inf = inflow_values of the group).
// NX: the ghost lies across an x-normal face (west or east); inward_pos: west or north side.
template <bool NX>
ITR_DEV void ghost_state(int code, float& h, float& qx, float& qy, float hstage, float2 inf, bool inward_pos) {
  if (code == 0) {
    if (NX) qx = -qx; else qy = -qy;
  } else if (code == 2) {
    h = hstage;
  } else if (code >= 3) {
    h = h > inf.y ? h : inf.y;   // NaN h gives the critical depth, as f64::max does
    const float qn = inward_pos ? inf.x : -inf.x;
    if (NX) { qx = qn; qy = 0.0f; } else { qx = 0.0f; qy = qn; }
  }
}

// Ghost wetness of the padded rows for a step whose inflow group values are `inf` (the dry-row
// test of step_fused, kernel.rs:590-612, takes a row with a wet ghost as wet): a stage ghost
// holds water when its depth is > 0, an inflow ghost when the group's critical depth is > 0;
// wall and transmissive ghosts copy their interior cell, so they hold water only beside a wet
// row and need no flag. gw[j], j = 0 .. ny + 1 (0 and ny + 1: the north and south ghost rows,
// 1 .. ny: the west and east ghosts of grid row j - 1). bc: device codes (2 stage, 3 + group
// inflow) north[nx], south[nx], west[ny], east[ny]; bh: stage depths indexed like bc (or NULL).
// One warp, all 32 lanes.
ITR_DEV void ghost_row_wet(const uint8_t* bc, int nx, int ny, const float* bh, const float2* inf, uint8_t* gw, int lane) {
  auto wet = [&](int p) -> bool {
    const int code = bc[p];
    return (code == 2 && bh && bh[p] > 0.0f) || (code >= 3 && inf[code - 3].y > 0.0f);
  };
  for (int e = 0; e < 2; ++e) {   // the north and south ghost rows
    bool w = false;
    for (int c = lane; c < nx; c += 32) w = w || wet(e * nx + c);
    w = __any_sync(0xffffffffu, w);
    if (lane == 0) gw[e == 0 ? 0 : ny + 1] = w ? 1 : 0;
  }
  for (int j = 1 + lane; j <= ny; j += 32) gw[j] = (wet(2 * nx + j - 1) || wet(2 * nx + ny + j - 1)) ? 1 : 0;
}

// Run-wide scalars of one call.
struct RunParams {
  double duration, sync, cfl, dt_max, h_dry, h_eps, infil, initial_depth;
  double dx, dy, g, area, wet_count;
  uint32_t n_sync;
  int skip_dry;
  int rain_sorted;   // breakpoints non-decreasing in time: the cursor path is exact
  Rain rain;
  Inflow inflow;
  // step-invariant f32 constants (solver.rs:269-285), rounded once on the host
  float g_f, g_half_f, inv_dx_f, inv_dy_f, h_dry_f, heps2_f, q_min_f;
  float nz;   // -0.0f, supplied at run time (see mul2)
};

ITR_DEV double dmin_num(double a, double b) { return a < b ? a : b; }  // operands never NaN here

// One step's scalar schedule from the previous state of the integrator.
struct StepPlan {
  double dt, t_new, rain;
  bool hits;
};

ITR_DEV StepPlan plan_step(const RunParams& P, double t, uint32_t sync_index, double dt_cfl) {
  StepPlan s;
  double t_sync = dmin_num((double)(sync_index + 1) * P.sync, P.duration);
  double dt = dmin_num(dt_cfl, P.dt_max);
  s.hits = t + dt >= t_sync - 1e-9 * P.sync;
  if (s.hits) dt = t_sync - t;
  s.rain = rain_integral(P.rain, t, t + dt);
  s.t_new = s.hits ? t_sync : t + dt;
  s.dt = dt;
  return s;
}

ITR_DEV StepPlan plan_step_c(const RunParams& P, double t, uint32_t sync_index, double dt_cfl, RainCursor& cu) {
  StepPlan s;
  double t_sync = dmin_num((double)(sync_index + 1) * P.sync, P.duration);
  double dt = dmin_num(dt_cfl, P.dt_max);
  s.hits = t + dt >= t_sync - 1e-9 * P.sync;
  if (s.hits) dt = t_sync - t;
  s.rain = P.rain_sorted ? rain_integral_c(P.rain, t, t + dt, cu) : rain_integral(P.rain, t, t + dt);
  s.t_new = s.hits ? t_sync : t + dt;
  s.dt = dt;
  return s;
}

// plan_step for a step whose dt before the sync clip is given (the baseline-locked dt).
ITR_DEV StepPlan plan_step_dt(const RunParams& P, double t, uint32_t sync_index, double dt) {
  StepPlan s;
  double t_sync = dmin_num((double)(sync_index + 1) * P.sync, P.duration);
  s.hits = t + dt >= t_sync - 1e-9 * P.sync;
  if (s.hits) dt = t_sync - t;
  s.rain = rain_integral(P.rain, t, t + dt);
  s.t_new = s.hits ? t_sync : t + dt;
  s.dt = dt;
  return s;
}

// plan_step_c for a step whose dt before the sync clip is given: the baseline-locked dt
// (solver.rs:452-456 sets dt from the schedule, then :484-487 clip it to the sync instant).
ITR_DEV StepPlan plan_step_dt_c(const RunParams& P, double t, uint32_t sync_index, double dt, RainCursor& cu) {
  StepPlan s;
  double t_sync = dmin_num((double)(sync_index + 1) * P.sync, P.duration);
  s.hits = t + dt >= t_sync - 1e-9 * P.sync;
  if (s.hits) dt = t_sync - t;
  s.rain = P.rain_sorted ? rain_integral_c(P.rain, t, t + dt, cu) : rain_integral(P.rain, t, t + dt);
  s.t_new = s.hits ? t_sync : t + dt;
  s.dt = dt;
  return s;
}

// Per-step constants from the host-rounded invariants and this step's dt and rain.
ITR_DEV StepK step_consts(const RunParams& P, double dt, double rain) {
  StepK k;
  k.g = P.g_f; k.g_half = P.g_half_f; k.inv_dx = P.inv_dx_f; k.inv_dy = P.inv_dy_f;
  k.h_dry = P.h_dry_f; k.heps2 = P.heps2_f; k.q_min = P.q_min_f;
  k.dt = (float)dt;
  k.dtdx = (float)(dt / P.dx);
  k.dtdy = (float)(dt / P.dy);
  k.rain = (float)rain;
  k.cap = (float)(P.infil * dt);
  k.nz = P.nz;
  k.exact = 0u;
  return k;
}

ITR_DEV StepK make_consts(const RunParams& P, double dt, double rain) {
  StepK k;
  k.g = (float)P.g;
  k.g_half = (float)(0.5 * P.g);
  k.dt = (float)dt;
  k.dtdx = (float)(dt / P.dx);
  k.dtdy = (float)(dt / P.dy);
  k.inv_dx = (float)(1.0 / P.dx);
  k.inv_dy = (float)(1.0 / P.dy);
  k.h_dry = (float)P.h_dry;
  k.heps2 = (float)(P.h_eps * P.h_eps);
  k.q_min = (float)1e-30;
  k.rain = (float)rain;
  k.cap = (float)(P.infil * dt);
  k.nz = P.nz;
  k.exact = 0u;
  return k;
}

// Objective on the device (objective.rs:94-149), for the incumbent abort and J.
struct DevObjective {
  int n_assets;
  const int* asset_off;
  const int* asset_pos;
  const double* asset_thr;
  const double* asset_w;
  int n_guard;
  const int* guard_pos;
  const double* baseline;  // per monitor or null
  double tol, tau, cut_cost, fill_cost, earth_w;
  int require, guard_abort, has_incumbent;
  double incumbent;
  int enabled;
};

// Per-design scalar results written by the kernels.
// A design's warm start (Solver::run_impl from a Checkpoint, solver.rs:354-378): the
// baseline's state at a checkpoint and its integrator there. state == NULL: cold start.
struct WarmStart {
  const float* state;   // [4][nx*ny]: h, qx, qy, running peak depth
  double t, dt_cfl, acc_rain, v0, volume, rel_res;
  double tot_infil, tot_fix, tot_in, tot_out;   // ledger totals (infil, fix per unit area)
  unsigned long long step;
  unsigned sync_index;
  int n_rows;
};

struct DesignOut {
  unsigned long long steps;
  double t_end;
  unsigned int sync_count;
  int status;
  unsigned int breach_cell;
  unsigned int breach_sync;
  double violation;
  double lower_bound;
  double v0;
  double volume;
  double rel_residual;
  int n_rows;
  int pad;
  unsigned long long rows_skipped;   // dry rows skipped (kernel.rs:605-612)
};

}  // namespace itr

// --------------------------------------------------------------- two cells at once ----
// The same arithmetic on pairs of cells: every add and multiply is a paired FP32
// instruction (__fadd2_rn / __fmul2_rn: each component is the IEEE round-to-nearest
// result of the scalar operation), every compare, select, square root and reciprocal is
// done per component. Association order is the scalar code's, so each component has the
// same bits as the scalar path (and as the reference's f32 kernel).
namespace itr {

struct B2 { bool x, y; };
struct Face2 { float2 m, nl, nr, t; };

ITR_DEV float2 f2(float a) { return make_float2(a, a); }
// Packed FP32 pairs through PTX with an explicit .rn rounding modifier: such instructions are
// never contracted into fused multiply-adds (the float2 intrinsics may be), so each component
// is exactly the scalar IEEE result.
ITR_DEV unsigned long long pk2(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
ITR_DEV float2 upk2(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
ITR_DEV float2 add2(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(r);
}
ITR_DEV float2 sub2(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(r);
}
// Paired product as fma(a, b, -0): exactly round(a*b) for every input (x + -0 == x, zeros
// keep their sign). The -0 must not be a compile-time constant, else the compiler turns the
// fma back into a multiply and fuses it with the next add (observed on sm_100a), which
// would round once instead of twice; it is the kernel parameter StepK::nz.
ITR_DEV float2 mul2(float2 a, float2 b, float nz) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)), "l"(pk2(make_float2(nz, nz))));
  return upk2(r);
}
ITR_DEV float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
ITR_DEV float2 sel2(B2 c, float2 a, float2 b) { return make_float2(c.x ? a.x : b.x, c.y ? a.y : b.y); }
ITR_DEV float2 max2(float2 a, float2 b) { return make_float2(rmax(a.x, b.x), rmax(a.y, b.y)); }
ITR_DEV float2 min2(float2 a, float2 b) { return make_float2(rmin(a.x, b.x), rmin(a.y, b.y)); }
ITR_DEV B2 gt2(float2 a, float b) { return B2{a.x > b, a.y > b}; }
ITR_DEV B2 ge2(float2 a, float b) { return B2{a.x >= b, a.y >= b}; }
ITR_DEV B2 le2(float2 a, float b) { return B2{a.x <= b, a.y <= b}; }
ITR_DEV B2 lt2(float2 a, float b) { return B2{a.x < b, a.y < b}; }
ITR_DEV B2 not2(B2 a) { return B2{!a.x, !a.y}; }
ITR_DEV B2 and2(B2 a, B2 b) { return B2{a.x && b.x, a.y && b.y}; }
ITR_DEV B2 or2(B2 a, B2 b) { return B2{a.x || b.x, a.y || b.y}; }
ITR_DEV float2 sqrt2(float2 a) { return make_float2(sqrt_rn(a.x), sqrt_rn(a.y)); }
ITR_DEV float2 rcp2(float2 a) { return make_float2(rcp(a.x), rcp(a.y)); }
ITR_DEV float2 fma2(float2 a, float2 b, float2 c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)), "l"(pk2(c)));
  return upk2(r);
}

// ---- Reciprocal without the IEEE routine's per-lane slow-path branch ----
// 1/x as one Newton step from the hardware estimate (textbook FMA refinement: P. Markstein,
// IBM J. Res. Dev. 34(1), 1990; J.-M. Muller et al., Handbook of Floating-Point Arithmetic,
// 2nd ed., 2018, ch. 4): y = est(1/x); e = fma(-x, y, 1); y + y e. Checked against CUDA's
// IEEE reciprocal on every 32-bit input with |x| in [2^-125, 2^126): identical. An operand
// outside that range (zero, infinity, NaN, tiny or huge) sends the whole warp through the
// IEEE routine for that call, as does k.exact; the branch is warp-uniform, so the common
// path carries no divergence point. Results are the IEEE ones for every input. The step
// kernel's reciprocals (HLL denominator, friction, velocity) are in range for every
// healthy state: the fallback is for NaN/infinite states and for checking.
ITR_DEV float rcp_est(float x) { float r; asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
// In range: |x| in [2^-125, 2^126), i.e. biased exponent 2 .. 252. Two compares of |x| (the
// absolute value is an operand modifier); NaN, zero and infinity fail them.
ITR_DEV bool rcp_in(float x) { return fabsf(x) >= 0x1p-125f && fabsf(x) < 0x1p126f; }

ITR_DEV float2 rcp2f(float2 x, unsigned exact) {
  const float2 y = make_float2(rcp_est(x.x), rcp_est(x.y));
  const float2 e = fma2(neg2(x), y, f2(1.0f));
  float2 r = fma2(y, e, y);
  if (__any_sync(0xffffffffu, !(rcp_in(x.x) && rcp_in(x.y)) || exact)) r = rcp2(x);
  return r;
}
// canon (a == 0 ? +0 : a) as one paired add of +0: x + 0 is x for every x except -0, which
// rounds to +0; a NaN stays a NaN (its payload may differ, which no result depends on).
ITR_DEV float2 canon2(float2 a) { return add2(a, f2(0.0f)); }
// max(a, 0) with the reference's NaN rule (a > 0 ? a : 0): the hardware maximum with +0 gives
// the same bits for all 2^32 inputs of each component (checked exhaustively on the B200,
// NaN and -0 included), in one instruction per component instead of a compare and a select.
ITR_DEV float2 max2z(float2 a) { return make_float2(fmaxf(a.x, 0.0f), fmaxf(a.y, 0.0f)); }
ITR_DEV float2 abs2(float2 a) { return make_float2(rabs(a.x), rabs(a.y)); }

ITR_DEV float2 rcbrt2(float2 x, float nz) {
  float2 r = make_float2(__uint_as_float(0x54A23280u - __float_as_uint(x.x) / 3u),
                         __uint_as_float(0x54A23280u - __float_as_uint(x.y) / 3u));
  const float2 x3 = mul2(x, f2((float)(1.0 / 3.0)), nz);
  const float2 c43 = f2((float)(4.0 * (1.0 / 3.0)));
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float2 r2 = mul2(r, r, nz);
    r = sub2(mul2(r, c43, nz), mul2(x3, mul2(r2, r2, nz), nz));
  }
  return r;
}

// hll (numerics.rs:56-93) on two faces.
ITR_DEV Face2 hll2(float2 hl, float2 ul, float2 tl, float2 cl, float2 hr, float2 ur, float2 tr, float2 cr, float g_half, float nz,
                   unsigned exact) {
  const float NZ = nz;
  const B2 dry_l = not2(gt2(hl, 0.0f));
  const B2 dry_r = not2(gt2(hr, 0.0f));
  const float2 ustar = sub2(add2(mul2(f2(0.5f), add2(ul, ur), NZ), cl), cr);
  const float2 cstar = add2(mul2(f2(0.5f), add2(cl, cr), NZ), mul2(f2(0.25f), sub2(ul, ur), NZ));
  const float2 ul_cl = sub2(ul, cl);
  const float2 ur_cr = add2(ur, cr);
  const float2 slw = min2(ul_cl, sub2(ustar, cstar));
  const float2 srw = max2(ur_cr, add2(ustar, cstar));
  const float2 sl = sel2(dry_l, sub2(ur, mul2(f2(2.0f), cr, NZ)), sel2(dry_r, ul_cl, slw));
  const float2 sr = sel2(dry_l, ur_cr, sel2(dry_r, add2(ul, mul2(f2(2.0f), cl, NZ)), srw));
  const float2 ml = mul2(hl, ul, NZ);
  const float2 mr = mul2(hr, ur, NZ);
  const float2 gh = f2(g_half);
  const float2 pl_ = mul2(mul2(gh, hl, NZ), hl, NZ);
  const float2 pr_ = mul2(mul2(gh, hr, NZ), hr, NZ);
  const float2 pl = add2(mul2(ml, ul, NZ), pl_);
  const float2 pr = add2(mul2(mr, ur, NZ), pr_);
  const B2 both_dry = and2(dry_l, dry_r);
  const B2 use_l = ge2(sl, 0.0f);
  const B2 use_r = le2(sr, 0.0f);
  const B2 trivial = or2(or2(both_dry, use_l), use_r);
  const float2 den = sel2(trivial, f2(1.0f), sub2(sr, sl));
  const float2 inv = rcp2f(den, exact);
  const float2 slsr = mul2(sl, sr, NZ);
  const float2 fm_star = mul2(add2(sub2(mul2(sr, ml, NZ), mul2(sl, mr, NZ)), mul2(slsr, sub2(hr, hl), NZ)), inv, NZ);
  const float2 fn_star = mul2(add2(sub2(mul2(sr, pl, NZ), mul2(sl, pr, NZ)), mul2(slsr, sub2(mr, ml), NZ)), inv, NZ);
  const float2 fm = sel2(both_dry, f2(0.0f), sel2(use_l, ml, sel2(use_r, mr, fm_star)));
  const float2 fn = sel2(both_dry, f2(0.0f), sel2(use_l, pl, sel2(use_r, pr, fn_star)));
  Face2 f;
  f.m = fm;
  f.nl = sub2(fn, pl_);
  f.nr = sub2(fn, pr_);
  f.t = mul2(fm, sel2(gt2(fm, 0.0f), tl, tr), NZ);
  return f;
}

// face_signed / face_crest (numerics.rs:95-129) on two faces; (ul,vl,cl) of the low side.
template <bool NORMAL_X, bool CREST>
ITR_DEV Face2 face2(float2 hl, float2 ul, float2 vl, float2 cl, float2 hr, float2 ur, float2 vr, float2 cr,
                    float2 d0, float2 d1, const StepK& k) {
  const float NZ = k.nz;
  float2 hsl, hsr, csl, csr;
  if (!CREST) {
    const B2 pos = gt2(d0, 0.0f);
    hsl = max2z(sub2(hl, max2z(d0)));
    hsr = max2z(sub2(hr, max2z(neg2(d0))));
    const float2 cred = sqrt2(mul2(f2(k.g), sel2(pos, hsl, hsr), NZ));
    csl = sel2(pos, cred, cl);
    csr = sel2(pos, cr, cred);
  } else {
    hsl = max2z(sub2(hl, d0));
    hsr = max2z(sub2(hr, d1));
    const B2 pl = gt2(d0, 0.0f), pr = gt2(d1, 0.0f);
    const float2 sl = sqrt2(mul2(f2(k.g), hsl, NZ)), sr = sqrt2(mul2(f2(k.g), hsr, NZ));
    csl = sel2(pl, sl, cl);
    csr = sel2(pr, sr, cr);
  }
  if (NORMAL_X) return hll2(hsl, ul, vl, csl, hsr, ur, vr, csr, k.g_half, NZ, k.exact);
  return hll2(hsl, vl, ul, csl, hsr, vr, ur, csr, k.g_half, NZ, k.exact);
}

struct CellNew2 {
  float2 h, qx, qy, s, infil, fix, c;
  B2 bad;
};

// flux_update then sources (numerics.rs:144-195) on two cells.
ITR_DEV CellNew2 update_cell2(float2 h, float2 qx, float2 qy, const Face2& w, const Face2& e, const Face2& n,
                              const Face2& s, float2 wet, float2 gn2, const StepK& k) {
  const float NZ = k.nz;
  const float2 dtdx = f2(k.dtdx), dtdy = f2(k.dtdy);
  float2 h1 = sub2(sub2(h, mul2(dtdx, sub2(e.m, w.m), NZ)), mul2(dtdy, sub2(s.m, n.m), NZ));
  const float2 qx1 = sub2(sub2(qx, mul2(dtdx, sub2(e.nl, w.nr), NZ)), mul2(dtdy, sub2(s.t, n.t), NZ));
  const float2 qy1 = sub2(sub2(qy, mul2(dtdx, sub2(e.t, w.t), NZ)), mul2(dtdy, sub2(s.nl, n.nr), NZ));
  CellNew2 o;
  B2 bad = not2(B2{h1.x >= -k.h_dry, h1.y >= -k.h_dry});
  const B2 neg = lt2(h1, 0.0f);
  o.fix = max2z(neg2(h1));   // h1 < 0 ? -h1 : 0, the same bits for every h1
  h1 = sel2(neg, f2(0.0f), h1);
  const float2 h2 = add2(h1, mul2(f2(k.rain), wet, NZ));
  o.infil = min2(mul2(f2(k.cap), wet, NZ), h2);
  const float2 h3 = sub2(h2, o.infil);
  const B2 dry = lt2(h3, k.h_dry);
  const float2 r = rcbrt2(sel2(dry, f2(1.0f), h3), NZ);
  const float2 r3 = mul2(mul2(r, r, NZ), r, NZ);
  const float2 r7 = mul2(mul2(r3, r3, NZ), r, NZ);
  const float2 qm = sqrt2(add2(mul2(qx1, qx1, NZ), mul2(qy1, qy1, NZ)));
  const float2 inv = rcp2f(add2(f2(1.0f), mul2(mul2(mul2(f2(k.dt), gn2, NZ), qm, NZ), r7, NZ)), k.exact);
  const float2 keep = sel2(dry, f2(0.0f), f2(1.0f));
  float2 qx2 = mul2(mul2(qx1, inv, NZ), keep, NZ);
  float2 qy2 = mul2(mul2(qy1, inv, NZ), keep, NZ);
  qx2 = sel2(lt2(abs2(qx2), k.q_min), f2(0.0f), qx2);
  qy2 = sel2(lt2(abs2(qy2), k.q_min), f2(0.0f), qy2);
  const float2 c = sqrt2(mul2(f2(k.g), h3, NZ));
  o.s = add2(mul2(add2(mul2(abs2(qx2), r3, NZ), c), f2(k.inv_dx), NZ), mul2(add2(mul2(abs2(qy2), r3, NZ), c), f2(k.inv_dy), NZ));
  o.bad = B2{bad.x || !(qm.x == qm.x), bad.y || !(qm.y == qm.y)};
  o.h = canon2(h3);
  o.qx = canon2(qx2);
  o.qy = canon2(qy2);
  o.c = c;
  return o;
}

}  // namespace itr
