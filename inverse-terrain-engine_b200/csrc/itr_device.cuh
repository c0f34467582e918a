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
};

// A face flux tuple: mass, normal momentum seen from the low-index (n_l) and high-index
// (n_r) cell with the hydrostatic pressure correction folded in, tangential momentum.
struct FaceF { float m, nl, nr, t; };

// Desingularised velocity and celerity of a cell.
ITR_DEV void cell_vel(float h, float qx, float qy, float g, float heps2, float& u, float& v, float& c) {
  float h2 = h * h;
  float inv = 1.0f / (h2 + rmax(h2, heps2));
  float t = (h + h) * inv;
  u = qx * t;
  v = qy * t;
  c = sqrtf(g * h);
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
  float inv = 1.0f / den;
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
  float cred = sqrtf(g * hred);
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
  float csl = d_l > 0.0f ? sqrtf(g * hsl) : cl;
  float csr = d_r > 0.0f ? sqrtf(g * hsr) : cr;
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
  float qm = sqrtf(qx1 * qx1 + qy1 * qy1);
  float inv = 1.0f / (1.0f + k.dt * gn2 * qm * r7);
  float keep = dry ? 0.0f : 1.0f;
  float qx2 = qx1 * inv * keep;
  float qy2 = qy1 * inv * keep;
  if (rabs(qx2) < k.q_min) qx2 = 0.0f;
  if (rabs(qy2) < k.q_min) qy2 = 0.0f;
  float c = sqrtf(k.g * h3);
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

// Run-wide scalars of one call.
struct RunParams {
  double duration, sync, cfl, dt_max, h_dry, h_eps, infil, initial_depth;
  double dx, dy, g, area, wet_count;
  uint32_t n_sync;
  int skip_dry;
  Rain rain;
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
};

}  // namespace itr
