// itr_oracle.hpp — CPU restatement of the reference solver, test infrastructure only: the results the tests compare with.
//
// TEST INFRASTRUCTURE. This header is the parity oracle for the B200 batched forward
// operator. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
// load it (through oracle/liboracle.so). No product code includes or links it.
//
// It restates, in operation order, the reference crates (paths relative to the
// reference project root):
//   crates/itr-core/src/real.rs        rcbrt (f32/f64), FixedSum, max_slice, NaN-aware max/min
//   crates/itr-core/src/scenario.rs    Hyetograph::{rate, integral}        (:540-585)
//   crates/itr-hydro/src/numerics.rs   cell_vel, hll, face_signed, face_crest,
//                                      flux_update, sources                (:38-213)
//   crates/itr-hydro/src/terrain.rs    TerrainBase::build, coarsen, face_x/face_y,
//                                      PreparedTerrain::apply_edit          (:262-514)
//   crates/itr-hydro/src/boundary.rs   fill_ghosts (wall, transmissive, stage, inflow)
//   crates/itr-hydro/src/kernel.rs     step_oracle (:503) and step_fused with dry-row
//                                      skipping (:573), row accounting and monitors
//   crates/itr-hydro/src/solver.rs     consts, init_state, initial_smax, run_impl (:269-660)
//   crates/itr-core/src/objective.rs   evaluate, guard_breach, running_lower_bound
//   crates/itr-core/src/design.rs      Primitive::profile, materialize     (:95-385)
//   crates/itr-hydro/src/validation.rs the 8 analytic cases (x f32/f64 = 16)
//
// Compile with -ffp-contract=off -fno-fast-math: the reference's rule is "IEEE + - * / sqrt
// only, no FMA" (spec.md:618), so the f32 path here is bit-for-bit the reference's.
#pragma once
#include <cstdint>
#include <cstring>
#include <cmath>
#include <vector>
#include <string>
#include <algorithm>
#include <limits>
#include "itr_math.h"   // shared exp/log1p (inverse-terrain-engine_b200/csrc)

namespace orc {

// ---------------------------------------------------------------- real.rs ----------
template <class T> struct RealT;
template <> struct RealT<float> { using U = uint32_t; static constexpr const char* NAME = "f32"; };
template <> struct RealT<double> { using U = uint64_t; static constexpr const char* NAME = "f64"; };

// Real::max / Real::min (real.rs:44-51): `a > b ? a : b`; a NaN operand yields `b`.
template <class T> inline T rmax(T a, T b) { return a > b ? a : b; }
template <class T> inline T rmin(T a, T b) { return a < b ? a : b; }
// Real::abs (real.rs:38-41): -x only for x < 0, so -0.0 stays -0.0.
template <class T> inline T rabs(T a) { return a < T(0) ? -a : a; }
// Real::canon_zero (real.rs:55-58).
template <class T> inline T canon_zero(T a) { return a == T(0) ? T(0) : a; }

// Rust's inherent f64::min / f64::max (IEEE minNum/maxNum): the non-NaN operand wins.
inline double fmin_num(double a, double b) { if (a != a) return b; if (b != b) return a; return a < b ? a : b; }
inline double fmax_num(double a, double b) { if (a != a) return b; if (b != b) return a; return a > b ? a : b; }

// Real::rcbrt for f32 (real.rs:116-130): bit seed 0x54A23280 - bits/3, 3 short Newton steps.
inline float rcbrt(float x) {
  uint32_t bits; std::memcpy(&bits, &x, 4);
  uint32_t rb = 0x54A23280u - bits / 3u;
  float r; std::memcpy(&r, &rb, 4);
  const float x3 = x * (float)(1.0 / 3.0);
  const float c43 = (float)(4.0 * (1.0 / 3.0));
  for (int i = 0; i < 3; ++i) { float r2 = r * r; r = r * c43 - x3 * (r2 * r2); }
  return r;
}
// Real::rcbrt for f64 (real.rs:81-95): seed offset scaled to the f64 mantissa, 4 steps.
inline double rcbrt(double x) {
  const uint64_t K = 0x5540000000000000ull - (0x8782Bull << 29);
  uint64_t bits; std::memcpy(&bits, &x, 8);
  uint64_t rb = K - bits / 3u;
  double r; std::memcpy(&r, &rb, 8);
  const double third = 1.0 / 3.0;
  const double x3 = x * third;
  const double c43 = 4.0 * third;
  for (int i = 0; i < 4; ++i) { double r2 = r * r; r = r * c43 - x3 * (r2 * r2); }
  return r;
}

// FixedSum (real.rs:132-175): 16 lanes indexed by column & 15, fixed pairwise total.
template <class T> struct FixedSum {
  T acc[16];
  FixedSum() { for (int l = 0; l < 16; ++l) acc[l] = T(0); }
  void add(size_t col, T v) { acc[col & 15] += v; }
  // add_slice: element k has column k.
  void add_slice(const T* v, size_t n) { for (size_t k = 0; k < n; ++k) acc[k & 15] += v[k]; }
  T total() const {
    T l8[8];
    for (int k = 0; k < 8; ++k) l8[k] = acc[2 * k] + acc[2 * k + 1];
    T l4[4] = {l8[0] + l8[1], l8[2] + l8[3], l8[4] + l8[5], l8[6] + l8[7]};
    return (l4[0] + l4[1]) + (l4[2] + l4[3]);
  }
};

// max_slice (real.rs:177-191).
template <class T> inline T max_slice(const T* v, size_t n) {
  T m[16];
  for (int l = 0; l < 16; ++l) m[l] = T(0);
  for (size_t k = 0; k < n; ++k) m[k & 15] = rmax(m[k & 15], v[k]);
  T a = T(0);
  for (int l = 0; l < 16; ++l) a = rmax(a, m[l]);
  return a;
}

// ------------------------------------------------------------ scenario.rs ----------
// Hyetograph (scenario.rs:526-586): piecewise-linear (t [s], rate [m/s]), constant
// extrapolation, exact trapezoid integral split at breakpoints.
struct Hyetograph {
  std::vector<double> t, r;
  double rate(double x) const {
    size_t n = t.size();
    if (n == 0) return 0.0;
    if (x <= t[0]) return r[0];
    for (size_t k = 0; k + 1 < n; ++k) {
      if (x <= t[k + 1]) {
        double t0 = t[k], r0 = r[k], t1 = t[k + 1], r1 = r[k + 1];
        if (t1 == t0) return r1;
        return r0 + (r1 - r0) * (x - t0) / (t1 - t0);
      }
    }
    return r[n - 1];
  }
  double integral(double a, double b) const {
    if (b <= a) return 0.0;
    if (t.empty()) return 0.0;
    double total = 0.0, tt = a, rr = rate(a);
    for (size_t k = 0; k < t.size(); ++k) {
      double tk = t[k];
      if (tk > a && tk < b) {
        double rk = rate(tk);
        total += 0.5 * (rr + rk) * (tk - tt);
        tt = tk; rr = rk;
      }
    }
    double rb = rate(b);
    total += 0.5 * (rr + rb) * (b - tt);
    return total;
  }
  bool is_zero() const { for (double v : r) if (v != 0.0) return false; return true; }
};

// ------------------------------------------------------------ numerics.rs ----------
template <class T> struct StepConsts {
  T g, g_half, dt, dtdx, dtdy, inv_dx, inv_dy, h_dry, heps2, q_min, rain, cap;
};
template <class T> struct Vel { T u, v, c; };
template <class T> struct Face { T m, n_l, n_r, t; };

// cell_vel (numerics.rs:36-43).
template <class T> inline Vel<T> cell_vel(T h, T qx, T qy, const StepConsts<T>& k) {
  T h2 = h * h;
  T inv = T(1) / (h2 + rmax(h2, k.heps2));
  T t = (h + h) * inv;
  return Vel<T>{qx * t, qy * t, std::sqrt(k.g * h)};
}

// hll (numerics.rs:56-93).
template <class T>
inline Face<T> hll(T hl, T ul, T tl, T cl, T hr, T ur, T tr, T cr, const StepConsts<T>& k) {
  const T z = T(0), half = T(0.5), quarter = T(0.25), two = T(2.0);
  bool dry_l = !(hl > z), dry_r = !(hr > z);
  T ustar = half * (ul + ur) + cl - cr;
  T cstar = half * (cl + cr) + quarter * (ul - ur);
  T slw = rmin(ul - cl, ustar - cstar);
  T srw = rmax(ur + cr, ustar + cstar);
  T sl = dry_l ? ur - two * cr : (dry_r ? ul - cl : slw);
  T sr = dry_l ? ur + cr : (dry_r ? ul + two * cl : srw);
  T ml = hl * ul, mr = hr * ur;
  T pl_ = k.g_half * hl * hl, pr_ = k.g_half * hr * hr;
  T pl = ml * ul + pl_, pr = mr * ur + pr_;
  bool both_dry = dry_l && dry_r;
  bool use_l = sl >= z, use_r = sr <= z;
  T den = (both_dry || use_l || use_r) ? T(1) : sr - sl;
  T inv = T(1) / den;
  T slsr = sl * sr;
  T fm_star = (sr * ml - sl * mr + slsr * (hr - hl)) * inv;
  T fn_star = (sr * pl - sl * pr + slsr * (mr - ml)) * inv;
  T fm = both_dry ? z : (use_l ? ml : (use_r ? mr : fm_star));
  T fn = both_dry ? z : (use_l ? pl : (use_r ? pr : fn_star));
  T ft = fm * (fm > z ? tl : tr);
  return Face<T>{fm, fn - pl_, fn - pr_, ft};
}

// face_signed (numerics.rs:95-112).
template <class T>
inline Face<T> face_signed(T hl, Vel<T> vl, T hr, Vel<T> vr, T dz, bool normal_x, const StepConsts<T>& k) {
  const T z = T(0);
  bool pos = dz > z;
  T hsl = rmax(hl - rmax(dz, z), z);
  T hsr = rmax(hr - rmax(-dz, z), z);
  T hred = pos ? hsl : hsr;
  T cred = std::sqrt(k.g * hred);
  T csl = pos ? cred : vl.c;
  T csr = pos ? vr.c : cred;
  if (normal_x) return hll(hsl, vl.u, vl.v, csl, hsr, vr.u, vr.v, csr, k);
  return hll(hsl, vl.v, vl.u, csl, hsr, vr.v, vr.u, csr, k);
}

// face_crest (numerics.rs:114-129).
template <class T>
inline Face<T> face_crest(T hl, Vel<T> vl, T hr, Vel<T> vr, T d_l, T d_r, bool normal_x, const StepConsts<T>& k) {
  const T z = T(0);
  T hsl = rmax(hl - d_l, z);
  T hsr = rmax(hr - d_r, z);
  T csl = d_l > z ? std::sqrt(k.g * hsl) : vl.c;
  T csr = d_r > z ? std::sqrt(k.g * hsr) : vr.c;
  if (normal_x) return hll(hsl, vl.u, vl.v, csl, hsr, vr.u, vr.v, csr, k);
  return hll(hsl, vl.v, vl.u, csl, hsr, vr.v, vr.u, csr, k);
}

template <class T> struct CellOut { T h, qx, qy, s, infil, fix; bool bad; };

// flux_update (numerics.rs:144-153).
template <class T>
inline void flux_update(T h, T qx, T qy, const Face<T>& w, const Face<T>& e, const Face<T>& n,
                        const Face<T>& s, const StepConsts<T>& k, T& h1, T& qx1, T& qy1) {
  h1 = h - k.dtdx * (e.m - w.m) - k.dtdy * (s.m - n.m);
  qx1 = qx - k.dtdx * (e.n_l - w.n_r) - k.dtdy * (s.t - n.t);
  qy1 = qy - k.dtdx * (e.t - w.t) - k.dtdy * (s.n_l - n.n_r);
}

// sources (numerics.rs:155-195).
template <class T>
inline CellOut<T> sources(T h1, T qx1, T qy1, T wet, T gn2, const StepConsts<T>& k) {
  const T z = T(0);
  bool bad = !(h1 >= -k.h_dry);
  T fix = h1 < z ? -h1 : z;
  if (h1 < z) h1 = z;
  T h2 = h1 + k.rain * wet;
  T infil = rmin(k.cap * wet, h2);
  T h3 = h2 - infil;
  bool dry = h3 < k.h_dry;
  T r = rcbrt(dry ? T(1) : h3);
  T r3 = r * r * r;
  T r7 = r3 * r3 * r;
  T qm = std::sqrt(qx1 * qx1 + qy1 * qy1);
  T inv = T(1) / (T(1) + k.dt * gn2 * qm * r7);
  T keep = dry ? z : T(1);
  T qx2 = qx1 * inv * keep;
  T qy2 = qy1 * inv * keep;
  if (rabs(qx2) < k.q_min) qx2 = z;
  if (rabs(qy2) < k.q_min) qy2 = z;
  T c = std::sqrt(k.g * h3);
  T s_rate = (rabs(qx2) * r3 + c) * k.inv_dx + (rabs(qy2) * r3 + c) * k.inv_dy;
  bad = bad || !(qm == qm);
  return CellOut<T>{canon_zero(h3), canon_zero(qx2), canon_zero(qy2), s_rate, infil, fix, bad};
}

// -------------------------------------------------------- aligned.rs / terrain -----
// Padded row-major layout with a 1-cell ghost ring (aligned.rs:149-183). Alignment does not
// change results, so the stride here is simply nx + 2; padded column 0 is the west ghost.
struct Layout {
  size_t nx = 0, ny = 0, stride = 0;
  Layout() {}
  Layout(size_t nx_, size_t ny_) : nx(nx_), ny(ny_), stride(nx_ + 2) {}
  size_t at(size_t i, size_t j) const { return j * stride + i; }
  size_t row(size_t j) const { return j * stride; }
  size_t len() const { return (ny + 2) * stride; }
};

enum GhostKind : int { GH_WALL = 0, GH_TRANSMISSIVE = 1, GH_STAGE = 2, GH_INFLOW = 3 };
struct Ghost { int kind = GH_WALL; double stage = 0.0; int hydro = 0; double inv_len = 0.0; };

struct Boundaries {
  std::vector<Ghost> north, south, west, east;
  std::vector<Hyetograph> hydrographs;
};

// BoundarySegment (scenario.rs) restated: kind 0 stage, 1 inflow, 2 transmissive.
struct Segment {
  int kind = 2;  // 0 stage, 1 inflow, 2 transmissive
  int side = 0;  // 0 north, 1 south, 2 west, 3 east
  bool has_range = false; double r0 = 0, r1 = 0;
  double stage_m = 0;
  std::vector<double> ht, hq;  // inflow hydrograph (t, m3/s)
};

// Boundaries::from_segments (terrain.rs:151-187).
inline Boundaries boundaries_from_segments(const std::vector<Segment>& segs, size_t nx, size_t ny,
                                           double dx, double dy, double z_ref) {
  Boundaries b;
  b.north.assign(nx, Ghost{}); b.south.assign(nx, Ghost{});
  b.west.assign(ny, Ghost{}); b.east.assign(ny, Ghost{});
  for (const Segment& s : segs) {
    size_t n = (s.side <= 1) ? nx : ny;
    double d = (s.side <= 1) ? dx : dy;
    size_t a = 0, e = n;
    if (s.has_range) {
      double fa = std::floor(s.r0 / d); if (fa < 0) fa = 0;
      double fe = std::ceil(s.r1 / d); if (fe < 0) fe = 0;
      a = std::min((size_t)fa, n); e = std::min((size_t)fe, n);
    }
    double len_m = (double)(e > a ? e - a : 0) * d;
    Ghost g;
    if (s.kind == 0) { g.kind = GH_STAGE; g.stage = s.stage_m - z_ref; }
    else if (s.kind == 2) { g.kind = GH_TRANSMISSIVE; }
    else {
      Hyetograph h; h.t = s.ht; h.r = s.hq;
      b.hydrographs.push_back(h);
      g.kind = GH_INFLOW; g.hydro = (int)b.hydrographs.size() - 1;
      g.inv_len = len_m > 0.0 ? 1.0 / len_m : 0.0;
    }
    std::vector<Ghost>& v = s.side == 0 ? b.north : s.side == 1 ? b.south : s.side == 2 ? b.west : b.east;
    for (size_t x = a; x < e && x < v.size(); ++x) v[x] = g;
  }
  return b;
}

// FineTerrain (terrain.rs:190-235).
struct FineTerrain {
  size_t nx = 0, ny = 0;
  double origin_x = 0, origin_y = 0, dx = 1, dy = 1;
  std::vector<double> z;   // re-based
  std::vector<uint8_t> wall;
  double z_ref = 0, z_wall = 0;
  std::vector<double> n;   // Manning n
};

inline FineTerrain fine_terrain(size_t nx, size_t ny, double ox, double oy, double dx, double dy,
                                const double* dem, const uint8_t* walls, const double* manning) {
  FineTerrain f;
  f.nx = nx; f.ny = ny; f.origin_x = ox; f.origin_y = oy; f.dx = dx; f.dy = dy;
  double zmin = std::numeric_limits<double>::max(), zmax = std::numeric_limits<double>::lowest();
  for (size_t i = 0; i < nx * ny; ++i)
    if (!walls[i] && std::isfinite(dem[i])) { zmin = fmin_num(zmin, dem[i]); zmax = fmax_num(zmax, dem[i]); }
  if (zmin > zmax) { zmin = 0; zmax = 0; }
  f.z_ref = std::floor(zmin);
  f.z_wall = (zmax - f.z_ref) + 100.0;
  f.z.resize(nx * ny); f.wall.resize(nx * ny); f.n.assign(manning, manning + nx * ny);
  for (size_t i = 0; i < nx * ny; ++i) {
    bool w = walls[i] || !std::isfinite(dem[i]);
    f.wall[i] = w;
    f.z[i] = w ? f.z_wall : dem[i] - f.z_ref;
  }
  return f;
}

// Sparse fine-resolution edit (design.rs:144-178).
struct TerrainEdit {
  size_t c0 = 0, r0 = 0, w = 0, h = 0;
  std::vector<double> dz;
  double cut_m3 = 0, fill_m3 = 0;
  bool is_empty() const {
    if (w == 0 || h == 0) return true;
    for (double v : dz) if (v != 0.0) return false;
    return true;
  }
  double get(size_t col, size_t row) const {
    if (col < c0 || row < r0 || col >= c0 + w || row >= r0 + h) return 0.0;
    return dz[(row - r0) * w + (col - c0)];
  }
};

enum FaceMode { SIGNED = 0, CREST = 1 };

inline double fine_z(const FineTerrain& f, size_t c, size_t r, const TerrainEdit* e) {
  return f.z[r * f.nx + c] + (e ? e->get(c, r) : 0.0);
}

// coarse_cell (terrain.rs:357-373).
inline void coarse_cell(const FineTerrain& f, size_t lv, size_t c, size_t r, const TerrainEdit* e,
                        double& zz, bool& wall, double& nn) {
  double s = 0, sn = 0, sn_all = 0; size_t cnt = 0, tot = 0;
  for (size_t rr = r * lv; rr < std::min((r + 1) * lv, f.ny); ++rr)
    for (size_t cc = c * lv; cc < std::min((c + 1) * lv, f.nx); ++cc) {
      tot += 1;
      sn_all += f.n[rr * f.nx + cc];
      if (!f.wall[rr * f.nx + cc]) { s += fine_z(f, cc, rr, e); sn += f.n[rr * f.nx + cc]; cnt += 1; }
    }
  if (cnt == 0) { zz = f.z_wall; wall = true; nn = sn_all / (double)tot; }
  else { zz = s / (double)cnt; wall = false; nn = sn / (double)cnt; }
}

// face_x / face_y (terrain.rs:375-429).
inline void face_x(const FineTerrain& f, size_t lv, FaceMode mode, double zl, double zr, size_t i,
                   size_t r, const TerrainEdit* e, double& a, double& b) {
  if (mode == SIGNED) { a = zr - zl; b = 0.0; return; }
  size_t cl = i * lv - 1, cr = std::min(i * lv, f.nx - 1);
  double crest = std::numeric_limits<double>::lowest(); bool all_wall = true;
  for (size_t rr = r * lv; rr < std::min((r + 1) * lv, f.ny); ++rr)
    for (size_t cc : {cl, cr})
      if (!f.wall[rr * f.nx + cc]) { all_wall = false; crest = fmax_num(crest, fine_z(f, cc, rr, e)); }
  if (all_wall) crest = f.z_wall;
  double zf = fmax_num(fmax_num(crest, zl), zr);
  a = zf - zl; b = zf - zr;
}
inline void face_y(const FineTerrain& f, size_t lv, FaceMode mode, double zt, double zb, size_t c,
                   size_t rb, const TerrainEdit* e, double& a, double& b) {
  if (mode == SIGNED) { a = zb - zt; b = 0.0; return; }
  size_t rt_f = rb * lv - 1, rb_f = std::min(rb * lv, f.ny - 1);
  double crest = std::numeric_limits<double>::lowest(); bool all_wall = true;
  for (size_t cc = c * lv; cc < std::min((c + 1) * lv, f.nx); ++cc)
    for (size_t rr : {rt_f, rb_f})
      if (!f.wall[rr * f.nx + cc]) { all_wall = false; crest = fmax_num(crest, fine_z(f, cc, rr, e)); }
  if (all_wall) crest = f.z_wall;
  double zf = fmax_num(fmax_num(crest, zt), zb);
  a = zf - zt; b = zf - zb;
}

// TerrainBase (terrain.rs:237-332): full padded arrays (no row dedupe; results identical).
template <class T> struct TerrainBase {
  Layout layout;
  size_t level = 1;
  double dx = 1, dy = 1, g = 9.81;
  FaceMode mode = SIGNED;
  const FineTerrain* fine = nullptr;
  std::vector<double> z;        // level z, unpadded nx*ny
  std::vector<uint8_t> wall;    // level walls
  std::vector<T> fx0, fx1, fy0, fy1, wet, gn2;   // padded
  size_t wet_count = 0;
  Boundaries bnd;
};

static const double G_ACC = 9.81;  // terrain.rs:259

template <class T>
inline void terrain_build(TerrainBase<T>& tb, const FineTerrain& fine, size_t level, const std::vector<Segment>& segs) {
  size_t lv = std::max<size_t>(level, 1);
  size_t nx = (fine.nx + lv - 1) / lv, ny = (fine.ny + lv - 1) / lv;
  tb.fine = &fine; tb.level = lv;
  tb.dx = fine.dx * (double)lv; tb.dy = fine.dy * (double)lv; tb.g = G_ACC;
  tb.layout = Layout(nx, ny);
  tb.mode = lv == 1 ? SIGNED : CREST;
  tb.z.assign(nx * ny, 0.0); tb.wall.assign(nx * ny, 0);
  std::vector<double> nv(nx * ny, 0.0);
  for (size_t r = 0; r < ny; ++r)
    for (size_t c = 0; c < nx; ++c) {
      double zz, nn; bool w;
      coarse_cell(fine, lv, c, r, nullptr, zz, w, nn);
      tb.z[r * nx + c] = zz; tb.wall[r * nx + c] = w; nv[r * nx + c] = nn;
    }
  const Layout& L = tb.layout;
  size_t len = L.len();
  tb.fx0.assign(len, T(0)); tb.fx1.assign(len, T(0)); tb.fy0.assign(len, T(0)); tb.fy1.assign(len, T(0));
  auto zc = [&](size_t c, size_t r) { return tb.z[r * nx + c]; };
  for (size_t j = 1; j <= ny; ++j)
    for (size_t i = 1; i < nx; ++i) {
      double a, b; face_x(fine, lv, tb.mode, zc(i - 1, j - 1), zc(i, j - 1), i, j - 1, nullptr, a, b);
      tb.fx0[L.at(i, j)] = (T)a; tb.fx1[L.at(i, j)] = (T)b;
    }
  for (size_t j = 1; j < ny; ++j)
    for (size_t i = 1; i <= nx; ++i) {
      double a, b; face_y(fine, lv, tb.mode, zc(i - 1, j - 1), zc(i - 1, j), i - 1, j, nullptr, a, b);
      tb.fy0[L.at(i, j)] = (T)a; tb.fy1[L.at(i, j)] = (T)b;
    }
  tb.wet.assign(len, T(0)); tb.gn2.assign(len, T(0)); tb.wet_count = 0;
  for (size_t j = 1; j <= ny; ++j)
    for (size_t i = 1; i <= nx; ++i) {
      size_t k = (j - 1) * nx + (i - 1);
      bool w = !tb.wall[k];
      tb.wet[L.at(i, j)] = w ? T(1) : T(0);
      tb.wet_count += w;
      tb.gn2[L.at(i, j)] = (T)(G_ACC * nv[k] * nv[k]);
    }
  tb.bnd = boundaries_from_segments(segs, nx, ny, tb.dx, tb.dy, fine.z_ref);
}

// PreparedTerrain: base + private face arrays (copy of the base's; apply_edit rewrites
// the faces it touches, terrain.rs:458-505).
template <class T> struct PreparedTerrain {
  const TerrainBase<T>* base = nullptr;
  std::vector<T> fx0, fx1, fy0, fy1;
  std::vector<std::pair<size_t, double>> z_over;
  void reset(const TerrainBase<T>& b) {
    base = &b; fx0 = b.fx0; fx1 = b.fx1; fy0 = b.fy0; fy1 = b.fy1; z_over.clear();
  }
  std::vector<double> z_level() const {
    std::vector<double> z = base->z;
    for (auto& p : z_over) z[p.first] = p.second;
    return z;
  }
  void apply_edit(const TerrainEdit& e) {
    reset(*base);
    if (e.is_empty()) return;
    const TerrainBase<T>& b = *base;
    size_t lv = b.level, nx = b.layout.nx, ny = b.layout.ny;
    size_t c0 = e.c0 / lv, r0 = e.r0 / lv;
    size_t c1 = std::min((e.c0 + e.w + lv - 1) / lv, nx), r1 = std::min((e.r0 + e.h + lv - 1) / lv, ny);
    std::vector<double> zl = b.z;
    for (size_t r = r0; r < r1; ++r)
      for (size_t c = c0; c < c1; ++c) {
        double zz, nn; bool w;
        coarse_cell(*b.fine, lv, c, r, &e, zz, w, nn);
        zl[r * nx + c] = zz;
        z_over.push_back({r * nx + c, zz});
      }
    auto zc = [&](size_t c, size_t r) { return zl[r * nx + c]; };
    const Layout& L = b.layout;
    for (size_t r = r0; r < r1; ++r)
      for (size_t cl = (c0 > 0 ? c0 - 1 : 0); cl < std::min(c1, nx - 1); ++cl) {
        size_t i = cl + 1; double a, bb;
        face_x(*b.fine, lv, b.mode, zc(cl, r), zc(cl + 1, r), i, r, &e, a, bb);
        fx0[L.at(i, r + 1)] = (T)a;
        if (b.mode == CREST) fx1[L.at(i, r + 1)] = (T)bb;
      }
    for (size_t rt = (r0 > 0 ? r0 - 1 : 0); rt < std::min(r1, ny - 1); ++rt)
      for (size_t c = c0; c < c1; ++c) {
        double a, bb;
        face_y(*b.fine, lv, b.mode, zc(c, rt), zc(c, rt + 1), c, rt + 1, &e, a, bb);
        fy0[L.at(c + 1, rt + 1)] = (T)a;
        if (b.mode == CREST) fy1[L.at(c + 1, rt + 1)] = (T)bb;
      }
  }
};

// --------------------------------------------------------------- design.rs ---------
enum PrimKind { BERM = 0, SWALE = 1, CUT = 2, MOUND = 3 };
struct Primitive { int kind = BERM; double cx = 0, cy = 0, length = 0, width = 1, angle_deg = 0, height = 0; };

inline void prim_segment(const Primitive& p, double& x0, double& y0, double& x1, double& y1) {
  if (p.kind == MOUND) { x0 = x1 = p.cx; y0 = y1 = p.cy; return; }
  double a = p.angle_deg * (3.141592653589793 / 180.0);   // f64::to_radians
  double s = std::sin(a), c = std::cos(a);   // libm sin/cos, as libm::sin/cos
  double hl = 0.5 * p.length;
  x0 = p.cx - c * hl; y0 = p.cy - s * hl; x1 = p.cx + c * hl; y1 = p.cy + s * hl;
}
// Primitive::profile (design.rs:107-134).
inline double prim_profile(const Primitive& p, double x, double y) {
  double x0, y0, x1, y1; prim_segment(p, x0, y0, x1, y1);
  double vx = x1 - x0, vy = y1 - y0;
  double l2 = vx * vx + vy * vy;
  double t = 0.0;
  if (l2 > 0.0) { t = ((x - x0) * vx + (y - y0) * vy) / l2; t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t); }
  double px = x0 + t * vx - x, py = y0 + t * vy - y;
  double d = std::sqrt(px * px + py * py);
  double s = d / (0.5 * p.width);
  if (s >= 1.0) return 0.0;
  if (p.kind == CUT) {
    if (s <= 0.5) return 1.0;
    double u = (s - 0.5) / 0.5; double w = 1.0 - u * u; return w * w;
  }
  double w = 1.0 - s * s; return w * w;
}
inline void prim_bbox(const Primitive& p, double& a, double& b, double& c, double& d) {
  double x0, y0, x1, y1; prim_segment(p, x0, y0, x1, y1);
  double r = 0.5 * p.width;
  a = fmin_num(x0, x1) - r; b = fmin_num(y0, y1) - r; c = fmax_num(x0, x1) + r; d = fmax_num(y0, y1) + r;
}

// DesignSpace::materialize (design.rs:316-385).
inline TerrainEdit materialize(const std::vector<Primitive>& prims, double ox, double oy, double dx, double dy,
                               size_t nx, size_t ny, const uint8_t* editable, double max_abs_dz) {
  TerrainEdit e;
  size_t c0 = SIZE_MAX, r0 = SIZE_MAX, c1 = 0, r1 = 0;
  auto fl = [](double v) { v = std::floor(v); return v < 0 ? 0.0 : v; };
  auto ce = [](double v) { v = std::ceil(v); return v < 0 ? 0.0 : v; };
  for (const Primitive& p : prims) {
    if (p.height == 0.0) continue;
    double x0, y0, x1, y1; prim_bbox(p, x0, y0, x1, y1);
    double fc0 = (x0 - ox) / dx, fr1 = (oy - y0) / dy;
    double fc1 = (x1 - ox) / dx, fr0 = (oy - y1) / dy;
    size_t a = std::min((size_t)fl(fc0), nx), b = std::min((size_t)fl(fr0), ny);
    size_t c = std::min((size_t)ce(fc1), nx), d = std::min((size_t)ce(fr1), ny);
    if (a < c && b < d) { c0 = std::min(c0, a); r0 = std::min(r0, b); c1 = std::max(c1, c); r1 = std::max(r1, d); }
  }
  if (c0 >= c1 || r0 >= r1) return e;
  size_t w = c1 - c0, h = r1 - r0;
  std::vector<double> dz(w * h, 0.0);
  const size_t S = 4; const double inv = 1.0 / (double)(S * S);
  for (size_t r = 0; r < h; ++r)
    for (size_t c = 0; c < w; ++c) {
      size_t col = c0 + c, row = r0 + r;
      if (!editable[row * nx + col]) continue;
      double acc = 0.0;
      for (const Primitive& p : prims) {
        if (p.height == 0.0) continue;
        double s = 0.0;
        for (size_t sy = 0; sy < S; ++sy)
          for (size_t sx = 0; sx < S; ++sx) {
            double x = ox + ((double)col + ((double)sx + 0.5) / (double)S) * dx;
            double y = oy - ((double)row + ((double)sy + 0.5) / (double)S) * dy;
            s += prim_profile(p, x, y);
          }
        acc += p.height * s * inv;
      }
      dz[r * w + c] = acc < -max_abs_dz ? -max_abs_dz : (acc > max_abs_dz ? max_abs_dz : acc);
    }
  double a = dx * dy;
  for (double v : dz) { if (v > 0.0) e.fill_m3 += v * a; else e.cut_m3 -= v * a; }
  e.c0 = c0; e.r0 = r0; e.w = w; e.h = h; e.dz = dz;
  return e;
}

// ------------------------------------------------------------- objective.rs --------
struct Asset { std::vector<size_t> pos; double threshold = 0, weight = 1; };
struct Objective {
  std::vector<Asset> assets;
  std::vector<size_t> guard_pos;   // positions in the monitor list, in guard-cell order
  std::vector<uint32_t> mon_cells; // monitor cell ids (for the breach cell id)
  double guard_tol = 0.02, tau = 0.02, cut_cost = 1, fill_cost = 1, earth_weight = 1e-5;
  bool require_no_worsening = true;
};

// softplus (objective.rs:70-75) on the shared exp/log1p restatement.
inline double softplus(double x) { return itr_math::softplus(x); }

struct ObjReport { double j = 0, j_risk = 0, j_earth = 0, worst = 0, violation = 0; bool feasible = true; std::vector<double> peaks; };

// Objective::evaluate (objective.rs:94-128).
inline ObjReport obj_evaluate(const Objective& o, const double* mm, double cut, double fill, const double* baseline) {
  ObjReport r;
  for (const Asset& a : o.assets) {
    double pk = 0.0;
    for (size_t k : a.pos) pk = fmax_num(pk, mm[k]);
    r.peaks.push_back(pk);
    r.j_risk += a.weight * o.tau * softplus((pk - a.threshold) / o.tau);
  }
  r.j_earth = o.cut_cost * cut + o.fill_cost * fill;
  r.j = r.j_risk + o.earth_weight * r.j_earth;
  if (baseline) {
    double worst = 0.0;
    for (size_t k : o.guard_pos) worst = fmax_num(worst, mm[k] - baseline[k]);
    r.worst = worst;
    if (o.require_no_worsening && worst > o.guard_tol) r.violation = worst - o.guard_tol;
  }
  r.feasible = r.violation == 0.0;
  return r;
}

// ---------------------------------------------------------------- solver ----------
struct Params {
  double duration = 60, sync = 10, cfl = 0.35, dt_max = 5, h_dry = 1e-6, h_eps = 1e-5;
  Hyetograph rain;
  double infil_capacity = 0, initial_depth = 0;
  bool has_stage = false; double initial_stage = 0;
  bool skip_dry = true;
  double inflow_scale = 1.0;
  // Baseline-locked dt (SolverParams::locked_dt / cfl_hard, solver.rs:42-46): the baseline's
  // dt per step, each verified against cfl_hard; n_locked == 0 means adaptive dt.
  const double* locked_dt = nullptr;
  size_t n_locked = 0;
  double cfl_hard = 0.5;
  bool record_dts = false;   // keep the dt of every step (BaselineRecord::dts, solver.rs:508)
};

enum Kernel { K_ORACLE = 0, K_FUSED = 1 };
enum Abort { AB_NONE = 0, AB_GUARD = 1, AB_INCUMBENT = 2, AB_UNHEALTHY = 3 };

struct LedgerRow { double t, volume, rain, inflow, outflow, infil, fix, residual; };

struct RunResult {
  double t_end = 0; uint64_t steps = 0; uint32_t sync_count = 0;
  int abort = AB_NONE; uint32_t abort_cell = 0; double abort_exceed = 0; uint32_t abort_sync = 0; double abort_lb = 0;
  std::vector<double> mon_max, mon_tmax;
  std::vector<LedgerRow> rows;
  double v0 = 0, rel_residual = 0;
  double dt_min = 0, dt_max = 0, dt_mean = 0;
  uint64_t cell_updates = 0, rows_skipped = 0;
  std::vector<double> peak;      // per-cell running max of h (f64 compare), all cells
  std::vector<uint64_t> peak_step;
  double dt_fallback_t = -1.0;   // locked dt: time at which the run fell back to adaptive dt
  std::vector<double> dts;       // with Params::record_dts: the dt of every step, in order
};

// Optional observer config (GuardObserver, evaluator.rs:88-108).
struct ObserverCfg {
  const Objective* obj = nullptr;
  const double* baseline = nullptr;   // per monitor
  bool has_incumbent = false; double incumbent = 0;
  double cut = 0, fill = 0;
};

template <class T> struct Monitors {
  size_t nx = 0;
  std::vector<uint32_t> cells;
  std::vector<size_t> row_start;
  std::vector<double> max, tmax;
  void init(const std::vector<uint32_t>& c, size_t nx_, size_t ny) {
    nx = nx_; cells = c;
    row_start.assign(ny + 1, 0);
    size_t k = 0;
    for (size_t r = 0; r < ny; ++r) {
      row_start[r] = k;
      while (k < cells.size() && (size_t)cells[k] / nx == r) ++k;
    }
    row_start[ny] = cells.size();
    max.assign(cells.size(), 0.0); tmax.assign(cells.size(), 0.0);
  }
};

template <class T> struct StepStats {
  double smax = 0, sum_s = 0, infil = 0, fix = 0, bnd_in = 0, bnd_out = 0;
  bool bad = false; uint64_t rows_skipped = 0;
};

template <class T> struct Solver {
  Params p;
  const TerrainBase<T>* tb = nullptr;
  const PreparedTerrain<T>* terr = nullptr;
  Layout L;
  std::vector<T> h, qx, qy;
  std::vector<uint8_t> row_dry, ghost_wet, new_dry;
  std::vector<double> zlev;
  Monitors<T> mon;
  bool track_peak = false;
  std::vector<double> peak; std::vector<uint64_t> peak_step;
  uint64_t step_no = 0;
  // row buffers
  std::vector<T> vu, vv, vc;        // velocities, full padded arrays (oracle) or 2 rows (fused)
  std::vector<T> fxm, fxnl, fxnr, fxt;   // x-face rows
  std::vector<T> gm, gnl, gnr, gt;       // y-face rows
  std::vector<T> rs_infil, rs_fix, rs_s;

  StepConsts<T> consts(double dt, double rain) const {
    StepConsts<T> k;
    k.g = (T)tb->g; k.g_half = (T)(0.5 * tb->g); k.dt = (T)dt;
    k.dtdx = (T)(dt / tb->dx); k.dtdy = (T)(dt / tb->dy);
    k.inv_dx = (T)(1.0 / tb->dx); k.inv_dy = (T)(1.0 / tb->dy);
    k.h_dry = (T)p.h_dry; k.heps2 = (T)(p.h_eps * p.h_eps); k.q_min = (T)1e-30;
    k.rain = (T)rain; k.cap = (T)(p.infil_capacity * dt);
    return k;
  }

  // fill_ghosts (boundary.rs:12-87).
  void fill_ghosts(double t) {
    size_t nx = L.nx, ny = L.ny;
    double g = tb->g;
    const Boundaries& b = tb->bnd;
    auto crit = [&](double q) -> double {
      double x = q * q / g;
      return x > 0.0 ? x * rcbrt(x) * rcbrt(x) : 0.0;
    };
    auto zl = [&](size_t c, size_t r) { return zlev[r * nx + c]; };
    std::fill(ghost_wet.begin(), ghost_wet.end(), 0);
    for (size_t j = 1; j <= ny; ++j) {
      for (int side = 0; side < 2; ++side) {
        size_t gi = side == 0 ? 0 : nx + 1, ii = side == 0 ? 1 : nx;
        double inward = side == 0 ? 1.0 : -1.0;
        const Ghost& s = side == 0 ? b.west[j - 1] : b.east[j - 1];
        size_t gk = L.at(gi, j), ik = L.at(ii, j);
        T hi = h[ik], qxi = qx[ik], qyi = qy[ik], hg, qxg, qyg;
        if (s.kind == GH_WALL) { hg = hi; qxg = -qxi; qyg = qyi; }
        else if (s.kind == GH_TRANSMISSIVE) { hg = hi; qxg = qxi; qyg = qyi; }
        else if (s.kind == GH_STAGE) { hg = (T)fmax_num(s.stage - zl(ii - 1, j - 1), 0.0); qxg = qxi; qyg = qyi; }
        else {
          double q = b.hydrographs[s.hydro].rate(t) * s.inv_len * p.inflow_scale;
          double hgd = fmax_num((double)hi, crit(q));
          hg = (T)hgd; qxg = (T)(inward * q); qyg = T(0);
        }
        h[gk] = hg; qx[gk] = qxg; qy[gk] = qyg;
        if (hg > T(0)) ghost_wet[j] = 1;
      }
    }
    for (size_t i = 1; i <= nx; ++i) {
      for (int side = 0; side < 2; ++side) {
        size_t gj = side == 0 ? 0 : ny + 1, ij = side == 0 ? 1 : ny;
        double inward = side == 0 ? 1.0 : -1.0;
        const Ghost& s = side == 0 ? b.north[i - 1] : b.south[i - 1];
        size_t gk = L.at(i, gj), ik = L.at(i, ij);
        T hi = h[ik], qxi = qx[ik], qyi = qy[ik], hg, qxg, qyg;
        if (s.kind == GH_WALL) { hg = hi; qxg = qxi; qyg = -qyi; }
        else if (s.kind == GH_TRANSMISSIVE) { hg = hi; qxg = qxi; qyg = qyi; }
        else if (s.kind == GH_STAGE) { hg = (T)fmax_num(s.stage - zl(i - 1, ij - 1), 0.0); qxg = qxi; qyg = qyi; }
        else {
          double q = b.hydrographs[s.hydro].rate(t) * s.inv_len * p.inflow_scale;
          double hgd = fmax_num((double)hi, crit(q));
          hg = (T)hgd; qxg = T(0); qyg = (T)(inward * q);
        }
        h[gk] = hg; qx[gk] = qxg; qy[gk] = qyg;
        if (hg > T(0)) ghost_wet[gj] = 1;
      }
    }
    size_t corners[4][2] = {{0, 0}, {nx + 1, 0}, {0, ny + 1}, {nx + 1, ny + 1}};
    for (auto& c : corners) { size_t k = L.at(c[0], c[1]); h[k] = T(0); qx[k] = T(0); qy[k] = T(0); }
  }

  void vel_row(size_t j, T* u, T* v, T* c, const StepConsts<T>& k) {
    size_t o = L.row(j);
    for (size_t i = 0; i < L.nx + 2; ++i) {
      Vel<T> w = cell_vel(h[o + i], qx[o + i], qy[o + i], k);
      u[i] = w.u; v[i] = w.v; c[i] = w.c;
    }
  }
  // xface_row (kernel.rs:128-149): faces 0..=nx of padded row j.
  void xface_row(size_t j, const T* u, const T* v, const T* c, T* om, T* onl, T* onr, T* ot, const StepConsts<T>& k) {
    size_t o = L.row(j);
    const T* f0 = &terr->fx0[o]; const T* f1 = &terr->fx1[o];
    for (size_t i = 0; i <= L.nx; ++i) {
      Vel<T> a{u[i], v[i], c[i]}, b{u[i + 1], v[i + 1], c[i + 1]};
      Face<T> f = tb->mode == CREST ? face_crest(h[o + i], a, h[o + i + 1], b, f0[i], f1[i], true, k)
                                    : face_signed(h[o + i], a, h[o + i + 1], b, f0[i], true, k);
      om[i] = f.m; onl[i] = f.n_l; onr[i] = f.n_r; ot[i] = f.t;
    }
  }
  // yface_row (kernel.rs:151-179): faces between padded rows j and j+1, columns 1..=nx.
  void yface_row(size_t j, const T* ut, const T* vt, const T* ct, const T* ub, const T* vb, const T* cb,
                 T* om, T* onl, T* onr, T* ot, const StepConsts<T>& k) {
    size_t ot_ = L.row(j), ob = L.row(j + 1);
    const T* f0 = &terr->fy0[ot_]; const T* f1 = &terr->fy1[ot_];
    for (size_t i = 1; i <= L.nx; ++i) {
      Vel<T> a{ut[i], vt[i], ct[i]}, b{ub[i], vb[i], cb[i]};
      Face<T> f = tb->mode == CREST ? face_crest(h[ot_ + i], a, h[ob + i], b, f0[i], f1[i], false, k)
                                    : face_signed(h[ot_ + i], a, h[ob + i], b, f0[i], false, k);
      om[i] = f.m; onl[i] = f.n_l; onr[i] = f.n_r; ot[i] = f.t;
    }
  }

  struct RowAcc { double infil = 0, fix = 0, bnd_in = 0, bnd_out = 0, smax = 0, sum_s = 0; bool wet = false, bad = false, skipped = false; };

  // update_row (kernel.rs:238-309) + x_boundary + monitors_row.
  RowAcc update_row(size_t j, const T* xm, const T* xnl, const T* xnr, const T* xt,
                    const T* nm, const T* nnl, const T* nnr, const T* nt,
                    const T* sm, const T* snl, const T* snr, const T* st,
                    const StepConsts<T>& k, bool want_sum_s, double dt_dy, double t_new) {
    (void)nnl; (void)snr;
    size_t nx = L.nx, o = L.row(j);
    const T* wet = &tb->wet[o]; const T* gn2 = &tb->gn2[o];
    // Loop 1: flux divergence (values pass through memory at working precision).
    for (size_t i = 1; i <= nx; ++i) {
      Face<T> fw{xm[i - 1], T(0), xnr[i - 1], xt[i - 1]};
      Face<T> fe{xm[i], xnl[i], T(0), xt[i]};
      Face<T> fn{nm[i], T(0), nnr[i], nt[i]};
      Face<T> fs{sm[i], snl[i], T(0), st[i]};
      T a, b, c; flux_update(h[o + i], qx[o + i], qy[o + i], fw, fe, fn, fs, k, a, b, c);
      h[o + i] = a; qx[o + i] = b; qy[o + i] = c;
    }
    RowAcc acc; bool bad = false;
    for (size_t i = 1; i <= nx; ++i) {
      CellOut<T> r = sources(h[o + i], qx[o + i], qy[o + i], wet[i], gn2[i], k);
      h[o + i] = r.h; qx[o + i] = r.qx; qy[o + i] = r.qy;
      rs_infil[i] = r.infil; rs_fix[i] = r.fix; rs_s[i] = r.s;
      bad = bad || r.bad;
    }
    size_t n = nx + 2;
    FixedSum<T> si; si.add_slice(rs_infil.data(), n);
    FixedSum<T> sf; sf.add_slice(rs_fix.data(), n);
    if (want_sum_s) { FixedSum<T> ss; ss.add_slice(rs_s.data(), n); acc.sum_s = (double)ss.total(); }
    acc.wet = max_slice(&h[o + 1], n - 2) > T(0);
    acc.infil = (double)si.total(); acc.fix = (double)sf.total();
    acc.smax = (double)max_slice(rs_s.data(), n);
    acc.bad = bad;
    // x_boundary (kernel.rs:435-450)
    double w = (double)xm[0] * dt_dy, e = (double)xm[nx] * dt_dy;
    if (w > 0.0) acc.bnd_in += w; else acc.bnd_out -= w;
    if (e > 0.0) acc.bnd_out += e; else acc.bnd_in -= e;
    // monitors_row (kernel.rs:311-321)
    for (size_t q = mon.row_start[j - 1]; q < mon.row_start[j]; ++q) {
      size_t col = mon.cells[q] % nx;
      double v = (double)h[o + col + 1];
      if (v > mon.max[q]) { mon.max[q] = v; mon.tmax[q] = t_new; }
    }
    if (track_peak) {
      for (size_t i = 1; i <= nx; ++i) {
        double v = (double)h[o + i];
        size_t cidx = (j - 1) * nx + (i - 1);
        if (v > peak[cidx]) { peak[cidx] = v; peak_step[cidx] = step_no + 1; }
      }
    }
    return acc;
  }

  // y_boundary (kernel.rs:452-472).
  std::pair<double, double> y_boundary(const T* m, double dt_dx, bool top) const {
    FixedSum<double> s;
    for (size_t i = 1; i <= L.nx; ++i) s.add(i, (double)m[i]);
    double v = s.total() * dt_dx, fin = 0, fout = 0;
    if (top) { if (v > 0.0) fin = v; else fout = -v; }
    else { if (v > 0.0) fout = v; else fin = -v; }
    return {fin, fout};
  }

  // step_oracle (kernel.rs:502-570): full arrays, no skipping.
  StepStats<T> step_oracle(const StepConsts<T>& k, double dt, double t_new, bool want_sum_s) {
    size_t nx = L.nx, ny = L.ny, W = nx + 2;
    std::vector<T> U((ny + 2) * W), V((ny + 2) * W), C((ny + 2) * W);
    for (size_t j = 0; j < ny + 2; ++j) vel_row(j, &U[j * W], &V[j * W], &C[j * W], k);
    std::vector<T> XM((ny + 2) * W), XNL((ny + 2) * W), XNR((ny + 2) * W), XT((ny + 2) * W);
    for (size_t j = 1; j <= ny; ++j)
      xface_row(j, &U[j * W], &V[j * W], &C[j * W], &XM[j * W], &XNL[j * W], &XNR[j * W], &XT[j * W], k);
    std::vector<T> YM((ny + 1) * W, T(0)), YNL((ny + 1) * W, T(0)), YNR((ny + 1) * W, T(0)), YT((ny + 1) * W, T(0));
    for (size_t j = 0; j <= ny; ++j)
      yface_row(j, &U[j * W], &V[j * W], &C[j * W], &U[(j + 1) * W], &V[(j + 1) * W], &C[(j + 1) * W],
                &YM[j * W], &YNL[j * W], &YNR[j * W], &YT[j * W], k);
    double dt_dy = dt * tb->dy, dt_dx = dt * tb->dx;
    StepStats<T> st;
    std::vector<RowAcc> accs;
    std::vector<double> ssr(ny, 0.0);
    for (size_t j = 1; j <= ny; ++j) {
      RowAcc a = update_row(j, &XM[j * W], &XNL[j * W], &XNR[j * W], &XT[j * W],
                            &YM[(j - 1) * W], &YNL[(j - 1) * W], &YNR[(j - 1) * W], &YT[(j - 1) * W],
                            &YM[j * W], &YNL[j * W], &YNR[j * W], &YT[j * W], k, want_sum_s, dt_dy, t_new);
      row_dry[j] = !a.wet;
      ssr[j - 1] = a.sum_s;
      accs.push_back(a);
    }
    row_dry[0] = 1; row_dry[ny + 1] = 1;
    auto top = y_boundary(&YM[0], dt_dx, true);
    auto bot = y_boundary(&YM[ny * W], dt_dx, false);
    return finalize(accs, top, bot, ssr);
  }

  StepStats<T> finalize(const std::vector<RowAcc>& accs, std::pair<double, double> top,
                        std::pair<double, double> bot, const std::vector<double>& ssr) {
    StepStats<T> st;
    st.bnd_in = top.first + bot.first; st.bnd_out = top.second + bot.second;
    for (const RowAcc& a : accs) {
      st.infil += a.infil; st.fix += a.fix; st.bnd_in += a.bnd_in; st.bnd_out += a.bnd_out;
      st.smax = fmax_num(st.smax, a.smax); st.bad = st.bad || a.bad; st.rows_skipped += a.skipped;
    }
    for (double s : ssr) st.sum_s += s;
    return st;
  }

  // step_fused (kernel.rs:590-727), single strip: in-place row sweep, carried y-face row,
  // dry-row skipping. Bitwise identical to step_oracle (checked by the tests).
  // Buffers of the fused sweep, allocated once per run (the reference's fused kernel makes
  // no heap allocation in steady state, crates/itr-hydro/tests/equivalence.rs:186-207).
  struct FusedBufs {
    std::vector<uint8_t> dry;
    std::vector<T> tu, tv, tc, bu, bv, bcv;
    std::vector<T> top_m, top_nl, top_nr, top_t, bot_m, bot_nl, bot_nr, bot_t;
    std::vector<T> cu, cv, cc, nu, nv, nc;
    std::vector<T> pm, pnl, pnr, pt, qm, qnl, qnr, qt;
    std::vector<T> xm, xnl, xnr, xt;
    std::vector<RowAcc> accs;
    std::vector<double> ssr;
    void init(size_t nx, size_t ny) {
      size_t W = nx + 2;
      dry.assign(ny + 2, 0);
      for (auto* v : {&tu, &tv, &tc, &bu, &bv, &bcv, &top_m, &top_nl, &top_nr, &top_t, &bot_m, &bot_nl, &bot_nr, &bot_t,
                      &cu, &cv, &cc, &nu, &nv, &nc, &pm, &pnl, &pnr, &pt, &qm, &qnl, &qnr, &qt, &xm, &xnl, &xnr, &xt})
        v->assign(W, T(0));
      accs.assign(ny, RowAcc());
      ssr.assign(ny, 0.0);
    }
  } fb;

  // step_fused (kernel.rs:590-727), single strip: in-place row sweep, carried y-face row,
  // dry-row skipping. Bitwise identical to step_oracle (checked by the tests).
  StepStats<T> step_fused(const StepConsts<T>& k, double dt, double t_new, bool want_sum_s) {
    size_t ny = L.ny;
    FusedBufs& B = fb;
    bool rain_zero = !(k.rain > T(0));
    for (size_t j = 0; j < ny + 2; ++j) B.dry[j] = row_dry[j] && !ghost_wet[j];
    auto skippable = [&](size_t j) { return p.skip_dry && rain_zero && B.dry[j - 1] && B.dry[j] && B.dry[j + 1]; };
    // Pre-phase: boundary y-face rows (top = face 0, bottom = face ny), old state.
    vel_row(0, B.tu.data(), B.tv.data(), B.tc.data(), k); vel_row(1, B.bu.data(), B.bv.data(), B.bcv.data(), k);
    yface_row(0, B.tu.data(), B.tv.data(), B.tc.data(), B.bu.data(), B.bv.data(), B.bcv.data(), B.top_m.data(), B.top_nl.data(),
              B.top_nr.data(), B.top_t.data(), k);
    vel_row(ny, B.tu.data(), B.tv.data(), B.tc.data(), k); vel_row(ny + 1, B.bu.data(), B.bv.data(), B.bcv.data(), k);
    yface_row(ny, B.tu.data(), B.tv.data(), B.tc.data(), B.bu.data(), B.bv.data(), B.bcv.data(), B.bot_m.data(), B.bot_nl.data(),
              B.bot_nr.data(), B.bot_t.data(), k);
    double dt_dy = dt * tb->dy, dt_dx = dt * tb->dx;
    auto top = y_boundary(B.top_m.data(), dt_dx, true);
    auto bot = y_boundary(B.bot_m.data(), dt_dx, false);
    B.pm = B.top_m; B.pnl = B.top_nl; B.pnr = B.top_nr; B.pt = B.top_t;   // g_prev
    bool cur_valid = false;
    for (size_t j = 1; j <= ny; ++j) {
      if (skippable(j)) {
        RowAcc a; a.skipped = true; B.accs[j - 1] = a;
        new_dry[j] = 1; B.ssr[j - 1] = 0.0;
        std::fill(B.qm.begin(), B.qm.end(), T(0)); std::fill(B.qnl.begin(), B.qnl.end(), T(0));
        std::fill(B.qnr.begin(), B.qnr.end(), T(0)); std::fill(B.qt.begin(), B.qt.end(), T(0));
        std::swap(B.pm, B.qm); std::swap(B.pnl, B.qnl); std::swap(B.pnr, B.qnr); std::swap(B.pt, B.qt);
        cur_valid = false;
        continue;
      }
      if (!cur_valid) vel_row(j, B.cu.data(), B.cv.data(), B.cc.data(), k);
      if (j + 1 <= ny) {
        vel_row(j + 1, B.nu.data(), B.nv.data(), B.nc.data(), k);
        yface_row(j, B.cu.data(), B.cv.data(), B.cc.data(), B.nu.data(), B.nv.data(), B.nc.data(), B.qm.data(), B.qnl.data(),
                  B.qnr.data(), B.qt.data(), k);
        cur_valid = true;
      } else {
        B.qm = B.bot_m; B.qnl = B.bot_nl; B.qnr = B.bot_nr; B.qt = B.bot_t;
        cur_valid = false;
      }
      xface_row(j, B.cu.data(), B.cv.data(), B.cc.data(), B.xm.data(), B.xnl.data(), B.xnr.data(), B.xt.data(), k);
      RowAcc a = update_row(j, B.xm.data(), B.xnl.data(), B.xnr.data(), B.xt.data(), B.pm.data(), B.pnl.data(), B.pnr.data(),
                            B.pt.data(), B.qm.data(), B.qnl.data(), B.qnr.data(), B.qt.data(), k, want_sum_s, dt_dy, t_new);
      new_dry[j] = !a.wet; B.ssr[j - 1] = a.sum_s; B.accs[j - 1] = a;
      std::swap(B.pm, B.qm); std::swap(B.pnl, B.qnl); std::swap(B.pnr, B.qnr); std::swap(B.pt, B.qt);
      if (cur_valid) { std::swap(B.cu, B.nu); std::swap(B.cv, B.nv); std::swap(B.cc, B.nc); }
    }
    new_dry[0] = 1; new_dry[ny + 1] = 1;
    std::swap(row_dry, new_dry);
    return finalize(B.accs, top, bot, B.ssr);
  }

  double volume(double area) const {
    double v = 0.0;
    for (size_t j = 1; j <= L.ny; ++j) {
      FixedSum<T> s;
      for (size_t i = 1; i <= L.nx; ++i) s.add(i, h[L.at(i, j)]);
      v += (double)s.total();
    }
    return v * area;
  }

  double initial_smax() const {
    double g = tb->g, dx = tb->dx, dy = tb->dy, s = 0.0;
    for (size_t j = 1; j <= L.ny; ++j)
      for (size_t i = 1; i <= L.nx; ++i) {
        size_t k = L.at(i, j);
        double hh = (double)h[k];
        if (hh <= p.h_dry) continue;
        double c = std::sqrt(g * hh);
        double r = (std::fabs((double)qx[k]) / hh + c) / dx + (std::fabs((double)qy[k]) / hh + c) / dy;
        s = fmax_num(s, r);
      }
    return s;
  }

  // init_state (solver.rs:287-312); h0 overrides the initial depth when given.
  void init_state(const T* h0) {
    size_t nx = L.nx, ny = L.ny;
    std::fill(h.begin(), h.end(), T(0)); std::fill(qx.begin(), qx.end(), T(0)); std::fill(qy.begin(), qy.end(), T(0));
    for (size_t r = 0; r < ny; ++r)
      for (size_t c = 0; c < nx; ++c) {
        size_t k = r * nx + c;
        if (h0) { h[L.at(c + 1, r + 1)] = h0[k]; continue; }
        if (tb->wall[k]) continue;
        double d = p.initial_depth;
        if (p.has_stage) d = fmax_num(d, p.initial_stage - tb->fine->z_ref - zlev[k]);
        h[L.at(c + 1, r + 1)] = canon_zero((T)fmax_num(d, 0.0));
      }
    for (size_t j = 0; j < ny + 2; ++j) {
      bool all0 = true;
      for (size_t i = 0; i < nx + 2; ++i) if (!(h[L.at(i, j)] == T(0))) { all0 = false; break; }
      row_dry[j] = all0;
    }
  }

  // Sync snapshot of everything the run loop carries, for the locked-dt fallback
  // (Checkpoint, solver.rs:78-92; taken at the start and at every sync, solver.rs:444-447,611-614).
  struct Snap {
    std::vector<T> h, qx, qy; std::vector<uint8_t> row_dry;
    std::vector<double> mmax, mtmax, peak; std::vector<uint64_t> peak_step;
    double t = 0, dt_cfl = 0, s_cur = 0; uint64_t step = 0; uint32_t sync_index = 0;
    double acc[5] = {0, 0, 0, 0, 0}; double dmin = 0, dmax = 0, dsum = 0;
    uint64_t cell_updates = 0, rows_skipped = 0; size_t n_rows = 0;
  };

  // run_impl (solver.rs:346-660) without warm start or replay; with locked dt when
  // p.n_locked > 0 (solver.rs:436-483).
  // Optional custom start (the Ritter validation case builds a checkpoint by hand,
  // validation.rs:125-151): padded depth, all rows wet, given dt_next and v0.
  struct Start { std::vector<T> h; double dt_next = 0; double v0 = 0; };

  RunResult run(const PreparedTerrain<T>& pt, const std::vector<uint32_t>& monitors, Kernel kern,
                const ObserverCfg* obs, const T* h0 = nullptr, bool want_peak = false,
                const Start* start = nullptr) {
    terr = &pt; tb = pt.base; L = tb->layout;
    size_t nx = L.nx, ny = L.ny;
    h.assign(L.len(), T(0)); qx.assign(L.len(), T(0)); qy.assign(L.len(), T(0));
    row_dry.assign(ny + 2, 0); ghost_wet.assign(ny + 2, 0); new_dry.assign(ny + 2, 0);
    rs_infil.assign(nx + 2, T(0)); rs_fix.assign(nx + 2, T(0)); rs_s.assign(nx + 2, T(0));
    fb.init(nx, ny);
    zlev = pt.z_level();
    mon.init(monitors, nx, ny);
    track_peak = want_peak;
    if (want_peak) { peak.assign(nx * ny, 0.0); peak_step.assign(nx * ny, 0); }
    double area = tb->dx * tb->dy;
    RunResult R;
    double dt_cfl, s_cur;
    if (start) {
      h = start->h;
      std::fill(row_dry.begin(), row_dry.end(), 0);
      R.v0 = start->v0;
      dt_cfl = start->dt_next;
      s_cur = initial_smax();
    } else {
      init_state(h0);
      R.v0 = volume(area);
      double s0 = initial_smax();
      s_cur = s0;
      dt_cfl = s0 > 0.0 ? fmin_num(p.cfl / s0, p.dt_max) : p.dt_max;
    }
    double t = 0.0; uint64_t step = 0; uint32_t sync_index = 0;
    double acc_rain = 0, acc_in = 0, acc_out = 0, acc_infil = 0, acc_fix = 0;
    double dmin = std::numeric_limits<double>::max(), dmax = 0, dsum = 0;
    uint64_t cells = (uint64_t)nx * ny;
    uint32_t n_sync = (uint32_t)std::ceil(p.duration / p.sync);
    bool locked = p.n_locked > 0;
    Snap snap;
    auto save = [&]() {
      snap.h = h; snap.qx = qx; snap.qy = qy; snap.row_dry = row_dry;
      snap.mmax = mon.max; snap.mtmax = mon.tmax; snap.peak = peak; snap.peak_step = peak_step;
      snap.t = t; snap.dt_cfl = dt_cfl; snap.s_cur = s_cur; snap.step = step; snap.sync_index = sync_index;
      snap.acc[0] = acc_rain; snap.acc[1] = acc_in; snap.acc[2] = acc_out; snap.acc[3] = acc_infil; snap.acc[4] = acc_fix;
      snap.dmin = dmin; snap.dmax = dmax; snap.dsum = dsum;
      snap.cell_updates = R.cell_updates; snap.rows_skipped = R.rows_skipped; snap.n_rows = R.rows.size();
    };
    if (locked) save();
    while (t < p.duration && sync_index < n_sync) {
      double t_sync = fmin_num((double)(sync_index + 1) * p.sync, p.duration);
      double dt = fmin_num(dt_cfl, p.dt_max);
      if (locked) {
        // the recorded dt, verified against the hard CFL limit; otherwise restart adaptively
        // from the last sync snapshot (solver.rs:452-482)
        if (step < p.n_locked && p.locked_dt[step] * s_cur <= p.cfl_hard) {
          dt = p.locked_dt[step];
        } else {
          h = snap.h; qx = snap.qx; qy = snap.qy; row_dry = snap.row_dry;
          mon.max = snap.mmax; mon.tmax = snap.mtmax; peak = snap.peak; peak_step = snap.peak_step;
          acc_rain = snap.acc[0]; acc_in = snap.acc[1]; acc_out = snap.acc[2]; acc_infil = snap.acc[3]; acc_fix = snap.acc[4];
          dmin = snap.dmin; dmax = snap.dmax; dsum = snap.dsum;
          R.cell_updates = snap.cell_updates; R.rows_skipped = snap.rows_skipped; R.rows.resize(snap.n_rows);
          t = snap.t; step = snap.step; sync_index = snap.sync_index; dt_cfl = snap.dt_cfl; s_cur = snap.s_cur;
          R.dt_fallback_t = t;
          locked = false;
          continue;
        }
      }
      bool hits = t + dt >= t_sync - 1e-9 * p.sync;
      if (hits) dt = t_sync - t;
      double rain = p.rain.integral(t, t + dt);
      double t_new = hits ? t_sync : t + dt;
      fill_ghosts(t);
      if (p.record_dts) R.dts.push_back(dt);
      StepConsts<T> k = consts(dt, rain);
      step_no = step;
      StepStats<T> st = kern == K_ORACLE ? step_oracle(k, dt, t_new, hits) : step_fused(k, dt, t_new, hits);
      step += 1; t = t_new;
      acc_rain += rain * area * (double)tb->wet_count;
      acc_in += st.bnd_in; acc_out += st.bnd_out;
      acc_infil += st.infil * area; acc_fix += st.fix * area;
      dmin = fmin_num(dmin, dt); dmax = fmax_num(dmax, dt); dsum += dt;
      R.cell_updates += cells - st.rows_skipped * nx;
      R.rows_skipped += st.rows_skipped;
      if (st.bad) { R.abort = AB_UNHEALTHY; break; }
      dt_cfl = st.smax > 0.0 ? p.cfl / st.smax : p.dt_max;
      s_cur = st.smax;
      if (hits) {
        sync_index += 1;
        double v = volume(area);
        double expected = R.v0 + acc_rain + acc_in - acc_out - acc_infil + acc_fix;
        R.rows.push_back(LedgerRow{t, v, acc_rain, acc_in, acc_out, acc_infil, acc_fix, v - expected});
        if (obs && obs->obj) {
          const Objective& o = *obs->obj;
          // guard_breach (objective.rs:132-145)
          if (o.require_no_worsening && obs->baseline) {
            bool found = false; double wv = 0; uint32_t wc = 0;
            for (size_t q : o.guard_pos) {
              double w = mon.max[q] - obs->baseline[q] - o.guard_tol;
              if (w > 0.0 && (!found || w > wv)) { found = true; wv = w; wc = o.mon_cells[q]; }
            }
            if (found) { R.abort = AB_GUARD; R.abort_cell = wc; R.abort_exceed = wv; R.abort_sync = sync_index; break; }
          }
          if (obs->has_incumbent) {
            double lb = obj_evaluate(o, mon.max.data(), obs->cut, obs->fill, nullptr).j;
            if (lb >= obs->incumbent) { R.abort = AB_INCUMBENT; R.abort_lb = lb; break; }
          }
        }
        if (locked) save();
      }
    }
    R.t_end = t; R.steps = step; R.sync_count = sync_index;
    R.mon_max = mon.max; R.mon_tmax = mon.tmax;
    if (!R.rows.empty()) {
      double gross = R.v0 + R.rows.back().rain + R.rows.back().inflow;
      R.rel_residual = std::fabs(R.rows.back().residual) / fmax_num(gross, 1e-300);
    }
    R.dt_min = dmin == std::numeric_limits<double>::max() ? 0.0 : dmin;
    R.dt_max = dmax; R.dt_mean = step > 0 ? dsum / (double)step : 0.0;
    if (want_peak) { R.peak = peak; R.peak_step = peak_step; }
    return R;
  }
};

}  // namespace orc
