// itr_plain.cuh — the plain forward: one design per launch sequence, global-memory ping-pong.
//
// This is the straightforward CUDA form of the reference's GPU backend structure
// (crates/itr-gpu/src/shader.wgsl:135-365, lib.rs:302-328): per step one tiled `update`
// kernel (16x16 cells, 18x18 halo in shared memory, faces computed once per tile) and one
// single-warp `finalize` kernel that advances the f64 integrator on the device; the host
// polls a control word every `steps_per_submit` steps. Designs run one after another.
// It is the baseline the batched kernel is measured against, and it uses the same
// per-cell arithmetic (itr_device.cuh), so its results are bit-identical to the batched
// kernel's and to the f32 CPU oracle's.
#pragma once
#include "itr_device.cuh"

namespace itr {

constexpr int kTile = 16;

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
};

struct PlainArgs {
  RunParams P;
  int nx, ny, mode;
  const float* wet;
  const float* gn2;
  const uint8_t* bc;
  const float* dzx;   // this design
  const float* dzy;
  const float* dzx2;
  const float* dzy2;
  const float* h0;    // this design
  double cut, fill;
  int n_mon;
  const unsigned* mon_cells;
  DevObjective obj;
  float* H;           // [2][nx*ny]
  float* QX;
  float* QY;
  float* PK;          // nx*ny
  double* part;       // per block: [5] (infil, fix, in, out, vol)
  PlainCtl* ctl;
  double* ledger;     // max_rows*8
  int max_rows;
  unsigned long long max_steps;
};

// Old state of padded cell (gx, gy) with ghost cells outside (boundary.rs:36-87).
ITR_DEV void plain_load(const PlainArgs& A, int par, int gx, int gy, float& h, float& qx, float& qy) {
  const int nx = A.nx, ny = A.ny;
  const bool ox = gx < 0 || gx >= nx, oy = gy < 0 || gy >= ny;
  if (ox && oy) { h = 0.0f; qx = 0.0f; qy = 0.0f; return; }
  int sx = gx < 0 ? 0 : (gx >= nx ? nx - 1 : gx);
  int sy = gy < 0 ? 0 : (gy >= ny ? ny - 1 : gy);
  size_t i = (size_t)par * nx * ny + (size_t)sy * nx + sx;
  h = A.H[i]; qx = A.QX[i]; qy = A.QY[i];
  if (ox) { int code = gx < 0 ? A.bc[2 * nx + sy] : A.bc[2 * nx + ny + sy]; if (code == 0) qx = -qx; }
  else if (oy) { int code = gy < 0 ? A.bc[sx] : A.bc[nx + sx]; if (code == 0) qy = -qy; }
}

template <bool CREST>
__global__ void __launch_bounds__(256) k_plain_update(const PlainArgs A) {
  __shared__ float sh[18 * 18], su[18 * 18], sv[18 * 18], sc[18 * 18], sqx[18 * 18], sqy[18 * 18];
  __shared__ FaceF fx[16 * 17], fy[17 * 16];
  __shared__ float wmax[8];
  __shared__ unsigned wbad[8];
  __shared__ double wsum[8][5];
  const PlainCtl& cl = *A.ctl;
  if (cl.done) return;
  const int par = cl.par;
  const StepK k = cl.k;
  const bool hits = cl.pl.hits;
  const double dt_dx = cl.pl.dt * A.P.dx, dt_dy = cl.pl.dt * A.P.dy;
  const int nx = A.nx, ny = A.ny;
  const int gx0 = blockIdx.x * kTile, gy0 = blockIdx.y * kTile;
  const int li = threadIdx.x;
  for (int e = li; e < 324; e += 256) {
    int hx = e % 18, hy = e / 18;
    float h, qx, qy;
    plain_load(A, par, gx0 - 1 + hx, gy0 - 1 + hy, h, qx, qy);
    float u, v, c;
    cell_vel(h, qx, qy, k.g, k.heps2, u, v, c);
    sh[e] = h; sqx[e] = qx; sqy[e] = qy; su[e] = u; sv[e] = v; sc[e] = c;
  }
  __syncthreads();
  for (int e = li; e < 272; e += 256) {
    {  // x-faces: 16 rows x 17
      int fyr = e / 17, fxc = e % 17;
      int row = gy0 + fyr, f = gx0 + fxc;
      if (row < ny && f <= nx) {
        int a = (fyr + 1) * 18 + fxc;
        size_t o = (size_t)row * (nx + 1) + f;
        float d0 = A.dzx[o], d1 = CREST ? A.dzx2[o] : 0.0f;
        fx[e] = face<true, CREST>(sh[a], su[a], sv[a], sc[a], sh[a + 1], su[a + 1], sv[a + 1], sc[a + 1], d0, d1, k);
      }
    }
    {  // y-faces: 17 rows x 16
      int fyr = e / 16, fxc = e % 16;
      int c = gx0 + fxc, f = gy0 + fyr;
      if (c < nx && f <= ny) {
        int a = fyr * 18 + fxc + 1, b = a + 18;
        size_t o = (size_t)f * nx + c;
        float d0 = A.dzy[o], d1 = CREST ? A.dzy2[o] : 0.0f;
        fy[e] = face<false, CREST>(sh[a], su[a], sv[a], sc[a], sh[b], su[b], sv[b], sc[b], d0, d1, k);
      }
    }
  }
  __syncthreads();
  float smax = 0.0f;
  bool bad = false;
  double acc[5] = {0, 0, 0, 0, 0};
  const int lx = li % 16, ly = li / 16;
  const int gx = gx0 + lx, gy = gy0 + ly;
  if (gx < nx && gy < ny) {
    const FaceF w = fx[ly * 17 + lx], e = fx[ly * 17 + lx + 1];
    const FaceF n = fy[ly * 16 + lx], s = fy[(ly + 1) * 16 + lx];
    const int a = (ly + 1) * 18 + lx + 1;
    const size_t gi = (size_t)gy * nx + gx;
    CellNew o = update_cell(sh[a], sqx[a], sqy[a], w, e, n, s, A.wet[gi], A.gn2[gi], k);
    const size_t wo = (size_t)(par ^ 1) * nx * ny + gi;
    A.H[wo] = o.h; A.QX[wo] = o.qx; A.QY[wo] = o.qy;
    if (o.h > A.PK[gi]) A.PK[gi] = o.h;
    smax = o.s;
    bad = o.bad;
    acc[0] = (double)o.infil; acc[1] = (double)o.fix;
    if (hits) acc[4] = (double)o.h;
    // boundary faces (kernel.rs:435-472), per face
    if (gx == 0) { double v = (double)w.m * dt_dy; if (v > 0.0) acc[2] += v; else acc[3] -= v; }
    if (gx == nx - 1) { double v = (double)e.m * dt_dy; if (v > 0.0) acc[3] += v; else acc[2] -= v; }
    if (gy == 0) { double v = (double)n.m * dt_dx; if (v > 0.0) acc[2] += v; else acc[3] -= v; }
    if (gy == ny - 1) { double v = (double)s.m * dt_dx; if (v > 0.0) acc[3] += v; else acc[2] -= v; }
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
  if (li == 0) {
    float mm = 0.0f; unsigned bb = 0u; double ss[5] = {0, 0, 0, 0, 0};
    for (int w = 0; w < 8; ++w) { mm = rmax(mm, wmax[w]); bb |= wbad[w]; for (int j = 0; j < 5; ++j) ss[j] += wsum[w][j]; }
    if (mm > 0.0f) atomicMax(&A.ctl->smax_bits, __float_as_uint(mm));
    if (bb) atomicOr(&A.ctl->bad, 1u);
    double* p = A.part + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 5;
    for (int j = 0; j < 5; ++j) p[j] = ss[j];
  }
}

// Advance the integrator after a step (or plan the first step when `first`).
__global__ void k_plain_finalize(const PlainArgs A, int n_blocks, int first) {
  PlainCtl& c = *A.ctl;
  const int lane = threadIdx.x;
  const RunParams& P = A.P;
  if (c.done) return;
  if (!first) {
    // sum block partials in block order
    double tot[5] = {0, 0, 0, 0, 0};
    for (int b = lane; b < n_blocks; b += 32)
      for (int j = 0; j < 5; ++j) tot[j] += A.part[(size_t)b * 5 + j];
    for (int j = 0; j < 5; ++j)
      for (int o = 16; o > 0; o >>= 1) tot[j] += __shfl_xor_sync(0xffffffffu, tot[j], o);
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
        if (c.n_rows < A.max_rows && A.ledger) {
          double* o = A.ledger + (size_t)c.n_rows * 8;
          o[0] = c.t; o[1] = v; o[2] = c.acc_rain; o[3] = c.tot_in; o[4] = c.tot_out; o[5] = infil; o[6] = fix; o[7] = v - expected;
        }
        c.n_rows += 1;
        const DevObjective& ob = A.obj;
        if (ob.enabled) {
          if (ob.guard_abort && ob.require && ob.baseline) {
            double best = 0.0; int bk = -1;
            for (int g = 0; g < ob.n_guard; ++g) {
              int mp = ob.guard_pos[g];
              double w = (double)A.PK[A.mon_cells[mp]] - ob.baseline[mp] - ob.tol;
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
                double x = (double)A.PK[A.mon_cells[ob.asset_pos[m]]];
                pk = pk > x ? pk : x;
              }
              jr += ob.asset_w[a] * ob.tau * itr_math::softplus((pk - ob.asset_thr[a]) / ob.tau);
            }
            const double lb = jr + ob.earth_w * (ob.cut_cost * A.cut + ob.fill_cost * A.fill);
            if (lb >= ob.incumbent) { decision = 2; c.lower_bound = lb; }
          }
        }
        if (decision) { c.status = decision; c.done = 1; }
      }
      __syncwarp();
      if (c.done) return;
    }
  }
  if (lane == 0) {
    if (!(c.t < P.duration && c.sync_index < P.n_sync)) { c.done = 1; return; }
    if (c.step >= A.max_steps) { c.status = 4; c.done = 1; return; }
    c.pl = plan_step(P, c.t, c.sync_index, c.dt_cfl);
    c.k = step_consts(P, c.pl.dt, c.pl.rain);
  }
}

// Initial state and the first dt (solver.rs:381-390).
__global__ void k_plain_init(const PlainArgs A) {
  const int nx = A.nx, ny = A.ny, n = nx * ny;
  const RunParams& P = A.P;
  __shared__ double ss[32], sv[32];
  double s0 = 0.0, v0 = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    float h = A.h0[i];
    A.H[i] = h; A.QX[i] = 0.0f; A.QY[i] = 0.0f; A.PK[i] = 0.0f;
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
    *A.ctl = c;
  }
}

}  // namespace itr
