// itr_design.cuh — designs materialised on the device: primitives -> dz -> cell levels ->
// face jumps, for a fidelity level 1 grid (signed faces).
//
// Restates, per design and in f64:
//   * Primitive::profile (crates/itr-core/src/design.rs:107-134): distance to the primitive's
//     segment over half its width, (1 - s^2)^2 ridge or a flat-bottomed cut;
//   * DesignSpace::materialize (design.rs:316-385): 4x4 sub-sample quadrature per cell in the
//     union bounding box of the primitives, sum of height * mean profile over primitives,
//     masked by the editable cells, clamped to +-max_abs_dz; cut and fill volumes summed
//     over the box in row-major order;
//   * PreparedTerrain::apply_edit (crates/itr-hydro/src/terrain.rs:460-505) at level 1: cell
//     level z + dz (walls stay at z_wall) and every interior face jump f32(z_right - z_left),
//     the jumps of TerrainBase::build (terrain.rs:276-289) on the edited levels.
// The host evaluates each primitive's segment end points (sin and cos of its angle) with the
// same libm calls the reference makes, so every value here is an IEEE f64 add, multiply,
// divide or square root in the reference's order: the jumps equal the host path's bit for bit.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace itr {

// One primitive with its segment end points (Primitive::segment, design.rs:101-106).
struct MatPrim {
  double x0, y0, x1, y1;   // segment end points (equal for a mound)
  double width, height;
  double length;           // Primitive::length (the adjoint chain's d(end point)/dL)
  int kind;                // 0 berm, 1 swale, 2 cut, 3 mound
  int pad;
};

// One design: primitives [p0, p1) and the union bounding box, columns [c0, c1), rows [r0, r1)
// (empty when c0 >= c1 or r0 >= r1).
struct MatDesign {
  int p0, p1;
  int c0, r0, c1, r1;
};

struct MatArgs {
  int nx, ny, n;
  double ox, oy, dx, dy;   // GeoTransform of the grid
  double z_wall, max_abs_dz;
  const double* z;         // nx*ny base levels (walls at z_wall)
  const uint8_t* wall;     // nx*ny
  const uint8_t* editable; // nx*ny
  const MatPrim* prims;
  const MatDesign* des;
  double* dz;              // n * nx*ny
  double* ze;              // n * nx*ny edited levels
  float* dzx;              // n * ny*(nx+1)
  float* dzy;              // n * (ny+1)*nx
  double* cut;             // n
  double* fill;            // n
  const uint8_t* bc;       // boundary codes (ITR_BC_*) when stage depths are wanted, else NULL
  const double* stage;     // stage levels, indexed like bc
  float* bh;               // n * (2nx+2ny) stage-ghost depths
};

// Primitive::profile (design.rs:107-134).
__device__ __forceinline__ double mat_profile(const MatPrim& p, double x, double y) {
  const double vx = p.x1 - p.x0, vy = p.y1 - p.y0;
  const double l2 = vx * vx + vy * vy;
  double t = 0.0;
  if (l2 > 0.0) {
    t = ((x - p.x0) * vx + (y - p.y0) * vy) / l2;
    t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
  }
  const double px = p.x0 + t * vx - x, py = p.y0 + t * vy - y;
  const double d = sqrt(px * px + py * py);
  const double s = d / (0.5 * p.width);
  if (s >= 1.0) return 0.0;
  if (p.kind == 2) {   // cut: flat bottom, then a (1 - u^2)^2 bank
    if (s <= 0.5) return 1.0;
    const double u = (s - 0.5) / 0.5;
    const double w = 1.0 - u * u;
    return w * w;
  }
  const double w = 1.0 - s * s;
  return w * w;
}

// dz and the edited level of every cell of every design (grid: cells / 256 x designs).
__global__ void k_materialize(const MatArgs M) {
  const int d = blockIdx.y;
  const size_t N = (size_t)M.nx * M.ny;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int r = (int)(i / M.nx), c = (int)(i % M.nx);
  const MatDesign D = M.des[d];
  double dz = 0.0;
  if (c >= D.c0 && c < D.c1 && r >= D.r0 && r < D.r1 && M.editable[i]) {
    double acc = 0.0;
    for (int q = D.p0; q < D.p1; ++q) {
      const MatPrim p = M.prims[q];
      if (p.height == 0.0) continue;
      double s = 0.0;
      for (int sy = 0; sy < 4; ++sy)
        for (int sx = 0; sx < 4; ++sx) {
          const double x = M.ox + ((double)c + ((double)sx + 0.5) / 4.0) * M.dx;
          const double y = M.oy - ((double)r + ((double)sy + 0.5) / 4.0) * M.dy;
          s += mat_profile(p, x, y);
        }
      acc += p.height * s * (1.0 / 16.0);
    }
    dz = acc < -M.max_abs_dz ? -M.max_abs_dz : (acc > M.max_abs_dz ? M.max_abs_dz : acc);
  }
  M.dz[(size_t)d * N + i] = dz;
  M.ze[(size_t)d * N + i] = M.wall[i] ? M.z_wall : M.z[i] + dz;
}

// Face jumps of the edited levels (domain-edge faces 0), and the stage ghosts' depths
// f32(max(stage - z, 0)) behind stage cells (grid: max(ny*(nx+1), (ny+1)*nx) / 256 x designs).
__global__ void k_mat_jumps(const MatArgs M) {
  const int d = blockIdx.y;
  const int nx = M.nx, ny = M.ny;
  const size_t N = (size_t)nx * ny;
  const double* ze = M.ze + (size_t)d * N;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < (size_t)ny * (nx + 1)) {
    const int r = (int)(i / (nx + 1)), f = (int)(i % (nx + 1));
    M.dzx[(size_t)d * ny * (nx + 1) + i] =
        (f >= 1 && f <= nx - 1) ? (float)(ze[(size_t)r * nx + f] - ze[(size_t)r * nx + f - 1]) : 0.0f;
  }
  if (i < (size_t)(ny + 1) * nx) {
    const int f = (int)(i / nx), c = (int)(i % nx);
    M.dzy[(size_t)d * (ny + 1) * nx + i] =
        (f >= 1 && f <= ny - 1) ? (float)(ze[(size_t)f * nx + c] - ze[(size_t)(f - 1) * nx + c]) : 0.0f;
  }
  const size_t NB = 2 * (size_t)(nx + ny);
  if (M.bh && i < NB) {
    // boundary cell i: north[nx], south[nx], west[ny], east[ny]
    size_t cell;
    if (i < (size_t)nx) cell = i;
    else if (i < 2 * (size_t)nx) cell = (size_t)(ny - 1) * nx + (i - nx);
    else if (i < 2 * (size_t)nx + ny) cell = (i - 2 * (size_t)nx) * nx;
    else cell = (i - 2 * (size_t)nx - ny) * nx + nx - 1;
    float h = 0.0f;
    if (M.bc[i] == 2) {
      const double v = M.stage[i] - ze[cell];
      h = (float)(v > 0.0 ? v : 0.0);
    }
    M.bh[(size_t)d * NB + i] = h;
  }
}

// Cut and fill volumes of each design's edit (design.rs:376-383), summed over its bounding
// box in row-major order as the reference does. One warp per design: the lanes load 32
// consecutive cells of a row at once, and every lane runs the sum over them in column order
// (values broadcast by shuffle), so the f64 sums are the sequential ones, bit for bit.
__global__ void k_mat_volumes(const MatArgs M) {
  const int lane = threadIdx.x & 31;
  const int d = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (d >= M.n) return;   // (whole warps)
  const MatDesign D = M.des[d];
  const size_t N = (size_t)M.nx * M.ny;
  const double a = M.dx * M.dy;
  double cut = 0.0, fill = 0.0;
  for (int r = D.r0; r < D.r1; ++r)
    for (int c0 = D.c0; c0 < D.c1; c0 += 32) {
      const int c = c0 + lane, m = D.c1 - c0 < 32 ? D.c1 - c0 : 32;
      const double mine = c < D.c1 ? M.dz[(size_t)d * N + (size_t)r * M.nx + c] : 0.0;
      for (int k = 0; k < m; ++k) {
        const double v = __shfl_sync(0xffffffffu, mine, k);
        if (v > 0.0) fill += v * a; else cut -= v * a;
      }
    }
  if (lane == 0) {
    M.cut[d] = cut;
    M.fill[d] = fill;
  }
}

// ---- the design chain of the adjoint: dJ/d(height, width, length) per primitive ----
// dJ/d(dz) per cell from the face-jump gradients (level 1: each interior jump is the
// difference of its two cells' levels, the edge jumps stay 0, walls keep z_wall), then per
// primitive the derivative of the materialisation, written out from Primitive::profile
// (design.rs:107-134), contracted with it, plus the earthwork term lambda (cut_cost dV_cut +
// fill_cost dV_fill) (objective.rs:95-128).

// dJ/d(dz) of every cell of every design (grid: cells / 256 x designs).
__global__ void k_mat_gdz(int nx, int ny, const double* gx, const double* gy, const uint8_t* wall, double* gdz) {
  const int d = blockIdx.y;
  const size_t N = (size_t)nx * ny;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int r = (int)(i / nx), c = (int)(i % nx);
  const double* X = gx + (size_t)d * ny * (nx + 1) + (size_t)r * (nx + 1);
  const double* Y = gy + (size_t)d * (ny + 1) * nx;
  const double a = (c >= 1) ? X[c] : 0.0, b = (c + 1 <= nx - 1) ? X[c + 1] : 0.0;
  const double e = (r >= 1) ? Y[(size_t)r * nx + c] : 0.0, f = (r + 1 <= ny - 1) ? Y[(size_t)(r + 1) * nx + c] : 0.0;
  gdz[(size_t)d * N + i] = wall[i] ? 0.0 : ((a - b) + e) - f;
}

// The profile at (x, y) and its derivatives with respect to the primitive's width and length
// at fixed centre and angle. With s = d / (w / 2):
//   ridge P = (1 - s^2)^2, dP/ds = -4 s (1 - s^2);
//   cut   P = 1 for s <= 1/2, else (1 - u^2)^2 with u = 2 s - 1, dP/ds = -8 u (1 - u^2);
//   ds/dw = -s / w;  ds/dL = (2 / w) dd/dL, dd/dL = 0 beside the segment and, beyond an end,
//   the end's displacement (+-(cos a, sin a) / 2 per unit length) projected on the unit
//   vector from the sample to it.
__device__ __forceinline__ void mat_profile_d(const MatPrim& p, double x, double y, double& P, double& dw, double& dl) {
  P = 0.0; dw = 0.0; dl = 0.0;
  const double vx = p.x1 - p.x0, vy = p.y1 - p.y0;
  const double l2 = vx * vx + vy * vy;
  double t = 0.0;
  int end = 0;
  if (l2 > 0.0) {
    t = ((x - p.x0) * vx + (y - p.y0) * vy) / l2;
    if (t < 0.0) { t = 0.0; end = -1; }
    else if (t > 1.0) { t = 1.0; end = 1; }
  }
  const double px = p.x0 + t * vx - x, py = p.y0 + t * vy - y;
  const double d = sqrt(px * px + py * py);
  const double half = 0.5 * p.width;
  const double s = d / half;
  if (s >= 1.0) return;
  double dPds;
  if (p.kind == 2) {
    if (s <= 0.5) { P = 1.0; dPds = 0.0; }
    else { const double u = (s - 0.5) / 0.5, w = 1.0 - u * u; P = w * w; dPds = -8.0 * u * w; }
  } else {
    const double w = 1.0 - s * s;
    P = w * w; dPds = -4.0 * s * w;
  }
  dw = dPds * (-s / p.width);
  if (end != 0 && d > 0.0 && p.kind != 3 && p.length > 0.0) {
    const double ex = vx / (2.0 * p.length), ey = vy / (2.0 * p.length);
    dl = dPds * ((double)end * (px * ex + py * ey) / d) / half;
  }
}

// One primitive of one design: its own box of cells (materialize's box of that primitive).
struct MatJob {
  int design, prim;           // prim indexes the job's primitive table
  int c0, r0, c1, r1;
  int out;                    // output index (3 per primitive: height, width, length)
  int pad;
};

// One block per primitive: over its box, d(dz)/d(height, width, length) of every editable cell
// whose dz is not clamped, contracted with dJ/d(dz) plus the earthwork weight (the side of 0
// the cell's dz lies on; the mean of both sides at 0, as a central difference would see it).
__global__ void k_mat_dgrad(const MatArgs M, const MatPrim* jp, const MatJob* jobs, const double* dz, const double* gdz,
                            double earth_w, double cut_cost, double fill_cost, double* out) {
  const MatJob J = jobs[blockIdx.x];
  const MatPrim p = jp[J.prim];
  const int w = J.c1 - J.c0, h = J.r1 - J.r0;
  const size_t N = (size_t)M.nx * M.ny;
  const double area = M.dx * M.dy;
  double s[3] = {0, 0, 0};
  for (int k = threadIdx.x; w > 0 && h > 0 && k < w * h; k += blockDim.x) {
    const int r = J.r0 + k / w, c = J.c0 + k % w;
    const size_t i = (size_t)r * M.nx + c;
    const double z = dz[(size_t)J.design * N + i];
    if (!M.editable[i] || !(z > -M.max_abs_dz && z < M.max_abs_dz)) continue;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int sy = 0; sy < 4; ++sy)
      for (int sx = 0; sx < 4; ++sx) {
        const double x = M.ox + ((double)c + ((double)sx + 0.5) / 4.0) * M.dx;
        const double y = M.oy - ((double)r + ((double)sy + 0.5) / 4.0) * M.dy;
        double P, dw, dl;
        mat_profile_d(p, x, y, P, dw, dl);
        a0 += P; a1 += dw; a2 += dl;
      }
    const double we = area * (z > 0.0 ? fill_cost : (z < 0.0 ? -cut_cost : 0.5 * (fill_cost - cut_cost)));
    const double g = gdz[(size_t)J.design * N + i] + earth_w * we;
    s[0] += g * a0 * (1.0 / 16.0);
    s[1] += g * p.height * a1 * (1.0 / 16.0);
    s[2] += g * p.height * a2 * (1.0 / 16.0);
  }
  __shared__ double red[32][3];
  for (int j = 0; j < 3; ++j)
    for (int o = 16; o > 0; o >>= 1) s[j] += __shfl_xor_sync(0xffffffffu, s[j], o);
  if ((threadIdx.x & 31) == 0)
    for (int j = 0; j < 3; ++j) red[threadIdx.x >> 5][j] = s[j];
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[3] = {0, 0, 0};
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q)
      for (int j = 0; j < 3; ++j) t[j] += red[q][j];
    for (int j = 0; j < 3; ++j) out[J.out + j] = t[j];
  }
}

}  // namespace itr
