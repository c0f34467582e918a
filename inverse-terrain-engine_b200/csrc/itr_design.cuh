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
// box in row-major order as the reference does (one thread per design).
__global__ void k_mat_volumes(const MatArgs M) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= M.n) return;
  const MatDesign D = M.des[d];
  const size_t N = (size_t)M.nx * M.ny;
  const double a = M.dx * M.dy;
  double cut = 0.0, fill = 0.0;
  for (int r = D.r0; r < D.r1; ++r)
    for (int c = D.c0; c < D.c1; ++c) {
      const double v = M.dz[(size_t)d * N + (size_t)r * M.nx + c];
      if (v > 0.0) fill += v * a; else cut -= v * a;
    }
  M.cut[d] = cut;
  M.fill[d] = fill;
}

}  // namespace itr
