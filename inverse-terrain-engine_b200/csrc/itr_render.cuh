// itr_render.cuh — headless map image of a run's results (the viewer's map, presentation).
//
// Restates the fragment shader of the reference's result viewer (viewer/viewer.js:72-100,
// colour ramps :55-71) as one CUDA thread per output pixel writing RGBA8 into device memory:
// a grey hillshade of the terrain (central-difference gradient times the vertical
// exaggeration, lit from the north-west), a logarithmic blue depth ramp for depths above
// 5 mm (mode 0) or a diverging ramp for depth differences beyond 5 mm (mode 1), and hatching
// of cells whose peak depth rose by more than 1 cm. The ramp colours are the shader's
// constants (the hex colours to four decimals, as the viewer writes them into GLSL); the
// arithmetic is f32, as the shader's highp float. Pixels map to cells like the viewer's
// vertex shader at `scale` pixels per cell: pixel (px, py) sees cell coordinate
// ((px + 0.5) / scale, (py + 0.5) / scale), row 0 the northern row.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace itr {

struct RenderArgs {
  int nx, ny, scale, mode, worse;
  float vex, cs;
  const float* z;       // nx*ny terrain level (NaN: no data)
  const float* value;   // nx*ny depth (mode 0) or depth difference (mode 1)
  const float* dz;      // nx*ny peak-depth rise for the hatching, or NULL
  uchar4* out;          // (scale nx) x (scale ny)
};

__constant__ float kDepthRamp[8][3] = {
    {0.8706f, 0.9216f, 0.9686f}, {0.7765f, 0.8588f, 0.9373f}, {0.6196f, 0.7922f, 0.8824f}, {0.4196f, 0.6824f, 0.8392f},
    {0.2588f, 0.5725f, 0.7765f}, {0.1294f, 0.4431f, 0.7098f}, {0.0314f, 0.3176f, 0.6118f}, {0.0314f, 0.1882f, 0.4196f}};
__constant__ float kDiffRamp[7][3] = {
    {0.1294f, 0.4000f, 0.6745f}, {0.4039f, 0.6627f, 0.8118f}, {0.8196f, 0.8980f, 0.9412f}, {0.9686f, 0.9686f, 0.9686f},
    {0.9922f, 0.8588f, 0.7804f}, {0.9373f, 0.5412f, 0.3843f}, {0.6980f, 0.0941f, 0.1686f}};

// mix(a, b, f) = a (1 - f) + b f (the GLSL definition).
__device__ __forceinline__ float mixf(float a, float b, float f) { return a * (1.0f - f) + b * f; }

// glslRamp (viewer.js:65-70): x = clamp(t, 0, 1) (n - 1), i = min(floor(x), n - 2), mix.
__device__ __forceinline__ float3 ramp(const float (*C)[3], int n, float t) {
  const float x = fminf(fmaxf(t, 0.0f), 1.0f) * (float)(n - 1);
  const int i = min((int)floorf(x), n - 2);
  const float f = x - (float)i;
  return make_float3(mixf(C[i][0], C[i + 1][0], f), mixf(C[i][1], C[i + 1][1], f), mixf(C[i][2], C[i + 1][2], f));
}

// Z(c) of the shader: clamped to the grid, no data as 1e9.
__device__ __forceinline__ float render_z(const RenderArgs& A, int cx, int cy) {
  cx = min(max(cx, 0), A.nx - 1);
  cy = min(max(cy, 0), A.ny - 1);
  const float v = A.z[(size_t)cy * A.nx + cx];
  return v != v ? 1e9f : v;
}

__device__ __forceinline__ uint8_t unorm8(float v) { return (uint8_t)__float2int_rn(fminf(fmaxf(v, 0.0f), 1.0f) * 255.0f); }

__global__ void k_render_map(const RenderArgs A) {
  const int W = A.nx * A.scale, H = A.ny * A.scale;
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= W || py >= H) return;
  const float cxf = ((float)px + 0.5f) / (float)A.scale, cyf = ((float)py + 0.5f) / (float)A.scale;
  const int cx = (int)cxf, cy = (int)cyf;
  const size_t i = (size_t)cy * A.nx + cx;
  float3 col;
  const float zc = A.z[i];
  if (zc != zc || zc > 1e8f) {
    col = make_float3(0.87f, 0.87f, 0.87f);
  } else {
    float gx = (render_z(A, cx + 1, cy) - render_z(A, cx - 1, cy)) / (2.0f * A.cs) * A.vex;
    float gy = (render_z(A, cx, cy + 1) - render_z(A, cx, cy - 1)) / (2.0f * A.cs) * A.vex;
    if (fabsf(gx) > 1e6f) gx = 0.0f;
    if (fabsf(gy) > 1e6f) gy = 0.0f;
    const float nl = sqrtf(gx * gx + gy * gy + 1.0f);   // normalize(vec3(-gx, gy, 1))
    const float nx_ = -gx / nl, ny_ = gy / nl, nz_ = 1.0f / nl;
    const float ll = sqrtf(0.25f + 0.25f + 0.49f);      // normalize(vec3(-.5, .5, .7))
    const float lx = -0.5f / ll, ly = 0.5f / ll, lz = 0.7f / ll;
    const float shade = fminf(fmaxf(nx_ * lx + ny_ * ly + nz_ * lz, 0.0f), 1.0f);
    const float g = 0.3f + 0.6f * shade;
    col = make_float3(g, g, g);
    const float v = A.value[i];
    if (A.mode == 0) {
      if (v > 0.0050f) col = ramp(kDepthRamp, 8, logf(v / 0.0050f) / logf(400.0f));
    } else if (fabsf(v) > 0.005f) {
      col = ramp(kDiffRamp, 7, fminf(fmaxf(v / 0.20f, -1.0f), 1.0f) * 0.5f + 0.5f);
    }
    if (A.worse && A.dz) {
      const float d = A.dz[i];
      const float s = (cxf + cyf) * 0.5f;
      if (d > 0.01f && s - floorf(s) < 0.5f) col = make_float3(mixf(col.x, 0.0f, 0.7f), mixf(col.y, 0.0f, 0.7f), mixf(col.z, 0.0f, 0.7f));
    }
  }
  A.out[(size_t)py * W + px] = make_uchar4(unorm8(col.x), unorm8(col.y), unorm8(col.z), 255);
}

}  // namespace itr
