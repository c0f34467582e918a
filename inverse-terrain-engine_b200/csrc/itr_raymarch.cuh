// itr_raymarch.cuh — headless render of a flood scene: the video's height-field ray march
// (presentation, not on the solver's path).
//
// Restates the reference's SkSL fragment shader video/src/shaders/terrain.sksl (uniforms set
// by video/src/lib.rs:52-77, textures packed as in video/src/data.rs:89-96) as one CUDA thread
// per output pixel writing RGBA8 into device memory; the reference runs it through Skia on
// Metal, which has no counterpart here. Per pixel: the ray through the pixel centre, its
// entry into the terrain block, up to 260 relaxed march steps over the water surface and 7
// bisection steps, then the cut face of the block, or the ground lit by the sun with a soft
// shadow (28 steps) and procedural grass / soil / fill / roof albedo, or the flood water
// (turbid body over the lit bed, flow-advected and rain-ring ripples on its normal, Fresnel
// sky reflection), aerial perspective, the ACES-fit tone map and the 1/2.2 encode. Debug
// modes 1-3 and the top-down map view (uOrtho) are kept.
//
// Texture reads follow Skia's image shader at texel centres: texel (floor(x), floor(y)),
// clamped to the image, each channel byte / 255; so `c * 255` of the shader is the byte.
// The arithmetic is f32 in the shader's operation order (GLSL definitions of mix, clamp,
// smoothstep, fract, step, reflect; min / max return the second operand when it compares
// below / above the first); the sRGB-ish result is rounded to 8 bits directly (the shader's
// half4 output is not rounded to half first). The shader leaves sin, exp and pow to the
// platform; here they are itr_math's deterministic sinf_ref / expf_ref / powf_ref, so the
// image is the same bits on every device and on the CPU oracle (which calls the same ones):
// the procedural noise's fract(sin(.) * 43758.5) magnifies a last-bit difference in sin
// into a different pattern.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>
#include "itr_math.h"

namespace itr {

struct SceneArgs {
  const uchar4* terrain;   // tw x th texels: RG elevation code (16 bit), B material code
  const uchar4* depth;     // nx x ny: RG depth code (16 bit), B 255 where wet
  const uchar4* vel;       // nx x ny: RG velocity u, v (128 = 0, +-vel_max)
  int tw, th, nx, ny;
  int width, height;
  float cam_pos[3], cam_fwd[3], cam_right[3], cam_up[3];
  float focal;
  float dom_w, dom_h, cell;
  float z_span, up, depth_span, ve, time, rain, wet, overcast, vel_max, base;
  int ortho, debug;
  uchar4* out;             // width x height, row 0 the top
};

namespace rm {

struct V2 { float x, y; };
struct V3 { float x, y, z; };

__device__ __forceinline__ V2 v2(float x, float y) { return V2{x, y}; }
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 v3s(float s) { return V3{s, s, s}; }
__device__ __forceinline__ V2 operator+(V2 a, V2 b) { return v2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ V2 operator-(V2 a, V2 b) { return v2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ V2 operator*(V2 a, float s) { return v2(a.x * s, a.y * s); }
__device__ __forceinline__ V2 operator*(V2 a, V2 b) { return v2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ V2 operator/(V2 a, float s) { return v2(a.x / s, a.y / s); }
__device__ __forceinline__ V2 operator+(V2 a, float s) { return v2(a.x + s, a.y + s); }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator/(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }

__device__ __forceinline__ float mn(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float mx(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return mn(mx(x, lo), hi); }
__device__ __forceinline__ float lerp(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ V3 mix3(V3 a, V3 b, float t) { return v3(lerp(a.x, b.x, t), lerp(a.y, b.y, t), lerp(a.z, b.z, t)); }
__device__ __forceinline__ float fractf(float x) { return x - floorf(x); }
__device__ __forceinline__ float smooth(float e0, float e1, float x) {
  const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ float dot2(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len2(V2 a) { return sqrtf(dot2(a, a)); }
__device__ __forceinline__ V3 norm3(V3 a) { const float l = sqrtf(dot3(a, a)); return v3(a.x / l, a.y / l, a.z / l); }
__device__ __forceinline__ float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

// ------------------------------------------------------------------ textures ----------
// Skia's image shader at (x, y): texel (floor(x), floor(y)), clamped to the image
__device__ __forceinline__ uchar4 texel(const uchar4* t, int w, int h, float x, float y) {
  float fx = floorf(x), fy = floorf(y);
  fx = fx >= 0.0f ? fx : 0.0f;   // NaN too
  fy = fy >= 0.0f ? fy : 0.0f;
  const int i = fx < (float)(w - 1) ? (int)fx : w - 1;
  const int j = fy < (float)(h - 1) ? (int)fy : h - 1;
  return __ldg(t + (size_t)j * w + i);
}
__device__ __forceinline__ float dec16(uchar4 c) { return ((float)c.x * 256.0f + (float)c.y) / 65535.0f; }

// bilinTerrain / bilinDepth: manual bilinear filter, texel centres at i + 0.5
__device__ __forceinline__ float bilin(const uchar4* t, int w, int h, V2 tc) {
  const V2 f = tc + (-0.5f);
  const V2 i0 = v2(floorf(f.x), floorf(f.y));
  const V2 wt = f - i0;
  const float a = dec16(texel(t, w, h, i0.x + 0.5f, i0.y + 0.5f));
  const float b = dec16(texel(t, w, h, i0.x + 1.5f, i0.y + 0.5f));
  const float c = dec16(texel(t, w, h, i0.x + 0.5f, i0.y + 1.5f));
  const float d = dec16(texel(t, w, h, i0.x + 1.5f, i0.y + 1.5f));
  return lerp(lerp(a, b, wt.x), lerp(c, d, wt.x), wt.y);
}

struct Scene {
  const SceneArgs& A;
  __device__ V2 simTc(V2 xy) const { return v2(xy.x, A.dom_h - xy.y) / A.cell; }
  __device__ float groundH(V2 xy) const { return bilin(A.terrain, A.tw, A.th, simTc(xy) * A.up) * A.z_span * A.ve; }
  __device__ float depthM(V2 xy) const { return bilin(A.depth, A.nx, A.ny, simTc(xy)) * A.depth_span; }
  __device__ float waterH(V2 xy) const { return groundH(xy) + depthM(xy) * A.ve; }
  __device__ float surfaceH(V2 xy) const { return waterH(xy); }
  __device__ float material(V2 xy) const {
    const V2 s = simTc(xy) * A.up;
    const uchar4 c = texel(A.terrain, A.tw, A.th, floorf(s.x) + 0.5f, floorf(s.y) + 0.5f);
    return (float)c.z;
  }
  __device__ V2 velocity(V2 xy) const {
    const V2 s = simTc(xy);
    const uchar4 c = texel(A.vel, A.nx, A.ny, s.x, s.y);
    return v2(((float)c.x - 128.0f) / 127.0f * A.vel_max, ((float)c.y - 128.0f) / 127.0f * A.vel_max);
  }

  // ---------------------------------------------------------------- noise
  __device__ static float hash(V2 p) { return fractf(itr_math::sinf_ref(dot2(p, v2(127.1f, 311.7f))) * 43758.5453f); }
  __device__ static float vnoise(V2 p) {
    const V2 i = v2(floorf(p.x), floorf(p.y));
    const V2 f = v2(fractf(p.x), fractf(p.y));
    const V2 u = f * f * (v2(3.0f, 3.0f) - f * 2.0f);
    return lerp(lerp(hash(i), hash(i + v2(1.0f, 0.0f)), u.x), lerp(hash(i + v2(0.0f, 1.0f)), hash(i + v2(1.0f, 1.0f)), u.x), u.y);
  }
  __device__ static float fbm(V2 p) {
    float s = 0.0f, a = 0.5f;
    for (int i = 0; i < 5; ++i) {
      s += a * vnoise(p);
      p = p * 2.03f + v2(17.1f, 9.7f);
      a *= 0.5f;
    }
    return s;
  }

  // ---------------------------------------------------------------- sky and light
  __device__ static V3 sunDir() { return norm3(v3(-0.72f, 0.28f, 0.62f)); }
  __device__ V3 skyColor(V3 rd) const {
    const float upz = clampf(rd.z, -0.2f, 1.0f);
    const V3 clear = mix3(v3(0.62f, 0.72f, 0.84f), v3(0.20f, 0.36f, 0.66f), itr_math::powf_ref(mx(upz, 0.0f), 0.6f));
    const V3 storm = mix3(v3(0.42f, 0.45f, 0.49f), v3(0.22f, 0.25f, 0.30f), itr_math::powf_ref(mx(upz, 0.0f), 0.7f));
    V3 c = mix3(clear, storm, A.overcast);
    const float sd = mx(dot3(rd, sunDir()), 0.0f);
    const V3 glare = v3(1.0f, 0.85f, 0.6f) * itr_math::powf_ref(sd, 600.0f) * 18.0f + v3(1.0f, 0.8f, 0.55f) * itr_math::powf_ref(sd, 8.0f) * 0.18f;
    return c + glare * (1.0f - A.overcast);
  }
  __device__ V3 sunColor() const { return mix3(v3(2.9f, 2.6f, 2.2f), v3(0.35f, 0.36f, 0.38f), A.overcast); }
  __device__ V3 ambientColor() const { return mix3(v3(0.42f, 0.52f, 0.66f), v3(0.62f, 0.65f, 0.70f), A.overcast); }

  __device__ float softShadow(V3 p) const {
    if (A.overcast > 0.97f) return 1.0f;
    const V3 l = sunDir();
    float res = 1.0f, t = 0.6f;
    for (int i = 0; i < 28; ++i) {
      const V3 q = p + l * t;
      if (q.x < 0.0f || q.y < 0.0f || q.x > A.dom_w || q.y > A.dom_h) break;
      const float d = q.z - groundH(v2(q.x, q.y));
      res = mn(res, 10.0f * d / t);
      if (res < 0.0f) break;
      t += clampf(d * 0.6f, 0.6f, 24.0f);
    }
    return lerp(clampf(res, 0.0f, 1.0f), 1.0f, A.overcast);
  }

  __device__ V3 groundNormal(V2 xy) const {
    const float e = A.cell / A.up;
    const float hx = groundH(xy + v2(e, 0.0f)) - groundH(xy - v2(e, 0.0f));
    const float hy = groundH(xy + v2(0.0f, e)) - groundH(xy - v2(0.0f, e));
    return norm3(v3(-hx, -hy, 2.0f * e));
  }

  __device__ V3 albedo(V2 xy, V3 n, float m) const {
    const float g = fbm(xy * 0.08f);
    const float fine = fbm(xy * 0.9f);
    V3 grass = mix3(v3(0.07f, 0.12f, 0.035f), v3(0.11f, 0.135f, 0.05f), smooth(0.3f, 0.8f, g));
    grass = grass * (0.88f + 0.24f * fine);
    const float slope = 1.0f - n.z;
    const V3 dirt = v3(0.17f, 0.13f, 0.09f) * (0.85f + 0.3f * fine);
    V3 a = mix3(grass, dirt, smooth(0.08f * A.ve, 0.35f * A.ve, slope));
    if (m >= 250.0f) {
      a = (n.z > 0.35f) ? v3(0.11f, 0.10f, 0.10f) * (0.9f + 0.2f * fine) : v3(0.52f, 0.47f, 0.40f);
    } else if (m >= 1.0f && m <= 120.0f) {
      a = mix3(a, v3(0.24f, 0.16f, 0.10f) * (0.9f + 0.2f * fine), clampf(m / 15.0f, 0.0f, 1.0f));
    } else if (m > 120.0f && m <= 200.0f) {
      a = mix3(a, v3(0.20f, 0.14f, 0.09f), clampf((m - 120.0f) / 15.0f, 0.0f, 1.0f));
    }
    return a * lerp(1.0f, 0.62f, A.wet * (m >= 250.0f ? 0.5f : 1.0f));
  }

  __device__ V3 litSurface(V3 p, V3 n, V3 a, V3 rd) const {
    const V3 l = sunDir();
    const float sh = softShadow(p + n * 0.3f);
    const float ao = 0.6f + 0.4f * clampf(n.z, 0.0f, 1.0f);
    V3 col = a * (sunColor() * mx(dot3(n, l), 0.0f) * sh + ambientColor() * ao * (0.55f + 0.45f * n.z));
    const V3 h = norm3(l - rd);
    col = col + v3s(0.25f) * (A.wet * (1.0f - A.overcast) * sh) * itr_math::powf_ref(mx(dot3(n, h), 0.0f), 60.0f);   // s * float3(0.25) * pow
    return col;
  }

  // ---------------------------------------------------------------- water surface detail
  __device__ V2 rainRipple(V2 xy) const {
    const V2 g = xy / 0.7f;
    V2 acc = v2(0.0f, 0.0f);
    for (int j = -1; j <= 1; ++j) {
      for (int i = -1; i <= 1; ++i) {
        const V2 c = v2(floorf(g.x), floorf(g.y)) + v2((float)i, (float)j);
        const float r = hash(c);
        const V2 o = c + 0.5f + v2(hash(c + 3.1f) - 0.5f, hash(c + 7.7f) - 0.5f) * 0.35f;
        const float ph = fractf(A.time * 0.9f + r);
        const V2 d = g - o;
        const float dist = len2(d);
        const float ring = itr_math::sinf_ref(3.14159265f * 2.0f * (dist - ph * 0.9f) * 3.0f) * (1.0f - ph) *
                           smooth(0.9f, 0.0f, fabsf(dist - ph * 0.9f) * 3.0f);
        const float st = (A.rain * 1.2f < r) ? 0.0f : 1.0f;   // step(r, uRain * 1.2)
        acc = acc + (dist > 1e-3f ? d / dist : v2(0.0f, 0.0f)) * ring * st;
      }
    }
    return acc * 0.12f;
  }

  __device__ V2 flowRipple(V2 xy, V2 v) const {
    const float period = 2.5f;
    const float p0 = fractf(A.time / period);
    const float p1 = fractf(A.time / period + 0.5f);
    const float w0 = 1.0f - fabsf(p0 * 2.0f - 1.0f);
    const float e = 0.15f;
    const V2 q0 = xy * 1.6f - v * p0 * period * 1.6f;
    const V2 q1 = xy * 1.6f - v * p1 * period * 1.6f + 0.37f;
    const V2 g0 = v2(vnoise(q0 + v2(e, 0.0f)) - vnoise(q0 - v2(e, 0.0f)), vnoise(q0 + v2(0.0f, e)) - vnoise(q0 - v2(0.0f, e)));
    const V2 g1 = v2(vnoise(q1 + v2(e, 0.0f)) - vnoise(q1 - v2(e, 0.0f)), vnoise(q1 + v2(0.0f, e)) - vnoise(q1 - v2(0.0f, e)));
    const float speed = clampf(len2(v) / 0.6f, 0.0f, 1.0f);
    return (g0 * w0 + g1 * (1.0f - w0)) * (0.15f + 0.85f * speed) * 0.9f;
  }

  __device__ V3 shadeWater(V3 p, V3 rd, float dW, float t) const {
    const V2 xy = v2(p.x, p.y);
    const float e = A.cell * 0.5f;
    const float hx = waterH(xy + v2(e, 0.0f)) - waterH(xy - v2(e, 0.0f));
    const float hy = waterH(xy + v2(0.0f, e)) - waterH(xy - v2(0.0f, e));
    const V2 v = velocity(xy);
    V2 slope = v2(hx, hy) / (2.0f * e);
    const float detail = clampf(1.0f - t / 900.0f, 0.25f, 1.0f);
    slope = slope + (flowRipple(xy, v) + rainRipple(xy)) * detail * clampf(dW / 0.01f, 0.0f, 1.0f);
    const V3 n = norm3(v3(-slope.x, -slope.y, 1.0f));
    const V3 gn = groundNormal(xy);
    const V3 bed = litSurface(v3(xy.x, xy.y, groundH(xy)), gn, albedo(xy, groundNormal(xy), 0.0f) * 0.8f, rd);
    const V3 sigma = v3(9.0f, 11.0f, 15.0f);
    const float path = dW * (1.0f + 1.0f / mx(-rd.z, 0.15f));
    const V3 sp = sigma * (-path);
    const V3 trans = v3(itr_math::expf_ref(sp.x), itr_math::expf_ref(sp.y), itr_math::expf_ref(sp.z));
    const V3 silt = v3(0.085f, 0.062f, 0.038f);
    const V3 light = sunColor() * mx(sunDir().z, 0.0f) * softShadow(p + v3(0.0f, 0.0f, 0.2f)) + ambientColor();
    const V3 body = bed * trans + silt * light * (v3s(1.0f) - trans);
    const float cosi = clampf(dot3(-rd, n), 0.0f, 1.0f);
    const float F = 0.02f + 0.98f * itr_math::powf_ref(1.0f - cosi, 5.0f);
    const V3 r = rd - n * (2.0f * dot3(n, rd));   // reflect(rd, n)
    const V3 refl = skyColor(r);
    return mix3(body, refl, F);
  }
};

__device__ __forceinline__ uint8_t to_u8(float v) { return (uint8_t)__float2int_rn(clampf(v, 0.0f, 1.0f) * 255.0f); }

}  // namespace rm

__global__ void __launch_bounds__(256) k_render_scene(const SceneArgs A) {
  using namespace rm;
  const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= A.width || py >= A.height) return;
  const Scene S{A};
  const V2 fc = v2((float)px + 0.5f, (float)py + 0.5f);
  const float RX = (float)A.width, RY = (float)A.height;
  uchar4& out = A.out[(size_t)py * A.width + px];
  if (A.debug == 1) { out = make_uchar4(to_u8(fc.x / RX), to_u8(fc.y / RY), 0, 255); return; }
  if (A.debug == 2) {
    const V2 xy = v2(fc.x / RX * A.dom_w, (1.0f - fc.y / RY) * A.dom_h);
    const float v = bilin(A.terrain, A.tw, A.th, S.simTc(xy) * A.up);
    out = make_uchar4(to_u8(v), to_u8(fractf(v * 20.0f)), to_u8(S.material(xy) / 255.0f), 255);
    return;
  }
  if (A.debug == 3) {
    const V2 xy = v2(fc.x / RX * A.dom_w, (1.0f - fc.y / RY) * A.dom_h);
    out = make_uchar4(0, 0, to_u8(clampf(S.depthM(xy) * 5.0f, 0.0f, 1.0f)), 255);
    return;
  }
  V2 uv = v2((fc.x - 0.5f * RX) / RY, (fc.y - 0.5f * RY) / RY);
  uv.y = -uv.y;
  const V3 fwd = v3(A.cam_fwd[0], A.cam_fwd[1], A.cam_fwd[2]);
  const V3 right = v3(A.cam_right[0], A.cam_right[1], A.cam_right[2]);
  const V3 upv = v3(A.cam_up[0], A.cam_up[1], A.cam_up[2]);
  V3 rd = norm3(fwd * A.focal + right * uv.x + upv * uv.y);
  V3 ro = v3(A.cam_pos[0], A.cam_pos[1], A.cam_pos[2]);

  const float top = A.z_span * A.ve;
  const V3 bmin = v3(0.0f, 0.0f, -A.base * A.ve);
  const V3 bmax = v3(A.dom_w, A.dom_h, top);
  const V3 inv = v3(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
  const V3 t0 = (bmin - ro) * inv;
  const V3 t1 = (bmax - ro) * inv;
  const V3 tsm = v3(mn(t0.x, t1.x), mn(t0.y, t1.y), mn(t0.z, t1.z));
  const V3 tbg = v3(mx(t0.x, t1.x), mx(t0.y, t1.y), mx(t0.z, t1.z));
  const float tn = mx(mx(tsm.x, tsm.y), tsm.z);
  const float tf = mn(mn(tbg.x, tbg.y), tbg.z);

  V3 col = S.skyColor(rd);
  float tHit = -1.0f;
  bool side = false;
  auto clampDom = [&](V2 q) { return v2(clampf(q.x, 0.01f, A.dom_w - 0.01f), clampf(q.y, 0.01f, A.dom_h - 0.01f)); };
  if (A.ortho) {
    const V2 xy = v2(fc.x / RX * A.dom_w, (1.0f - fc.y / RY) * A.dom_h);
    rd = v3(0.0f, 0.0f, -1.0f);
    ro = v3(xy.x, xy.y, top + 40.0f);
    tHit = ro.z - S.surfaceH(xy);
  } else if (tf > mx(tn, 0.0f)) {
    float t = mx(tn, 0.0f);
    V3 p = ro + rd * t;
    const bool sideEntry = tn > 0.0f && (tsm.x >= mx(tsm.y, tsm.z) || tsm.y >= mx(tsm.x, tsm.z));
    if (sideEntry && p.z < S.surfaceH(clampDom(v2(p.x, p.y)))) {
      side = true;
      tHit = t;
    } else {
      float tPrev = t;
      for (int i = 0; i < 260; ++i) {
        p = ro + rd * t;
        const float d = p.z - S.surfaceH(v2(p.x, p.y));
        if (d < 0.0f) { tHit = t; break; }
        tPrev = t;
        t += mx(d * 0.42f, 0.04f + t * 0.0012f);
        if (t > tf) break;
      }
      if (tHit > 0.0f) {
        float a = tPrev, b = tHit;
        for (int k = 0; k < 7; ++k) {
          const float m = 0.5f * (a + b);
          const V3 q = ro + rd * m;
          if (q.z - S.surfaceH(v2(q.x, q.y)) < 0.0f) b = m; else a = m;
        }
        tHit = b;
      }
    }
  }

  if (tHit > 0.0f) {
    const V3 p = ro + rd * tHit;
    if (side) {
      const V2 xy = clampDom(v2(p.x, p.y));
      const float below = (S.surfaceH(xy) - p.z) / A.ve;
      V3 a = mix3(v3(0.16f, 0.11f, 0.07f), v3(0.30f, 0.22f, 0.14f), smooth(0.3f, 1.2f, below));
      a = mix3(a, v3(0.22f, 0.20f, 0.17f), smooth(4.0f, 7.0f, below)) *
          (0.85f + 0.3f * Scene::fbm(v2(p.x + p.y, p.z / A.ve) * 0.6f));
      const V3 n = fabsf(tsm.x - tn) < 1e-4f ? v3(signf(-rd.x), 0.0f, 0.0f) : v3(0.0f, signf(-rd.y), 0.0f);
      col = a * (S.sunColor() * mx(dot3(n, Scene::sunDir()), 0.0f) + S.ambientColor() * 0.75f);
    } else {
      const V2 xy = v2(p.x, p.y);
      const float dm = S.depthM(xy);
      const V3 n = S.groundNormal(xy);
      const float m = S.material(xy);
      const V3 a = S.albedo(xy, n, m);
      const float open = m >= 250.0f ? 0.0f : smooth(0.005f, 0.03f, dm);
      const float soak = clampf(dm / 0.005f, 0.0f, 1.0f);
      col = S.litSurface(p, n, a * lerp(1.0f, 0.7f, soak), rd);
      if (open > 0.0f) col = mix3(col, S.shadeWater(p, rd, dm, tHit), open);
    }
    const float fog = 1.0f - itr_math::expf_ref(-tHit * (0.00008f + 0.00025f * A.rain));
    col = mix3(col, S.skyColor(norm3(v3(rd.x, rd.y, 0.02f))), fog);
  }

  col = col * 1.1f;
  const V3 num = col * (col * 2.51f + v3s(0.03f));
  const V3 den = col * (col * 2.43f + v3s(0.59f)) + v3s(0.14f);
  const V3 tm = num / den;
  col = v3(clampf(tm.x, 0.0f, 1.0f), clampf(tm.y, 0.0f, 1.0f), clampf(tm.z, 0.0f, 1.0f));
  const float g = 1.0f / 2.2f;
  out = make_uchar4(to_u8(itr_math::powf_ref(col.x, g)), to_u8(itr_math::powf_ref(col.y, g)), to_u8(itr_math::powf_ref(col.z, g)), 255);
}

}  // namespace itr
