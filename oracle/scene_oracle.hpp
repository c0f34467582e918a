// scene_oracle.hpp — CPU restatement of the video's height-field ray marcher
// (video/src/shaders/terrain.sksl), the oracle for itr_gpu_render_scene.
//
// TEST INFRASTRUCTURE: included by oracle_capi.cpp only. f32 arithmetic in the shader's
// operation order, compiled without FMA contraction (oracle/Makefile), with the GLSL
// definitions of mix, clamp, smoothstep, fract, step, reflect and min / max; sin, exp and pow
// from itr_math.h (sinf_ref, expf_ref, powf_ref: the ones the device calls, deterministic
// double-precision restatements), square roots and divisions IEEE. Texture
// reads: the texel under the coordinate, clamped to the image; a channel's `c * 255` is its
// byte. Output rounded to 8 bits from f32.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstddef>
#include "itr_math.h"

namespace orc_scene {

struct F2 { float x, y; };
struct F3 { float x, y, z; };

static inline F2 f2(float x, float y) { F2 r; r.x = x; r.y = y; return r; }
static inline F3 f3(float x, float y, float z) { F3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline F2 add(F2 a, F2 b) { return f2(a.x + b.x, a.y + b.y); }
static inline F2 sub(F2 a, F2 b) { return f2(a.x - b.x, a.y - b.y); }
static inline F2 muls(F2 a, float s) { return f2(a.x * s, a.y * s); }
static inline F2 adds(F2 a, float s) { return f2(a.x + s, a.y + s); }
static inline F2 divs(F2 a, float s) { return f2(a.x / s, a.y / s); }
static inline F3 add(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline F3 sub(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline F3 mul(F3 a, F3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline F3 muls(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }

static inline float gmin(float a, float b) { return b < a ? b : a; }   // GLSL min
static inline float gmax(float a, float b) { return a < b ? b : a; }   // GLSL max
static inline float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
static inline float gmix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
static inline F3 gmix(F3 a, F3 b, float t) { return f3(gmix(a.x, b.x, t), gmix(a.y, b.y, t), gmix(a.z, b.z, t)); }
static inline float gfract(float x) { return x - std::floor(x); }
static inline float gsmooth(float e0, float e1, float x) {
  float t = gclamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
static inline float dot(F2 a, F2 b) { return a.x * b.x + a.y * b.y; }
static inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float length(F2 a) { return std::sqrt(dot(a, a)); }
static inline F3 normalize(F3 a) { float l = std::sqrt(dot(a, a)); return f3(a.x / l, a.y / l, a.z / l); }
static inline float gsign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

struct View {
  float cam_pos[3], cam_fwd[3], cam_right[3], cam_up[3], focal;
  float W, H, cell, z_lo, z_span, up, depth_span, ve, time, rain, wet, overcast, vel_max, base;
  int ortho, debug;
};

struct Tex { const uint8_t* p; int w, h; };

static inline const uint8_t* fetch(const Tex& t, float x, float y) {
  float fx = std::floor(x), fy = std::floor(y);
  if (!(fx >= 0.0f)) fx = 0.0f;
  if (!(fy >= 0.0f)) fy = 0.0f;
  int i = fx < (float)(t.w - 1) ? (int)fx : t.w - 1;
  int j = fy < (float)(t.h - 1) ? (int)fy : t.h - 1;
  return t.p + ((size_t)j * t.w + i) * 4;
}
static inline float dec16(const uint8_t* c) { return ((float)c[0] * 256.0f + (float)c[1]) / 65535.0f; }
static inline float bilin(const Tex& t, F2 tc) {
  F2 f = sub(tc, f2(0.5f, 0.5f));
  F2 i0 = f2(std::floor(f.x), std::floor(f.y));
  F2 w = sub(f, i0);
  float a = dec16(fetch(t, i0.x + 0.5f, i0.y + 0.5f));
  float b = dec16(fetch(t, i0.x + 1.5f, i0.y + 0.5f));
  float c = dec16(fetch(t, i0.x + 0.5f, i0.y + 1.5f));
  float d = dec16(fetch(t, i0.x + 1.5f, i0.y + 1.5f));
  return gmix(gmix(a, b, w.x), gmix(c, d, w.x), w.y);
}

struct Shader {
  View u;
  Tex terrain, depth, vel;

  F2 simTc(F2 xy) const { return divs(f2(xy.x, u.H - xy.y), u.cell); }
  float groundH(F2 xy) const { return bilin(terrain, muls(simTc(xy), u.up)) * u.z_span * u.ve; }
  float depthM(F2 xy) const { return bilin(depth, simTc(xy)) * u.depth_span; }
  float waterH(F2 xy) const { return groundH(xy) + depthM(xy) * u.ve; }
  float surfaceH(F2 xy) const { return waterH(xy); }
  float material(F2 xy) const {
    F2 s = muls(simTc(xy), u.up);
    return (float)fetch(terrain, std::floor(s.x) + 0.5f, std::floor(s.y) + 0.5f)[2];
  }
  F2 velocity(F2 xy) const {
    F2 s = simTc(xy);
    const uint8_t* c = fetch(vel, s.x, s.y);
    return f2(((float)c[0] - 128.0f) / 127.0f * u.vel_max, ((float)c[1] - 128.0f) / 127.0f * u.vel_max);
  }

  static float hash(F2 p) { return gfract(itr_math::sinf_ref(dot(p, f2(127.1f, 311.7f))) * 43758.5453f); }
  static float vnoise(F2 p) {
    F2 i = f2(std::floor(p.x), std::floor(p.y));
    F2 f = f2(gfract(p.x), gfract(p.y));
    F2 uu = f2(f.x * f.x * (3.0f - 2.0f * f.x), f.y * f.y * (3.0f - 2.0f * f.y));
    return gmix(gmix(hash(i), hash(add(i, f2(1, 0))), uu.x), gmix(hash(add(i, f2(0, 1))), hash(add(i, f2(1, 1))), uu.x), uu.y);
  }
  static float fbm(F2 p) {
    float s = 0.0f, a = 0.5f;
    for (int i = 0; i < 5; i++) {
      s += a * vnoise(p);
      p = add(muls(p, 2.03f), f2(17.1f, 9.7f));
      a *= 0.5f;
    }
    return s;
  }

  static F3 sunDir() { return normalize(f3(-0.72f, 0.28f, 0.62f)); }
  F3 skyColor(F3 rd) const {
    float upz = gclamp(rd.z, -0.2f, 1.0f);
    F3 clear = gmix(f3(0.62f, 0.72f, 0.84f), f3(0.20f, 0.36f, 0.66f), itr_math::powf_ref(gmax(upz, 0.0f), 0.6f));
    F3 storm = gmix(f3(0.42f, 0.45f, 0.49f), f3(0.22f, 0.25f, 0.30f), itr_math::powf_ref(gmax(upz, 0.0f), 0.7f));
    F3 c = gmix(clear, storm, u.overcast);
    float sd = gmax(dot(rd, sunDir()), 0.0f);
    F3 g1 = muls(muls(f3(1.0f, 0.85f, 0.6f), itr_math::powf_ref(sd, 600.0f)), 18.0f);
    F3 g2 = muls(muls(f3(1.0f, 0.8f, 0.55f), itr_math::powf_ref(sd, 8.0f)), 0.18f);
    return add(c, muls(add(g1, g2), 1.0f - u.overcast));
  }
  F3 sunColor() const { return gmix(f3(2.9f, 2.6f, 2.2f), f3(0.35f, 0.36f, 0.38f), u.overcast); }
  F3 ambientColor() const { return gmix(f3(0.42f, 0.52f, 0.66f), f3(0.62f, 0.65f, 0.70f), u.overcast); }

  float softShadow(F3 p) const {
    if (u.overcast > 0.97f) return 1.0f;
    F3 l = sunDir();
    float res = 1.0f, t = 0.6f;
    for (int i = 0; i < 28; i++) {
      F3 q = add(p, muls(l, t));
      if (q.x < 0.0f || q.y < 0.0f || q.x > u.W || q.y > u.H) break;
      float d = q.z - groundH(f2(q.x, q.y));
      res = gmin(res, 10.0f * d / t);
      if (res < 0.0f) break;
      t += gclamp(d * 0.6f, 0.6f, 24.0f);
    }
    return gmix(gclamp(res, 0.0f, 1.0f), 1.0f, u.overcast);
  }

  F3 groundNormal(F2 xy) const {
    float e = u.cell / u.up;
    float hx = groundH(add(xy, f2(e, 0))) - groundH(sub(xy, f2(e, 0)));
    float hy = groundH(add(xy, f2(0, e))) - groundH(sub(xy, f2(0, e)));
    return normalize(f3(-hx, -hy, 2.0f * e));
  }

  F3 albedo(F2 xy, F3 n, float m) const {
    float g = fbm(muls(xy, 0.08f));
    float fine = fbm(muls(xy, 0.9f));
    F3 grass = gmix(f3(0.07f, 0.12f, 0.035f), f3(0.11f, 0.135f, 0.05f), gsmooth(0.3f, 0.8f, g));
    grass = muls(grass, 0.88f + 0.24f * fine);
    float slope = 1.0f - n.z;
    F3 dirt = muls(f3(0.17f, 0.13f, 0.09f), 0.85f + 0.3f * fine);
    F3 a = gmix(grass, dirt, gsmooth(0.08f * u.ve, 0.35f * u.ve, slope));
    if (m >= 250.0f) {
      a = (n.z > 0.35f) ? muls(f3(0.11f, 0.10f, 0.10f), 0.9f + 0.2f * fine) : f3(0.52f, 0.47f, 0.40f);
    } else if (m >= 1.0f && m <= 120.0f) {
      a = gmix(a, muls(f3(0.24f, 0.16f, 0.10f), 0.9f + 0.2f * fine), gclamp(m / 15.0f, 0.0f, 1.0f));
    } else if (m > 120.0f && m <= 200.0f) {
      a = gmix(a, f3(0.20f, 0.14f, 0.09f), gclamp((m - 120.0f) / 15.0f, 0.0f, 1.0f));
    }
    return muls(a, gmix(1.0f, 0.62f, u.wet * (m >= 250.0f ? 0.5f : 1.0f)));
  }

  F3 litSurface(F3 p, F3 n, F3 a, F3 rd) const {
    F3 l = sunDir();
    float sh = softShadow(add(p, muls(n, 0.3f)));
    float ao = 0.6f + 0.4f * gclamp(n.z, 0.0f, 1.0f);
    F3 sun = muls(muls(sunColor(), gmax(dot(n, l), 0.0f)), sh);
    F3 amb = muls(muls(ambientColor(), ao), 0.55f + 0.45f * n.z);
    F3 col = mul(a, add(sun, amb));
    F3 h = normalize(sub(l, rd));
    float s = u.wet * (1.0f - u.overcast) * sh;
    return add(col, muls(f3(s * 0.25f, s * 0.25f, s * 0.25f), itr_math::powf_ref(gmax(dot(n, h), 0.0f), 60.0f)));
  }

  F2 rainRipple(F2 xy) const {
    F2 g = divs(xy, 0.7f);
    F2 acc = f2(0.0f, 0.0f);
    for (int j = -1; j <= 1; j++) {
      for (int i = -1; i <= 1; i++) {
        F2 c = add(f2(std::floor(g.x), std::floor(g.y)), f2((float)i, (float)j));
        float r = hash(c);
        F2 o = add(adds(c, 0.5f), muls(f2(hash(adds(c, 3.1f)) - 0.5f, hash(adds(c, 7.7f)) - 0.5f), 0.35f));
        float ph = gfract(u.time * 0.9f + r);
        F2 d = sub(g, o);
        float dist = length(d);
        float ring = itr_math::sinf_ref(3.14159265f * 2.0f * (dist - ph * 0.9f) * 3.0f) * (1.0f - ph) *
                     gsmooth(0.9f, 0.0f, std::fabs(dist - ph * 0.9f) * 3.0f);
        float st = u.rain * 1.2f < r ? 0.0f : 1.0f;
        F2 dir = dist > 1e-3f ? divs(d, dist) : f2(0.0f, 0.0f);
        acc = add(acc, muls(muls(dir, ring), st));
      }
    }
    return muls(acc, 0.12f);
  }

  F2 flowRipple(F2 xy, F2 v) const {
    float period = 2.5f;
    float p0 = gfract(u.time / period);
    float p1 = gfract(u.time / period + 0.5f);
    float w0 = 1.0f - std::fabs(p0 * 2.0f - 1.0f);
    float e = 0.15f;
    F2 q0 = sub(muls(xy, 1.6f), muls(muls(muls(v, p0), period), 1.6f));
    F2 q1 = adds(sub(muls(xy, 1.6f), muls(muls(muls(v, p1), period), 1.6f)), 0.37f);
    F2 g0 = f2(vnoise(add(q0, f2(e, 0))) - vnoise(sub(q0, f2(e, 0))), vnoise(add(q0, f2(0, e))) - vnoise(sub(q0, f2(0, e))));
    F2 g1 = f2(vnoise(add(q1, f2(e, 0))) - vnoise(sub(q1, f2(e, 0))), vnoise(add(q1, f2(0, e))) - vnoise(sub(q1, f2(0, e))));
    float speed = gclamp(length(v) / 0.6f, 0.0f, 1.0f);
    return muls(muls(add(muls(g0, w0), muls(g1, 1.0f - w0)), 0.15f + 0.85f * speed), 0.9f);
  }

  F3 shadeWater(F3 p, F3 rd, float dW, float t) const {
    F2 xy = f2(p.x, p.y);
    float e = u.cell * 0.5f;
    float hx = waterH(add(xy, f2(e, 0))) - waterH(sub(xy, f2(e, 0)));
    float hy = waterH(add(xy, f2(0, e))) - waterH(sub(xy, f2(0, e)));
    F2 v = velocity(xy);
    F2 slope = divs(f2(hx, hy), 2.0f * e);
    float detail = gclamp(1.0f - t / 900.0f, 0.25f, 1.0f);
    slope = add(slope, muls(muls(add(flowRipple(xy, v), rainRipple(xy)), detail), gclamp(dW / 0.01f, 0.0f, 1.0f)));
    F3 n = normalize(f3(-slope.x, -slope.y, 1.0f));
    F3 bed = litSurface(f3(xy.x, xy.y, groundH(xy)), groundNormal(xy), muls(albedo(xy, groundNormal(xy), 0.0f), 0.8f), rd);
    float path = dW * (1.0f + 1.0f / gmax(-rd.z, 0.15f));
    F3 trans = f3(itr_math::expf_ref(-9.0f * path), itr_math::expf_ref(-11.0f * path), itr_math::expf_ref(-15.0f * path));
    F3 silt = f3(0.085f, 0.062f, 0.038f);
    F3 light = add(muls(muls(sunColor(), gmax(sunDir().z, 0.0f)), softShadow(add(p, f3(0, 0, 0.2f)))), ambientColor());
    F3 body = add(mul(bed, trans), mul(mul(silt, light), sub(f3(1, 1, 1), trans)));
    float cosi = gclamp(dot(f3(-rd.x, -rd.y, -rd.z), n), 0.0f, 1.0f);
    float F = 0.02f + 0.98f * itr_math::powf_ref(1.0f - cosi, 5.0f);
    F3 r = sub(rd, muls(n, 2.0f * dot(n, rd)));
    return gmix(body, skyColor(r), F);
  }
};

static inline uint8_t unorm8(float v) { return (uint8_t)std::nearbyint(gclamp(v, 0.0f, 1.0f) * 255.0f); }

// One pixel of main(fc) at fc = (px + 0.5, py + 0.5).
static inline void pixel(const Shader& S, int px, int py, int width, int height, uint8_t* o) {
  const View& u = S.u;
  F2 fc = f2((float)px + 0.5f, (float)py + 0.5f);
  float RX = (float)width, RY = (float)height;
  o[3] = 255;
  if (u.debug == 1) { o[0] = unorm8(fc.x / RX); o[1] = unorm8(fc.y / RY); o[2] = 0; return; }
  if (u.debug == 2 || u.debug == 3) {
    F2 xy = f2(fc.x / RX * u.W, (1.0f - fc.y / RY) * u.H);
    if (u.debug == 2) {
      float v = bilin(S.terrain, muls(S.simTc(xy), u.up));
      o[0] = unorm8(v); o[1] = unorm8(gfract(v * 20.0f)); o[2] = unorm8(S.material(xy) / 255.0f);
    } else {
      o[0] = 0; o[1] = 0; o[2] = unorm8(gclamp(S.depthM(xy) * 5.0f, 0.0f, 1.0f));
    }
    return;
  }
  F2 uv = f2((fc.x - 0.5f * RX) / RY, (fc.y - 0.5f * RY) / RY);
  uv.y = -uv.y;
  F3 fwd = f3(u.cam_fwd[0], u.cam_fwd[1], u.cam_fwd[2]);
  F3 right = f3(u.cam_right[0], u.cam_right[1], u.cam_right[2]);
  F3 upv = f3(u.cam_up[0], u.cam_up[1], u.cam_up[2]);
  F3 rd = normalize(add(add(muls(fwd, u.focal), muls(right, uv.x)), muls(upv, uv.y)));
  F3 ro = f3(u.cam_pos[0], u.cam_pos[1], u.cam_pos[2]);
  float top = u.z_span * u.ve;
  F3 bmin = f3(0.0f, 0.0f, -u.base * u.ve), bmax = f3(u.W, u.H, top);
  F3 inv = f3(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
  F3 t0 = mul(sub(bmin, ro), inv), t1 = mul(sub(bmax, ro), inv);
  F3 tsm = f3(gmin(t0.x, t1.x), gmin(t0.y, t1.y), gmin(t0.z, t1.z));
  F3 tbg = f3(gmax(t0.x, t1.x), gmax(t0.y, t1.y), gmax(t0.z, t1.z));
  float tn = gmax(gmax(tsm.x, tsm.y), tsm.z);
  float tf = gmin(gmin(tbg.x, tbg.y), tbg.z);
  F3 col = S.skyColor(rd);
  float tHit = -1.0f;
  bool side = false;
  auto inner = [&](F2 q) { return f2(gclamp(q.x, 0.01f, u.W - 0.01f), gclamp(q.y, 0.01f, u.H - 0.01f)); };
  if (u.ortho) {
    F2 xy = f2(fc.x / RX * u.W, (1.0f - fc.y / RY) * u.H);
    rd = f3(0.0f, 0.0f, -1.0f);
    ro = f3(xy.x, xy.y, top + 40.0f);
    tHit = ro.z - S.surfaceH(xy);
  } else if (tf > gmax(tn, 0.0f)) {
    float t = gmax(tn, 0.0f);
    F3 p = add(ro, muls(rd, t));
    bool sideEntry = tn > 0.0f && (tsm.x >= gmax(tsm.y, tsm.z) || tsm.y >= gmax(tsm.x, tsm.z));
    if (sideEntry && p.z < S.surfaceH(inner(f2(p.x, p.y)))) {
      side = true;
      tHit = t;
    } else {
      float tPrev = t;
      for (int i = 0; i < 260; i++) {
        p = add(ro, muls(rd, t));
        float d = p.z - S.surfaceH(f2(p.x, p.y));
        if (d < 0.0f) { tHit = t; break; }
        tPrev = t;
        t += gmax(d * 0.42f, 0.04f + t * 0.0012f);
        if (t > tf) break;
      }
      if (tHit > 0.0f) {
        float a = tPrev, b = tHit;
        for (int k = 0; k < 7; k++) {
          float m = 0.5f * (a + b);
          F3 q = add(ro, muls(rd, m));
          if (q.z - S.surfaceH(f2(q.x, q.y)) < 0.0f) b = m; else a = m;
        }
        tHit = b;
      }
    }
  }
  if (tHit > 0.0f) {
    F3 p = add(ro, muls(rd, tHit));
    if (side) {
      F2 xy = inner(f2(p.x, p.y));
      float below = (S.surfaceH(xy) - p.z) / u.ve;
      F3 a = gmix(f3(0.16f, 0.11f, 0.07f), f3(0.30f, 0.22f, 0.14f), gsmooth(0.3f, 1.2f, below));
      a = muls(gmix(a, f3(0.22f, 0.20f, 0.17f), gsmooth(4.0f, 7.0f, below)),
               0.85f + 0.3f * Shader::fbm(muls(f2(p.x + p.y, p.z / u.ve), 0.6f)));
      F3 n = std::fabs(tsm.x - tn) < 1e-4f ? f3(gsign(-rd.x), 0, 0) : f3(0, gsign(-rd.y), 0);
      col = mul(a, add(muls(S.sunColor(), gmax(dot(n, Shader::sunDir()), 0.0f)), muls(S.ambientColor(), 0.75f)));
    } else {
      F2 xy = f2(p.x, p.y);
      float dm = S.depthM(xy);
      F3 n = S.groundNormal(xy);
      float m = S.material(xy);
      F3 a = S.albedo(xy, n, m);
      float open = m >= 250.0f ? 0.0f : gsmooth(0.005f, 0.03f, dm);
      float soak = gclamp(dm / 0.005f, 0.0f, 1.0f);
      col = S.litSurface(p, n, muls(a, gmix(1.0f, 0.7f, soak)), rd);
      if (open > 0.0f) col = gmix(col, S.shadeWater(p, rd, dm, tHit), open);
    }
    float fog = 1.0f - itr_math::expf_ref(-tHit * (0.00008f + 0.00025f * u.rain));
    col = gmix(col, S.skyColor(normalize(f3(rd.x, rd.y, 0.02f))), fog);
  }
  col = muls(col, 1.1f);
  float c3[3] = {col.x, col.y, col.z};
  for (int k = 0; k < 3; ++k) {
    float c = c3[k];
    float v = gclamp((c * (2.51f * c + 0.03f)) / (c * (2.43f * c + 0.59f) + 0.14f), 0.0f, 1.0f);
    o[k] = unorm8(itr_math::powf_ref(v, 1.0f / 2.2f));
  }
}

}  // namespace orc_scene
