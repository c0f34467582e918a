"""Headless flood-scene render (itr_gpu_render_scene): the video's height-field ray marcher
(video/src/shaders/terrain.sksl, uniforms from video/src/lib.rs:52-77) computed on the device.
Presentation only; the reference runs it through Skia on Metal, which has no counterpart here.

CPU: the deterministic sin and pow the restatement uses (itr_math.h) against numpy; the
oracle's image against values worked out by hand from the shader: the debug views, a sky
seen from above the block, and the top-down map of a flat cut under a storm sky (no shadow,
no glare, a known albedo). GPU: the device image equals the oracle's bit for bit in every
view (sunlit and storm perspectives with water, rain rings and flow ripples, the block's cut
face, the map view, the debug views); both use the same f32 operation order and the same
sin / exp / pow.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle_ref as orc
from itr_gpu.scene_render import (MAT_BUILDING, MAT_CUT, MAT_FILL, SceneView, depth_texture, look, terrain_texture,
                                  velocity_texture)
from itr_gpu.scenes import valley_field

NX, NY, CELL = 45, 35, 10.0        # the valley scene at 10 m: 450 x 350 m
W_M, H_M = NX * CELL, NY * CELL


def scene(up=2, ve=2.0):
    """Textures of the 10 m valley: terrain refined `up` times with a building, a fill and a
    cut, water on the valley floor, flow along the valley."""
    zf = valley_field(20261203 + 1)
    tw, th = NX * up, NY * up
    x = (np.arange(tw) + 0.5) * CELL / up
    y = H_M - (np.arange(th) + 0.5) * CELL / up
    z = zf(*np.meshgrid(x, y))
    mat = np.zeros((th, tw), np.uint8)
    mat[10:14, 20:26] = MAT_BUILDING
    z[10:14, 20:26] += 6.0
    mat[30:36, 40:50] = MAT_FILL
    z[30:36, 40:50] += 0.8
    mat[50:56, 60:70] = MAT_CUT
    z[50:56, 60:70] -= 0.5
    trgba, z_lo, z_span = terrain_texture(z, mat)
    xc = (np.arange(NX) + 0.5) * CELL
    yc = H_M - (np.arange(NY) + 0.5) * CELL
    zc = zf(*np.meshgrid(xc, yc))
    depth = np.clip(zc.min() + 1.4 - zc, 0.0, None)
    drgba = depth_texture(depth, 4.0)
    vrgba = velocity_texture(np.where(depth > 0, 0.7, 0.0), np.where(depth > 0, 0.15, 0.0), 2.0)
    base = dict(domain=(W_M, H_M, CELL), z_lo=z_lo, z_span=z_span, up=float(up), depth_span=4.0, ve=ve, vel_max=2.0)
    return trgba, drgba, vrgba, base


def view(base, pos, target, fov=50.0, **kw):
    fwd, right, upv, focal = look(pos, target, fov)
    return SceneView(cam_pos=tuple(pos), cam_fwd=fwd, cam_right=right, cam_up=upv, focal=focal, **base, **kw)


def views(base):
    top = base["z_span"] * base["ve"]
    return {
        "sunlit": view(base, (-80.0, -60.0, top + 90.0), (225.0, 175.0, 0.3 * top), time=610.0, rain=0.6, wet=0.4,
                       overcast=0.2),
        "storm": view(base, (520.0, 420.0, top + 60.0), (200.0, 160.0, 0.2 * top), fov=60.0, time=1200.0, rain=1.0,
                      wet=1.0, overcast=0.98),
        "side": view(base, (225.0, -140.0, 0.2 * top), (225.0, 175.0, 0.1 * top), fov=70.0, time=30.0, overcast=0.5),
        "map": SceneView(**base, ortho=True, time=300.0, rain=0.3, wet=0.2, overcast=0.4),
        "debug1": SceneView(**base, debug=1),
        "debug2": SceneView(**base, debug=2),
        "debug3": SceneView(**base, debug=3),
    }


def u8(v):
    return int(np.rint(min(max(v, 0.0), 1.0) * 255.0))


def tone(c):
    c = np.asarray(c, np.float64) * 1.1
    v = np.clip((c * (2.51 * c + 0.03)) / (c * (2.43 * c + 0.59) + 0.14), 0.0, 1.0)
    return [u8(x) for x in v ** (1.0 / 2.2)]


def test_texture_codes_and_camera():
    """The packers invert as video/src/data.rs:94-96 decodes (16-bit codes within half a code
    step), the velocity code as terrain.sksl:84-87 reads it, and look() builds Camera::look's
    frame (video/src/lib.rs:35-42): unit forward, horizontal right, up = right x forward."""
    rng = np.random.default_rng(3)
    z = rng.uniform(3.0, 27.0, (20, 30))
    t, lo, span = terrain_texture(z, np.full((20, 30), 60))
    back = (t[..., 0].astype(np.float64) * 256 + t[..., 1]) / 65535.0 * span + lo
    assert np.abs(back - z).max() <= 0.5 * span / 65535.0 + 1e-12 and np.all(t[..., 2] == 60)
    d = rng.uniform(0.0, 3.0, (20, 30))
    d[0, 0] = 0.0
    dt_ = depth_texture(d, 4.0)
    back = (dt_[..., 0].astype(np.float64) * 256 + dt_[..., 1]) / 65535.0 * 4.0
    assert np.abs(back - d).max() <= 0.5 * 4.0 / 65535.0 + 1e-12
    assert dt_[0, 0, 2] == 0 and np.all(dt_[d > 0][:, 2] == 255)
    u, v = rng.uniform(-2, 2, (20, 30)), rng.uniform(-2, 2, (20, 30))
    vt = velocity_texture(u, v, 2.0)
    assert np.abs((vt[..., 0].astype(np.float64) - 128.0) / 127.0 * 2.0 - u).max() <= 0.5 * 2.0 / 127.0 + 1e-12
    assert np.abs((vt[..., 1].astype(np.float64) - 128.0) / 127.0 * 2.0 - v).max() <= 0.5 * 2.0 / 127.0 + 1e-12
    fwd, right, up, focal = look((-80.0, -60.0, 120.0), (225.0, 175.0, 10.0), 50.0)
    f, r, w = np.array(fwd), np.array(right), np.array(up)
    assert abs(np.linalg.norm(f) - 1) < 1e-6 and abs(np.linalg.norm(r) - 1) < 1e-6 and abs(r[2]) < 1e-7
    assert np.allclose(w, np.cross(r, f), atol=1e-6) and w[2] > 0 and abs(f @ r) < 1e-6
    assert abs(focal - 0.5 / math.tan(math.radians(25.0))) < 1e-6


def test_deterministic_sin_and_pow():
    rng = np.random.default_rng(5)
    xs = np.concatenate([rng.uniform(-10, 10, 2000), rng.uniform(-4e6, 4e6, 2000), [0.0, math.pi / 2, -math.pi]])
    got = np.array([orc.lib().orc_sin_ref(float(x)) for x in xs])
    np.testing.assert_allclose(got, np.sin(xs), rtol=0, atol=1e-15)
    xs32 = rng.uniform(0, 1, 2000).astype(np.float32)
    ys32 = rng.uniform(0.1, 600, 2000).astype(np.float32)
    got = np.array([orc.lib().orc_powf_ref(float(x), float(y)) for x, y in zip(xs32, ys32)], np.float32)
    want = (xs32.astype(np.float64) ** ys32.astype(np.float64)).astype(np.float32)
    np.testing.assert_allclose(got, want, rtol=2e-7, atol=1e-38)
    assert orc.lib().orc_powf_ref(0.0, 0.6) == 0.0 and orc.lib().orc_powf_ref(1.0, 5.0) == 1.0


def test_oracle_debug_views():
    t, d, v, base = scene()
    w, h = 64, 36
    img = orc.render_scene(t, d, v, SceneView(**base, debug=1), w, h)
    for px, py in ((0, 0), (63, 35), (17, 9)):
        assert tuple(img[py, px]) == (u8((px + 0.5) / w), u8((py + 0.5) / h), 0, 255)
    # a constant terrain code and material, a constant depth
    code, m = 40000, 160
    tc = np.zeros_like(t)
    tc[..., 0], tc[..., 1], tc[..., 2], tc[..., 3] = code >> 8, code & 255, m, 255
    img = orc.render_scene(tc, d, v, SceneView(**base, debug=2), w, h)
    val = ((code >> 8) * 256.0 + (code & 255)) / 65535.0
    assert tuple(img[5, 7]) == (u8(val), u8(val * 20.0 - math.floor(val * 20.0)), m, 255)
    dc = depth_texture(np.full((NY, NX), 0.1), 4.0)
    img = orc.render_scene(t, dc, v, SceneView(**base, debug=3), w, h)
    dv = (int(dc[0, 0, 0]) * 256 + int(dc[0, 0, 1])) / 65535.0 * 4.0
    assert tuple(img[20, 30]) == (0, 0, u8(dv * 5.0), 255)


def test_oracle_sky_from_above():
    """Looking up from above the block: every ray leaves the box, the pixel is skyColor(rd)."""
    t, d, v, base = scene()
    top = base["z_span"] * base["ve"]
    vw = SceneView(**base, cam_pos=(200.0, 150.0, top + 50.0), cam_fwd=(0.0, 0.6, 0.8), cam_right=(1.0, 0.0, 0.0),
                   cam_up=(0.0, -0.8, 0.6), focal=0.9, overcast=0.3)
    w, h = 48, 27
    img = orc.render_scene(t, d, v, vw, w, h)
    sun = np.array([-0.72, 0.28, 0.62]) / np.linalg.norm([-0.72, 0.28, 0.62])
    for px, py in ((0, 0), (47, 26), (24, 13), (5, 20)):
        uvx = (px + 0.5 - 0.5 * w) / h
        uvy = -(py + 0.5 - 0.5 * h) / h
        rd = np.array(vw.cam_fwd) * vw.focal + np.array(vw.cam_right) * uvx + np.array(vw.cam_up) * uvy
        rd /= np.linalg.norm(rd)
        upz = min(max(rd[2], -0.2), 1.0)
        clear = np.array([0.62, 0.72, 0.84]) * (1 - max(upz, 0) ** 0.6) + np.array([0.20, 0.36, 0.66]) * max(upz, 0) ** 0.6
        storm = np.array([0.42, 0.45, 0.49]) * (1 - max(upz, 0) ** 0.7) + np.array([0.22, 0.25, 0.30]) * max(upz, 0) ** 0.7
        c = clear * (1 - vw.overcast) + storm * vw.overcast
        sd = max(float(rd @ sun), 0.0)
        c = c + (1 - vw.overcast) * (np.array([1.0, 0.85, 0.6]) * sd ** 600 * 18 + np.array([1.0, 0.8, 0.55]) * sd ** 8 * 0.18)
        want = tone(c)
        assert all(abs(int(a) - b) <= 1 for a, b in zip(img[py, px, :3], want)), (px, py, img[py, px], want)


def test_oracle_flat_cut_map():
    """Top-down map of a flat cut (material 200: albedo (0.20, 0.14, 0.09), no noise) under a
    storm sky (overcast 1: no shadow, no glare), dry and unsoaked."""
    t, d, v, base = scene()
    code = 30000
    tc = np.zeros_like(t)
    tc[..., 0], tc[..., 1], tc[..., 2], tc[..., 3] = code >> 8, code & 255, 200, 255
    dry = depth_texture(np.zeros((NY, NX)), 4.0)
    vw = SceneView(**base, ortho=True, overcast=1.0, wet=0.0, rain=0.0)
    img = orc.render_scene(tc, dry, v, vw, 40, 30)
    sun = np.array([-0.72, 0.28, 0.62]) / np.linalg.norm([-0.72, 0.28, 0.62])
    a = np.array([0.20, 0.14, 0.09])
    col = a * (np.array([0.35, 0.36, 0.38]) * sun[2] + np.array([0.62, 0.65, 0.70]))
    top = base["z_span"] * base["ve"]
    g = code / 65535.0 * base["z_span"] * base["ve"]
    fog = 1.0 - math.exp(-(top + 40.0 - g) * 0.00008)
    col = col * (1 - fog) + np.array([0.22, 0.25, 0.30]) * fog
    want = tone(col)
    for px, py in ((3, 3), (20, 15), (39, 29)):
        assert all(abs(int(x) - y) <= 1 for x, y in zip(img[py, px, :3], want)), (img[py, px], want)


@pytest.fixture(scope="module")
def gpu():
    from itr_gpu import GpuSolver
    g = GpuSolver()
    yield g
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sunlit", "storm", "side", "map", "debug1", "debug2", "debug3"])
def test_device_image_matches_oracle(gpu, name):
    t, d, v, base = scene()
    vw = views(base)[name]
    w, h = 192, 108
    dev = gpu.render_scene(t, d, v, vw, w, h)
    ref = orc.render_scene(t, d, v, vw, w, h)
    if not np.array_equal(dev, ref):
        diff = np.abs(dev.astype(int) - ref.astype(int))
        raise AssertionError(f"{name}: {(diff > 0).sum()} channels differ, max {diff.max()}")
    if name in ("sunlit", "storm", "side", "map"):
        assert len(np.unique(dev.reshape(-1, 4), axis=0)) > 200   # a real picture, not one colour


@pytest.mark.gpu
def test_device_full_hd_frame(gpu):
    """A 1920 x 1080 frame (the video's size, lib.rs:13-14), with its device time."""
    t, d, v, base = scene(up=4)
    vw = views(base)["sunlit"]
    img = gpu.render_scene(t, d, v, vw, 1920, 1080)
    ms = gpu.last_timing()["kernel_ms"]
    print(f"1920x1080 frame: {ms:.2f} ms on the device")
    assert img.shape == (1080, 1920, 4) and np.all(img[..., 3] == 255)
    assert len(np.unique(img.reshape(-1, 4), axis=0)) > 1000
