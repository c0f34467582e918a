"""Inputs of the headless flood-scene render (itr_gpu_render_scene, presentation only).

The reference's video ray-marches every recorded frame with an SkSL shader through Skia
(video/src/shaders/terrain.sksl). Its inputs are three packed textures (video/src/data.rs:89-96)
and the uniforms that video/src/lib.rs:52-77 sets. This module builds the same inputs from
arrays: a camera from a position and a target (Camera::look, lib.rs:35-42), and the terrain,
depth and velocity textures with their 16-bit and 8-bit codes.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib

MAT_GROUND, MAT_FILL, MAT_CUT, MAT_BUILDING = 0, 60, 160, 250   # material codes the shader tells apart


@dataclass
class SceneView:
    """The shader's uniforms (terrain.sksl:13-31), in the field order of itr_scene_view."""
    cam_pos: tuple = (0.0, 0.0, 100.0)
    cam_fwd: tuple = (0.0, 1.0, 0.0)
    cam_right: tuple = (1.0, 0.0, 0.0)
    cam_up: tuple = (0.0, 0.0, 1.0)
    focal: float = 1.0
    domain: tuple = (1.0, 1.0, 1.0)     # width, height, cell size (m)
    z_lo: float = 0.0
    z_span: float = 1.0
    up: float = 1.0                     # terrain texels per simulation cell
    depth_span: float = 4.0
    ve: float = 1.0
    time: float = 0.0
    rain: float = 0.0
    wet: float = 0.0
    overcast: float = 0.1
    vel_max: float = 2.0
    base: float = 9.0                   # lib.rs:75
    ortho: bool = False
    debug: int = 0

    def to_c(self) -> _lib.SceneView:
        f3 = C.c_float * 3
        return _lib.SceneView(f3(*self.cam_pos), f3(*self.cam_fwd), f3(*self.cam_right), f3(*self.cam_up), self.focal,
                              f3(*self.domain), self.z_lo, self.z_span, self.up, self.depth_span, self.ve, self.time,
                              self.rain, self.wet, self.overcast, self.vel_max, self.base, 1 if self.ortho else 0,
                              int(self.debug))

    def floats(self) -> np.ndarray:
        """The 27 floats of the view in itr_scene_view order (the CPU oracle's argument)."""
        return np.array(list(self.cam_pos) + list(self.cam_fwd) + list(self.cam_right) + list(self.cam_up) + [self.focal]
                        + list(self.domain) + [self.z_lo, self.z_span, self.up, self.depth_span, self.ve, self.time,
                                               self.rain, self.wet, self.overcast, self.vel_max, self.base],
                        dtype=np.float32)


def look(pos, target, fov_deg: float):
    """Camera::look (video/src/lib.rs:35-42) in f32: forward, right (forward x z), up
    (right x forward) and the focal length 0.5 / tan(fov / 2) in image-height units."""
    f32 = np.float32
    p, t = np.asarray(pos, f32), np.asarray(target, f32)

    def norm(v):
        return (v / f32(math.sqrt(float(np.dot(v, v))))).astype(f32)

    fwd = norm(t - p)
    right = norm(np.cross(fwd, np.array([0, 0, 1], f32)).astype(f32))
    up = np.cross(right, fwd).astype(f32)
    focal = f32(0.5) / f32(math.tan(math.radians(fov_deg) / 2.0))
    return tuple(map(float, fwd)), tuple(map(float, right)), tuple(map(float, up)), float(focal)


def _code16(v01: np.ndarray) -> np.ndarray:
    return np.rint(np.clip(v01, 0.0, 1.0) * 65535.0).astype(np.uint32)


def terrain_texture(z: np.ndarray, material: np.ndarray | None = None, z_lo: float | None = None,
                    z_span: float | None = None):
    """RGBA texture of the refined terrain (th, tw): R, G the 16-bit elevation code over
    [z_lo, z_lo + z_span], B the material code. Returns (rgba, z_lo, z_span)."""
    z = np.asarray(z, np.float64)
    lo = float(z.min()) if z_lo is None else z_lo
    span = float(z.max() - lo) * 1.02 + 1e-3 if z_span is None else z_span
    code = _code16((z - lo) / span)
    out = np.zeros(z.shape + (4,), np.uint8)
    out[..., 0] = code >> 8
    out[..., 1] = code & 255
    out[..., 2] = 0 if material is None else np.asarray(material, np.uint8)
    out[..., 3] = 255
    return out, lo, span


def depth_texture(depth: np.ndarray, depth_span: float) -> np.ndarray:
    """RGBA texture of the simulation grid's depth: R, G the 16-bit code over depth_span,
    B 255 where wet."""
    d = np.asarray(depth, np.float64)
    code = _code16(d / depth_span)
    out = np.zeros(d.shape + (4,), np.uint8)
    out[..., 0] = code >> 8
    out[..., 1] = code & 255
    out[..., 2] = np.where(d > 0.0, 255, 0)
    out[..., 3] = 255
    return out


def velocity_texture(u: np.ndarray, v: np.ndarray, vel_max: float) -> np.ndarray:
    """RGBA texture of the velocity: R, G = 128 + 127 u / vel_max (and v), clamped to 0..255."""
    def enc(a):
        return np.clip(np.rint(128.0 + 127.0 * np.asarray(a, np.float64) / vel_max), 0, 255).astype(np.uint8)
    u = np.asarray(u)
    out = np.zeros(u.shape + (4,), np.uint8)
    out[..., 0] = enc(u)
    out[..., 1] = enc(v)
    out[..., 3] = 255
    return out
