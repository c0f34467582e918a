"""Earthwork primitives and their materialisation into a fine-resolution edit.

Restates crates/itr-core/src/design.rs: Primitive::segment/profile/bbox (:95-142),
DesignSpace::q and decode quantisation (:259-296), materialize (:316-385). Trigonometry
and square roots are the C library's (Python's math module), as the reference's `libm`
calls are. Also the derivatives of the profile with respect to height, width and length
at a fixed quantised position, for the adjoint chain dJ/d(height, width, length).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .terrain import GeoTransform, TerrainEdit

BERM, SWALE, CUT, MOUND = 0, 1, 2, 3
KIND_NAMES = {"berm": BERM, "swale": SWALE, "cut": CUT, "mound": MOUND}


@dataclass
class Primitive:
    kind: int
    cx: float
    cy: float
    length: float
    width: float
    angle_deg: float
    height: float

    def segment(self):
        if self.kind == MOUND:
            return (self.cx, self.cy), (self.cx, self.cy)
        a = self.angle_deg * (math.pi / 180.0)   # f64::to_radians
        s, c = math.sin(a), math.cos(a)
        hl = 0.5 * self.length
        return (self.cx - c * hl, self.cy - s * hl), (self.cx + c * hl, self.cy + s * hl)

    def profile(self, x: float, y: float) -> float:
        (x0, y0), (x1, y1) = self.segment()
        vx, vy = x1 - x0, y1 - y0
        l2 = vx * vx + vy * vy
        t = 0.0
        if l2 > 0.0:
            t = ((x - x0) * vx + (y - y0) * vy) / l2
            t = 0.0 if t < 0.0 else (1.0 if t > 1.0 else t)
        px, py = x0 + t * vx - x, y0 + t * vy - y
        d = math.sqrt(px * px + py * py)
        s = d / (0.5 * self.width)
        if s >= 1.0:
            return 0.0
        if self.kind == CUT:
            if s <= 0.5:
                return 1.0
            u = (s - 0.5) / 0.5
            w = 1.0 - u * u
            return w * w
        w = 1.0 - s * s
        return w * w

    def bbox(self):
        (x0, y0), (x1, y1) = self.segment()
        r = 0.5 * self.width
        return min(x0, x1) - r, min(y0, y1) - r, max(x0, x1) + r, max(y0, y1) + r

    def as_row(self):
        return [float(self.kind), self.cx, self.cy, self.length, self.width, self.angle_deg, self.height]


def quantize(v: float, step: float) -> float:
    """DesignSpace::q (design.rs:259-261)."""
    return round_half_away(v / step) * step if step > 0.0 else v


def round_half_away(x: float) -> float:
    """Rust f64::round: half-way cases away from zero. Rounds |x| through its exact
    fractional part (|x| - floor(|x|) is exact in f64), so no x + 0.5 rounding step can
    carry 0.49999999999999994 up to 1 or an odd integer above 2^52 to the next even one."""
    if not math.isfinite(x):
        return x
    a = abs(x)
    r = math.floor(a)
    if a - r >= 0.5:
        r += 1.0
    return math.copysign(r, x)


def materialize(prims: list[Primitive], geo: GeoTransform, nx: int, ny: int, editable: np.ndarray,
                max_abs_dz: float) -> TerrainEdit:
    """DesignSpace::materialize (design.rs:316-385): 4x4 sub-sample quadrature per cell."""
    e = TerrainEdit()
    c0 = r0 = 1 << 62
    c1 = r1 = 0
    for p in prims:
        if p.height == 0.0:
            continue
        x0, y0, x1, y1 = p.bbox()
        fc0, fr1 = (x0 - geo.origin_x) / geo.dx, (geo.origin_y - y0) / geo.dy
        fc1, fr0 = (x1 - geo.origin_x) / geo.dx, (geo.origin_y - y1) / geo.dy
        a = min(int(max(math.floor(fc0), 0.0)), nx)
        b = min(int(max(math.floor(fr0), 0.0)), ny)
        c = min(int(max(math.ceil(fc1), 0.0)), nx)
        d = min(int(max(math.ceil(fr1), 0.0)), ny)
        if a < c and b < d:
            c0, r0, c1, r1 = min(c0, a), min(r0, b), max(c1, c), max(r1, d)
    if c0 >= c1 or r0 >= r1:
        return e
    w, h = c1 - c0, r1 - r0
    dz = np.zeros(w * h)
    S = 4
    inv = 1.0 / (S * S)
    for r in range(h):
        for c in range(w):
            col, row = c0 + c, r0 + r
            if not editable[row, col]:
                continue
            acc = 0.0
            for p in prims:
                if p.height == 0.0:
                    continue
                s = 0.0
                for sy in range(S):
                    for sx in range(S):
                        x = geo.origin_x + (col + (sx + 0.5) / S) * geo.dx
                        y = geo.origin_y - (row + (sy + 0.5) / S) * geo.dy
                        s += p.profile(x, y)
                acc += p.height * s * inv
            dz[r * w + c] = -max_abs_dz if acc < -max_abs_dz else (max_abs_dz if acc > max_abs_dz else acc)
    a = geo.dx * geo.dy
    for v in dz:
        if v > 0.0:
            e.fill_m3 += v * a
        else:
            e.cut_m3 -= v * a
    e.c0, e.r0, e.w, e.h, e.dz = c0, r0, w, h, dz
    return e


def random_design(rng: np.random.Generator, n_prims: int, box: tuple[float, float, float, float],
                  length=(20.0, 100.0), width=(3.0, 8.0), height=(-0.5, 0.5), quant=(0.01, 0.5, 0.5, 1.0)) -> list[Primitive]:
    """Seeded random quantised primitives: berm when height > 0, swale when < 0."""
    qh, qp, qw, qa = quant
    out = []
    for _ in range(n_prims):
        cx = quantize(rng.uniform(box[0], box[2]), qp)
        cy = quantize(rng.uniform(box[1], box[3]), qp)
        ln = quantize(rng.uniform(*length), qp)
        wd = max(quantize(rng.uniform(*width), qw), 1e-6)
        an = quantize(rng.uniform(0.0, 180.0), qa)
        if an >= 180.0:
            an -= 180.0
        ht = quantize(rng.uniform(*height), qh)
        kind = BERM if ht >= 0.0 else SWALE
        out.append(Primitive(kind, cx, cy, ln, wd, an, ht))
    return out
