"""Chain rule from the device adjoint to design parameters (host side).

itr_gpu_vjp gives dJ/d(face jump) for every face of a design. At fidelity level 1 (signed
faces) a cell's bed is z = z_fine + dz (walls keep z_wall) and every interior jump is the
difference of its two cells' beds (terrain.rs:460-505: dzx[r][i] = z[r][i] - z[r][i-1],
dzy[r][c] = z[r][c] - z[r-1][c]; the domain-edge jumps stay 0), so

    dJ/d(dz[r][c]) = gx[r][c] - gx[r][c+1] + gy[r][c] - gy[r+1][c]   (interior faces only).

dz comes from the design's primitives through DesignSpace::materialize (design.rs:316-385):
a 4x4 sub-sample quadrature of each primitive's profile times its height, clamped to
+-max_abs_dz and masked by the editable area. dJ/d(height, width, length) of a primitive at
fixed quantized centre and angle is the dz gradient contracted with d(dz)/d(theta), plus the
earthwork term's derivative lambda (cut_cost dV_cut + fill_cost dV_fill) (objective.rs:95-128).
d(dz)/d(theta) is the derivative of the quadrature, written out from Primitive::profile
(design.rs:107-134): with s = d / (w / 2) the distance to the segment over the half width,
  ridge P = (1 - s^2)^2           dP/ds = -4 s (1 - s^2)
  cut   P = 1 (s <= 1/2), else (1 - u^2)^2 with u = 2 s - 1,   dP/ds = -8 u (1 - u^2)
  ds/dw = -s / w,   ds/dL = (2 / w) dd/dL,
where dd/dL is 0 beside the segment and (p - e) . de/dL / d beyond an end e, whose end points
move by +-(cos a, sin a) / 2 per unit of length. The profile is C1 in w and L (its derivative
vanishes at s = 1 and is continuous at s = 1/2), so the quadrature's derivative is the sum of
the samples' derivatives; a cell whose dz is clamped to +-max_abs_dz has none.
primitive_gradient_fd keeps the central differences of the f64 materialize as the check.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .design import CUT, MOUND, Primitive, materialize

PARAMS = ("height", "width", "length")
STEPS = {"height": 1e-4, "width": 1e-3, "length": 1e-3}


def dz_gradient(base, gx: np.ndarray, gy: np.ndarray) -> np.ndarray:
    """dJ/d(dz) per cell (ny, nx) from the face-jump gradients (ny, nx+1) and (ny+1, nx)."""
    nx, ny = base.nx, base.ny
    gx = np.asarray(gx, np.float64).reshape(ny, nx + 1).copy()
    gy = np.asarray(gy, np.float64).reshape(ny + 1, nx).copy()
    gx[:, 0] = 0.0; gx[:, nx] = 0.0       # domain-edge jumps do not follow the bed
    gy[0, :] = 0.0; gy[ny, :] = 0.0
    g = gx[:, :nx] - gx[:, 1:] + gy[:ny, :] - gy[1:, :]
    if base.level == 1:
        g[base.fine.wall] = 0.0            # walls keep z_wall
    return g


def _dz_full(prims, geo, nx, ny, editable, max_abs_dz):
    e = materialize(prims, geo, nx, ny, editable, max_abs_dz)
    full = np.zeros((ny, nx))
    if not e.is_empty():
        full[e.r0:e.r0 + e.h, e.c0:e.c0 + e.w] = e.dz.reshape(e.h, e.w)
    return full, e.cut_m3, e.fill_m3


def profile_derivatives(p: Primitive, x: float, y: float):
    """Primitive::profile at (x, y) and its derivatives with respect to width and length."""
    (x0, y0), (x1, y1) = p.segment()
    vx, vy = x1 - x0, y1 - y0
    l2 = vx * vx + vy * vy
    t, end = 0.0, 0
    if l2 > 0.0:
        t = ((x - x0) * vx + (y - y0) * vy) / l2
        if t < 0.0:
            t, end = 0.0, -1
        elif t > 1.0:
            t, end = 1.0, 1
    px, py = x0 + t * vx - x, y0 + t * vy - y
    d = math.sqrt(px * px + py * py)
    half = 0.5 * p.width
    s = d / half
    if s >= 1.0:
        return 0.0, 0.0, 0.0
    if p.kind == CUT:
        if s <= 0.5:
            P, dPds = 1.0, 0.0
        else:
            u = (s - 0.5) / 0.5
            w = 1.0 - u * u
            P, dPds = w * w, -8.0 * u * w
    else:
        w = 1.0 - s * s
        P, dPds = w * w, -4.0 * s * w
    dP_dw = dPds * (-s / p.width)
    dP_dL = 0.0
    if end != 0 and d > 0.0 and p.kind != MOUND and p.length > 0.0:
        ex, ey = vx / (2.0 * p.length), vy / (2.0 * p.length)   # d(end point)/dL at the far end
        dP_dL = dPds * (end * (px * ex + py * ey) / d) / half
    return P, dP_dw, dP_dL


def _prim_box(p: Primitive, geo, nx, ny):
    x0, y0, x1, y1 = p.bbox()
    a = min(int(max(math.floor((x0 - geo.origin_x) / geo.dx), 0.0)), nx)
    b = min(int(max(math.floor((geo.origin_y - y1) / geo.dy), 0.0)), ny)
    c = min(int(max(math.ceil((x1 - geo.origin_x) / geo.dx), 0.0)), nx)
    d = min(int(max(math.ceil((geo.origin_y - y0) / geo.dy), 0.0)), ny)
    return a, b, c, d


def primitive_gradient(base, geo, editable, max_abs_dz: float, prims: list[Primitive], gx: np.ndarray, gy: np.ndarray,
                       objective_def=None) -> np.ndarray:
    """dJ/d(height, width, length) per primitive, shape (len(prims), 3), from the written-out
    derivative of the quadrature. objective_def (an ObjectiveDef) adds the earthwork term;
    without it only the asset term is differentiated."""
    if base.level != 1:
        raise ValueError("the design chain is written for fidelity level 1 (signed faces)")
    nx, ny = base.nx, base.ny
    gdz = dz_gradient(base, gx, gy)
    dz, _, _ = _dz_full(prims, geo, nx, ny, editable, max_abs_dz)
    lam = 0.0 if objective_def is None else objective_def.earth_weight
    cc = 0.0 if objective_def is None else objective_def.cut_cost
    fc = 0.0 if objective_def is None else objective_def.fill_cost
    area = geo.dx * geo.dy
    out = np.zeros((len(prims), len(PARAMS)))
    S = 4
    for i, p in enumerate(prims):
        a, b, c, d = _prim_box(p, geo, nx, ny)
        acc = np.zeros(3)
        for row in range(b, d):
            for col in range(a, c):
                z = dz[row, col]
                if not editable[row, col] or not (-max_abs_dz < z < max_abs_dz):
                    continue
                s0 = s1 = s2 = 0.0
                for sy in range(S):
                    for sx in range(S):
                        x = geo.origin_x + (col + (sx + 0.5) / S) * geo.dx
                        y = geo.origin_y - (row + (sy + 0.5) / S) * geo.dy
                        P, dw, dL = profile_derivatives(p, x, y)
                        s0 += P; s1 += dw; s2 += dL
                ddz = np.array([s0, p.height * s1, p.height * s2]) / (S * S)
                we = area * (fc if z > 0.0 else (-cc if z < 0.0 else 0.5 * (fc - cc)))
                acc += (gdz[row, col] + lam * we) * ddz
        out[i] = acc
    return out


def primitive_gradient_fd(base, geo, editable, max_abs_dz: float, prims: list[Primitive], gx: np.ndarray, gy: np.ndarray,
                          objective_def=None) -> np.ndarray:
    """primitive_gradient by central differences of the f64 materialize (the check)."""
    nx, ny = base.nx, base.ny
    gdz = dz_gradient(base, gx, gy)
    lam = 0.0 if objective_def is None else objective_def.earth_weight
    out = np.zeros((len(prims), len(PARAMS)))
    for i, p in enumerate(prims):
        for k, name in enumerate(PARAMS):
            h = STEPS[name]
            up = [dataclasses.replace(q, **{name: getattr(q, name) + h}) if j == i else q for j, q in enumerate(prims)]
            dn = [dataclasses.replace(q, **{name: getattr(q, name) - h}) if j == i else q for j, q in enumerate(prims)]
            zu, cu, fu = _dz_full(up, geo, nx, ny, editable, max_abs_dz)
            zd, cd, fd = _dz_full(dn, geo, nx, ny, editable, max_abs_dz)
            d = float(np.sum(gdz * (zu - zd))) / (2 * h)
            if lam:
                d += lam * (objective_def.cut_cost * (cu - cd) + objective_def.fill_cost * (fu - fd)) / (2 * h)
            out[i, k] = d
    return out


def face_jumps_f64(base, dz: np.ndarray):
    """Signed face jumps of base + dz in f64 (level 1), the f64 oracle's input for finite
    differences through the design chain."""
    nx, ny = base.nx, base.ny
    z = np.where(base.fine.wall, base.fine.z_wall, base.fine.z + dz).astype(np.float64)
    dzx = np.zeros((ny, nx + 1))
    dzy = np.zeros((ny + 1, nx))
    dzx[:, 1:nx] = z[:, 1:] - z[:, :-1]
    dzy[1:ny, :] = z[1:, :] - z[:-1, :]
    return dzx, dzy
