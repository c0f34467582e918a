"""Chain rule from the device adjoint to design parameters (host side).

itr_gpu_vjp gives dJ/d(face jump) for every face of a design. At fidelity level 1 (signed
faces) a cell's bed is z = z_fine + dz (walls keep z_wall) and every interior jump is the
difference of its two cells' beds (terrain.rs:460-505: dzx[r][i] = z[r][i] - z[r][i-1],
dzy[r][c] = z[r][c] - z[r-1][c]; the domain-edge jumps stay 0), so

    dJ/d(dz[r][c]) = gx[r][c] - gx[r][c+1] + gy[r][c] - gy[r+1][c]   (interior faces only).

dz comes from the design's primitives through DesignSpace::materialize (design.rs:316-385):
a 4x4 sub-sample quadrature of each primitive's profile times its height, clamped to
+-max_abs_dz and masked by the editable area. dJ/d(height, width, length) of a primitive at
fixed quantized centre and angle is the dz gradient contracted with d(dz)/d(theta), taken
by central differences of the f64 materialize (it is linear in height, and the (1 - s^2)^2
profile is C1 in width and length), plus the earthwork term's derivative
lambda (cut_cost dV_cut + fill_cost dV_fill) (objective.rs:95-128).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .design import Primitive, materialize

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


def primitive_gradient(base, geo, editable, max_abs_dz: float, prims: list[Primitive], gx: np.ndarray, gy: np.ndarray,
                       objective_def=None) -> np.ndarray:
    """dJ/d(height, width, length) per primitive, shape (len(prims), 3). objective_def (an
    ObjectiveDef) adds the earthwork term; without it only the asset term is differentiated."""
    if base.level != 1:
        raise ValueError("the design chain is written for fidelity level 1 (signed faces)")
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
