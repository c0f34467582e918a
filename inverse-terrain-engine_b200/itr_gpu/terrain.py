"""Prepared terrain: the inputs of one batch call, built the way the reference builds them.

Restates crates/itr-hydro/src/terrain.rs (TerrainBase::build :262-321, coarsen/coarse_cell
:336-373, face_x/face_y :375-429, PreparedTerrain::apply_edit :458-505, Boundaries
::from_segments :151-187) and FineTerrain::new (:204-235) in numpy float64, rounding each
face jump to float32 once, so the packed arrays are bit-identical to the reference's rows.
The packed layout is the one lib.rs:177-201 uploads: dzx[r, f] for x-face f (0..nx) of row
r, dzy[f, c] for y-face f (0..ny) of column c, wet/gn2 per cell.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from ._lib import BC_INFLOW, BC_STAGE, BC_TRANSMISSIVE, BC_WALL, FACE_CREST, FACE_SIGNED

G = 9.81  # terrain.rs:259

SIDES = {"north": 0, "south": 1, "west": 2, "east": 3}


@dataclass
class Segment:
    """BoundarySegment (scenario.rs): kind 'stage' | 'inflow' | 'transmissive'."""
    kind: str
    side: str
    range_m: tuple[float, float] | None = None
    stage_m: float = 0.0
    hydrograph: list[tuple[float, float]] = field(default_factory=list)


@dataclass
class GeoTransform:
    origin_x: float
    origin_y: float
    dx: float
    dy: float

    def cell_center(self, col, row):
        return self.origin_x + (col + 0.5) * self.dx, self.origin_y - (row + 0.5) * self.dy


class FineTerrain:
    """FineTerrain::new (terrain.rs:204-235): re-based elevations, walls at z_wall."""

    def __init__(self, dem: np.ndarray, walls: np.ndarray, manning: np.ndarray, geo: GeoTransform):
        dem = np.asarray(dem, dtype=np.float64)
        walls = np.asarray(walls, dtype=bool)
        self.ny, self.nx = dem.shape
        self.geo = geo
        ok = (~walls) & np.isfinite(dem)
        if ok.any():
            zmin, zmax = float(dem[ok].min()), float(dem[ok].max())
        else:
            zmin = zmax = 0.0
        self.z_ref = math.floor(zmin)
        self.z_wall = (zmax - self.z_ref) + 100.0
        self.wall = walls | ~np.isfinite(dem)
        self.z = np.where(self.wall, self.z_wall, dem - self.z_ref)
        self.n = np.asarray(manning, dtype=np.float64) * np.ones_like(dem)


class TerrainBase:
    """TerrainBase<f32>::build (terrain.rs:262-321) for fidelity level `level`."""

    def __init__(self, fine: FineTerrain, level: int = 1, segments: list[Segment] | None = None):
        lv = max(int(level), 1)
        self.fine = fine
        self.level = lv
        self.nx = -(-fine.nx // lv)
        self.ny = -(-fine.ny // lv)
        self.dx = fine.geo.dx * lv
        self.dy = fine.geo.dy * lv
        self.g = G
        self.mode = FACE_SIGNED if lv == 1 else FACE_CREST
        self.z, self.wall, nvals = _coarsen(fine, lv, None)
        self.dzx, self.dzx2, self.dzy, self.dzy2 = _faces(fine, lv, self.mode, self.z, None, None)
        self.wet = np.where(self.wall, 0.0, 1.0).astype(np.float32)
        self.gn2 = (G * nvals * nvals).astype(np.float32)
        self.wet_count = int((~self.wall).sum())
        (self.bc, self.bc_stage, self.hydrographs, self.bc_inflow,
         self.bc_inv_len) = _boundaries(segments or [], self.nx, self.ny, self.dx, self.dy, fine.z_ref)

    @property
    def has_stage(self) -> bool:
        return bool((self.bc == BC_STAGE).any())

    @property
    def has_inflow(self) -> bool:
        return bool((self.bc == BC_INFLOW).any())

    def cell_area(self) -> float:
        return self.dx * self.dy


def _coarse_cell_block(fine, lv, c, r, z):
    """coarse_cell (terrain.rs:357-373) for one block, sequential sums as in the reference."""
    s = 0.0
    sn = 0.0
    sn_all = 0.0
    cnt = 0
    tot = 0
    for rr in range(r * lv, min((r + 1) * lv, fine.ny)):
        for cc in range(c * lv, min((c + 1) * lv, fine.nx)):
            tot += 1
            sn_all += float(fine.n[rr, cc])
            if not fine.wall[rr, cc]:
                s += float(z[rr, cc])
                sn += float(fine.n[rr, cc])
                cnt += 1
    if cnt == 0:
        return fine.z_wall, True, sn_all / tot
    return s / cnt, False, sn / cnt


def _coarsen(fine, lv, zfine):
    z = fine.z if zfine is None else zfine
    if lv == 1:
        zc = np.where(fine.wall, fine.z_wall, z).astype(np.float64)
        return zc, fine.wall.copy(), fine.n.astype(np.float64).copy()
    nx, ny = -(-fine.nx // lv), -(-fine.ny // lv)
    zc = np.zeros((ny, nx))
    wall = np.zeros((ny, nx), dtype=bool)
    nv = np.zeros((ny, nx))
    for r in range(ny):
        for c in range(nx):
            zc[r, c], wall[r, c], nv[r, c] = _coarse_cell_block(fine, lv, c, r, z)
    return zc, wall, nv


def _crest_x(fine, lv, zfine, i, r, zl, zr):
    cl = i * lv - 1
    cr = min(i * lv, fine.nx - 1)
    crest = -math.inf
    all_wall = True
    for rr in range(r * lv, min((r + 1) * lv, fine.ny)):
        for cc in (cl, cr):
            if not fine.wall[rr, cc]:
                all_wall = False
                crest = max(crest, float(zfine[rr, cc]))
    if all_wall:
        crest = fine.z_wall
    zf = max(max(crest, zl), zr)
    return zf - zl, zf - zr


def _crest_y(fine, lv, zfine, c, rb, zt, zb):
    rt_f = rb * lv - 1
    rb_f = min(rb * lv, fine.ny - 1)
    crest = -math.inf
    all_wall = True
    for cc in range(c * lv, min((c + 1) * lv, fine.nx)):
        for rr in (rt_f, rb_f):
            if not fine.wall[rr, cc]:
                all_wall = False
                crest = max(crest, float(zfine[rr, cc]))
    if all_wall:
        crest = fine.z_wall
    zf = max(max(crest, zt), zb)
    return zf - zt, zf - zb


def _faces(fine, lv, mode, zc, zfine, rows_cols):
    """All face jumps of a level (terrain.rs:276-289); float64 differences, one f32 rounding."""
    ny, nx = zc.shape
    dzx = np.zeros((ny, nx + 1), dtype=np.float32)
    dzy = np.zeros((ny + 1, nx), dtype=np.float32)
    dzx2 = np.zeros_like(dzx) if mode == FACE_CREST else None
    dzy2 = np.zeros_like(dzy) if mode == FACE_CREST else None
    if mode == FACE_SIGNED:
        dzx[:, 1:nx] = (zc[:, 1:] - zc[:, :-1]).astype(np.float32)
        dzy[1:ny, :] = (zc[1:, :] - zc[:-1, :]).astype(np.float32)
        return dzx, dzx2, dzy, dzy2
    zf = fine.z if zfine is None else zfine
    for r in range(ny):
        for i in range(1, nx):
            a, b = _crest_x(fine, lv, zf, i, r, float(zc[r, i - 1]), float(zc[r, i]))
            dzx[r, i] = np.float32(a)
            dzx2[r, i] = np.float32(b)
    for j in range(1, ny):
        for c in range(nx):
            a, b = _crest_y(fine, lv, zf, c, j, float(zc[j - 1, c]), float(zc[j, c]))
            dzy[j, c] = np.float32(a)
            dzy2[j, c] = np.float32(b)
    return dzx, dzx2, dzy, dzy2


def edge_values(a: np.ndarray) -> np.ndarray:
    """Values of the interior cells behind the boundary cells, in boundary-code order:
    north row, south row, west column, east column."""
    return np.concatenate([a[0, :], a[-1, :], a[:, 0], a[:, -1]])


def _boundaries(segs, nx, ny, dx, dy, z_ref):
    """Boundaries::from_segments (terrain.rs:151-187) as per-side-cell codes, with each
    stage cell's level above the datum and each inflow cell's hydrograph index and
    1 / segment length (0 for an empty segment)."""
    codes = {s: np.full(nx if s in ("north", "south") else ny, BC_WALL, dtype=np.uint8) for s in SIDES}
    stage = {s: np.zeros(len(codes[s])) for s in SIDES}
    inflow = {s: np.full(len(codes[s]), -1, dtype=np.int64) for s in SIDES}
    inv_len = {s: np.zeros(len(codes[s])) for s in SIDES}
    hydros = []
    for sg in segs:
        n, d = (nx, dx) if sg.side in ("north", "south") else (ny, dy)
        if sg.range_m is not None:
            a = min(int(max(math.floor(sg.range_m[0] / d), 0.0)), n)
            e = min(int(max(math.ceil(sg.range_m[1] / d), 0.0)), n)
        else:
            a, e = 0, n
        if sg.kind == "stage":
            codes[sg.side][a:e] = BC_STAGE
            stage[sg.side][a:e] = sg.stage_m - z_ref
        elif sg.kind == "transmissive":
            codes[sg.side][a:e] = BC_TRANSMISSIVE
        elif sg.kind == "inflow":
            hydros.append(list(sg.hydrograph))
            codes[sg.side][a:e] = BC_INFLOW
            inflow[sg.side][a:e] = len(hydros) - 1
            len_m = (e - a if e > a else 0) * d
            inv_len[sg.side][a:e] = 1.0 / len_m if len_m > 0.0 else 0.0
        else:
            raise ValueError(f"unknown boundary kind {sg.kind}")
    bc = np.concatenate([codes["north"], codes["south"], codes["west"], codes["east"]]).astype(np.uint8)
    st = np.concatenate([stage["north"], stage["south"], stage["west"], stage["east"]])
    inf = np.concatenate([inflow["north"], inflow["south"], inflow["west"], inflow["east"]])
    il = np.concatenate([inv_len["north"], inv_len["south"], inv_len["west"], inv_len["east"]])
    return bc, st, hydros, inf, il


@dataclass
class TerrainEdit:
    """Sparse fine-resolution edit (design.rs:144-178)."""
    c0: int = 0
    r0: int = 0
    w: int = 0
    h: int = 0
    dz: np.ndarray | None = None
    cut_m3: float = 0.0
    fill_m3: float = 0.0

    def is_empty(self) -> bool:
        return self.w == 0 or self.h == 0 or self.dz is None or not np.any(self.dz != 0.0)


class PreparedTerrain:
    """Per-candidate terrain: shared base + private face arrays (terrain.rs:431-505)."""

    def __init__(self, base: TerrainBase):
        self.base = base
        self.dzx = base.dzx.copy()
        self.dzy = base.dzy.copy()
        self.dzx2 = None if base.dzx2 is None else base.dzx2.copy()
        self.dzy2 = None if base.dzy2 is None else base.dzy2.copy()
        self.z = base.z.copy()
        self.cut_m3 = 0.0
        self.fill_m3 = 0.0

    def apply_edit(self, e: TerrainEdit) -> "PreparedTerrain":
        b = self.base
        self.__init__(b)
        self.cut_m3, self.fill_m3 = e.cut_m3, e.fill_m3
        if e.is_empty():
            return self
        lv, nx, ny, fine = b.level, b.nx, b.ny, b.fine
        zfine = fine.z.copy()
        sub = zfine[e.r0:e.r0 + e.h, e.c0:e.c0 + e.w]
        zfine[e.r0:e.r0 + e.h, e.c0:e.c0 + e.w] = sub + e.dz.reshape(e.h, e.w)   # fine_z: z + edit.get
        c0, r0 = e.c0 // lv, e.r0 // lv
        c1 = min(-(-(e.c0 + e.w) // lv), nx)
        r1 = min(-(-(e.r0 + e.h) // lv), ny)
        for r in range(r0, r1):
            for c in range(c0, c1):
                if lv == 1:
                    self.z[r, c] = fine.z_wall if fine.wall[r, c] else zfine[r, c]
                else:
                    self.z[r, c] = _coarse_cell_block(fine, lv, c, r, zfine)[0]
        zc = self.z
        for r in range(r0, r1):
            for cl in range(max(c0 - 1, 0), min(c1, nx - 1)):
                i = cl + 1
                if b.mode == FACE_SIGNED:
                    self.dzx[r, i] = np.float32(zc[r, cl + 1] - zc[r, cl])
                else:
                    a, bb = _crest_x(fine, lv, zfine, i, r, float(zc[r, cl]), float(zc[r, cl + 1]))
                    self.dzx[r, i] = np.float32(a)
                    self.dzx2[r, i] = np.float32(bb)
        for rt in range(max(r0 - 1, 0), min(r1, ny - 1)):
            for c in range(c0, c1):
                if b.mode == FACE_SIGNED:
                    self.dzy[rt + 1, c] = np.float32(zc[rt + 1, c] - zc[rt, c])
                else:
                    a, bb = _crest_y(fine, lv, zfine, c, rt + 1, float(zc[rt, c]), float(zc[rt + 1, c]))
                    self.dzy[rt + 1, c] = np.float32(a)
                    self.dzy2[rt + 1, c] = np.float32(bb)
        return self

    def z_level(self) -> np.ndarray:
        return self.z

    def z_edge(self) -> np.ndarray:
        """z level of the cells behind the boundary cells (itr_design.z_edge)."""
        return edge_values(self.z)

    def initial_depth(self, initial_depth: float, initial_stage: float | None = None) -> np.ndarray:
        """init_state (solver.rs:287-306): depth per cell, 0 on walls."""
        d = np.full(self.z.shape, float(initial_depth))
        if initial_stage is not None:
            d = np.maximum(d, initial_stage - self.base.fine.z_ref - self.z)
        h = np.maximum(d, 0.0).astype(np.float32)
        h[self.base.wall] = 0.0
        return h + np.float32(0.0)   # canon_zero


def synthetic_terrain(nx, ny, dx, zfun, wallfun=None, n=0.03, segments=None, level=1) -> TerrainBase:
    """validation::terrain (validation.rs:43-65): z and walls from functions of the cell centre."""
    geo = GeoTransform(0.0, ny * dx, dx, dx)
    cols, rows = np.meshgrid(np.arange(nx), np.arange(ny))
    x = geo.origin_x + (cols + 0.5) * dx
    y = geo.origin_y - (rows + 0.5) * dx
    dem = np.vectorize(zfun, otypes=[np.float64])(x, y) if not hasattr(zfun, "vectorized") else zfun(x, y)
    walls = np.zeros((ny, nx), dtype=bool) if wallfun is None else np.vectorize(wallfun, otypes=[bool])(cols, rows)
    fine = FineTerrain(dem, walls, np.full((ny, nx), n), geo)
    return TerrainBase(fine, level, segments)
