"""Test helpers: packed inputs of a TerrainBase for the CPU oracle, bitwise comparisons."""
from __future__ import annotations

import numpy as np


def base_arrays(base):
    return (base.nx, base.ny, base.dx, base.dy, base.mode, base.wet, base.gn2, base.bc)


def design_dict(t, params=None):
    h0 = None
    if params is not None and params.initial_stage is not None:
        h0 = t.initial_depth(params.initial_depth, params.initial_stage)
    elif params is not None and params.initial_depth > 0:
        h0 = t.initial_depth(params.initial_depth)
    return dict(dzx=t.dzx, dzy=t.dzy, dzx2=t.dzx2, dzy2=t.dzy2, h0=h0, cut=t.cut_m3, fill=t.fill_m3)


def bits32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32)).view(np.uint32)


def assert_bitwise(a, b, what):
    a32, b32 = bits32(a), bits32(b)
    if not np.array_equal(a32, b32):
        diff = np.flatnonzero(a32.ravel() != b32.ravel())
        k = diff[0]
        raise AssertionError(f"{what}: {len(diff)} values differ; first at {k}: {np.asarray(a).ravel()[k]!r} vs "
                             f"{np.asarray(b).ravel()[k]!r}; max |d| = {np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)))}")
