"""Headless map image (itr_gpu_render_map): the result viewer's fragment shader
(viewer/viewer.js:72-100, colour ramps :55-71) computed on the device. Presentation only.

CPU: the oracle's restatement against values worked out by hand from the shader (flat
hillshade, the depth ramp's ends and middle, no-data grey, hatching). GPU: the device image
against the oracle's on a run's peak depths and a depth difference; f32 log and square root
may round differently, so a channel may differ by one level.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle_ref as orc


def flat_grey():
    l = math.sqrt(0.99)
    return round(255 * (0.3 + 0.6 * (0.7 / l)))


def test_oracle_known_values():
    ny, nx = 4, 6
    z = np.zeros((ny, nx), np.float32)
    v = np.zeros((ny, nx), np.float32)
    v[0, 0] = 2.0                      # D_MAX: the ramp's last colour, #08306b
    v[0, 1] = 0.1                      # sqrt(D_MIN D_MAX): halfway, mix of #6baed6 and #4292c6
    v[0, 2] = 0.004                    # below D_MIN: hillshade only
    z[3, 5] = np.nan                   # no data: grey 0.87
    img = orc.render_map(z, v, 5.0)
    g = flat_grey()
    assert tuple(img[1, 1, :3]) == (g, g, g)
    assert tuple(img[0, 0, :3]) == (round(255 * 0.0314), round(255 * 0.1882), round(255 * 0.4196))
    mid = [round(255 * (0.5 * a + 0.5 * b)) for a, b in zip((0.4196, 0.6824, 0.8392), (0.2588, 0.5725, 0.7765))]
    assert all(abs(int(x) - y) <= 1 for x, y in zip(img[0, 1, :3], mid))
    assert tuple(img[0, 2, :3]) == (g, g, g)
    assert tuple(img[3, 5, :3]) == (round(255 * 0.87),) * 3
    assert np.all(img[..., 3] == 255)
    # difference mode: 0 stays grey, +0.2 the last colour, -0.2 the first
    d = np.zeros((ny, nx), np.float32)
    d[0, 0], d[0, 1] = 0.2, -0.2
    img = orc.render_map(z, d, 5.0, mode=1)
    assert tuple(img[0, 0, :3]) == (round(255 * 0.6980), round(255 * 0.0941), round(255 * 0.1686))
    assert tuple(img[0, 1, :3]) == (round(255 * 0.1294), round(255 * 0.4000), round(255 * 0.6745))
    assert tuple(img[2, 2, :3]) == (g, g, g)
    # hatching of a worsened cell at 2 pixels per cell: the pixel whose (x + y) / 2 has a
    # fractional part below 1/2 is darkened to 30 % (cell (1, 1): pixels 2..3; only (2, 2))
    w = np.zeros((ny, nx), np.float32)
    w[1, 1] = 0.05
    img = orc.render_map(z, v, 5.0, scale=2, worse_dz=w)
    dark = 255 * 0.3 * (0.3 + 0.6 * 0.7 / math.sqrt(0.99))
    assert abs(int(img[2, 2, 0]) - dark) <= 1
    assert img[2, 3, 0] == g and img[3, 2, 0] == g and img[3, 3, 0] == g


@pytest.mark.gpu
@pytest.mark.parametrize("mode,scale", [(0, 1), (0, 3), (1, 2)])
def test_device_image_matches_oracle(mode, scale):
    from itr_gpu import GpuSolver
    from itr_gpu.scenes import valley_scene
    sc = valley_scene(10.0)
    sc.params.duration_s = 1200.0
    ts = [t for _, _, t in sc.designs(2)]
    g = GpuSolver()
    try:
        runs = g.run_batch(sc.params, ts, sc.monitors, want_peak=True)
        z = ts[0].z.astype(np.float32)
        value = runs[0].peak if mode == 0 else runs[1].peak - runs[0].peak
        worse = runs[1].peak - runs[0].peak
        dev = g.render_map(z, value, sc.base.dx, mode=mode, vex=3.0, scale=scale, worse_dz=worse)
    finally:
        g.close()
    ref = orc.render_map(z, value, sc.base.dx, mode=mode, vex=3.0, scale=scale, worse_dz=worse)
    diff = np.abs(dev.astype(int) - ref.astype(int))
    assert diff.max() <= 1, diff.max()
    assert (diff == 0).mean() >= 0.999
    assert len(np.unique(dev.reshape(-1, 4), axis=0)) > 20   # a real picture, not one colour
