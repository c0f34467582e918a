"""The design chain of the adjoint on the CPU: the written-out derivative of
Primitive::profile and of DesignSpace::materialize's quadrature (crates/itr-core/src/
design.rs:107-134, 316-385) against central differences of the f64 reference restatement.

* profile_derivatives: d(profile)/d(width) and d(profile)/d(length) at random points around
  a berm, a cut (flat bottom then a bank) and a mound, against central differences with a
  1e-6 m step;
* primitive_gradient (the host mirror of the device's k_mat_dgrad) against
  primitive_gradient_fd (central differences of the whole f64 materialize, the host chain
  this replaced) on seeded valley designs with random face-jump gradients and the earthwork
  term: within 1e-3 relative (the finite differences' own truncation error near the profile's
  support edge), identical in height (the quadrature is linear in it).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from itr_gpu.adjoint import primitive_gradient, primitive_gradient_fd, profile_derivatives
from itr_gpu.design import BERM, CUT, MOUND, Primitive
from itr_gpu.scenes import valley_scene


@pytest.mark.parametrize("kind", [BERM, CUT, MOUND])
def test_profile_derivatives_vs_central_differences(kind):
    rng = np.random.default_rng(11 + kind)
    p = Primitive(kind, 100.0, 80.0, 40.0, 6.0, 30.0, 0.4)
    h = 1e-6
    worst = 0.0
    for _ in range(400):
        x, y = 100.0 + rng.uniform(-30.0, 30.0), 80.0 + rng.uniform(-15.0, 15.0)
        P, dw, dl = profile_derivatives(p, x, y)
        assert P == p.profile(x, y)
        fw = (dataclasses.replace(p, width=p.width + h).profile(x, y) - dataclasses.replace(p, width=p.width - h).profile(x, y)) / (2 * h)
        fl = (dataclasses.replace(p, length=p.length + h).profile(x, y) - dataclasses.replace(p, length=p.length - h).profile(x, y)) / (2 * h)
        worst = max(worst, abs(fw - dw), abs(fl - dl))
    assert worst < 1e-7, worst


def test_primitive_gradient_vs_materialize_central_differences():
    sc = valley_scene(10.0)
    rng = np.random.default_rng(5)
    nx, ny = sc.base.nx, sc.base.ny
    for prims, _, _ in sc.designs(4):
        gx = rng.normal(size=(ny, nx + 1))
        gy = rng.normal(size=(ny + 1, nx))
        a = primitive_gradient(sc.base, sc.geo, sc.editable, 1.0, prims, gx, gy, sc.objective.d)
        b = primitive_gradient_fd(sc.base, sc.geo, sc.editable, 1.0, prims, gx, gy, sc.objective.d)
        scale = np.maximum(np.abs(b), 1e-2 * np.max(np.abs(b)))
        assert np.max(np.abs(a - b) / scale) < 1e-3, (a, b)
        np.testing.assert_allclose(a[:, 0], b[:, 0], rtol=1e-7)
