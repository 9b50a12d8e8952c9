"""FAST_FP32 start radii (kernels.h FastStart): away from the boundary a FAST
solve starts its walks from a conservative FP32 bound of the distance
instead of the exact FP64 query; where the exact value decides something
(the boundary class, a start inside the epsilon shell) it still takes the
exact query.  So a FAST solve classifies every point exactly as the
PLAIN_FP64 solve does, and its walks that start inside the shell return the
same boundary value at the same nearest point."""
from __future__ import annotations

import numpy as np
import pytest

from walk_on_spheres_b200 import meshes

pytestmark = pytest.mark.gpu


def _near_boundary_points(rng, dim, n, eps):
    """Points at radius 1 +- up to 3 eps (the unit circle / sphere meshes),
    so many start inside the epsilon shell and many just outside it, plus
    points spread over the interior."""
    d = rng.normal(size=(n, dim))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    radial = 1.0 + rng.choice([-1.0, 1.0], size=n) * rng.uniform(0.0, 3.0 * eps, size=n)
    inner = rng.normal(size=(n // 4, dim))
    inner *= (rng.uniform(0.0, 0.95, size=(n // 4, 1)) /
              np.linalg.norm(inner, axis=1, keepdims=True))
    return np.vstack([d * radial[:, None], inner])


@pytest.mark.parametrize("mname", ["circle1024", "sphere"])
def test_fast_start_keeps_locations_and_shell_starts(solver, mname):
    m = meshes.circle(segments=1024) if mname == "circle1024" else meshes.uv_sphere()
    solver.set_mesh(m)
    eps = 1e-2
    rng = np.random.default_rng(31)
    pts = _near_boundary_points(rng, m.dim, 4000, eps)
    kw = dict(N_walks=64, epsilon=eps, seed=11)
    fast = solver.solve_points("laplace", pts, method="fast", **kw)
    plain = solver.solve_points("laplace", pts, method="plain", **kw)
    assert np.array_equal(fast.location, plain.location)
    exact, _, _ = solver.closest_points(pts, precision=64)
    ins = fast.location == 1
    shell = ins & (exact <= eps)
    assert shell.sum() > 300 and (ins & (exact > eps) & (exact < 3 * eps)).sum() > 300
    # a start inside the shell takes no step and returns g at the exact
    # nearest point, in both methods (each kernel evaluates g in its own FP64
    # rounding: the fast kernels may fuse multiply-adds, the exact ones not)
    assert np.allclose(fast.mean[shell], plain.mean[shell], rtol=1e-12, atol=1e-14)
    assert np.all(fast.variance[shell] == 0.0)
    assert np.all(fast.mean_steps[shell] == 0) and np.all(plain.mean_steps[shell] == 0)
    # every other inside point walks
    assert np.all(fast.mean_steps[ins & ~shell] >= 1)
