"""GPU results against closed-form FP64 solutions.

Stated error: |mean - u| <= 5 SE + eps * max|grad u| + h, where the second
term bounds the bias of stopping at distance <= eps and evaluating g at the
nearest boundary point, and h (1e-6) covers the polygon-vs-circle geometry
error (O(1/n^2) for n segments).

* Annulus 0.5 < r < 1 (2 x 128 segments), g = x^2 - y^2 on the outer loop
  (boundary_id 0) and 0 on the inner loop (src/equations/laplace.cpp:16-18):
  u = (16/15 r^2 - 1/(15 r^2)) cos 2 theta, max|grad u| <= 2.2.
* Unit disk (1024 segments), f = 0.1 on r <= a = 0.15, g = 0
  (src/equations/poisson.cpp:22-51):
  u = f/4 (a^2 - r^2) + f a^2/2 ln(1/a) for r <= a, f a^2/2 ln(1/r) outside;
  max|grad u| = f a / 2 = 0.0075.
"""
from __future__ import annotations

import numpy as np
import pytest

from walk_on_spheres_b200 import meshes

pytestmark = pytest.mark.gpu


def grid_points(solver, n):
    b = solver.bbox
    xs = np.array([b[0] + (b[1] - b[0]) * i / (n - 1) for i in range(n)])
    ys = np.array([b[2] + (b[3] - b[2]) * j / (n - 1) for j in range(n)])
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    return X, Y


def annulus_u(X, Y):
    r2 = X * X + Y * Y
    return (16.0 / 15.0 * r2 - 1.0 / (15.0 * r2)) * (X * X - Y * Y) / r2


def disk_u(X, Y, f=0.1, a=0.15):
    r = np.hypot(X, Y)
    inner = f / 4 * (a * a - r * r) + f * a * a / 2 * np.log(1 / a)
    outer = f * a * a / 2 * np.log(1 / np.maximum(r, 1e-300))
    return np.where(r <= a, inner, outer)


@pytest.mark.parametrize("method,walks", [("plain", 4000), ("fast", 40000), ("fast64", 20000)])
def test_annulus_laplace(solver, method, walks):
    solver.set_mesh(meshes.annulus())
    n = 32
    r = solver.solve_grid("laplace", n, n, N_walks=walks, seed=12345, method=method)
    X, Y = grid_points(solver, n)
    u = annulus_u(X, Y)
    ins = r.location[:, :, 0] == 1
    err = np.abs(r.mean[:, :, 0] - u)[ins]
    bound = 5 * r.standard_error[:, :, 0][ins] + 1e-2 * 2.2 + 1e-6
    assert (err <= bound).all(), (err - bound).max()
    # the bias is mostly sub-epsilon: the mean error is small
    assert abs((r.mean[:, :, 0] - u)[ins].mean()) < 2e-3


@pytest.mark.parametrize("mode", ["green", "uniform"])
@pytest.mark.parametrize("method", ["fast", "plain"])
def test_disk_poisson(solver, mode, method):
    solver.set_mesh(meshes.circle(segments=1024))
    n = 24
    walks = 4000 if method == "plain" else 40000
    r = solver.solve_grid("poisson", n, n, N_walks=walks, seed=7, source_mode=mode,
                          method=method)
    X, Y = grid_points(solver, n)
    u = disk_u(X, Y)
    ins = r.location[:, :, 0] == 1
    err = np.abs(r.mean[:, :, 0] - u)[ins]
    bound = 5 * r.standard_error[:, :, 0][ins] + 1e-2 * 0.0075 + 1e-6
    ok = err <= bound
    # uniform-ball sampling of a small source has heavy tails (rare large
    # Green values), so its standard-error estimate is loose at a few points
    assert ok.mean() >= (0.999 if mode == "green" else 0.98), ok.mean()
    assert np.median(err / np.maximum(r.standard_error[:, :, 0][ins], 1e-30)) < 1.5
