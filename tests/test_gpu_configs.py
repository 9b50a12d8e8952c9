"""GPU parity at the benchmark configurations' full sizes, against the
reference's own code (oracle/_ref: the reference sources compiled where they
lie, run here on every host core with the reference's per-point loop of
include/wos/runner.hpp:157-236).

* annulus Laplace: the whole 64 x 64 grid, 10 000 walks, eps 1e-2,
  seed 12345 (the reference defaults, src/main.cpp:95-97);
* disk Poisson: the 256 x 256 grid, 4096 walks, uniform and Green source
  sampling; the walks are compared on a seeded sample of 2000 grid points,
  the location codes on the whole grid;
* screened sphere: alpha 10 on the 16 128-triangle UV sphere, the 64^3 grid,
  1024 walks, seed 7; walks on a seeded sample of 1200 grid points,
  location codes on the whole grid.

Tolerances:
* location codes and the inside / ray counters: bit-exact;
* PLAIN_FP64 (the reference's streams): >= 98% of inside points to 1e-9
  relative, every point within 4 standard errors;
* FAST_FP32 / FAST_FP64 (other streams): >= 99% of points within 3 combined
  standard errors, the mean |z| at most 1 (1 SE on average; 0.80 is the
  expectation), and the mean z within 4/sqrt(n) of zero (no bias);
* closed-form solutions: |mean - u| <= 5 SE + eps max|grad u| + 1e-6.
"""
from __future__ import annotations

import numpy as np
import pytest

from walk_on_spheres_b200 import meshes
from walk_on_spheres_b200.parallel import grid_coords

pytestmark = pytest.mark.gpu


def _plain_bar(mean, se, ref_mean, ref_se):
    close = np.abs(mean - ref_mean) <= 1e-9 * np.maximum(1.0, np.abs(ref_mean))
    assert close.mean() >= 0.98, close.mean()
    far = ~close
    if far.any():
        z = np.abs(mean[far] - ref_mean[far]) / np.maximum(ref_se[far], 1e-300)
        assert (z <= 4.0).all(), z.max()


def _fast_bar(mean, se, ref_mean, ref_se):
    s = np.hypot(se, ref_se)
    live = s > 0
    z = (mean[live] - ref_mean[live]) / s[live]
    assert (np.abs(z) <= 3.0).mean() >= 0.99, (np.abs(z) > 3).mean()
    assert np.abs(z).mean() <= 1.0, np.abs(z).mean()
    assert abs(z.mean()) <= 4.0 / np.sqrt(z.size), z.mean()
    assert np.allclose(mean[~live], ref_mean[~live], rtol=1e-5, atol=1e-12)


def _sample(n_grid, k, seed):
    return np.sort(np.random.default_rng(seed).choice(n_grid, size=k, replace=False))


# ------------------------------------------------------------------ annulus


@pytest.fixture(scope="module")
def annulus_ref(reference):
    from oracle.oracle import Solve
    return reference.solve_grid("laplace", Solve(meshes.annulus(), 64, 64, N_walks=10000,
                                                 epsilon=1e-2, seed=12345))


def _annulus_u(x, y):
    r2 = x * x + y * y
    return (16.0 / 15.0 * r2 - 1.0 / (15.0 * r2)) * (x * x - y * y) / r2


@pytest.mark.parametrize("method", ["plain", "fast", "fast64"])
def test_annulus_64sq_10000_walks(solver, annulus_ref, method):
    solver.set_mesh(meshes.annulus())
    r = solver.solve_grid("laplace", 64, 64, N_walks=10000, epsilon=1e-2, seed=12345,
                          method=method)
    ref = annulus_ref
    loc = r.location.ravel()
    assert np.array_equal(loc, ref.location)
    ins = loc == 1
    assert r.counters["inside_points"] == ref.counters["inside_points"]
    mean, se = r.mean.ravel()[ins], r.standard_error.ravel()[ins]
    if method == "plain":
        assert r.counters["max_steps_hits"] == ref.counters["max_steps_hits"]
        _plain_bar(mean, se, ref.mean[ins], ref.standard_error[ins])
    else:
        _fast_bar(mean, se, ref.mean[ins], ref.standard_error[ins])
    bnd = loc == 2
    assert np.allclose(r.mean.ravel()[bnd], ref.mean[bnd], rtol=1e-13, atol=1e-15)
    # the closed-form harmonic solution (outer loop written first: g = x^2 - y^2 on r = 1)
    xy = grid_coords(solver.grid_over_mesh(64, 64), 2, np.flatnonzero(ins))
    u = _annulus_u(xy[:, 0], xy[:, 1])
    assert (np.abs(mean - u) <= 5 * se + 1e-2 * 2.2 + 1e-6).all()


# --------------------------------------------------------------------- disk


@pytest.fixture(scope="module")
def disk_ref(reference):
    from oracle.oracle import Solve
    mesh = meshes.circle(segments=1024)
    pts = _sample(256 * 256, 2000, 256)
    out = {"points": pts}
    for mode in (0, 1):
        out[mode] = reference.solve_grid("poisson", Solve(mesh, 256, 256, N_walks=4096,
                                                          epsilon=1e-2, seed=12345,
                                                          source_mode=mode, points=pts))
    # location codes of the whole grid (one walk per point)
    out["location"] = reference.solve_grid("poisson", Solve(mesh, 256, 256, N_walks=1,
                                                            seed=12345)).location
    return out


def _disk_u(x, y, f=0.1, a=0.15):
    r = np.hypot(x, y)
    return np.where(r <= a, f / 4 * (a * a - r * r) + f * a * a / 2 * np.log(1 / a),
                    f * a * a / 2 * np.log(1 / np.maximum(r, 1e-300)))


@pytest.mark.parametrize("mode", ["uniform", "green"])
@pytest.mark.parametrize("method", ["plain", "fast"])
def test_disk_256sq_4096_walks(solver, disk_ref, method, mode):
    solver.set_mesh(meshes.circle(segments=1024))
    grid = solver.grid_over_mesh(256, 256)
    pts = disk_ref["points"]
    ref = disk_ref[0 if mode == "uniform" else 1]
    kw = dict(N_walks=4096, epsilon=1e-2, seed=12345, source_mode=mode, method=method)
    if method == "plain":
        # the reference estimator on the sampled points, seeded by their grid index
        r = solver.solve_points("poisson", grid_coords(grid, 2, pts),
                                point_index=pts.astype(np.uint64), **kw)
        loc, mean, se = r.location, r.mean, r.standard_error
    else:
        r = solver.solve_grid("poisson", 256, 256, **kw)
        assert np.array_equal(r.location.ravel(), disk_ref["location"])
        loc = r.location.ravel()[pts]
        mean, se = r.mean.ravel()[pts], r.standard_error.ravel()[pts]
    assert np.array_equal(loc, ref.location[pts])
    ins = loc == 1
    rm, rs = ref.mean[pts][ins], ref.standard_error[pts][ins]
    if method == "plain":
        _plain_bar(mean[ins], se[ins], rm, rs)
    else:
        _fast_bar(mean[ins], se[ins], rm, rs)
    xy = grid_coords(grid, 2, pts[ins])
    err = np.abs(mean[ins] - _disk_u(xy[:, 0], xy[:, 1]))
    ok = err <= 5 * se[ins] + 1e-2 * 0.0075 + 1e-6
    # uniform-ball samples of the small source have heavy tails
    assert ok.mean() >= (0.999 if mode == "green" else 0.98), ok.mean()


# ------------------------------------------------------------------- sphere


@pytest.fixture(scope="module")
def sphere_ref(reference):
    from oracle.oracle import Solve
    mesh = meshes.uv_sphere()
    pts = _sample(64 ** 3, 1200, 64)
    out = {"points": pts}
    out["walks"] = reference.solve_grid("screened_poisson", Solve(
        mesh, 64, 64, 64, N_walks=1024, epsilon=1e-2, seed=7, alpha=10.0, points=pts))
    out["classes"] = reference.solve_grid("screened_poisson", Solve(
        mesh, 64, 64, 64, N_walks=1, epsilon=1e-2, seed=7, alpha=10.0))
    return out


@pytest.mark.parametrize("method,leaf", [("plain", 4), ("plain", 2), ("fast", 4),
                                         ("fast", 8), ("fast64", 4)])
def test_screened_sphere_64cube_1024_walks(solver, sphere_ref, method, leaf):
    solver.set_mesh(meshes.uv_sphere(), leaf_size=leaf)
    grid = solver.grid_over_mesh(64, 64, 64)
    pts = sphere_ref["points"]
    ref = sphere_ref["walks"]
    kw = dict(N_walks=1024, epsilon=1e-2, seed=7, alpha=10.0, method=method)
    if method == "plain":
        r = solver.solve_points("screened_poisson", grid_coords(grid, 3, pts),
                                point_index=pts.astype(np.uint64), **kw)
        loc, mean, se = r.location, r.mean, r.standard_error
    else:
        r = solver.solve_grid("screened_poisson", 64, 64, 64, **kw)
        cls = sphere_ref["classes"]
        # whole-grid classification: codes and the reference's ray counters
        assert np.array_equal(r.location.ravel(), cls.location)
        assert r.counters["ambiguous_ray_retries"] == cls.counters["ambiguous_ray_retries"]
        assert r.counters["indeterminate_points"] == cls.counters["indeterminate_points"]
        assert r.counters["effective_epsilon"] == 0.005  # min(eps, 0.05 / alpha)
        loc = r.location.ravel()[pts]
        mean, se = r.mean.ravel()[pts], r.standard_error.ravel()[pts]
    assert np.array_equal(loc, ref.location[pts])
    ins = loc == 1
    assert ins.sum() > 500
    if method == "plain":
        _plain_bar(mean[ins], se[ins], ref.mean[pts][ins], ref.standard_error[pts][ins])
    else:
        _fast_bar(mean[ins], se[ins], ref.mean[pts][ins], ref.standard_error[pts][ins])
