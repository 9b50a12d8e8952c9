"""Solve batches (wos_batch_*): every solve of a mixed batch reproduces the
same solve run alone through wos_solve_grid, with and without CUDA-graph
capture: identical locations, counters and per-point step counts (the walks
are the same), statistics equal to 1e-12 relative (the batch kernel may
round the terminal FP64 arithmetic differently); graph replays are
bit-for-bit deterministic; invalid solves and meshes are rejected."""
from __future__ import annotations

import numpy as np
import pytest

from walk_on_spheres_b200 import meshes

pytestmark = pytest.mark.gpu

FIELDS = ("mean", "variance", "standard_error", "mean_steps", "location")


def _specs():
    rng = np.random.default_rng(42)
    star = meshes.star_polygon(rng, 300)
    psph = meshes.perturbed_sphere(rng, 40, 20)
    return [
        (star, "laplace", (23, 19, 1), dict(N_walks=700, seed=1, method="fast")),
        (meshes.circle(segments=256), "poisson", (20, 20, 1),
         dict(N_walks=1500, seed=2, source_mode="green", method="fast")),
        (meshes.annulus(), "screened_poisson", (18, 21, 1),
         dict(N_walks=300, seed=3, alpha=7.0, method="fast64")),
        (star, "helmholtz", (16, 16, 1), dict(N_walks=256, seed=4, method="fast")),
        (meshes.uv_sphere(lon=32, lat=16), "laplace", (9, 8, 7),
         dict(N_walks=1100, seed=5, method="fast")),
        (psph, "screened_poisson", (8, 9, 10), dict(N_walks=400, seed=6, alpha=12.0,
                                                    method="fast")),
        (meshes.uv_sphere(lon=24, lat=12), "poisson", (7, 7, 7),
         dict(N_walks=200, seed=7, source_mode="uniform", method="fast64")),
    ]


def _assert_same(a, b):
    """Bit-for-bit equality (graph replays of one batch)."""
    for k in FIELDS:
        x, y = getattr(a, k), getattr(b, k)
        if k == "location":
            assert np.array_equal(x, y), k
        else:
            assert np.array_equal(x, y, equal_nan=True), k


def _assert_reproduces(a, b):
    """A batched solve against the same solve alone: same walks."""
    assert np.array_equal(a.location, b.location)
    assert np.array_equal(a.mean_steps, b.mean_steps, equal_nan=True)
    for k in ("mean", "variance", "standard_error"):
        x, y = getattr(a, k), getattr(b, k)
        both = np.isnan(x) & np.isnan(y)
        assert not (np.isnan(x) ^ np.isnan(y)).any(), k
        assert np.allclose(x[~both], y[~both], rtol=1e-12, atol=1e-15), k


@pytest.mark.parametrize("use_graph", [False, True], ids=["stream", "graph"])
def test_batch_equals_individual_solves(solver, use_graph):
    from walk_on_spheres_b200.batch import Batch
    specs = _specs()
    b = Batch(solver)
    ids = []
    mesh_ids = {}
    for mesh, eq, (nx, ny, nz), kw in specs:
        key = id(mesh)
        if key not in mesh_ids:
            mesh_ids[key] = b.add_mesh(mesh)
        ids.append(b.add_solve(mesh_ids[key], eq, nx, ny, nz, **kw))
    ms = b.run(use_graph=use_graph)
    assert ms > 0
    info = b.info()
    assert info["solves"] == len(specs)
    walks = 0
    for sid, (mesh, eq, (nx, ny, nz), kw) in zip(ids, specs):
        got = b.result(sid)
        solver.set_mesh(mesh)
        want = solver.solve_grid(eq, nx, ny, nz, **kw)
        _assert_reproduces(got, want)
        for c in ("inside_points", "max_steps_hits", "ambiguous_ray_retries",
                  "indeterminate_points", "total_walks", "total_steps"):
            assert got.counters[c] == want.counters[c], c
        assert np.isclose(got.counters["sum_variance"], want.counters["sum_variance"],
                          rtol=1e-12)
        walks += want.counters["total_walks"]
    assert info["walks"] == walks
    b.close()


def test_graph_replay_is_deterministic_and_tuning_rebuilds(solver):
    from walk_on_spheres_b200.batch import Batch
    specs = _specs()[:5]
    b = Batch(solver)
    ids = []
    for mesh, eq, (nx, ny, nz), kw in specs:
        ids.append(b.add_solve(b.add_mesh(mesh), eq, nx, ny, nz, **kw))
    b.run(use_graph=True)
    first = [b.result(i) for i in ids]
    b.run(use_graph=True)
    for i, r in zip(ids, first):
        _assert_same(b.result(i), r)
    # another chunking re-plans and re-captures; it matches the single solve
    # under the same chunking
    b.set_tuning(chunk=128)
    b.run(use_graph=True)
    solver.set_tuning(chunk=128)
    try:
        for sid, (mesh, eq, (nx, ny, nz), kw) in zip(ids, specs):
            solver.set_mesh(mesh)
            _assert_reproduces(b.result(sid), solver.solve_grid(eq, nx, ny, nz, **kw))
    finally:
        solver.set_tuning(0, 0)
    b.close()


def test_batch_rejects_invalid_solves(solver):
    from walk_on_spheres_b200._lib import WosError
    from walk_on_spheres_b200.batch import Batch
    b = Batch(solver)
    m = b.add_mesh(meshes.annulus())
    with pytest.raises(WosError, match="FAST"):
        b.add_solve(m, "laplace", 8, 8, N_walks=10, method="plain")
    with pytest.raises(WosError, match="unknown mesh"):
        b.add_solve(m + 1, "laplace", 8, 8, N_walks=10, method="fast")
    with pytest.raises(WosError, match="alpha"):
        b.add_solve(m, "screened_poisson", 8, 8, N_walks=10, alpha=0.0, method="fast")
    # meshes are checked when added, with wos_set_mesh's messages
    from walk_on_spheres_b200.meshes import Mesh
    bad = Mesh(2, np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 0.0]]),
               np.array([[0, 1], [1, 2], [2, 0]], dtype=np.int32), np.zeros(3, dtype=np.int32))
    with pytest.raises(WosError, match="zero-length line segment"):
        b.add_mesh(bad)
    # prepare() builds the new meshes (in parallel) before the first run; the
    # solve then matches the same solve alone
    sid = b.add_solve(m, "laplace", 9, 9, N_walks=64, seed=3, method="fast")
    b.prepare()
    b.run(use_graph=False)
    solver.set_mesh(meshes.annulus())
    _assert_reproduces(b.result(sid), solver.solve_grid("laplace", 9, 9, N_walks=64, seed=3,
                                                        method="fast"))
    # an empty batch runs
    b2 = Batch(solver)
    b2.run(use_graph=True)
    assert b2.info()["solves"] == 0
    b.close()
    b2.close()
