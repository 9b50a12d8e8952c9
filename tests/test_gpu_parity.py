"""GPU parity: libwos_b200 (through its C ABI) against the reference's golden
vectors and the plain-C oracle.

Tolerances:
* PRNG streams, FP64 closest-point distances, location codes and ray
  counters: bit-exact.
* PLAIN_FP64 means / variances / mean steps: the device runs the reference's
  streams in the reference's order, so results differ only through the last
  bits of CUDA's versus glibc's sin/cos/log/exp; at least 98% of inside
  points must agree to 1e-9 relative and every point within 4 standard
  errors.
* FAST_FP32 / FAST_FP64 use other (counter-based) streams: per-point means
  within 4.5 combined standard errors for >= 99% of points, and the mean of
  the standardised differences within 4/sqrt(n) of zero.
"""
from __future__ import annotations

import numpy as np
import pytest

from tests.golden.make_golden import GRID_CASES
from tests.helpers import mesh_by_name

pytestmark = pytest.mark.gpu


def test_device_prng_bit_exact(solver, golden):
    got = solver.prng_u64(golden["prng_seeds"], golden["prng_u64"].shape[1])
    assert np.array_equal(got, golden["prng_u64"])


@pytest.mark.parametrize("mname", ["annulus", "sphere"])
def test_closest_points_fp64_bit_exact(solver, golden, mname):
    m = mesh_by_name(mname)
    solver.set_mesh(m)
    d, near, bid = solver.closest_points(golden[f"npq_{mname}_points"], precision=64)
    assert np.array_equal(d, golden[f"npq_{mname}_dist"])
    assert np.abs(near - golden[f"npq_{mname}_nearest"]).max() <= 4e-16
    if m.dim == 2:
        assert np.array_equal(bid, golden[f"npq_{mname}_bid"])


@pytest.mark.parametrize("mname", ["annulus", "sphere"])
def test_closest_points_fp32(solver, golden, mname):
    m = mesh_by_name(mname)
    solver.set_mesh(m)
    d, near, _ = solver.closest_points(golden[f"npq_{mname}_points"], precision=32)
    assert np.abs(d - golden[f"npq_{mname}_dist"]).max() <= 2e-6


def _solve(solver, case, method, walks=None):
    name, eq, mname, (nx, ny, nz), n_walks, seed, extra = case
    solver.set_mesh(mesh_by_name(mname))
    return solver.solve_grid(eq, nx, ny, nz, N_walks=walks or n_walks, seed=seed, method=method,
                             **extra)


@pytest.mark.parametrize("case", GRID_CASES, ids=[c[0] for c in GRID_CASES])
def test_plain_fp64_matches_reference(solver, golden, case):
    name = case[0]
    res = _solve(solver, case, "plain")
    pre = f"grid_{name}_"
    loc = golden[pre + "location"].reshape(res.location.shape)
    assert np.array_equal(res.location, loc)
    ins = loc == 1
    c = golden[pre + "counters"]
    assert res.counters["inside_points"] == c[0]
    assert res.counters["max_steps_hits"] == c[1]
    assert res.counters["ambiguous_ray_retries"] == c[2]
    assert res.counters["indeterminate_points"] == c[3]
    mean = golden[pre + "mean"].reshape(loc.shape)
    se = golden[pre + "standard_error"].reshape(loc.shape)
    if ins.any():
        got = res.mean[ins]
        close = np.abs(got - mean[ins]) <= 1e-9 * np.maximum(1.0, np.abs(mean[ins]))
        assert close.mean() >= 0.98, close.mean()
        far = ~close
        if far.any():
            z = np.abs(got[far] - mean[ins][far]) / np.maximum(se[ins][far], 1e-300)
            assert (z <= 4.0).all(), z.max()
        steps = golden[pre + "mean_steps"].reshape(loc.shape)
        assert (np.abs(res.mean_steps[ins] - steps[ins]) <= 1e-9 * steps[ins]).mean() >= 0.98
        if res.counters["total_walks"] == res.counters["inside_points"]:
            # one walk per point: the variance is 0, as the reference defines it
            assert np.all(res.variance[ins] == 0.0)
    # boundary / outside points
    bnd = loc == 2
    assert np.allclose(res.mean[bnd], mean[bnd], rtol=1e-13, atol=1e-15)
    out = (loc == 0) | (loc == 3)
    assert np.isnan(res.mean[out]).all()


@pytest.mark.parametrize("method", ["fast", "fast64"])
@pytest.mark.parametrize("case", [c for c in GRID_CASES if c[0] in (
    "annulus_laplace", "circle_poisson_uniform", "circle_poisson_green",
    "annulus_screened_uniform", "annulus_screened_green", "circle_helmholtz",
    "sphere_laplace", "sphere_screened", "sphere_poisson")], ids=lambda c: c[0])
def test_fast_statistically_equal(solver, oracle, case, method):
    from oracle.oracle import Solve
    name, eq, mname, (nx, ny, nz), _, seed, extra = case
    walks = 2000
    res = _solve(solver, case, method, walks=walks)
    ref = oracle.solve_grid(eq, Solve(mesh_by_name(mname), nx, ny, nz, N_walks=walks, seed=seed,
                                      **extra))
    loc = ref.location.reshape(res.location.shape)
    assert np.array_equal(res.location, loc)
    ins = loc == 1
    m_o = ref.mean.reshape(loc.shape)[ins]
    s_o = ref.standard_error.reshape(loc.shape)[ins]
    m_f, s_f = res.mean[ins], res.standard_error[ins]
    scale = np.sqrt(s_o ** 2 + s_f ** 2)
    live = scale > 0
    z = (m_f[live] - m_o[live]) / scale[live]
    assert (np.abs(z) <= 4.5).mean() >= 0.99, np.abs(z).max()
    assert abs(z.mean()) <= 4.0 / np.sqrt(max(1, z.size)), z.mean()
    # no standard error where the oracle has none (constant walks)
    assert np.all(np.abs(m_f[~live] - m_o[~live]) <= 1e-5 * np.maximum(1.0, np.abs(m_o[~live])))
    # walk lengths: FAST_FP64 takes the oracle's balls (mean steps within 5%);
    # FAST_FP32 may take lattice-bound balls, at least 1/2 of the upper bound
    # of the distance, so its walks are longer, but never shorter
    st_o = ref.mean_steps.reshape(loc.shape)[ins].mean()
    ratio = res.mean_steps[ins].mean() / st_o
    if method == "fast64":
        assert abs(ratio - 1.0) <= 0.05, ratio
    else:
        assert 0.95 <= ratio <= 1.6, ratio


def test_solve_points_matches_grid(solver):
    m = mesh_by_name("annulus")
    solver.set_mesh(m)
    g = solver.solve_grid("laplace", 12, 12, N_walks=300, seed=77, method="plain")
    box = solver.bbox
    xs = np.linspace(box[0], box[1], 12)
    ys = np.linspace(box[2], box[3], 12)
    # the grid formula min + (max-min)*i/(N-1), evaluated as the reference does
    xs = np.array([box[0] + (box[1] - box[0]) * i / 11 for i in range(12)])
    ys = np.array([box[2] + (box[3] - box[2]) * j / 11 for j in range(12)])
    pts = np.array([(x, y) for x in xs for y in ys])
    r = solver.solve_points("laplace", pts, point_index=np.arange(144, dtype=np.uint64),
                            N_walks=300, seed=77, method="plain")
    assert np.array_equal(r.location, g.location.ravel())
    ins = r.location == 1
    assert np.array_equal(r.mean[ins], g.mean.ravel()[ins])


def test_solve_points_rejects_non_finite_points(solver):
    """A NaN or infinite start point (or heat probe) is refused on the host
    with a clear message, before anything reaches the device."""
    from walk_on_spheres_b200._lib import WosError
    from walk_on_spheres_b200.heat import HeatProblem
    solver.set_mesh(mesh_by_name("annulus"))
    for bad in (np.nan, np.inf):
        pts = np.array([[0.5, 0.0], [bad, 0.1]])
        with pytest.raises(WosError, match="point coordinates must be finite"):
            solver.solve_points("laplace", pts, N_walks=16, method="fast")
        with pytest.raises(WosError, match="probe coordinates must be finite"):
            HeatProblem(solver, pts, N_walks=16).forward(1.0, (0.5, 0.0), 0.1)
    # the context stays usable
    r = solver.solve_points("laplace", np.array([[0.5, 0.0]]), N_walks=16, method="fast")
    assert r.location[0] in (0, 1, 2)


def test_sharded_solver_matches_grid(solver):
    """The per-shard GPU solver (walk_on_spheres_b200.parallel) reproduces the
    grid sweep point for point: same coordinates, same global-index seeds."""
    import os
    import socket
    import torch.distributed as dist
    from walk_on_spheres_b200 import parallel
    solver.set_mesh(mesh_by_name("annulus"))
    grid = solver.grid_over_mesh(20, 18, 1)
    g = solver.solve_grid("laplace", grid=grid, N_walks=200, seed=3, method="fast")
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        out = parallel.solve_grid_sharded(
            parallel.gpu_shard_solver(solver, "laplace", grid, N_walks=200, seed=3, method="fast"),
            parallel.grid_size(grid, 2))
    finally:
        dist.destroy_process_group()
    assert np.array_equal(out["location"], g.location.ravel())
    ins = out["location"] == 1
    assert np.allclose(out["mean"][ins], g.mean.ravel()[ins], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("method", ["fast", "fast64"])
def test_fast_edge_cases(solver, golden, method):
    """The FAST methods on the reference's edge cases: a grid row with no
    inside point (nothing to walk, boundary values exact), one walk per point
    (variance 0, as the reference defines it), and walks cut at max_steps
    (hits counted, no walk longer than the cap)."""
    by = {c[0]: c for c in GRID_CASES}
    pre = "grid_annulus_laplace_row_"
    r = _solve(solver, by["annulus_laplace_row"], method)
    loc = golden[pre + "location"].reshape(r.location.shape)
    assert np.array_equal(r.location, loc)
    assert r.counters["inside_points"] == 0 and r.counters["total_walks"] == 0
    bnd = loc == 2
    assert bnd.any()
    assert np.allclose(r.mean[bnd], golden[pre + "mean"].reshape(loc.shape)[bnd],
                       rtol=1e-13, atol=1e-15)
    assert np.isnan(r.mean[loc == 0]).all()

    r = _solve(solver, by["circle_poisson_one_walk"], method)
    ins = r.location == 1
    assert ins.sum() == golden["grid_circle_poisson_one_walk_counters"][0]
    assert np.all(r.variance[ins] == 0.0) and np.all(r.standard_error[ins] == 0.0)
    assert np.all(np.isfinite(r.mean[ins]))

    for name, cap in (("annulus_laplace_max_steps", 3), ("sphere_laplace_max_steps", 2)):
        r = _solve(solver, by[name], method)
        ins = r.location == 1
        assert r.counters["max_steps_hits"] > 0
        assert np.all(r.mean_steps[ins] <= cap) and np.all(np.isfinite(r.mean[ins]))
