"""GPU heat source and its adjoint (kernels_adjoint.cu through the C ABI).

Source modes: uniform, Green and Green-source MIS.

Tolerances:
* replay: the adjoint's replayed probe values equal the forward's bit for
  bit (same kernel, same seeds).
* CRN central differences of the forward (h = 1e-4 relative per parameter)
  against the adjoint's per-probe derivatives: relative 1e-4 of the largest
  derivative (truncation only: the walks are identical), and the summed
  gradient within the 2% target by a wide margin.
* linearity in the vertex data: relative 1e-9 (FP64 sums of FP64 weights;
  the scatter-add order varies).
* FAST_FP32 / FAST_FP64 against the FP64 oracle (other streams): per-probe
  values and derivatives within 4.5 combined standard errors for >= 97% of
  probes.
* quadrature references at the centre of a disk / ball: 4 standard errors
  plus 2e-3 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

from tests.heat_reference import centre_value
from walk_on_spheres_b200 import meshes

pytestmark = pytest.mark.gpu

SLAB_X0 = (0.05, 0.025, 0.01)
THETA = np.array([1e3, *SLAB_X0, 2e-3])


@pytest.fixture(scope="module")
def slab_mesh():
    return meshes.slab_box(target_triangles=20000)


def _slab_probes(n, seed=0, spread=0.008):
    rng = np.random.default_rng(seed)
    c = np.array(SLAB_X0)
    return c + rng.uniform([-spread, -spread, -0.009], [spread, spread, -0.001], size=(n, 3))


def _heat(solver, mesh, probes, **kw):
    from walk_on_spheres_b200.heat import HeatProblem
    solver.set_mesh(mesh)
    args = dict(N_walks=512, epsilon=1e-5, seed=7, source_mode="green", method="fast")
    args.update(kw)
    return HeatProblem(solver, probes, **args)


@pytest.mark.parametrize("method", ["fast", "fast64"])
def test_adjoint_replays_forward_bit_for_bit(solver, slab_mesh, method):
    heat = _heat(solver, slab_mesh, _slab_probes(64), method=method)
    g = np.random.default_rng(1).normal(size=heat.n_verts)
    f = heat.forward(THETA[0], THETA[1:4], THETA[4], g)
    a = heat.adjoint(THETA[0], THETA[1:4], THETA[4], g)
    assert (f.location == 1).all()
    assert np.array_equal(f.mean, a.replayed_mean)
    assert f.counters["total_steps"] == a.counters["total_steps"]


@pytest.mark.parametrize("mode", ["uniform", "green", "mis"])
def test_adjoint_matches_crn_central_differences(solver, slab_mesh, mode):
    # the MIS proposal is held fixed while the source parameters move
    heat = _heat(solver, slab_mesh, _slab_probes(96, seed=2), source_mode=mode,
                 proposal=(SLAB_X0, 2e-3))
    a = heat.adjoint(THETA[0], THETA[1:4], THETA[4])
    for k in range(5):
        h = 1e-4 * abs(THETA[k])
        tp, tm = THETA.copy(), THETA.copy()
        tp[k] += h
        tm[k] -= h
        fd = (heat.forward(tp[0], tp[1:4], tp[4]).mean -
              heat.forward(tm[0], tm[1:4], tm[4]).mean) / (2 * h)
        jac = a.jacobian[:, k]
        assert np.abs(fd - jac).max() <= 1e-4 * np.abs(jac).max(), k
        # the summed gradient (grad_u = 1) against the summed differences; the
        # L1 norm guards sums that cancel across probes
        assert abs(a.grad_source[k] - fd.sum()) <= 0.02 * np.abs(fd).sum(), k


def test_adjoint_is_linear_in_vertex_values(solver, slab_mesh):
    heat = _heat(solver, slab_mesh, _slab_probes(80, seed=4, spread=0.02))
    rng = np.random.default_rng(9)
    g = rng.normal(size=heat.n_verts)
    w = rng.normal(size=heat.n)
    u_g = heat.forward(THETA[0], THETA[1:4], THETA[4], g).mean
    u_0 = heat.forward(THETA[0], THETA[1:4], THETA[4]).mean
    a = heat.adjoint(THETA[0], THETA[1:4], THETA[4], g, grad_u=w)
    lhs = float(w @ (u_g - u_0))
    rhs = float(a.grad_vertex_values @ g)
    assert abs(lhs - rhs) <= 1e-9 * max(1.0, np.abs(w) @ np.abs(u_g - u_0))
    assert abs(a.grad_vertex_values.sum() - w.sum()) <= 1e-9 * np.abs(w).sum()
    # weighted source gradient = weights against the per-probe Jacobian
    assert np.allclose(a.grad_source, w @ a.jacobian, rtol=1e-9, atol=0)


@pytest.mark.parametrize("method,mode", [("fast", "green"), ("fast64", "green"),
                                         ("fast", "mis")])
def test_heat_matches_fp64_oracle(solver, oracle, slab_mesh, method, mode):
    probes = _slab_probes(48, seed=5)
    g = np.random.default_rng(3).uniform(0.0, 1.0, size=slab_mesh.verts.shape[0])
    heat = _heat(solver, slab_mesh, probes, N_walks=4096, method=method, seed=21,
                 source_mode=mode)
    f = heat.forward(THETA[0], THETA[1:4], THETA[4], g)
    a = heat.adjoint(THETA[0], THETA[1:4], THETA[4], g)
    ref = oracle.heat_solve(slab_mesh, probes, THETA[0], THETA[1:4], THETA[4], vertex_values=g,
                            N_walks=4096, epsilon=1e-5, seed=21,
                            source_mode={"green": 1, "mis": 2}[mode], n_threads=8)
    assert np.array_equal(f.location, ref["location"])
    z = (f.mean - ref["mean"]) / np.hypot(f.standard_error, ref["standard_error"])
    assert (np.abs(z) <= 4.5).mean() >= 0.97, np.abs(z).max()
    for k in range(5):
        s = np.hypot(a.jacobian_se[:, k], ref["jacobian_se"][:, k])
        live = s > 0
        zk = (a.jacobian[live, k] - ref["jacobian"][live, k]) / s[live]
        assert (np.abs(zk) <= 4.5).mean() >= 0.97, (k, np.abs(zk).max())


@pytest.mark.parametrize("mode", ["green", "mis"])
@pytest.mark.parametrize("dim", [2, 3])
def test_heat_centre_value_matches_quadrature(solver, dim, mode):
    from walk_on_spheres_b200.heat import HeatProblem
    if dim == 2:
        mesh, x0 = meshes.circle(segments=1024), (0.2, -0.1)
    else:
        mesh, x0 = meshes.uv_sphere(lon=128, lat=64), (0.2, -0.1, 0.15)
    Q, sigma = 2.0, 0.3
    ref = centre_value(dim, 1.0, Q, x0, sigma)
    solver.set_mesh(mesh)
    heat = HeatProblem(solver, np.zeros((1, dim)), N_walks=200000, epsilon=1e-4, seed=8,
                       source_mode=mode)
    a = heat.adjoint(Q, x0, sigma)
    f = heat.forward(Q, x0, sigma)
    assert f.location[0] == 1
    assert abs(f.mean[0] - ref["u"]) <= 4 * f.standard_error[0] + 2e-3 * abs(ref["u"])
    for k in [0, 1, 2, 4] + ([3] if dim == 3 else []):
        err = abs(a.jacobian[0, k] - ref["jacobian"][k])
        assert err <= 4 * a.jacobian_se[0, k] + 2e-3 * np.abs(ref["jacobian"]).max(), k


def test_vertex_interpolation_reproduces_linear_data(solver):
    """g linear in space is harmonic and interpolated exactly on each triangle,
    so with Q = 0 every probe value is that linear function (up to the epsilon
    shell and Monte Carlo error)."""
    from walk_on_spheres_b200.heat import HeatProblem
    mesh = meshes.uv_sphere(lon=64, lat=32)
    solver.set_mesh(mesh)
    coef = np.array([0.3, -0.7, 0.5])
    g = mesh.verts @ coef + 1.0
    rng = np.random.default_rng(6)
    probes = rng.uniform(-0.5, 0.5, size=(64, 3))
    heat = HeatProblem(solver, probes, N_walks=4096, epsilon=1e-4, seed=3)
    f = heat.forward(0.0, (0.0, 0.0, 0.0), 1.0, g)
    want = probes @ coef + 1.0
    err = np.abs(f.mean - want)
    assert (err <= 4.5 * f.standard_error + 1e-4 * np.linalg.norm(coef)).mean() >= 0.97


def test_boundary_and_outside_probes(solver, slab_mesh):
    """A probe on the boundary returns the interpolated g and scatters its
    weight to the triangle's vertices; an outside probe is NaN and inert."""
    heat = _heat(solver, slab_mesh, np.array([[0.05, 0.025, 0.0], [0.2, 0.2, 0.2],
                                              [0.05, 0.02, 0.005]]))
    g = np.arange(heat.n_verts, dtype=np.float64) * 1e-3
    f = heat.forward(THETA[0], THETA[1:4], THETA[4], g)
    assert list(f.location) == [2, 0, 1]
    assert np.isnan(f.mean[1])
    a = heat.adjoint(THETA[0], THETA[1:4], THETA[4], g, grad_u=np.array([1.0, 5.0, 0.0]))
    assert abs(a.grad_vertex_values.sum() - 1.0) <= 1e-12
    assert abs(a.grad_vertex_values @ g - f.mean[0]) <= 1e-12
    assert np.all(a.jacobian[0] == 0.0) and np.all(np.isnan(a.jacobian[1]))


def test_autograd_function_matches_crn_differences(solver, slab_mesh):
    import torch
    from walk_on_spheres_b200.heat import heat_probe_values
    heat = _heat(solver, slab_mesh, _slab_probes(32, seed=8), N_walks=256)
    g0 = np.random.default_rng(2).uniform(size=heat.n_verts)
    Q = torch.tensor(THETA[0], dtype=torch.float64, requires_grad=True)
    x0 = torch.tensor(THETA[1:4], dtype=torch.float64, requires_grad=True)
    sigma = torch.tensor(THETA[4], dtype=torch.float64, requires_grad=True)
    g = torch.tensor(g0, dtype=torch.float64, requires_grad=True)
    u = heat_probe_values(heat, Q, x0, sigma, g)
    loss = (u ** 2).sum()
    loss.backward()

    def L(theta, gv):
        m = heat.forward(theta[0], theta[1:4], theta[4], gv).mean
        return float((m ** 2).sum())

    grads = [Q.grad.item(), *x0.grad.tolist(), sigma.grad.item()]
    for k in range(5):
        h = 1e-4 * abs(THETA[k])
        tp, tm = THETA.copy(), THETA.copy()
        tp[k] += h
        tm[k] -= h
        fd = (L(tp, g0) - L(tm, g0)) / (2 * h)
        assert abs(grads[k] - fd) <= 1e-3 * abs(fd) + 1e-30, (k, grads[k], fd)
    d = np.random.default_rng(4).normal(size=heat.n_verts)
    h = 1e-3
    fd = (L(THETA, g0 + h * d) - L(THETA, g0 - h * d)) / (2 * h)
    assert abs(float(g.grad.numpy() @ d) - fd) <= 1e-6 * abs(fd)


def test_mis_narrow_source_and_registry_rejection(solver):
    """MIS against Green sampling for a source much narrower than the balls
    around it (standard error several times smaller, same mean), and the
    registry equations' rejection of MIS (they have no source proposal, as in
    include/wos/wos.hpp:83-92)."""
    from walk_on_spheres_b200._lib import WosError
    from walk_on_spheres_b200.heat import HeatProblem
    solver.set_mesh(meshes.circle(segments=1024))
    ref = centre_value(2, 1.0, 2.0, (0.2, -0.1), 0.05)
    out = {}
    for mode in ("green", "mis"):
        heat = HeatProblem(solver, np.zeros((1, 2)), N_walks=100000, epsilon=1e-4, seed=5,
                           source_mode=mode)
        out[mode] = heat.forward(2.0, (0.2, -0.1), 0.05)
    assert out["mis"].standard_error[0] < out["green"].standard_error[0] / 3
    assert abs(out["mis"].mean[0] - ref["u"]) <= 4 * out["mis"].standard_error[0] + 2e-3 * ref["u"]
    with pytest.raises(WosError, match="GreenSourceMIS"):
        solver.solve_grid("poisson", 8, 8, N_walks=16, source_mode="mis", method="fast")
    with pytest.raises(WosError, match="MIS probability"):
        HeatProblem(solver, np.zeros((1, 2)), N_walks=16, source_mode="mis",
                    mis_green_probability=1.0).forward(2.0, (0.2, -0.1), 0.05)
