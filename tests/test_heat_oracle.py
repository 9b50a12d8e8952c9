"""The FP64 heat-source oracle (wo_heat_solve) on CPU: derivative formulas
against common-random-number central differences of its own forward values,
exact linearity in the per-vertex boundary data, and quadrature references
at the centre of a disk and a ball.

Source modes: uniform, Green and Green-source MIS (with the source's own
Gaussian as proposal).

Tolerances:
* CRN central differences (h = 1e-4 relative to each parameter, FP64 walks,
  same seeds): the walks are identical, so the difference quotient and the
  derivative sum differ by the O((h/sigma)^2) truncation terms only —
  relative 1e-4 of the largest derivative.
* linearity in g: rounding only — 1e-12 relative.
* quadrature references: within 4 standard errors plus 2e-3 relative (the
  1024-segment polygon / 128 x 64 UV sphere and the epsilon shell move the
  boundary by less than that).
"""
from __future__ import annotations

import numpy as np
import pytest

from tests.heat_reference import centre_value
from walk_on_spheres_b200 import meshes

SLAB_X0 = (0.05, 0.025, 0.01)


@pytest.fixture(scope="module")
def slab():
    return meshes.slab_box(target_triangles=2000)


def _slab_probes(n, seed=0):
    rng = np.random.default_rng(seed)
    # probes within 8 mm of the source centre, inside the slab
    c = np.array(SLAB_X0)
    p = c + rng.uniform([-0.008, -0.008, -0.009], [0.008, 0.008, -0.001], size=(n, 3))
    return p


@pytest.mark.parametrize("mode", [0, 1, 2], ids=["uniform", "green", "mis"])
def test_oracle_derivatives_match_crn_differences(oracle, slab, mode):
    probes = _slab_probes(6)
    # the MIS proposal stays fixed while the source parameters move
    base = dict(N_walks=200, epsilon=1e-5, seed=11, source_mode=mode, n_threads=4,
                proposal=(SLAB_X0, 2e-3))
    theta = np.array([1e3, *SLAB_X0, 2e-3])
    r = oracle.heat_solve(slab, probes, theta[0], theta[1:4], theta[4], **base)
    assert (r["location"] == 1).all()
    for k in range(5):
        h = 1e-4 * abs(theta[k])
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        up = oracle.heat_solve(slab, probes, tp[0], tp[1:4], tp[4], **base)["mean"]
        um = oracle.heat_solve(slab, probes, tm[0], tm[1:4], tm[4], **base)["mean"]
        fd = (up - um) / (2 * h)
        jac = r["jacobian"][:, k]
        tol = 1e-4 * np.abs(jac).max() + 1e-300
        assert np.abs(fd - jac).max() <= tol, (k, fd, jac)


def test_oracle_is_linear_in_vertex_values(oracle, slab):
    probes = _slab_probes(5, seed=3)
    rng = np.random.default_rng(5)
    g = rng.normal(size=slab.verts.shape[0])
    w = rng.normal(size=probes.shape[0])
    kw = dict(N_walks=100, epsilon=1e-5, seed=2, source_mode=1, n_threads=4)
    with_g = oracle.heat_solve(slab, probes, 1e3, SLAB_X0, 2e-3, vertex_values=g, weights=w, **kw)
    zero_g = oracle.heat_solve(slab, probes, 1e3, SLAB_X0, 2e-3, weights=w, **kw)
    lhs = float(w @ (with_g["mean"] - zero_g["mean"]))
    rhs = float(with_g["grad_vertex"] @ g)
    assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs))
    # each walk scatters weights summing to 1: sum_v grad_v = sum_p w_p
    assert abs(with_g["grad_vertex"].sum() - w.sum()) <= 1e-12 * np.abs(w).sum()


@pytest.mark.parametrize("mode", [1, 2], ids=["green", "mis"])
@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_centre_value_matches_quadrature(oracle, dim, mode):
    if dim == 2:
        mesh = meshes.circle(segments=1024)
        x0, N = (0.2, -0.1), 6000
    else:
        mesh = meshes.uv_sphere(lon=128, lat=64)
        x0, N = (0.2, -0.1, 0.15), 3000
    Q, sigma = 2.0, 0.3
    ref = centre_value(dim, 1.0, Q, x0, sigma)
    r = oracle.heat_solve(mesh, np.zeros((1, dim)), Q, x0, sigma, N_walks=N, epsilon=1e-4,
                          seed=4, source_mode=mode, n_threads=8)
    assert r["location"][0] == 1
    assert abs(r["mean"][0] - ref["u"]) <= 4 * r["standard_error"][0] + 2e-3 * abs(ref["u"])
    for k in [0, 1, 2, 4] + ([3] if dim == 3 else []):
        err = abs(r["jacobian"][0, k] - ref["jacobian"][k])
        assert err <= 4 * r["jacobian_se"][0, k] + 2e-3 * np.abs(ref["jacobian"]).max(), k


def test_oracle_mis_reduces_variance_for_a_narrow_source(oracle):
    """Green-source MIS (include/wos/source_sampling.hpp:35-78) with the source's
    own Gaussian as proposal: for a source much narrower than the balls that
    contain it, Green sampling rarely lands on it; the mixture does."""
    mesh = meshes.circle(segments=1024)
    kw = dict(N_walks=20000, epsilon=1e-4, seed=6, n_threads=8)
    ref = centre_value(2, 1.0, 2.0, (0.2, -0.1), 0.05)
    green = oracle.heat_solve(mesh, np.zeros((1, 2)), 2.0, (0.2, -0.1), 0.05, source_mode=1, **kw)
    mis = oracle.heat_solve(mesh, np.zeros((1, 2)), 2.0, (0.2, -0.1), 0.05, source_mode=2, **kw)
    assert mis["standard_error"][0] < green["standard_error"][0] / 3
    assert abs(mis["mean"][0] - ref["u"]) <= 4 * mis["standard_error"][0] + 2e-3 * ref["u"]
