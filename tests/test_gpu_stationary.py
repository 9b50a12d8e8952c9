"""Stationary plate heating (wos_stationary_solve) against the reference's own
level-1 program through tests/golden/stationary_golden.npz, written by
tests/golden/make_stationary_golden.py from oracle/_ref/wos_level1_ref.

Tolerances:
* PLAIN_FP64 follows the reference's seeds and streams: for each of the
  program's three solves, at least 98% of interior points agree with the
  reference to 1e-9 relative and every point within 4 of the reference's
  standard errors (CUDA's and glibc's transcendental functions differ in
  the last bit); the edge points are exactly 0.
* FAST_FP32 / FAST_FP64 (other streams) against PLAIN_FP64: >= 99% of
  interior points within 4.5 combined standard errors, and the reference's
  validation gates (apps/welding/tools/validate_level1.py, restated in
  oracle/fd_plate.py) against the finite-difference solution.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "stationary_golden.npz"
CASES = ["manufactured", "gaussian", "gaussian_mis"]


def _inner(a):
    return a[1:-1, 1:-1]


@pytest.fixture(scope="module")
def plain(solver):
    from walk_on_spheres_b200.stationary import LEVEL1_CASES, solve_stationary
    return {c: solve_stationary(solver, method="plain", **LEVEL1_CASES[c]) for c in CASES}


@pytest.mark.parametrize("case", CASES)
def test_plain_matches_reference_program(plain, case):
    g = np.load(GOLDEN)
    r = plain[case]
    ref, ref_se = g[f"{case}_mean"], g[f"{case}_se"]
    assert r.mean.shape == ref.shape == (49, 33)
    edge = np.ones(ref.shape, dtype=bool)
    edge[1:-1, 1:-1] = False
    for a in (r.mean, r.standard_error, r.variance, r.mean_steps):
        assert np.all(a[edge] == 0.0)
    got, want = _inner(r.mean), _inner(ref)
    close = np.abs(got - want) <= 1e-9 * np.maximum(1e-3, np.abs(want))
    assert close.mean() >= 0.98, close.mean()
    far = ~close
    if far.any():
        z = np.abs(got[far] - want[far]) / np.maximum(_inner(ref_se)[far], 1e-300)
        assert (z <= 4.0).all(), z.max()
    # same walks: identical mean step counts where the means agree
    steps_equal = _inner(r.mean_steps) == _inner(g[f"{case}_steps"])
    assert steps_equal[close].mean() >= 0.98
    assert r.max_steps_hits == 0


@pytest.mark.parametrize("method", ["fast", "fast64"])
@pytest.mark.parametrize("case", CASES)
def test_fast_agrees_with_plain(solver, plain, case, method):
    from walk_on_spheres_b200.stationary import LEVEL1_CASES, solve_stationary
    f = solve_stationary(solver, method=method, **LEVEL1_CASES[case])
    p = plain[case]
    se = np.hypot(_inner(p.standard_error), _inner(f.standard_error))
    z = np.abs(_inner(p.mean) - _inner(f.mean)) / se
    assert (z <= 4.5).mean() >= 0.99, z.max()
    assert abs(z.mean() - 0.798) < 4 * 0.6 / np.sqrt(z.size) + 0.05, z.mean()
    assert f.device_ms > 0 and f.max_steps_hits == 0


@pytest.mark.parametrize("case", ["gaussian", "gaussian_mis"])
def test_fast_passes_the_reference_validation_gates(solver, case):
    from oracle.fd_plate import fd_reference, level1_gates
    from walk_on_spheres_b200.stationary import LEVEL1_CASES, gaussian_summary, solve_stationary
    r = solve_stationary(solver, method="fast", **LEVEL1_CASES[case])
    gates = level1_gates(r.mean, r.standard_error, r.params, gaussian_summary(r),
                         fd_reference(r.params))
    assert gates["all"], gates


def test_manufactured_solution_within_error(solver):
    from walk_on_spheres_b200.stationary import (exact_manufactured, manufactured_summary,
                                                 solve_stationary)
    r = solve_stationary(solver, "manufactured", method="fast")
    err = np.abs(_inner(r.mean - exact_manufactured(r.params)))
    assert (err <= 4.0 * _inner(r.standard_error)).mean() >= 0.99
    # the reference's own run: RMSE 0.629 K, centre SE 0.678 K at 6000 walks
    s = manufactured_summary(r)
    assert s["field_rmse"] < 1.0 and s["center_absolute_error"] < 4 * s["center_standard_error"]


def test_mis_reduces_the_standard_error(solver):
    from walk_on_spheres_b200.stationary import solve_stationary
    g = solve_stationary(solver, "gaussian", method="fast", source_mode="green")
    m = solve_stationary(solver, "gaussian", method="fast", source_mode="mis")
    ratio = np.mean(_inner(m.standard_error)) / np.mean(_inner(g.standard_error))
    # the reference's own fields: 0.56 (tests/golden/stationary_golden.npz)
    assert ratio < 0.75, ratio


def test_rejects_the_reference_invalid_configurations(solver):
    from walk_on_spheres_b200._lib import WosError
    from walk_on_spheres_b200.stationary import solve_stationary
    with pytest.raises(WosError, match="requires a source proposal sampler and PDF"):
        solve_stationary(solver, "manufactured", source_mode="mis", walks=8)
    with pytest.raises(WosError, match="finite and in \\(0, 1\\)"):
        solve_stationary(solver, "gaussian", source_mode="mis", mis_green_probability=1.0)
    with pytest.raises(WosError, match="invalid Gaussian heat-source parameters"):
        solve_stationary(solver, "gaussian", efficiency=1.5)
    with pytest.raises(WosError, match="invalid Gaussian heat-source parameters"):
        solve_stationary(solver, "gaussian", source_x=0.2)


def test_proposal_cap_reports_the_reference_error(solver):
    # a Gaussian of sigma 1 m centred on a corner of the 0.12 x 0.08 m plate:
    # about 0.15% of its proposals land on the plate, so a cap of one
    # attempt runs out
    from walk_on_spheres_b200._lib import WosError
    from walk_on_spheres_b200.stationary import solve_stationary
    with pytest.raises(WosError, match="rejection sampler did not accept a point"):
        solve_stationary(solver, "gaussian", source_mode="mis", source_x=0.0, source_y=0.0,
                         sigma_x=1.0, sigma_y=1.0, max_proposal_attempts=1, walks=64,
                         nx=9, ny=7)
    # with the reference's cap the same problem solves
    r = solve_stationary(solver, "gaussian", source_mode="mis", source_x=0.0, source_y=0.0,
                         sigma_x=1.0, sigma_y=1.0, walks=64, nx=9, ny=7)
    assert np.isfinite(r.mean).all()
