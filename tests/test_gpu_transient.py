"""Transient plate heating (wos_transient_solve) against the reference's own
welding programs -- level 0 (cooling), level 2 (stationary source) and
level 3 (moving source) -- through tests/golden/transient_golden.npz, written
by tests/golden/make_transient_golden.py from oracle/_ref/wos_level*_ref.

Tolerances:
* PLAIN_FP64 follows the reference's seeds and streams step by step: at
  every stored step at least 98% of interior points agree with the
  reference to 1e-9 relative (level 0 prints six significant digits: 1e-5)
  and every point within 4 of the reference's standard errors (the rule of
  the single-solve parity tests; CUDA's and glibc's transcendental functions
  differ in the last bit).
* FAST_FP32 (other streams) against PLAIN_FP64 at step 1 (no history yet):
  >= 99% of interior points within 4.5 combined standard errors.  Later
  steps also carry the noise of the sampled history field, which the
  per-step standard error does not include, so they are compared through
  the field's total (2% at 2000 walks).
* graph replay and stream launch: bit-for-bit equal.
* FAST_FP32 / FAST_FP64 at the level-2 defaults, and FAST_FP32 at the
  level-3 configuration, pass the reference's own
  level-2 and level-3 validations (oracle/fd_transient.py).
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "transient_golden.npz"


def _cases():
    g = np.load(GOLDEN)
    return [(k[:-len("_config")], json.loads(str(g[k]))) for k in sorted(g.files)
            if k.endswith("_config")]


def params_for(cfg: dict) -> tuple[dict, np.ndarray | None]:
    """Library parameters (and initial field) of a reference program's options."""
    from walk_on_spheres_b200.transient import LEVEL0, LEVEL3
    level = cfg["level"]
    if level == 2:
        keys = ("nx", "ny", "dt", "total_time", "heat_on_time", "walks", "seed", "cubic")
        return {k: cfg[k] for k in keys}, None
    if level == 3:
        return dict(LEVEL3, walks=cfg["walks"], seed=cfg["seed"]), None
    n = cfg["grid"]
    p = dict(LEVEL0, nx=n, ny=n, dt=cfg["dt"], total_time=cfg["steps"] * cfg["dt"],
             walks=cfg["walks"], epsilon=cfg["epsilon"], seed=cfg["seed"],
             conductivity=cfg["diffusivity"])
    # sin(pi x) sin(pi y) with the C library's sin, as the reference computes it
    init = np.zeros((n, n))
    for i in range(1, n - 1):
        for j in range(1, n - 1):
            init[i, j] = math.sin(math.pi * (i / (n - 1))) * math.sin(math.pi * (j / (n - 1)))
    return p, init


@pytest.mark.parametrize("name,cfg", _cases(), ids=[c[0] for c in _cases()])
def test_plain_matches_reference_program(solver, name, cfg):
    from walk_on_spheres_b200.transient import solve_transient
    g = np.load(GOLDEN)
    steps, ref, ref_se = g[f"{name}_steps"], g[f"{name}_rise"], g[f"{name}_se"]
    params, init = params_for(cfg)
    r = solve_transient(solver, method="plain", use_graph=True, initial=init, **params)
    assert r.fields.shape[1:] == ref.shape[1:]
    rtol = 1e-5 if cfg["level"] == 0 else 1e-9
    interior = np.zeros(ref.shape[1:], dtype=bool)
    interior[1:-1, 1:-1] = True
    for k, s in enumerate(steps):
        assert np.all(r.fields[s][~interior] == 0.0)
        got, want = r.fields[s][interior], ref[k][interior]
        close = np.abs(got - want) <= rtol * np.maximum(1e-3, np.abs(want))
        assert close.mean() >= 0.98, (s, close.mean())
        far = ~close
        if far.any():
            z = np.abs(got[far] - want[far]) / np.maximum(ref_se[k][interior][far], 1e-300)
            assert (z <= 4.0).all(), (s, z.max())


@pytest.mark.parametrize("method", ["fast", "fast64"])
def test_fast_agrees_with_plain(solver, method):
    from walk_on_spheres_b200.transient import solve_transient
    opts = dict(nx=11, ny=9, dt=0.25, total_time=1.0, heat_on_time=0.5, walks=2000, seed=3)
    p = solve_transient(solver, method="plain", **opts)
    f = solve_transient(solver, method=method, **opts)
    inner = (slice(1, -1), slice(1, -1))
    s1 = np.hypot(p.standard_error[1][inner], f.standard_error[1][inner])
    z = np.abs(p.fields[1][inner] - f.fields[1][inner]) / s1
    assert (z <= 4.5).mean() >= 0.99, z.max()
    for s in range(2, p.fields.shape[0]):
        tp, tf = p.fields[s].sum(), f.fields[s].sum()
        assert abs(tf / tp - 1.0) <= 0.02, (s, tf, tp)


@pytest.mark.parametrize("method", ["plain", "fast"])
def test_graph_equals_stream(solver, method):
    from walk_on_spheres_b200.transient import solve_transient
    opts = dict(nx=9, ny=7, dt=0.5, total_time=2.0, heat_on_time=1.0, walks=200, seed=9,
                method=method)
    a = solve_transient(solver, use_graph=True, **opts)
    b = solve_transient(solver, use_graph=False, **opts)
    assert np.array_equal(a.fields, b.fields)
    assert np.array_equal(a.standard_error, b.standard_error)
    assert a.device_ms > 0


def test_rejects_the_reference_invalid_configurations(solver):
    from walk_on_spheres_b200._lib import WosError
    from walk_on_spheres_b200.transient import solve_transient
    with pytest.raises(WosError, match="odd integers"):
        solve_transient(solver, nx=10)
    with pytest.raises(WosError, match="smaller than --total-time"):
        solve_transient(solver, heat_on_time=10.0, total_time=10.0)
    with pytest.raises(WosError, match="integer multiple"):
        solve_transient(solver, dt=0.3, total_time=1.0, heat_on_time=0.5)


@pytest.mark.parametrize("method", ["fast", "fast64"])
def test_fast_passes_the_reference_level2_validation(solver, method):
    # apps/welding/tools/validate_level2.py restated in oracle/fd_transient.py:
    # at the reference's level-2 defaults (49 x 33, 100 steps, 500 walks)
    # every step's field is within 5% RMS and 10% at the centre of the
    # implicit finite-difference solution, relative to its peak
    from oracle.fd_transient import level2_gates
    from walk_on_spheres_b200.transient import defaults, solve_transient
    r = solve_transient(solver, method=method)
    params = defaults()
    g = level2_gates(r.fields, r.standard_error, params, r.max_steps_hits)
    assert g["passed"], g["failures"][:5]
    worst = max(row["normalized_rmse"] for row in g["rows"])
    assert worst < 0.05, worst


def test_fast_passes_the_reference_level3_validation(solver):
    # apps/welding/tools/validate_level3.py restated in oracle/fd_transient.py:
    # the moving source at its fixed configuration (97 x 65, 150 steps, 500
    # walks) within 1% RMS and 2% at the peak of a 4x-refined, 16-substep
    # finite-difference solution at every step, and the seven probes' peaks
    # within max(5 K, 2%).  The two argmax gates (peak at most one cell
    # away, probe peak time within one step) are applied in their 3-SE form:
    # where the field is flat near its peak, the reference's argmax differs
    # from the run's by less than the Monte Carlo error at 500 walks (e.g.
    # 0.06 K over six steps for the 10 mm transverse probe, against a
    # standard error of 0.16 K), so the strict gates pass or fail with the seed.
    from oracle.fd_transient import level3_gates
    from walk_on_spheres_b200.transient import LEVEL3, defaults, solve_transient
    params = dict(defaults())
    params.update(LEVEL3)
    for seed in (20260819, 7):
        r = solve_transient(solver, method="fast", seed=seed, **LEVEL3)
        g = level3_gates(r.fields, r.standard_error, params, r.max_steps_hits,
                         statistical_argmax=True)
        assert g["passed"], (seed, g["failures"][:5])
        assert max(row["normalized_rmse"] for row in g["rows"]) < 0.01


def test_fast_level0_matches_the_discrete_cooling_solution(solver):
    # the level-0 program's own check (apps/welding/src/level0_cooling.cpp:
    # 286-288, 394-400): after s implicit steps the field is
    # d^s sin(pi x) sin(pi y), d = 1 / (1 + 2 pi^2 kappa dt).  The walks
    # sample the previous field by bilinear interpolation of its grid values;
    # for this eigenfunction the interpolant averages (pi h)^2 / 12 below the
    # function per axis, so each step also scales the amplitude by
    # 1 - (pi h)^2 / 6 (0.64% on the 17 x 17 grid; the reference's own run in
    # tests/golden is 2.7% low at the centre after five steps).  At 20 000
    # walks FAST_FP32 must follow (d (1 - (pi h)^2 / 6))^s within 1% at the
    # centre and 2% RMS at every step.
    from walk_on_spheres_b200.transient import LEVEL0, level0_initial, solve_transient
    n = LEVEL0["nx"]
    init = level0_initial(n, n)
    r = solve_transient(solver, method="fast", initial=init, **dict(LEVEL0, walks=20000))
    d = 1.0 / (1.0 + 2.0 * math.pi**2 * LEVEL0["conductivity"] * LEVEL0["dt"])
    h = 1.0 / (n - 1)
    per_step = d * (1.0 - (math.pi * h) ** 2 / 6.0)
    for s in range(1, r.fields.shape[0]):
        amp = per_step**s
        err = (r.fields[s] - amp * init)[1:-1, 1:-1]
        assert np.sqrt(np.mean(err**2)) / amp < 0.02, (s, np.sqrt(np.mean(err**2)) / amp)
        assert abs(r.fields[s][n // 2, n // 2] / amp - 1.0) < 0.01, (s, r.fields[s][n // 2, n // 2] / amp)
