"""Stationary plate solver host logic (no GPU): the reference's Level1Config
defaults through the C ABI, the level-1 summary functions against the
reference program's own summary rows (applied to its own fields, from
tests/golden/stationary_golden.npz), and the finite-difference validator
(oracle/fd_plate.py) passing the reference's fields as the reference's
validator does."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from walk_on_spheres_b200.stationary import (LEVEL1_CASES, StationaryResult, defaults,
                                             exact_manufactured, gaussian_summary,
                                             make_params, manufactured_summary)

GOLDEN = Path(__file__).resolve().parent / "golden" / "stationary_golden.npz"


def _golden_result(case: str) -> tuple[StationaryResult, dict]:
    g = np.load(GOLDEN)
    summary = json.loads(str(g[f"{case}_summary"]))
    spec = LEVEL1_CASES[case]
    params = defaults(spec["source"])
    r = StationaryResult(g[f"{case}_mean"], g[f"{case}_variance"], g[f"{case}_se"],
                         g[f"{case}_steps"], int(summary["max_steps_hits"]), 0.0, params)
    return r, summary


def test_defaults_are_the_reference_level1_config():
    # Level1Config, apps/welding/src/level1_stationary_heat.cpp:42-61
    want = dict(nx=49, ny=33, walks=6000, max_steps=1000, epsilon=8e-6, seed=20260818,
                length_x=0.12, length_y=0.08, thickness=0.006, conductivity=35.0,
                electrical_power=800.0, efficiency=0.75, sigma_x=0.006, sigma_y=0.006,
                peak_rise=100.0, source_x=0.06, source_y=0.04, mis_green_probability=0.5,
                max_proposal_attempts=1_000_000)
    for source in ("manufactured", "gaussian"):
        d = defaults(source)
        for k, v in want.items():
            assert d[k] == v, (source, k)
    # the case streams of :599-600 and :623-624
    assert defaults("manufactured")["case_stream"] == 0x4C4556454C31414F
    assert defaults("gaussian")["case_stream"] == 0x4C4556454C314247
    assert make_params("gaussian", source_mode="mis").source_mode == 2
    with pytest.raises(TypeError):
        make_params("gaussian", source=0)
    with pytest.raises(ValueError):
        make_params("disk")


def test_manufactured_summary_matches_the_reference_row():
    r, ref = _golden_result("manufactured")
    s = manufactured_summary(r)
    for k in ("center_mean", "center_standard_error", "center_absolute_error"):
        assert s[k] == ref[k], k
    for k in ("field_rmse", "field_max_absolute_error", "mean_standard_error",
              "max_standard_error", "mean_steps"):
        assert s[k] == pytest.approx(ref[k], rel=1e-12, abs=0.0), k
    assert s["max_steps_hits"] == ref["max_steps_hits"] == 0
    # the exact solution vanishes on the plate edges and peaks at the centre
    u = exact_manufactured(r.params)
    assert u[24, 16] == pytest.approx(100.0, rel=1e-15)
    assert np.abs(u[0, :]).max() < 1e-12 and np.abs(u[:, -1]).max() < 1e-12


@pytest.mark.parametrize("case", ["gaussian", "gaussian_mis"])
def test_gaussian_summary_matches_the_reference_row(case):
    r, ref = _golden_result(case)
    s = gaussian_summary(r)
    for k in ("peak_temperature_rise", "peak_x", "peak_y", "peak_standard_error"):
        assert s[k] == ref[k], k
    for k in ("symmetry_max_relative_residual", "symmetry_rms_relative_residual",
              "symmetry_within_three_standard_errors_fraction", "mean_standard_error",
              "max_standard_error", "mean_steps"):
        assert s[k] == pytest.approx(ref[k], rel=1e-12, abs=0.0), k
    assert s["absorbed_power"] == ref["absorbed_power"] == 600.0
    # midpoint rule over 800 x 600 cells; numpy's exp may differ from the C
    # library's in the last bit, so the sum agrees to rounding
    assert s["integrated_power"] == pytest.approx(ref["integrated_power"], rel=1e-13)
    assert s["power_relative_error"] < 1e-6


@pytest.mark.parametrize("case", ["gaussian", "gaussian_mis"])
def test_fd_validator_passes_the_reference_fields(case):
    from oracle.fd_plate import fd_reference, level1_gates
    r, _ = _golden_result(case)
    ref = fd_reference(r.params)
    gates = level1_gates(r.mean, r.standard_error, r.params, gaussian_summary(r), ref)
    assert gates["all"], gates
    # MIS reduces the standard error of the same problem
    if case == "gaussian_mis":
        g, _ = _golden_result("gaussian")
        assert np.mean(r.standard_error[1:-1, 1:-1]) < np.mean(g.standard_error[1:-1, 1:-1])


def test_fd_validator_rejects_planted_errors():
    from oracle.fd_plate import fd_reference, level1_gates
    r, _ = _golden_result("gaussian")
    ref = fd_reference(r.params)

    def gates_of(mean):
        bad = StationaryResult(mean, r.variance, r.standard_error, r.mean_steps, 0, 0.0,
                               r.params)
        return level1_gates(bad.mean, bad.standard_error, bad.params, gaussian_summary(bad), ref)

    # 10% too hot: the centre gate fails
    g = gates_of(r.mean * 1.1)
    assert not g["centre"] and not g["all"]
    # a uniform offset of 10% of the peak inside the plate: the field gate fails
    off = r.mean.copy()
    off[1:-1, 1:-1] += 0.1 * ref.max()
    g = gates_of(off)
    assert not g["field_nrmse"] and not g["all"]
    # a hot spot away from the source: the peak-location gate fails
    spot = r.mean.copy()
    spot[5, 5] = 2.0 * r.mean.max()
    g = gates_of(spot)
    assert not g["peak_location"] and not g["all"]
