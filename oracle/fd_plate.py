"""Finite-difference reference of the stationary Gaussian plate problem and the
reference's level-1 validation gates.  TEST INFRASTRUCTURE ONLY: the oracle
of the stationary plate solver, never part of the product path.

Restates apps/welding/tools/validate_level1.py:21-187: the 5-point negative
Laplacian on a grid refined `refinement` times in each direction, solved
with conjugate gradients to a relative residual of 1e-11 with u = 0 on the
plate edges, sampled back at the coarse grid points; then the gates:
  power          the summary's relative power error < 1e-6
  field_nrmse    RMS interior error / FD peak < 0.05
  centre         |error at the centre| <= max(3 SE, 0.03 FD peak)
  peak_location  distance of the WoS peak from the source centre <= one
                 coarse-cell diagonal
  symmetry       RMS mirror residual < 0.02 and > 99% of mirror pairs
                 within 3 combined SE
  max_steps      no walk hit the step limit
"""
from __future__ import annotations

import numpy as np


def negative_laplacian(u: np.ndarray, hx: float, hy: float) -> np.ndarray:
    """validate_level1.py:35-41 (u holds interior values; zero outside)."""
    out = (2.0 / hx**2 + 2.0 / hy**2) * u
    out[1:, :] -= u[:-1, :] / hx**2
    out[:-1, :] -= u[1:, :] / hx**2
    out[:, 1:] -= u[:, :-1] / hy**2
    out[:, :-1] -= u[:, 1:] / hy**2
    return out


def conjugate_gradient(rhs: np.ndarray, hx: float, hy: float, rtol: float = 1e-11,
                       max_iterations: int = 20_000) -> tuple[np.ndarray, int, float]:
    """validate_level1.py:44-74."""
    x = np.zeros_like(rhs)
    r = rhs.copy()
    d = r.copy()
    rr = float(np.sum(r * r))
    norm0 = np.sqrt(rr)
    if norm0 == 0.0:
        return x, 0, 0.0
    for it in range(1, max_iterations + 1):
        ad = negative_laplacian(d, hx, hy)
        a = rr / float(np.sum(d * ad))
        x += a * d
        r -= a * ad
        rr_next = float(np.sum(r * r))
        rel = np.sqrt(rr_next) / norm0
        if rel <= rtol:
            return x, it, rel
        d = r + (rr_next / rr) * d
        rr = rr_next
    raise RuntimeError(f"finite-difference CG did not converge after {max_iterations} iterations")


def fd_reference(params: dict, refinement: int = 4) -> np.ndarray:
    """FD temperature rise of the finite-plate Gaussian on the coarse (nx, ny)
    grid (validate_level1.py:81-123)."""
    from math import erf, sqrt, pi
    nx, ny = params["nx"], params["ny"]
    lx, ly = params["length_x"], params["length_y"]
    fnx, fny = (nx - 1) * refinement + 1, (ny - 1) * refinement + 1
    fx, fy = np.linspace(0.0, lx, fnx), np.linspace(0.0, ly, fny)
    hx, hy = fx[1] - fx[0], fy[1] - fy[0]
    xx, yy = np.meshgrid(fx[1:-1], fy[1:-1], indexing="ij")

    def integral(lo, hi, c, s):
        return s * sqrt(pi / 2.0) * (erf((hi - c) / (sqrt(2.0) * s)) - erf((lo - c) / (sqrt(2.0) * s)))

    sx, sy, cx, cy = params["sigma_x"], params["sigma_y"], params["source_x"], params["source_y"]
    ix, iy = integral(0.0, lx, cx, sx), integral(0.0, ly, cy, sy)
    shape = np.exp(-0.5 * (((xx - cx) / sx) ** 2 + ((yy - cy) / sy) ** 2))
    absorbed = params["electrical_power"] * params["efficiency"]
    q = absorbed * shape / (params["thickness"] * ix * iy)
    u, _, _ = conjugate_gradient(q / params["conductivity"], hx, hy)
    fine = np.zeros((fnx, fny))
    fine[1:-1, 1:-1] = u
    return fine[::refinement, ::refinement]


def level1_gates(mean: np.ndarray, se: np.ndarray, params: dict, summary: dict,
                 reference: np.ndarray | None = None) -> dict:
    """validate_level1.py:125-187 for one WoS field; `summary` is the solve's
    gaussian summary (power_relative_error, peak_x, peak_y, symmetry, hits)."""
    if reference is None:
        reference = fd_reference(params)
    nx, ny = params["nx"], params["ny"]
    x = np.linspace(0.0, params["length_x"], nx)
    y = np.linspace(0.0, params["length_y"], ny)
    err = (mean - reference)[1:-1, 1:-1]
    ref_peak = float(np.max(reference))
    nrmse = float(np.sqrt(np.mean(err**2))) / ref_peak
    ci, cj = nx // 2, ny // 2
    centre_err = float(mean[ci, cj] - reference[ci, cj])
    centre_limit = max(3.0 * float(se[ci, cj]), 0.03 * ref_peak)
    peak_err = float(np.hypot(summary["peak_x"] - params["source_x"],
                              summary["peak_y"] - params["source_y"]))
    peak_limit = float(np.hypot(x[1] - x[0], y[1] - y[0]))
    gates = {
        "power": summary["power_relative_error"] < 1e-6,
        "field_nrmse": nrmse < 0.05,
        "centre": abs(centre_err) <= centre_limit,
        "peak_location": peak_err <= peak_limit,
        "symmetry": (summary["symmetry_rms_relative_residual"] < 0.02 and
                     summary["symmetry_within_three_standard_errors_fraction"] > 0.99),
        "max_steps": summary["max_steps_hits"] == 0,
    }
    gates["all"] = all(gates.values())
    gates["field_normalized_rmse"] = nrmse
    gates["centre_error"] = centre_err
    return gates
