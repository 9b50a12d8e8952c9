"""Finite-difference reference of the transient plate problem (welding level 2)
and the reference's level-2 validation gates.  TEST INFRASTRUCTURE ONLY: the
checker of the transient solver, never part of the product path.

Restates apps/welding/tools/validate_level2.py:108-330 (default options: the
WoS grid itself, one implicit step per WoS step):
  * the five-point Dirichlet Laplacian on the interior of the nx x ny grid,
    diagonalised by the sine transform, so an implicit Euler step
        (I - kappa dt Lap) u_{n+1} = u_n + dt f_n q / (rho c)
    is one division per mode;
  * q the stationary Gaussian at the plate centre, normalised on the finite
    plate, switched on for the share f_n of each step before heat_on_time;
  * gates at every stored step > 0: RMS interior error / FD peak <= 0.05,
    |centre error| / FD peak <= 0.10; all fields >= -1e-10; no walk at the
    step cap; injected energy = absorbed power x heat_on_time.
"""
from __future__ import annotations

import math

import numpy as np


def heating_fraction(t0: float, t1: float, heat_on: float) -> float:
    """Share of [t0, t1] before heat_on (level2_transient_heat.cpp:226-234)."""
    lo, hi = max(0.0, t0), min(t1, heat_on)
    return (hi - lo) / (t1 - t0) if hi > lo else 0.0


def gaussian_integral(lo: float, hi: float, c: float, s: float) -> float:
    r2 = math.sqrt(2.0)
    return s * math.sqrt(math.pi / 2.0) * (math.erf((hi - c) / (r2 * s)) -
                                           math.erf((lo - c) / (r2 * s)))


class SineModes:
    """Implicit-Euler solves of the interior five-point Laplacian (Dirichlet
    zero on the grid edges) in the sine basis (validate_level2.py:108-145)."""

    def __init__(self, nx: int, ny: int, dx: float, dy: float, coefficient: float):
        mx, my = nx - 2, ny - 2
        kx, ky = np.arange(1, mx + 1, dtype=float), np.arange(1, my + 1, dtype=float)
        self.sx = np.sin(math.pi * np.outer(kx, kx) / (mx + 1))
        self.sy = np.sin(math.pi * np.outer(ky, ky) / (my + 1))
        lx = 4.0 / dx**2 * np.sin(math.pi * kx / (2.0 * (mx + 1))) ** 2
        ly = 4.0 / dy**2 * np.sin(math.pi * ky / (2.0 * (my + 1))) ** 2
        self.denominator = 1.0 + coefficient * (lx[:, None] + ly[None, :])
        self.scale = 2.0 / (mx + 1) * 2.0 / (my + 1)

    def forward(self, f: np.ndarray) -> np.ndarray:
        return self.scale * (self.sx.T @ f @ self.sy)

    def inverse(self, c: np.ndarray) -> np.ndarray:
        return self.sx @ c @ self.sy.T


def fd_fields(params: dict) -> np.ndarray:
    """FD temperature rise at every step, shape (steps + 1, nx, ny), of a
    level-2 parameter set (wos_transient_params fields as a dict)."""
    nx, ny, dt = params["nx"], params["ny"], params["dt"]
    steps = int(round(params["total_time"] / dt))
    x0, y0 = params["plate_x0"], params["plate_y0"]
    lx, ly = params["length_x"], params["length_y"]
    x = np.linspace(x0, x0 + lx, nx)
    y = np.linspace(y0, y0 + ly, ny)
    kappa = params["conductivity"] / (params["density"] * params["specific_heat"])
    cx, cy = x0 + 0.5 * lx, y0 + 0.5 * ly
    sx, sy = params["sigma_x"], params["sigma_y"]
    absorbed = params["electrical_power"] * params["efficiency"]
    ix = gaussian_integral(x0, x0 + lx, cx, sx)
    iy = gaussian_integral(y0, y0 + ly, cy, sy)
    xx, yy = np.meshgrid(x[1:-1], y[1:-1], indexing="ij")
    q = absorbed / (params["thickness"] * ix * iy) * np.exp(
        -0.5 * (((xx - cx) / sx) ** 2 + ((yy - cy) / sy) ** 2))
    modes = SineModes(nx, ny, x[1] - x[0], y[1] - y[0], kappa * dt)
    rate = modes.forward(q / (params["density"] * params["specific_heat"]))
    c = np.zeros((nx - 2, ny - 2))
    out = np.zeros((steps + 1, nx, ny))
    for s in range(1, steps + 1):
        f = heating_fraction((s - 1) * dt, s * dt, params["heat_on_time"])
        c = (c + dt * f * rate) / modes.denominator
        out[s, 1:-1, 1:-1] = modes.inverse(c)
    return out


def level2_gates(fields: np.ndarray, standard_error: np.ndarray, params: dict,
                 max_steps_hits: int, reference: np.ndarray | None = None,
                 rmse_limit: float = 0.05, center_limit: float = 0.10) -> dict:
    """validate_level2.py:230-330 for the fields of one run (every step
    stored); returns the per-step figures and the list of failures."""
    if reference is None:
        reference = fd_fields(params)
    nx, ny = params["nx"], params["ny"]
    failures: list[str] = []
    if not np.isfinite(fields).all() or not np.isfinite(standard_error).all():
        failures.append("non-finite WoS values")
    if fields.min() < -1e-10:
        failures.append(f"negative temperature rise {fields.min():.3g}")
    if max_steps_hits != 0:
        failures.append("walks reached max_steps")
    dt = params["dt"]
    steps = fields.shape[0] - 1
    absorbed = params["electrical_power"] * params["efficiency"]
    energy = sum(absorbed * heating_fraction((s - 1) * dt, s * dt, params["heat_on_time"]) * dt
                 for s in range(1, steps + 1))
    if abs(energy - absorbed * params["heat_on_time"]) > 1e-10 * max(1.0, energy):
        failures.append("source energy mismatch")
    rows = []
    for s in range(1, steps + 1):
        err = fields[s, 1:-1, 1:-1] - reference[s, 1:-1, 1:-1]
        peak = float(reference[s].max())
        nrmse = float(np.sqrt(np.mean(err**2))) / peak if peak > 0 else 0.0
        centre = abs(float(fields[s, nx // 2, ny // 2] - reference[s, nx // 2, ny // 2]))
        ncentre = centre / peak if peak > 0 else 0.0
        cover = float(np.mean(np.abs(err) <= 3.0 * standard_error[s, 1:-1, 1:-1]))
        rows.append({"step": s, "normalized_rmse": nrmse, "normalized_center_error": ncentre,
                     "coverage_3se": cover})
        if nrmse > rmse_limit:
            failures.append(f"step {s}: normalized RMSE {nrmse:.3%}")
        if ncentre > center_limit:
            failures.append(f"step {s}: normalized centre error {ncentre:.3%}")
    return {"rows": rows, "failures": failures, "passed": not failures}
