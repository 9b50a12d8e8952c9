"""Finite-difference references of the transient plate problems (welding
levels 2 and 3) and the reference's validation gates.  TEST INFRASTRUCTURE
ONLY: the oracle of the transient solver, never part of the product path.

Level 3 (moving source): fd_fields_moving / level3_gates restate
apps/welding/tools/validate_level3.py:133-420 (below).

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


# ---------------------------------------------------------------- level 3

# the program's fixed probes (level3_moving_heat.cpp:85-93): name, x, y
LEVEL3_PROBES = (("centreline_m20", -0.020, 0.000), ("centreline_m10", -0.010, 0.000),
                 ("centreline_0", 0.000, 0.000), ("centreline_p10", 0.010, 0.000),
                 ("centreline_p20", 0.020, 0.000), ("transverse_p5", 0.000, 0.005),
                 ("transverse_p10", 0.000, 0.010))


def fd_fields_moving(params: dict, refinement: int = 4, substeps: int = 16) -> np.ndarray:
    """FD temperature rise of the moving-source problem at the WoS nodes of
    every step, shape (steps + 1, nx, ny) (validate_level3.py:133-240): a
    grid refined `refinement` times, `substeps` implicit steps per WoS step,
    the source sampled at each substep's midpoint while it is on."""
    nx, ny, dt = params["nx"], params["ny"], params["dt"]
    steps = int(round(params["total_time"] / dt))
    x0, y0 = params["plate_x0"], params["plate_y0"]
    lx, ly = params["length_x"], params["length_y"]
    rnx, rny = (nx - 1) * refinement + 1, (ny - 1) * refinement + 1
    rx, ry = np.linspace(x0, x0 + lx, rnx), np.linspace(y0, y0 + ly, rny)
    heat_capacity = params["density"] * params["specific_heat"]
    kappa = params["conductivity"] / heat_capacity
    rdt = dt / substeps
    modes = SineModes(rnx, rny, rx[1] - rx[0], ry[1] - ry[0], kappa * rdt)
    sx, sy = params["sigma_x"], params["sigma_y"]
    wy = params["weld_y"]
    absorbed = params["electrical_power"] * params["efficiency"]
    iy = gaussian_integral(y0, y0 + ly, wy, sy)
    proj_y = modes.sy.T @ np.exp(-0.5 * ((ry[1:-1] - wy) / sy) ** 2)
    c = np.zeros((rnx - 2, rny - 2))
    out = np.zeros((steps + 1, nx, ny))
    for s in range(1, steps + 1):
        for k in range(substeps):
            tm = (s - 1) * dt + (k + 0.5) * rdt
            if tm < params["heat_on_time"]:
                cx = params["source_start_x"] + params["weld_speed"] * tm
                ix = gaussian_integral(x0, x0 + lx, cx, sx)
                proj_x = modes.sx.T @ np.exp(-0.5 * ((rx[1:-1] - cx) / sx) ** 2)
                amp = absorbed / (params["thickness"] * ix * iy * heat_capacity)
                c = (c + rdt * modes.scale * amp * np.outer(proj_x, proj_y)) / modes.denominator
            else:
                c = c / modes.denominator
        fine = np.zeros((rnx, rny))
        fine[1:-1, 1:-1] = modes.inverse(c)
        out[s] = fine[::refinement, ::refinement]
    return out


def level3_gates(fields: np.ndarray, standard_error: np.ndarray, params: dict,
                 max_steps_hits: int, reference: np.ndarray | None = None,
                 rmse_limit: float = 0.01, peak_limit: float = 0.02,
                 statistical_argmax: bool = False) -> dict:
    """validate_level3.py:330-420 for the fields of one run (every step):
    per step normalised RMSE <= 1%, peak within 2% and at most one cell from
    the reference peak; per probe the peak rise within max(5 K, 2%) and its
    time within one step; no negative rise, no walk at the step cap.

    With statistical_argmax the two argmax gates (peak cell, probe peak
    time) fail only when the run's value at the reference's argmax lies more
    than 3 standard errors below the run's maximum.  Where the field is flat
    near its peak (late cooling, the 10 mm transverse probe), values a cell
    or a few steps apart differ by less than the Monte Carlo error at 500
    walks, so the argmax itself is noise."""
    if reference is None:
        reference = fd_fields_moving(params)
    nx, ny, dt = params["nx"], params["ny"], params["dt"]
    x = np.linspace(params["plate_x0"], params["plate_x0"] + params["length_x"], nx)
    y = np.linspace(params["plate_y0"], params["plate_y0"] + params["length_y"], ny)
    gate = max(x[1] - x[0], y[1] - y[0]) + 1e-12
    failures: list[str] = []
    if fields[:, 1:-1, 1:-1].min() < 0.0:
        failures.append("negative interior temperature rise")
    if max_steps_hits != 0:
        failures.append("walks reached max_steps")
    rows = []
    for s in range(1, fields.shape[0]):
        err = fields[s, 1:-1, 1:-1] - reference[s, 1:-1, 1:-1]
        rpeak, wpeak = float(reference[s].max()), float(fields[s].max())
        nrmse = float(np.sqrt(np.mean(err**2))) / rpeak if rpeak > 0 else 0.0
        ri, rj = np.unravel_index(int(np.argmax(reference[s])), reference[s].shape)
        wi, wj = np.unravel_index(int(np.argmax(fields[s])), fields[s].shape)
        loc = float(np.hypot(x[wi] - x[ri], y[wj] - y[rj]))
        rel = abs(wpeak - rpeak) / rpeak if rpeak > 0 else 0.0
        rows.append({"step": s, "normalized_rmse": nrmse, "peak_relative_error": rel,
                     "peak_location_error": loc})
        if nrmse > rmse_limit:
            failures.append(f"step {s}: normalized RMSE {nrmse:.3%}")
        if rel > peak_limit:
            failures.append(f"step {s}: peak relative error {rel:.3%}")
        far = loc > gate
        if far and statistical_argmax:
            se2 = float(np.hypot(standard_error[s][wi, wj], standard_error[s][ri, rj]))
            far = fields[s][ri, rj] < wpeak - 3.0 * se2
        if far:
            failures.append(f"step {s}: peak location error {loc * 1e3:.3f} mm")
    probes = []
    for name, px, py in LEVEL3_PROBES:
        i, j = int(np.argmin(np.abs(x - px))), int(np.argmin(np.abs(y - py)))
        wc, rc = fields[:, i, j], reference[:, i, j]
        wf, rf = int(np.argmax(wc)), int(np.argmax(rc))
        perr = float(wc[wf] - rc[rf])
        terr = (wf - rf) * dt
        probes.append({"probe": name, "peak_error": perr, "peak_time_error": terr})
        if abs(perr) > max(5.0, 0.02 * float(rc[rf])):
            failures.append(f"{name}: probe peak error {perr:.3f} K")
        late = abs(terr) > dt + 1e-12
        if late and statistical_argmax:
            se2 = float(np.hypot(standard_error[wf, i, j], standard_error[rf, i, j]))
            late = wc[rf] < wc[wf] - 3.0 * se2
        if late:
            failures.append(f"{name}: probe peak-time error {terr:.3f} s")
    return {"rows": rows, "probes": probes, "failures": failures, "passed": not failures}
