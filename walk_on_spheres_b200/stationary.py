"""Stationary plate heating (wos_stationary_* in include/wos_b200.h): the
reference's welding level 1 (apps/welding/src/level1_stationary_heat.cpp)
on the GPU.

    from walk_on_spheres_b200 import Solver
    from walk_on_spheres_b200.stationary import solve_stationary, gaussian_summary
    r = solve_stationary(Solver(0), source="gaussian", source_mode="mis")
    r.mean                  # temperature rise on the (nx, ny) grid, kelvin
    gaussian_summary(r)     # the reference's level-1 summary row

The three solves of the reference program are LEVEL1_CASES: the
manufactured Poisson problem (exact solution peak_rise sin(pi x/Lx)
sin(pi y/Ly)), and the finite-plate Gaussian heat source with Green and
with Green-source MIS sampling.  PLAIN_FP64 follows the reference's seeds
and streams.  The summary functions restate the reference's reporting
(manufactured_error :301-323, find_peak :402-420, symmetry_summary
:428-461, integrated_power_midpoint gaussian_heat_source.hpp:75-92).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .solver import METHODS, SOURCE_MODES, Solver, _enum, _ptr

SOURCES = {"manufactured": 0, "gaussian": 1}

LEVEL1_CASES = {
    "manufactured": dict(source="manufactured", source_mode="green"),
    "gaussian": dict(source="gaussian", source_mode="green"),
    "gaussian_mis": dict(source="gaussian", source_mode="mis"),
}
"""The reference program's three solves (level1_stationary_heat.cpp:591-650):
each with the Level1Config defaults and its own case stream."""


def make_params(source: str = "gaussian", **kw) -> _lib.StationaryParams:
    p = _lib.StationaryParams()
    _lib.lib().wos_stationary_defaults(C.byref(p), _enum(source, SOURCES, "source"))
    for k, v in kw.items():
        if k == "method":
            v = _enum(v, METHODS, "method")
        elif k == "source_mode":
            v = _enum(v, SOURCE_MODES, "source_mode")
        if not hasattr(p, k) or k == "source":
            raise TypeError(f"unknown stationary parameter {k!r}")
        setattr(p, k, v)
    return p


def defaults(source: str = "gaussian") -> dict:
    """The reference's Level1Config for `source` as a dict (plus method = "fast")."""
    p = make_params(source)
    d = {k: getattr(p, k) for k, _ in _lib.StationaryParams._fields_}
    d["method"] = "fast"
    return d


@dataclass
class StationaryResult:
    mean: np.ndarray            # (nx, ny) temperature rise
    variance: np.ndarray
    standard_error: np.ndarray
    mean_steps: np.ndarray
    max_steps_hits: int
    device_ms: float
    params: dict = field(repr=False)

    @property
    def x(self) -> np.ndarray:
        return grid_coordinates(0.0, self.params["length_x"], self.params["nx"])

    @property
    def y(self) -> np.ndarray:
        return grid_coordinates(0.0, self.params["length_y"], self.params["ny"])


def grid_coordinates(lo: float, hi: float, n: int) -> np.ndarray:
    """wos::grid_coordinate (include/wos/grid.hpp:12-18) for every index."""
    if n <= 1:
        return np.array([lo] * max(n, 0), dtype=np.float64)
    return np.array([lo + (hi - lo) * float(i) / float(n - 1) for i in range(n)])


def solve_stationary(solver: Solver, source: str = "gaussian", **kw) -> StationaryResult:
    """One stationary plate solve; keyword arguments override the Level1Config
    defaults (nx, ny, walks, epsilon, seed, source_mode, method, ...)."""
    L = solver._L
    p = make_params(source, **kw)
    shape = (max(p.nx, 0), max(p.ny, 0))
    out = [np.zeros(shape) for _ in range(4)]
    hits = C.c_longlong()
    ms = C.c_float()
    solver._check(L.wos_stationary_solve(solver._ctx, C.byref(p), *[_ptr(a) for a in out],
                                         C.byref(hits), C.byref(ms)))
    params = {k: getattr(p, k) for k, _ in _lib.StationaryParams._fields_}
    return StationaryResult(*out, hits.value, ms.value, params)


# ------------------------------------------------------ the reference's reports

def _interior(a: np.ndarray) -> np.ndarray:
    return a[1:-1, 1:-1]


def exact_manufactured(params: dict) -> np.ndarray:
    """ManufacturedPoisson2D::exact on the grid (:89-92)."""
    x = grid_coordinates(0.0, params["length_x"], params["nx"])
    y = grid_coordinates(0.0, params["length_y"], params["ny"])
    return params["peak_rise"] * np.outer(np.sin(np.pi * x / params["length_x"]),
                                          np.sin(np.pi * y / params["length_y"]))


def manufactured_summary(r: StationaryResult) -> dict:
    """The level-1A summary row (write_manufactured_outputs, :339-380)."""
    p = r.params
    err = _interior(r.mean - exact_manufactured(p))
    ci, cj = p["nx"] // 2, p["ny"] // 2
    return {
        "center_mean": float(r.mean[ci, cj]),
        "center_standard_error": float(r.standard_error[ci, cj]),
        "center_exact": float(p["peak_rise"]),
        "center_absolute_error": abs(float(r.mean[ci, cj]) - p["peak_rise"]),
        "field_rmse": float(np.sqrt(np.mean(err * err))),
        "field_max_absolute_error": float(np.max(np.abs(err))),
        "mean_standard_error": float(np.mean(_interior(r.standard_error))),
        "max_standard_error": float(np.max(_interior(r.standard_error))),
        "mean_steps": float(np.mean(_interior(r.mean_steps))),
        "max_steps_hits": r.max_steps_hits,
    }


def gaussian_integral(lower: float, upper: float, centre: float, sigma: float) -> float:
    """GaussianHeatSource2D::gaussian_integral (gaussian_heat_source.hpp:112-123)."""
    import math
    s2 = 1.41421356237309504880168872420969808
    return sigma * 1.25331413731550025120788264240552263 * (
        math.erf((upper - centre) / (s2 * sigma)) - math.erf((lower - centre) / (s2 * sigma)))


def volumetric_power_density(params: dict, x, y):
    """GaussianHeatSource2D::volumetric_power_density (:38-41), vectorised."""
    ix = gaussian_integral(0.0, params["length_x"], params["source_x"], params["sigma_x"])
    iy = gaussian_integral(0.0, params["length_y"], params["source_y"], params["sigma_y"])
    dx = (np.asarray(x) - params["source_x"]) / params["sigma_x"]
    dy = (np.asarray(y) - params["source_y"]) / params["sigma_y"]
    absorbed = params["electrical_power"] * params["efficiency"]
    return absorbed * np.exp(-0.5 * (dx * dx + dy * dy)) / (params["thickness"] * ix * iy)


def integrated_power_midpoint(params: dict, nx: int = 800, ny: int = 600) -> float:
    """thickness x the midpoint rule of q over the plate (gaussian_heat_source.hpp:75-92)."""
    dx = params["length_x"] / nx
    dy = params["length_y"] / ny
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dy
    q = volumetric_power_density(params, x[:, None], y[None, :])
    return float(params["thickness"] * np.cumsum(q.ravel())[-1] * dx * dy)


def gaussian_summary(r: StationaryResult) -> dict:
    """The level-1B summary row (write_gaussian_outputs, :463-546)."""
    p = r.params
    x, y = r.x, r.y
    inner = _interior(r.mean)
    k = int(np.argmax(inner))       # first maximum in (i, j) order, as find_peak
    pi, pj = k // inner.shape[1] + 1, k % inner.shape[1] + 1
    peak = float(r.mean[pi, pj])
    absorbed = p["electrical_power"] * p["efficiency"]
    power = integrated_power_midpoint(p)
    # symmetry_summary: every point against its x and y mirrors
    se = r.standard_error
    d = np.stack([np.abs(r.mean - r.mean[::-1, :]), np.abs(r.mean - r.mean[:, ::-1])], axis=-1)
    c = np.stack([np.hypot(se, se[::-1, :]), np.hypot(se, se[:, ::-1])], axis=-1)
    ok = (d <= 3.0 * c) | ((d == 0.0) & (c == 0.0))
    return {
        "absorbed_power": absorbed,
        "integrated_power": power,
        "power_relative_error": abs(power - absorbed) / absorbed,
        "peak_temperature_rise": peak,
        "peak_x": float(x[pi]),
        "peak_y": float(y[pj]),
        "peak_standard_error": float(r.standard_error[pi, pj]),
        "symmetry_max_relative_residual": float(d.max()) / peak,
        "symmetry_rms_relative_residual": float(np.sqrt(np.mean(d * d))) / peak,
        "symmetry_within_three_standard_errors_fraction": float(ok.mean()),
        "mean_standard_error": float(np.mean(_interior(r.standard_error))),
        "max_standard_error": float(np.max(_interior(r.standard_error))),
        "mean_steps": float(np.mean(_interior(r.mean_steps))),
        "max_steps_hits": r.max_steps_hits,
    }
