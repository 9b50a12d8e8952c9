"""Transient plate heating (wos_transient_* in include/wos_b200.h): the
reference's welding time loops on the GPU -- scenario 0, cooling
(apps/welding/src/level0_cooling.cpp), scenario 2, a stationary Gaussian
source (level2_transient_heat.cpp, the default), scenario 3, a moving
Gaussian source (level3_moving_heat.cpp).

    from walk_on_spheres_b200 import Solver
    from walk_on_spheres_b200.transient import solve_transient
    r = solve_transient(Solver(0), method="fast", walks=500)   # reference defaults otherwise
    r.fields[-1]            # final temperature rise on the (nx, ny) grid, kelvin
    r.standard_error[-1]

Every implicit-Euler step is one screened walk-on-spheres solve whose source
samples the previous step's field; the whole time loop runs as one launch
sequence (one CUDA graph with use_graph=True).  PLAIN_FP64 follows the
reference's seeds and streams step by step.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .solver import METHODS, Solver, _enum, _ptr


def defaults() -> dict:
    """The reference's Level2Config defaults as a dict (plus method = "fast")."""
    p = _lib.TransientParams()
    _lib.lib().wos_transient_defaults(C.byref(p))
    d = {k: getattr(p, k) for k, _ in _lib.TransientParams._fields_}
    d["method"] = "fast"
    return d


LEVEL0 = dict(scenario=0, nx=17, ny=17, dt=0.01, total_time=0.05, walks=2000,
              epsilon=1e-3, seed=12345, cubic=0, length_x=1.0, length_y=1.0, plate_x0=0.0,
              plate_y0=0.0, conductivity=1.0, density=1.0, specific_heat=1.0)
"""The reference's level-0 options (level0_cooling.cpp:37-47): unit square,
diffusivity 1, 5 steps of 0.01, bilinear history."""

LEVEL3 = dict(scenario=3, nx=97, ny=65, dt=0.1, total_time=15.0, heat_on_time=5.0,
              source_start_x=-0.05, weld_y=0.0, weld_speed=0.02, cubic=1)
"""The reference's level-3 configuration (Level3Config, level3_moving_heat.cpp:
44-76): heat_on_time is its heat_off_time."""


def level0_initial(nx: int = 17, ny: int = 17) -> np.ndarray:
    """sin(pi x) sin(pi y) on the interior of the unit-square grid, 0 on its edges
    (level0_cooling.cpp:177-179, 270-283)."""
    x = np.array([(i / (nx - 1)) for i in range(nx)])
    y = np.array([(j / (ny - 1)) for j in range(ny)])
    f = np.outer(np.sin(np.pi * x), np.sin(np.pi * y))
    f[0, :] = f[-1, :] = 0.0
    f[:, 0] = f[:, -1] = 0.0
    return f


def make_params(**kw) -> _lib.TransientParams:
    p = _lib.TransientParams()
    _lib.lib().wos_transient_defaults(C.byref(p))
    if ("length_x" in kw or "length_y" in kw) and "plate_x0" not in kw:
        kw.setdefault("plate_x0", -0.5 * kw.get("length_x", p.length_x))
        kw.setdefault("plate_y0", -0.5 * kw.get("length_y", p.length_y))
    for k, v in kw.items():
        if k == "method":
            v = _enum(v, METHODS, "method")
        elif k == "cubic":
            v = int(bool(v))
        if not hasattr(p, k):
            raise TypeError(f"unknown transient parameter {k!r}")
        setattr(p, k, v)
    return p


@dataclass
class TransientResult:
    fields: np.ndarray          # (steps + 1, nx, ny) temperature rise
    standard_error: np.ndarray  # (steps + 1, nx, ny)
    max_steps_hits: int
    device_ms: float
    steps: int


def solve_transient(solver: Solver, use_graph: bool = True, initial=None,
                    **kw) -> TransientResult:
    """Run a transient problem; `initial` is the (nx, ny) field at time 0 (zeros if
    None); keyword arguments override the level-2 defaults (see LEVEL0, LEVEL3)."""
    L = solver._L
    p = make_params(**kw)
    init = None
    if initial is not None:
        init = np.ascontiguousarray(initial, dtype=np.float64)
        if init.shape != (p.nx, p.ny):
            raise ValueError(f"initial field must have shape ({p.nx}, {p.ny})")
    steps = L.wos_transient_steps(C.byref(p))
    if steps < 0:
        # let the library report the reason
        steps = 0
    shape = (steps + 1, p.nx, p.ny)
    fields = np.empty(shape)
    se = np.empty(shape)
    hits = C.c_longlong()
    ms = C.c_float()
    solver._check(L.wos_transient_solve(solver._ctx, C.byref(p), _ptr(init), int(bool(use_graph)),
                                        _ptr(fields), _ptr(se), C.byref(hits), C.byref(ms)))
    return TransientResult(fields, se, hits.value, ms.value, steps)
