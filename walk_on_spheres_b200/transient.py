"""Transient plate heating (wos_transient_* in include/wos_b200.h): the
reference's level-2 welding baseline (apps/welding/src/level2_transient_heat.cpp)
on the GPU.

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


def make_params(**kw) -> _lib.TransientParams:
    p = _lib.TransientParams()
    _lib.lib().wos_transient_defaults(C.byref(p))
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


def solve_transient(solver: Solver, use_graph: bool = True, **kw) -> TransientResult:
    L = solver._L
    p = make_params(**kw)
    steps = L.wos_transient_steps(C.byref(p))
    if steps < 0:
        # let the library report the reason
        steps = 0
    shape = (steps + 1, p.nx, p.ny)
    fields = np.empty(shape)
    se = np.empty(shape)
    hits = C.c_longlong()
    ms = C.c_float()
    solver._check(L.wos_transient_solve(solver._ctx, C.byref(p), int(bool(use_graph)),
                                        _ptr(fields), _ptr(se), C.byref(hits), C.byref(ms)))
    return TransientResult(fields, se, hits.value, ms.value, steps)
