"""Transient solver host logic (no GPU): the reference's defaults and
parameter checks through the C ABI, and the golden fields' layout."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np

from walk_on_spheres_b200 import _lib
from walk_on_spheres_b200.transient import defaults, make_params

GOLDEN = Path(__file__).resolve().parent / "golden" / "transient_golden.npz"


def test_defaults_are_the_reference_level2_config():
    d = defaults()
    # Level2Config, apps/welding/src/level2_transient_heat.cpp:46-78
    want = dict(nx=49, ny=33, walks=500, max_steps=1000, cubic=1, dt=0.1, total_time=10.0,
                heat_on_time=3.0, epsilon=8e-6, seed=20260819, length_x=0.12, length_y=0.08,
                thickness=0.006, conductivity=35.0, density=7800.0, specific_heat=600.0,
                electrical_power=800.0, efficiency=0.75, sigma_x=0.006, sigma_y=0.006)
    for k, v in want.items():
        assert d[k] == v, k


def test_step_count_and_checks():
    L = _lib.lib()
    steps = lambda **kw: L.wos_transient_steps(C.byref(make_params(**kw)))  # noqa: E731
    assert steps() == 100
    assert steps(dt=0.25, total_time=1.0, heat_on_time=0.5) == 4
    assert steps(nx=10) == -1                 # even grid
    assert steps(ny=1) == -1
    assert steps(heat_on_time=10.0) == -1     # not before the end
    assert steps(dt=0.3, total_time=1.0, heat_on_time=0.5) == -1  # not a multiple
    assert steps(epsilon=0.05) == -1          # too large for the plate
    assert steps(efficiency=1.5) == -1


def test_golden_fields_layout():
    g = np.load(GOLDEN)
    for k in g.files:
        if not k.endswith("_config"):
            continue
        name, cfg = k[:-len("_config")], json.loads(str(g[k]))
        rise, steps = g[f"{name}_rise"], g[f"{name}_steps"]
        assert rise.shape[0] == steps.shape[0] and steps[0] == 0
        # zero temperature rise on the plate edges at every step
        assert np.all(rise[:, 0, :] == 0.0) and np.all(rise[:, -1, :] == 0.0)
        assert np.all(rise[:, :, 0] == 0.0) and np.all(rise[:, :, -1] == 0.0)
        c = (rise.shape[1] // 2, rise.shape[2] // 2)
        if cfg["level"] == 0:
            # cooling: the centre starts at sin(pi/2)^2 = 1 and decays
            assert abs(rise[0][c] - 1.0) < 1e-6 and rise[-1][c] < rise[0][c]
        else:
            assert np.all(rise[0] == 0.0) and rise[-1][c] > 0.0


def test_level_presets_are_valid():
    from walk_on_spheres_b200.transient import LEVEL0, LEVEL3, level0_initial
    L = _lib.lib()
    assert L.wos_transient_steps(C.byref(make_params(**LEVEL0))) == 5
    assert L.wos_transient_steps(C.byref(make_params(**LEVEL3))) == 150
    f = level0_initial()
    assert f.shape == (17, 17) and abs(f[8, 8] - 1.0) < 1e-15 and f[0].max() == 0.0
