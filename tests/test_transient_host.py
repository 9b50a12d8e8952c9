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


def test_fd_reference_modes_match_a_dense_solve():
    # the sine-mode implicit step equals a dense solve of
    # (I - c Lap_h) u = rhs with u = 0 on the grid edges
    from oracle.fd_transient import SineModes
    nx, ny, dx, dy, c = 9, 7, 0.1, 0.07, 0.03
    mx, my = nx - 2, ny - 2
    A = np.zeros((mx * my, mx * my))
    for i in range(mx):
        for j in range(my):
            r = i * my + j
            A[r, r] = 1.0 + c * (2.0 / dx**2 + 2.0 / dy**2)
            for di, dj, h in ((1, 0, dx), (-1, 0, dx), (0, 1, dy), (0, -1, dy)):
                ii, jj = i + di, j + dj
                if 0 <= ii < mx and 0 <= jj < my:
                    A[r, ii * my + jj] -= c / h**2
    rhs = np.random.default_rng(3).random((mx, my))
    want = np.linalg.solve(A, rhs.ravel()).reshape(mx, my)
    m = SineModes(nx, ny, dx, dy, c)
    got = m.inverse(m.forward(rhs) / m.denominator)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-13)


def test_fd_reference_heats_then_cools():
    # level-2 defaults: the FD field rises while the source is on and decays
    # after; the energy injected is the absorbed power times heat_on_time
    from oracle.fd_transient import fd_fields, heating_fraction
    p = defaults()
    f = fd_fields(p)
    steps = f.shape[0] - 1
    on = int(round(p["heat_on_time"] / p["dt"]))
    c = (p["nx"] // 2, p["ny"] // 2)
    assert f[on][c] > f[on // 2][c] > 0.0 and f[steps][c] < f[on][c]
    assert np.all(f[:, 0, :] == 0.0) and np.all(f[:, :, -1] == 0.0)
    absorbed = p["electrical_power"] * p["efficiency"]
    energy = sum(absorbed * heating_fraction((s - 1) * p["dt"], s * p["dt"], p["heat_on_time"])
                 * p["dt"] for s in range(1, steps + 1))
    assert abs(energy - absorbed * p["heat_on_time"]) < 1e-9


def test_fd_moving_reference_follows_the_source():
    # level-3 configuration: while the source is on, the FD peak rides on the
    # weld line behind the source centre x(t) = -0.05 + 0.02 t and advances
    # with it; after switch-off (5 s) the peak falls every step
    from oracle.fd_transient import fd_fields_moving
    from walk_on_spheres_b200.transient import LEVEL3
    p = dict(defaults())
    p.update(LEVEL3)
    f = fd_fields_moving(p, refinement=2, substeps=4)
    x = np.linspace(p["plate_x0"], p["plate_x0"] + p["length_x"], p["nx"])
    y = np.linspace(p["plate_y0"], p["plate_y0"] + p["length_y"], p["ny"])
    peak_x = []
    for s in (10, 25, 40):
        i, j = np.unravel_index(int(np.argmax(f[s])), f[s].shape)
        centre = p["source_start_x"] + p["weld_speed"] * s * p["dt"]
        assert abs(y[j] - p["weld_y"]) < 1e-12
        assert centre - 0.02 <= x[i] <= centre + 1e-12, (s, x[i], centre)
        peak_x.append(x[i])
    # 3 s apart the source moves 60 mm; the peak follows, its lag growing as
    # the thermal wake builds up (9 mm at 1 s, 12.5 mm at 2.5 s)
    assert 0.8 * 0.06 <= peak_x[2] - peak_x[0] <= 0.06 + (x[1] - x[0]), peak_x
    on = int(round(p["heat_on_time"] / p["dt"]))
    peaks = f[on + 1:].max(axis=(1, 2))
    assert np.all(np.diff(peaks) < 0.0)
    assert np.all(f[:, 0, :] == 0.0) and np.all(f[:, :, 0] == 0.0)
