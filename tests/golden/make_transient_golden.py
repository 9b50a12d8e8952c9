"""Generate the transient golden fields from the REFERENCE's own programs.

    make -C oracle ref        # builds oracle/_ref/wos_level{0,2,3}_ref from the reference sources
    python tests/golden/make_transient_golden.py

oracle/_ref/wos_level{0,2,3}_ref are the reference's apps/welding/src/
level0_cooling.cpp, level2_transient_heat.cpp and level3_moving_heat.cpp
compiled where they lie (one rank, no OpenMP).  Each case of CASES runs one
of them and stores the fields it writes to its history CSV as
<case>_rise / <case>_se arrays of shape (steps stored, nx, ny), the stored
step numbers as <case>_steps and the options as <case>_config, in
transient_golden.npz.  Level 2 and 3 print 17 significant digits, level 0
six.
"""
from __future__ import annotations

import csv
import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent
BIN = ROOT / "oracle" / "_ref"

# name -> (program level, command-line options, steps to store or None for all)
CASES = {
    "level2_cubic_9x7": (2, dict(nx=9, ny=7, dt=0.5, total_time=2.5, heat_on_time=1.0,
                                 walks=60, seed=5, cubic=1), None),
    "level2_bilinear_11x9": (2, dict(nx=11, ny=9, dt=0.25, total_time=1.0, heat_on_time=0.5,
                                     walks=40, seed=77, cubic=0), None),
    "level0_17": (0, dict(grid=17, steps=5, dt=0.01, diffusivity=1.0, walks=200,
                          epsilon=1e-3, seed=12345), None),
    "level3_97x65": (3, dict(walks=2, seed=20260819), [0, 1, 2, 50, 150]),
}


def command(level: int, opts: dict, prefix: Path) -> list[str]:
    exe = str(BIN / f"wos_level{level}_ref")
    if level == 0:
        return [exe, "--grid", str(opts["grid"]), "--steps", str(opts["steps"]),
                "--dt", str(opts["dt"]), "--diffusivity", str(opts["diffusivity"]),
                "--walks", str(opts["walks"]), "--epsilon", str(opts["epsilon"]),
                "--seed", str(opts["seed"]), "--output", str(prefix) + ".csv"]
    if level == 2:
        return [exe, "--nx", str(opts["nx"]), "--ny", str(opts["ny"]), "--dt", str(opts["dt"]),
                "--total-time", str(opts["total_time"]),
                "--heat-on-time", str(opts["heat_on_time"]), "--walks", str(opts["walks"]),
                "--seed", str(opts["seed"]),
                "--history-interpolation", "cubic" if opts["cubic"] else "bilinear",
                "--output-prefix", str(prefix)]
    return [exe, "--walks", str(opts["walks"]), "--seed", str(opts["seed"]),
            "--output-prefix", str(prefix)]


def read_history(path: Path, value_column: str, keep) -> dict[int, tuple]:
    fields: dict[int, list] = {}
    with open(path) as f:
        for r in csv.DictReader(f):
            s = int(r["step"])
            if keep is not None and s not in keep:
                continue
            fields.setdefault(s, []).append((float(r[value_column]),
                                             float(r["standard_error"])))
    return fields


def run_case(level: int, opts: dict, keep, workdir: Path):
    prefix = workdir / f"level{level}"
    subprocess.run(command(level, opts, prefix), check=True, capture_output=True)
    if level == 0:
        nx = ny = opts["grid"]
        hist = read_history(Path(str(prefix) + "_history.csv"), "numerical", keep)
    else:
        nx, ny = (opts["nx"], opts["ny"]) if level == 2 else (97, 65)
        hist = read_history(Path(str(prefix) + "_history.csv"), "temperature_rise", keep)
    steps = sorted(hist)
    rise = np.array([[v for v, _ in hist[s]] for s in steps]).reshape(len(steps), nx, ny)
    se = np.array([[e for _, e in hist[s]] for s in steps]).reshape(len(steps), nx, ny)
    return np.array(steps), rise, se


def main() -> int:
    g = {}
    with tempfile.TemporaryDirectory() as d:
        for name, (level, opts, keep) in CASES.items():
            steps, rise, se = run_case(level, opts, keep, Path(d))
            g[f"{name}_steps"] = steps
            g[f"{name}_rise"] = rise
            g[f"{name}_se"] = se
            g[f"{name}_config"] = np.array(json.dumps({"level": level, **opts}))
    np.savez_compressed(OUT / "transient_golden.npz", **g)
    print(f"wrote {OUT / 'transient_golden.npz'} ({len(g)} arrays)")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
