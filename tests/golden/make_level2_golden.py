"""Generate the transient golden fields from the REFERENCE's own program.

    make -C oracle ref        # builds oracle/_ref/wos_level2_ref from the reference sources
    python tests/golden/make_level2_golden.py

oracle/_ref/wos_level2_ref is the reference's apps/welding/src/
level2_transient_heat.cpp compiled where it lies (one rank, no OpenMP).  It
is run on small configurations (LEVEL2_CASES) and the fields it writes to
its history CSV (17 significant digits, every step) are stored, per case,
as <case>_rise and <case>_se arrays of shape (steps + 1, nx, ny) in
level2_golden.npz, with the configuration beside them.
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
BIN = ROOT / "oracle" / "_ref" / "wos_level2_ref"

# name -> command-line options of the reference program
LEVEL2_CASES = {
    "cubic_9x7": dict(nx=9, ny=7, dt=0.5, total_time=2.5, heat_on_time=1.0, walks=60,
                      seed=5, cubic=1),
    "bilinear_11x9": dict(nx=11, ny=9, dt=0.25, total_time=1.0, heat_on_time=0.5, walks=40,
                          seed=77, cubic=0),
}


def run_case(opts: dict, workdir: Path) -> tuple[np.ndarray, np.ndarray]:
    prefix = workdir / "case"
    cmd = [str(BIN), "--nx", str(opts["nx"]), "--ny", str(opts["ny"]), "--dt", str(opts["dt"]),
           "--total-time", str(opts["total_time"]), "--heat-on-time", str(opts["heat_on_time"]),
           "--walks", str(opts["walks"]), "--seed", str(opts["seed"]),
           "--history-interpolation", "cubic" if opts["cubic"] else "bilinear",
           "--output-prefix", str(prefix)]
    subprocess.run(cmd, check=True, capture_output=True)
    steps = int(round(opts["total_time"] / opts["dt"]))
    rise = np.full((steps + 1, opts["nx"], opts["ny"]), np.nan)
    se = np.full_like(rise, np.nan)
    with open(str(prefix) + "_history.csv") as f:
        rows = list(csv.DictReader(f))
    per_step = opts["nx"] * opts["ny"]
    for s in range(steps + 1):
        block = [r for r in rows if int(r["step"]) == s]
        assert len(block) == per_step, (s, len(block))
        # rows are written in (i, j) order, j fastest
        rise[s] = np.array([float(r["temperature_rise"]) for r in block]).reshape(
            opts["nx"], opts["ny"])
        se[s] = np.array([float(r["standard_error"]) for r in block]).reshape(
            opts["nx"], opts["ny"])
    return rise, se


def main() -> int:
    g = {}
    with tempfile.TemporaryDirectory() as d:
        for name, opts in LEVEL2_CASES.items():
            rise, se = run_case(opts, Path(d))
            g[f"{name}_rise"] = rise
            g[f"{name}_se"] = se
            g[f"{name}_config"] = np.array(json.dumps(opts))
    np.savez_compressed(OUT / "level2_golden.npz", **g)
    print(f"wrote {OUT / 'level2_golden.npz'} ({len(g)} arrays)")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
