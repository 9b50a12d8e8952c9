"""Generate the stationary plate golden fields from the REFERENCE's own program.

    make -C oracle ref        # builds oracle/_ref/wos_level1_ref from the reference sources
    python tests/golden/make_stationary_golden.py

oracle/_ref/wos_level1_ref is the reference's
apps/welding/src/level1_stationary_heat.cpp compiled where it lies (one rank).
It takes no options: it solves its built-in Level1Config case three times
(manufactured Poisson; finite-plate Gaussian with Green sampling; the same
with Green-source MIS) and writes CSV files with 17 significant digits under
data/ of its working directory.  This script runs it in a temporary
directory and stores, per case, the (nx, ny) fields <case>_mean, <case>_se,
<case>_variance, <case>_steps and the summary row as JSON <case>_summary in
stationary_golden.npz.  It takes about 80 s on one core.
"""
from __future__ import annotations

import csv
import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1].parent
OUT = Path(__file__).resolve().parent / "stationary_golden.npz"
EXE = ROOT / "oracle" / "_ref" / "wos_level1_ref"

# case -> (field CSV stem, field column of the temperature rise)
CASES = {
    "manufactured": ("level1_manufactured", "temperature_rise"),
    "gaussian": ("level1_gaussian", "temperature_rise"),
    "gaussian_mis": ("level1_gaussian_mis", "temperature_rise"),
}


def read_field(path: Path, column: str) -> dict[str, np.ndarray]:
    rows = list(csv.DictReader(open(path)))
    xs = sorted({float(r["x"]) for r in rows})
    ys = sorted({float(r["y"]) for r in rows})
    shape = (len(xs), len(ys))
    out = {k: np.zeros(shape) for k in ("mean", "se", "variance", "steps")}
    for r in rows:
        i, j = xs.index(float(r["x"])), ys.index(float(r["y"]))
        out["mean"][i, j] = float(r[column])
        out["se"][i, j] = float(r["standard_error"])
        out["variance"][i, j] = float(r["variance"])
        out["steps"][i, j] = float(r["mean_steps"])
    return out


def main() -> None:
    arrays = {}
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.run([str(EXE)], cwd=tmp, check=True, capture_output=True)
        data = Path(tmp) / "data"
        for case, (stem, column) in CASES.items():
            for k, v in read_field(data / f"{stem}_field.csv", column).items():
                arrays[f"{case}_{k}"] = v
            row = next(csv.DictReader(open(data / f"{stem}_summary.csv")))
            arrays[f"{case}_summary"] = np.array(json.dumps({k: float(v) for k, v in row.items()}))
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
