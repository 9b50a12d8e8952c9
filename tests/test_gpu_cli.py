"""The drop-in end to end: `wos <equation> Nx Ny [Nz] mesh.obj` (PLAIN_FP64,
the default method) against the reference's registry entry run on the same
OBJ file (src/equations/<eq>.cpp run_2D/run_3D through include/wos/runner.hpp,
its HDF5 datasets captured in memory).  Location codes, coordinates and every
/metadata scalar must be equal.  The fields are held to the same PLAIN parity
bar as the grid tests: at least 98% of points to 1e-9 relative, all within
4 standard errors."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from walk_on_spheres_b200 import h5lite, meshes

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
WOS = ROOT / "walk_on_spheres_b200" / "bin" / "wos"

# (equation, mesh, grid, walks, seed, extra options, reference alpha, source mode)
CASES = {
    "annulus_laplace": ("laplace", lambda: meshes.annulus(segments=64), (12, 12), 300, 5, [],
                        5.0, 0),
    "circle_poisson_green": ("poisson", lambda: meshes.circle(segments=128), (10, 10), 300, 11,
                             ["--source-mode", "green"], 5.0, 1),
    "sphere_screened": ("screened_poisson", lambda: meshes.uv_sphere(lon=16, lat=8), (6, 6, 6),
                        120, 7, ["--alpha", "10"], 10.0, 0),
}

META_TYPES = {"N_walks": np.int32, "epsilon": np.float64, "max_steps": np.int32,
              "max_steps_hits": np.int64, "seed": np.uint64, "max_ray_attempts": np.int32,
              "ambiguous_ray_retries": np.int64, "indeterminate_points": np.int64,
              "alpha": np.float64, "source_mode": np.int32}


@pytest.mark.parametrize("name", sorted(CASES))
def test_cli_file_matches_reference_registry(tmp_path, reference, name):
    eq, mesh_fn, grid, walks, seed, extra, alpha, mode = CASES[name]
    mesh = mesh_fn()
    obj = meshes.write_obj(mesh, tmp_path / "mesh.obj")
    out = tmp_path / "ours.h5"
    args = [str(WOS), "--seed", str(seed), "--walks", str(walks), "-o", str(out), *extra, eq,
            *[str(v) for v in grid], str(obj)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    nz = grid[2] if len(grid) == 3 else 1
    ref = reference.run_registry(eq, mesh.dim, str(obj), grid[0], grid[1], nz, walks, 1e-2,
                                 1000, 12, seed, alpha, mode)
    ours = h5lite.read(out)
    shape = (grid[0], grid[1], nz)
    assert set(ours) == set(ref)
    loc = ref["/location"].view(np.uint8).reshape(shape)
    assert np.array_equal(ours["/location"], loc)
    for axis in ("/x", "/y", "/z"):
        assert np.array_equal(ours[axis], ref[axis].view(np.float64))
    for key, dtype in META_TYPES.items():
        name_ = "/metadata/" + key
        if name_ in ref:
            want = ref[name_].view(dtype)[0]
            assert ours[name_] == want and ours[name_].dtype == dtype, key
    ins = loc == 1
    mean = ref["/mean"].view(np.float64).reshape(shape)
    se = ref["/standard_error"].view(np.float64).reshape(shape)
    got = ours["/mean"]
    close = np.abs(got[ins] - mean[ins]) <= 1e-9 * np.maximum(1.0, np.abs(mean[ins]))
    assert close.mean() >= 0.98, close.mean()
    far = ~close
    if far.any():
        z = np.abs(got[ins][far] - mean[ins][far]) / np.maximum(se[ins][far], 1e-300)
        assert (z <= 4.0).all(), z.max()
    steps = ref["/mean_steps"].view(np.float64).reshape(shape)
    assert (np.abs(ours["/mean_steps"][ins] - steps[ins]) <= 1e-9 * steps[ins]).mean() >= 0.98
    assert np.isnan(got[(loc == 0) | (loc == 3)]).all()
    # the printed summary carries the reference's lines (runner.hpp:265-290)
    assert "Random seed: %d (fixed by --seed)" % seed in r.stdout
    lines = [line.strip() for line in r.stdout.splitlines()]
    assert "number of inside points:       %d" % int(ins.sum()) in lines
    hits = int(ref["/metadata/max_steps_hits"].view(np.int64)[0])
    assert "paths reaching max steps:      %d" % hits in lines
    if mesh.dim == 3:
        retries = int(ref["/metadata/ambiguous_ray_retries"].view(np.int64)[0])
        assert "ambiguous ray retries:         %d" % retries in lines


def test_cli_file_opens_with_libhdf5(tmp_path):
    """Where h5py (libhdf5) is installed, a `wos` result file opens with it and
    holds the datasets the library's own reader sees."""
    h5py = pytest.importorskip("h5py")
    obj = meshes.write_obj(meshes.annulus(segments=32), tmp_path / "mesh.obj")
    out = tmp_path / "ours.h5"
    r = subprocess.run([str(WOS), "--walks", "50", "-o", str(out), "laplace", "8", "8",
                        str(obj)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    ours = h5lite.read(out)
    with h5py.File(out, "r") as f:
        for key, value in ours.items():
            assert np.array_equal(np.asarray(f[key][()]), value, equal_nan=True), key
