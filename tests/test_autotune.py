"""Autotuner host logic (CPU) and a tuning run on the GPU."""
from __future__ import annotations

import numpy as np
import pytest

from walk_on_spheres_b200 import autotune, meshes, parallel


class _Grid:
    def __init__(self, nx, ny, nz, box):
        self.Nx, self.Ny, self.Nz = nx, ny, nz
        self.xmin, self.xmax, self.ymin, self.ymax, self.zmin, self.zmax = box


def test_pick_prefers_the_fastest_finite_row():
    rows = [{"chunk": 128, "walks_per_s": 1.0}, {"chunk": 256, "walks_per_s": float("nan")},
            {"chunk": 512, "walks_per_s": 3.0}, {"chunk": 1024, "walks_per_s": 3.0}]
    assert autotune.pick(rows)["chunk"] == 512
    with pytest.raises(RuntimeError):
        autotune.pick([{"walks_per_s": None}])


def test_problem_key_groups_by_octave():
    a = autotune.problem_key(3, 17000, "laplace", "fast", 1024)
    b = autotune.problem_key(3, 20000, "laplace", "fast", 1024)
    c = autotune.problem_key(3, 40000, "laplace", "fast", 1024)
    assert a == b != c


def test_sample_points_match_the_grid_formula():
    g = _Grid(5, 4, 3, (-1.0, 2.0, 0.0, 1.5, -0.5, 0.5))
    pts, idx = autotune.sample_points(g, 3, 10, seed=4)
    assert len(set(idx.tolist())) == 10
    for p, i in zip(pts, idx):
        assert p.tolist() == parallel.grid_points(g, 3, int(i), int(i) + 1)[0].tolist()


@pytest.mark.gpu
def test_tuner_picks_a_schedule_and_caches_it(solver, tmp_path):
    m = meshes.annulus()
    t = autotune.Tuner(solver, cache_path=str(tmp_path / "tune.json"),
                       chunks=(128, 512), leaf_sizes=(2, 4), block_factors=(0, 1))
    r = t.tune(m, "laplace", (32, 32, 1), N_walks=1024, seed=3, method="fast")
    assert r.chunk in (128, 512) and r.leaf_size in (2, 4) and r.walks_per_s > 0
    assert len(r.table) >= 2 + 4
    # sampled probes give a result too
    ts = autotune.Tuner(solver, probe_points=256, chunks=(128, 512), leaf_sizes=(4,))
    assert ts.tune(m, "laplace", (32, 32, 1), use_cache=False, N_walks=1024, seed=3,
                   method="fast").chunk in (128, 512)
    # the tuned solver still solves the same problem
    res = solver.solve_grid("laplace", 16, 16, N_walks=256, seed=3, method="fast")
    assert np.isfinite(res.mean[res.location == 1]).all()
    # a second tuner reads the cache
    t2 = autotune.Tuner(solver, cache_path=str(tmp_path / "tune.json"))
    r2 = t2.tune(m, "laplace", (32, 32, 1), N_walks=1024, seed=3, method="fast")
    assert (r2.chunk, r2.blocks, r2.leaf_size) == (r.chunk, r.blocks, r.leaf_size)
    solver.set_tuning(0, 0)
