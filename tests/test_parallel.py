"""Multi-process sharding (walk_on_spheres_b200.parallel) on CPU with gloo,
world size 2.  The per-shard solver is the oracle (the reference restatement)
seeded by global linear indices, so the gathered fields must equal a
one-process sweep exactly — the decomposition independence the reference
promises (README.md:87-90)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from walk_on_spheres_b200 import meshes, parallel


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _Grid:
    def __init__(self, m, nx, ny, nz=1):
        b = m.bbox()
        self.Nx, self.Ny, self.Nz = nx, ny, nz
        self.xmin, self.xmax, self.ymin, self.ymax, self.zmin, self.zmax = b


def _oracle_shard_solver(mesh, eq, nx, ny, nz, kw):
    from oracle.oracle import Oracle, Solve
    o = Oracle()

    def solve(start, end):
        pts = np.arange(start, end, dtype=np.int64)
        r = o.solve_grid(eq, Solve(mesh, nx, ny, nz, points=pts, n_threads=1, **kw))
        out = {k: getattr(r, k)[start:end] for k in parallel.FIELDS}
        out["counters"] = r.counters
        return out

    return solve


def _worker(rank, world, port, case, results):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mesh, eq, (nx, ny, nz), kw = case
        n = nx * ny * nz
        out = parallel.solve_grid_sharded(_oracle_shard_solver(mesh, eq, nx, ny, nz, kw), n)
        if rank == 0:
            results.put({k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in out.items()})
    finally:
        dist.destroy_process_group()


CASES = {
    "annulus_laplace": (meshes.annulus(), "laplace", (13, 11, 1), dict(N_walks=60, seed=5)),
    "sphere_screened": (meshes.uv_sphere(lon=16, lat=8), "screened_poisson", (5, 6, 7),
                        dict(N_walks=30, seed=9, alpha=10.0)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_two_rank_gather_equals_single_process(name, oracle):
    from oracle.oracle import Solve
    case = CASES[name]
    mesh, eq, (nx, ny, nz), kw = case
    ctx = mp.get_context("spawn")
    results = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, case, results)) for r in range(2)]
    for p in procs:
        p.start()
    got = results.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = oracle.solve_grid(eq, Solve(mesh, nx, ny, nz, n_threads=1, **kw))
    loc = np.asarray(got["location"], dtype=np.uint8)
    assert np.array_equal(loc, ref.location)
    for k in ("mean", "variance", "standard_error", "mean_steps"):
        a, b = np.asarray(got[k]), getattr(ref, k)
        both_nan = np.isnan(a) & np.isnan(b)
        assert np.array_equal(a[~both_nan], b[~both_nan]), k
    assert got["counters"]["inside_points"] == ref.counters["inside_points"]
    assert got["counters"]["ambiguous_ray_retries"] == ref.counters["ambiguous_ray_retries"]


def test_shard_bounds_cover_the_grid():
    for n in (1, 7, 100, 65536):
        for world in (1, 2, 3, 8):
            spans = [parallel.shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            assert max(e - s for s, e in spans) - min(e - s for s, e in spans) <= 1


def test_grid_points_match_grid_coordinate():
    m = meshes.uv_sphere(lon=8, lat=4)
    g = _Grid(m, 4, 5, 6)
    pts = parallel.grid_points(g, 3, 0, 120)
    lin = 37
    i, j, k = lin // 30, (lin // 6) % 5, lin % 6
    want = [g.xmin + (g.xmax - g.xmin) * i / 3, g.ymin + (g.ymax - g.ymin) * j / 4,
            g.zmin + (g.zmax - g.zmin) * k / 5]
    assert pts[lin].tolist() == want
