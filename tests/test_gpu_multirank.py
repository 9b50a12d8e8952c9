"""The registry entries with several ranks, as under the reference's
`mpirun -np P wos ...` (README.md:32): two processes, each a rank on GPU 0
with its block of the grid (include/wos/runner.hpp:90-134), the collectives
backed by a gloo process group in place of MPI.  The result file they write
together must be byte-identical to the file of a one-rank run: every point
is seeded by its global index, so the split changes nothing, and the
metadata counters are the reduced totals."""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
from pathlib import Path

import pytest

from walk_on_spheres_b200 import meshes

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]

CASES = {
    "laplace2d": (0, 2, lambda: meshes.annulus(), (24, 20, 1), 300, 0.0),
    "screened3d": (2, 3, lambda: meshes.uv_sphere(lon=24, lat=12), (10, 9, 8), 100, 8.0),
}


def _rank_main(rank, world, port, case, mesh_path, out_path, method, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WOS_B200_DEVICE="0",
                      WOS_B200_METHOD=method)
    sys.path.insert(0, str(ROOT))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from walk_on_spheres_b200.parallel import TorchCollectives
    from walk_on_spheres_b200.solver import registry
    eq, dim, _, (nx, ny, nz), walks, alpha = CASES[case]
    entry = registry()[eq]
    run = entry.run_2D if dim == 2 else entry.run_3D
    with TorchCollectives():
        rc = run(rank, world, mesh_path, out_path, nx, ny, nz, walks, 1e-2, 1000, 12, 77,
                 alpha, 0)
    q.put((rank, rc))
    dist.destroy_process_group()


@pytest.mark.parametrize("method", ["plain", "fast"])
@pytest.mark.parametrize("case", list(CASES))
def test_two_ranks_write_the_one_rank_file(tmp_path, case, method):
    sys.path.insert(0, str(ROOT))
    import bench
    from walk_on_spheres_b200.solver import registry
    eq, dim, make_mesh, (nx, ny, nz), walks, alpha = CASES[case]
    mesh_path = str(meshes.write_obj(make_mesh(), tmp_path / "m.obj"))
    one = str(tmp_path / "one.h5")
    two = str(tmp_path / "two.h5")
    os.environ["WOS_B200_METHOD"] = method
    try:
        entry = registry()[eq]
        run = entry.run_2D if dim == 2 else entry.run_3D
        assert run(0, 1, mesh_path, one, nx, ny, nz, walks, 1e-2, 1000, 12, 77, alpha, 0) == 0
    finally:
        del os.environ["WOS_B200_METHOD"]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = bench.free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, case, mesh_path, two, method, q))
             for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 0), (1, 0)]
    assert Path(one).read_bytes() == Path(two).read_bytes()
