"""The registry entries under the reference's own launcher shape
(`mpirun -np P wos ...`): the reference's rank blocks
(include/wos/runner.hpp:90-134) and the caller-supplied collectives that
stand in for MPI.  CPU only: the decomposition and the failure paths end
before any GPU work; two gloo ranks back the collectives."""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
from pathlib import Path

import numpy as np
import pytest

from walk_on_spheres_b200 import meshes
from walk_on_spheres_b200.parallel import rank_block

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.parametrize("dim,shape,size", [
    (2, (64, 64, 1), 2), (2, (64, 64, 1), 4), (2, (64, 64, 1), 6), (2, (7, 5, 1), 8),
    (2, (256, 1, 1), 3), (3, (64, 64, 64), 8), (3, (64, 64, 64), 12), (3, (9, 1, 13), 6),
    (3, (10, 10, 1), 4), (3, (5, 6, 7), 30)])
def test_rank_blocks_tile_the_grid(dim, shape, size):
    nx, ny, nz = shape
    cover = np.zeros(shape, dtype=np.int32)
    dims0 = None
    for r in range(size):
        dims, off, cnt = rank_block(dim, nx, ny, nz, r, size)
        dims0 = dims0 or dims
        assert dims == dims0 and int(np.prod(dims)) == size
        # runner.hpp:116-131: cx = r / (dy dz), ...; start = N c / d
        c = (r // (dims[1] * dims[2]), (r // dims[2]) % dims[1], r % dims[2])
        for k in range(3):
            assert off[k] == shape[k] * c[k] // dims[k]
            assert off[k] + cnt[k] == shape[k] * (c[k] + 1) // dims[k]
        cover[off[0]:off[0] + cnt[0], off[1]:off[1] + cnt[1], off[2]:off[2] + cnt[2]] += 1
    assert (cover == 1).all()
    # axes of extent 1 are never split; the factors are non-increasing
    free = [d for d, n in zip(dims0, shape) if n > 1]
    assert all(d == 1 for d, n in zip(dims0, shape) if n == 1)
    assert free == sorted(free, reverse=True)


def test_balanced_decompositions():
    assert rank_block(2, 64, 64, 1, 0, 4)[0] == (2, 2, 1)
    assert rank_block(2, 64, 64, 1, 0, 8)[0] == (4, 2, 1)
    assert rank_block(3, 64, 64, 64, 0, 8)[0] == (2, 2, 2)
    assert rank_block(3, 64, 64, 64, 0, 12)[0] == (3, 2, 2)
    assert rank_block(3, 64, 64, 64, 0, 16)[0] == (4, 2, 2)


def test_rank_block_errors_carry_the_references_messages():
    with pytest.raises(ValueError, match=r"^Cannot assign 5 MPI ranks to only 4 grid points; "
                                         r"use fewer ranks or a larger grid$"):
        rank_block(2, 2, 2, 1, 0, 5)
    with pytest.raises(ValueError, match=r"^MPI decomposition 3 x 1 x 1 exceeds grid 2 x 2 x 1; "
                                         r"use fewer ranks or a larger grid$"):
        rank_block(2, 2, 2, 1, 0, 3)


def _rank_main(rank, world, port, mesh_path, out_path, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from walk_on_spheres_b200.parallel import TorchCollectives
    from walk_on_spheres_b200.solver import registry
    entry = registry()[0]
    with TorchCollectives():
        # 3 grid points for 2 ranks along x fits; a 1 x 1 grid does not
        rc_small = entry.run_2D(rank, world, mesh_path, out_path, 1, 1, 1, 10, 1e-2, 1000, 12,
                                1, 0.0, 0)
        # a mesh file that does not exist: every rank fails together
        rc_missing = entry.run_2D(rank, world, mesh_path + ".missing", out_path, 8, 8, 1, 10,
                                  1e-2, 1000, 12, 1, 0.0, 0)
    q.put((rank, rc_small, rc_missing))
    dist.destroy_process_group()


def test_two_gloo_ranks_fail_together_before_any_gpu_work(tmp_path):
    sys.path.insert(0, str(ROOT))
    import bench
    mesh_path = str(meshes.write_obj(meshes.annulus(segments=16), tmp_path / "a.obj"))
    out = str(tmp_path / "never.h5")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = bench.free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, mesh_path, out, q))
             for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == [(0, 1, 1), (1, 1, 1)]
    assert not Path(out).exists()
