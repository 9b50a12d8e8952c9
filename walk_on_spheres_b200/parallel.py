"""Sharding one grid sweep across processes (one per GPU) with torch.distributed.

The reference splits the grid into MPI blocks (include/wos/runner.hpp:90-134);
because every point is seeded from its global linear index
(runner.hpp:163-168) the fields do not depend on the split (README.md:87-90).
Here rank r solves the contiguous linear-index range
[n*r/world, n*(r+1)/world) of the grid — its own points, seeded by their
global index.  Either rank 0 gathers the fields and sums the counters
(solve_grid_sharded, the counterpart of runner.hpp:240-263), or every rank
writes its range straight into the result file after rank 0 creates it
(solve_grid_sharded_to_file, the counterpart of the collective HDF5 write,
include/wos/hdf5_io.hpp:51-171).  There is no collective inside the walk
loop; the only communication is a reduction of a few scalars at the end, and
the gather or two barriers.

    import torch.distributed as dist
    from walk_on_spheres_b200 import Solver, meshes, parallel
    dist.init_process_group("nccl")
    s = Solver(local_rank).set_mesh(meshes.circle())
    grid = s.grid_over_mesh(256, 256)
    out = parallel.solve_grid_sharded(parallel.gpu_shard_solver(s, "poisson", grid, N_walks=4096,
                                      seed=1), parallel.grid_size(grid, s.dim))
    # rank 0: out["mean"] etc. are the full (Nx*Ny*Nz,) fields
"""
from __future__ import annotations

import numpy as np

FIELDS = ("mean", "variance", "standard_error", "mean_steps", "location")
COUNTS = ("inside_points", "max_steps_hits", "ambiguous_ray_retries", "indeterminate_points",
          "total_walks", "total_steps", "exact_queries")


def grid_size(grid, dim: int) -> int:
    return int(grid.Nx) * int(grid.Ny) * (int(grid.Nz) if dim == 3 else 1)


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous linear-index range of `rank` (sizes differ by at most one)."""
    return n * rank // world, n * (rank + 1) // world


def grid_points(grid, dim: int, start: int, end: int) -> np.ndarray:
    """Coordinates of linear indices [start, end) of `grid`, computed like
    grid_coordinate (include/wos/grid.hpp:12-18): min + (max-min)*i/(N-1)."""
    return grid_coords(grid, dim, np.arange(start, end, dtype=np.int64))


def grid_coords(grid, dim: int, lin) -> np.ndarray:
    """Coordinates of the given linear indices of `grid` (row-major i, j, k)."""
    nx, ny = int(grid.Nx), int(grid.Ny)
    nz = int(grid.Nz) if dim == 3 else 1
    lin = np.asarray(lin, dtype=np.int64)
    i, j, k = lin // (ny * nz), (lin // nz) % ny, lin % nz

    def coord(lo, hi, idx, count):
        if count <= 1:
            return np.full(idx.shape, lo, dtype=np.float64)
        return lo + (hi - lo) * idx.astype(np.float64) / float(count - 1)

    cols = [coord(grid.xmin, grid.xmax, i, nx), coord(grid.ymin, grid.ymax, j, ny)]
    if dim == 3:
        cols.append(coord(grid.zmin, grid.zmax, k, nz))
    return np.stack(cols, axis=1)


def gpu_shard_solver(solver, equation: str, grid, **params):
    """Per-shard solve on this rank's GPU through wos_solve_points, each point
    seeded by its global linear index."""

    def solve(start: int, end: int) -> dict:
        pts = grid_points(grid, solver.dim, start, end)
        r = solver.solve_points(equation, pts, point_index=np.arange(start, end, dtype=np.uint64),
                                **params)
        out = {k: getattr(r, k) for k in FIELDS}
        out["counters"] = r.counters
        return out

    return solve


def solve_grid_sharded(solve_shard, n_points: int, group=None, device=None) -> dict | None:
    """Solve this rank's shard with `solve_shard(start, end)` and gather the full
    fields on rank 0 (other ranks return None).  `device` is where the
    collective tensors live (a CUDA device for NCCL, None / "cpu" for gloo)."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    start, end = shard_bounds(n_points, rank, world)
    local = solve_shard(start, end)
    m = end - start
    width = -(-n_points // world) + 1          # longest shard
    buf = np.full((len(FIELDS), width), np.nan)
    for f, name in enumerate(FIELDS):
        buf[f, :m] = np.asarray(local[name], dtype=np.float64)[:m]
    t = torch.from_numpy(buf)
    c = local.get("counters", {})
    counts = torch.tensor([float(c.get(k, 0)) for k in COUNTS], dtype=torch.float64)
    times = torch.tensor([float(c.get("total_ms", 0.0))], dtype=torch.float64)
    if device is not None and str(device) != "cpu":
        t, counts, times = t.to(device), counts.to(device), times.to(device)
    gathered = [torch.empty_like(t) for _ in range(world)] if rank == 0 else None
    dist.gather(t, gathered, dst=0, group=group)
    dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(times, op=dist.ReduceOp.MAX, group=group)
    if rank != 0:
        return None
    out = {}
    for f, name in enumerate(FIELDS):
        full = np.empty(n_points, dtype=np.float64)
        for r in range(world):
            s, e = shard_bounds(n_points, r, world)
            full[s:e] = gathered[r][f, :e - s].cpu().numpy()
        out[name] = full.astype(np.uint8) if name == "location" else full
    out["counters"] = {k: int(v) for k, v in zip(COUNTS, counts.cpu().tolist())}
    out["counters"]["total_ms_max_over_ranks"] = float(times.item())
    return out


def solve_grid_sharded_to_file(solve_shard, grid, path, meta, group=None,
                               device=None) -> dict:
    """Solve this rank's shard and write it straight into the result file at
    `path`: the reference's parallel HDF5 write (include/wos/hdf5_io.hpp:51-171),
    with no gather of the fields.  The counters are summed over the ranks
    first, as runner.hpp:240-263 does, and rank 0 creates the file with them in
    /metadata (`meta` gives the run settings; its counters are replaced).
    Then every rank writes its own linear-index range.  Every rank takes the
    same collective steps on failure too: a failed create or write raises on
    all ranks.  Returns the summed counters on every rank."""
    import dataclasses

    import torch
    import torch.distributed as dist

    from . import results

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    n_points = int(grid.Nx) * int(grid.Ny) * int(grid.Nz)
    start, end = shard_bounds(n_points, rank, world)
    local = solve_shard(start, end)
    c = local.get("counters", {})
    counts = torch.tensor([float(c.get(k, 0)) for k in COUNTS], dtype=torch.float64)
    times = torch.tensor([float(c.get("total_ms", 0.0))], dtype=torch.float64)
    on_device = device is not None and str(device) != "cpu"
    if on_device:
        counts, times = counts.to(device), times.to(device)
    dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(times, op=dist.ReduceOp.MAX, group=group)
    total = {k: int(v) for k, v in zip(COUNTS, counts.cpu().tolist())}
    total["total_ms_max_over_ranks"] = float(times.item())

    def agree(ok: bool, what: str):
        flag = torch.tensor([1 if ok else 0], dtype=torch.int32)
        if on_device:
            flag = flag.to(device)
        dist.all_reduce(flag, op=dist.ReduceOp.MIN, group=group)
        if int(flag.item()) == 0:
            raise RuntimeError(f"sharded HDF5 write: {what} failed on a rank")

    error = None
    if rank == 0:
        full = dataclasses.replace(meta, max_steps_hits=total["max_steps_hits"],
                                   ambiguous_ray_retries=total["ambiguous_ray_retries"],
                                   indeterminate_points=total["indeterminate_points"])
        try:
            results.create(path, grid, full)
        except (RuntimeError, OSError) as e:
            error = e
    agree(error is None, "creating the file")
    try:
        lay = results.layout(grid, meta.write_ray_metadata, meta.write_source_metadata)
        results.write_range(path, lay, grid, start,
                            {k: np.asarray(local[k])[:end - start] for k in FIELDS})
    except (RuntimeError, OSError, ValueError) as e:
        error = e
    agree(error is None, "writing a shard")
    return total


def rank_block(dim: int, Nx: int, Ny: int, Nz: int, rank: int, size: int):
    """(dims, offset, count) of `rank`'s block of the grid as the reference
    splits it over `size` MPI ranks (include/wos/runner.hpp:90-134); raises
    ValueError with the reference's message when the ranks do not fit."""
    import ctypes as C

    from . import _lib
    dims, off, cnt = (C.c_int * 3)(), (C.c_int * 3)(), (C.c_int * 3)()
    err = C.create_string_buffer(256)
    rc = _lib.lib().wos_rank_block(dim, Nx, Ny, Nz, rank, size, dims, off, cnt, err, 256)
    if rc != 0:
        raise ValueError(err.value.decode() or "invalid arguments")
    return tuple(dims), tuple(off), tuple(cnt)


class TorchCollectives:
    """Backs the registry's multi-rank collectives (wos_set_collectives) with a
    torch.distributed process group, in place of the reference's MPI: a
    registry entry called with (rank, size) on every rank of the group then
    solves its block and writes it into the shared result file.

        dist.init_process_group("gloo")       # or "nccl" with device=...
        with TorchCollectives():
            entry.run_2D(dist.get_rank(), dist.get_world_size(), mesh, out, ...)

    Reductions run on `device` (None / "cpu" for gloo)."""

    def __init__(self, group=None, device=None):
        import ctypes as C

        from . import _lib
        self.group, self.device = group, device
        self._C = C
        self._fns = (_lib.BARRIER_FN(self._barrier), _lib.ALLREDUCE_FN(self._allreduce),
                     _lib.DIMS_FN())
        self.struct = _lib.Collectives(self._fns[0], self._fns[1], self._fns[2], None)

    def _barrier(self, user) -> int:
        import torch.distributed as dist
        try:
            dist.barrier(group=self.group)
            return 0
        except Exception:
            return 1

    def _allreduce(self, values, n, op, user) -> int:
        import torch
        import torch.distributed as dist
        try:
            t = torch.tensor([values[i] for i in range(n)], dtype=torch.float64)
            if self.device is not None and str(self.device) != "cpu":
                t = t.to(self.device)
            dist.all_reduce(t, op=dist.ReduceOp.MAX if op == 1 else dist.ReduceOp.SUM,
                            group=self.group)
            for i, v in enumerate(t.cpu().tolist()):
                values[i] = v
            return 0
        except Exception:
            return 1

    def __enter__(self):
        from . import _lib
        _lib.check(_lib.lib().wos_set_collectives(self._C.byref(self.struct)))
        return self

    def __exit__(self, *exc):
        from . import _lib
        _lib.lib().wos_set_collectives(None)
