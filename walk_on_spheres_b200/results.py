"""Result files with the reference's HDF5 layout (include/wos/hdf5_io.hpp:15-338).

`write` writes a whole result at once (wos_write_hdf5).  The parallel path is
the reference's collective hyperslab write (hdf5_io.hpp:51-171) without
MPI-IO: one process calls `create` (coordinates and /metadata written, the
five fields' storage reserved), then every rank writes its own part of the
fields with `write_range` (a linear-index shard) or `write_block` (an x, y, z
block like the reference's rank blocks, include/wos/runner.hpp:90-134).
Writes of disjoint parts may run from many processes at once. Once every
point has been written, the file is byte-identical to `write` of the whole
fields.

    from walk_on_spheres_b200 import results
    meta = results.ResultMeta(N_walks=4096, epsilon=1e-2, max_steps=1000, seed=12345)
    results.write("r.h5", grid, {"mean": m, "variance": v, ...}, meta)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib

FIELDS = ("mean", "variance", "standard_error", "mean_steps", "location")


@dataclass(frozen=True)
class ResultMeta:
    """The /metadata scalars (hdf5_io.hpp:300-322).  The counters are totals
    over all ranks.  The ray counters are written when `write_ray_metadata`
    is set (3D runs), alpha and source_mode when `write_source_metadata` is."""
    N_walks: int
    epsilon: float
    max_steps: int
    max_steps_hits: int = 0
    write_ray_metadata: bool = False
    max_ray_attempts: int = 12
    ambiguous_ray_retries: int = 0
    indeterminate_points: int = 0
    seed: int = 0
    write_source_metadata: bool = False
    alpha: float = 0.0
    source_mode: int = 0

    def args(self) -> tuple:
        return (int(self.N_walks), float(self.epsilon), int(self.max_steps),
                int(self.max_steps_hits), int(bool(self.write_ray_metadata)),
                int(self.max_ray_attempts), int(self.ambiguous_ray_retries),
                int(self.indeterminate_points), int(self.seed),
                int(bool(self.write_source_metadata)), float(self.alpha), int(self.source_mode))


def run_meta(equation: str, dim: int, N_walks: int, effective_epsilon: float, max_steps: int,
             seed: int, alpha: float = 0.0, source_mode: int = 0, max_ray_attempts: int = 12,
             counters: dict | None = None) -> ResultMeta:
    """The /metadata a registry run writes (the equation files' run calls,
    src/equations/*.cpp): the effective epsilon (screened_poisson reduces it,
    screened_poisson.cpp:22-38); the ray counters in 3D; alpha and
    source_mode for poisson (alpha 0, poisson.cpp:126-134) and
    screened_poisson only.  `counters` are the run's totals."""
    c = counters or {}
    source = equation in ("poisson", "screened_poisson")
    return ResultMeta(N_walks=N_walks, epsilon=effective_epsilon, max_steps=max_steps,
                      max_steps_hits=int(c.get("max_steps_hits", 0)),
                      write_ray_metadata=dim == 3, max_ray_attempts=max_ray_attempts,
                      ambiguous_ray_retries=int(c.get("ambiguous_ray_retries", 0)),
                      indeterminate_points=int(c.get("indeterminate_points", 0)), seed=seed,
                      write_source_metadata=source,
                      alpha=alpha if equation == "screened_poisson" else 0.0,
                      source_mode=int(source_mode))


def _error(what: str, rc: int):
    msg = _lib.lib().wos_last_global_error().decode(errors="replace")
    raise RuntimeError(f"{what} failed (status {rc}): {msg}")


def _field_arrays(fields: dict, n: int) -> list[np.ndarray]:
    out = []
    for name in FIELDS:
        dtype = np.uint8 if name == "location" else np.float64
        a = np.ascontiguousarray(np.asarray(fields[name]).reshape(-1), dtype=dtype)
        if a.size != n:
            raise ValueError(f"field {name!r} has {a.size} values, expected {n}")
        out.append(a)
    return out


def _ptrs(arrays):
    return [a.ctypes.data_as(C.c_void_p) for a in arrays]


def _points(grid) -> int:
    return int(grid.Nx) * int(grid.Ny) * int(grid.Nz)


def write(path, grid, fields: dict, meta: ResultMeta) -> None:
    """Write a whole result file (wos_write_hdf5)."""
    arrays = _field_arrays(fields, _points(grid))
    rc = _lib.lib().wos_write_hdf5(str(path).encode(), C.byref(grid), *_ptrs(arrays),
                                   *meta.args())
    if rc != 0:
        _error("wos_write_hdf5", rc)


def layout(grid, write_ray_metadata: bool, write_source_metadata: bool) -> _lib.H5Layout:
    """The file layout of a result for `grid`, writing nothing."""
    lay = _lib.H5Layout()
    rc = _lib.lib().wos_hdf5_layout(C.byref(grid), int(bool(write_ray_metadata)),
                                    int(bool(write_source_metadata)), C.byref(lay))
    if rc != 0:
        _error("wos_hdf5_layout", rc)
    return lay


def create(path, grid, meta: ResultMeta) -> _lib.H5Layout:
    """Create the result file with every dataset but the fields' values."""
    lay = _lib.H5Layout()
    rc = _lib.lib().wos_hdf5_create(str(path).encode(), C.byref(grid), *meta.args(),
                                    C.byref(lay))
    if rc != 0:
        _error("wos_hdf5_create", rc)
    return lay


def write_range(path, lay: _lib.H5Layout, grid, start: int, fields: dict) -> None:
    """Write grid points start .. start + len - 1 (linear C order) of the fields."""
    n = np.asarray(fields["mean"]).size
    arrays = _field_arrays(fields, n)
    rc = _lib.lib().wos_hdf5_write_range(str(path).encode(), C.byref(lay), C.byref(grid),
                                         int(start), int(n), *_ptrs(arrays))
    if rc != 0:
        _error("wos_hdf5_write_range", rc)


def write_block(path, lay: _lib.H5Layout, grid, offset, fields: dict) -> None:
    """Write the block of grid points offset + [0, shape) along x, y, z; each
    field is an array of the block's shape (count_x, count_y, count_z)."""
    shape = np.shape(fields["mean"])
    if len(shape) != 3:
        raise ValueError("block fields must be 3-dimensional (x, y, z)")
    arrays = _field_arrays(fields, int(np.prod(shape)))
    off = (C.c_int * 3)(*[int(v) for v in offset])
    cnt = (C.c_int * 3)(*[int(v) for v in shape])
    rc = _lib.lib().wos_hdf5_write_block(str(path).encode(), C.byref(lay), C.byref(grid), off,
                                         cnt, *_ptrs(arrays))
    if rc != 0:
        _error("wos_hdf5_write_block", rc)
