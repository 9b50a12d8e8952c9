"""Many solves in one launch sequence (wos_batch_* in include/wos_b200.h).

    b = Batch(solver)
    m = b.add_mesh(meshes.star_polygon(rng, 512))
    s = b.add_solve(m, "poisson", 128, 128, N_walks=1024, seed=3, method="fast")
    ms = b.run(use_graph=True)          # device time of the whole batch
    r = b.result(s)                     # GridResult, as Solver.solve_grid returns

Each solve means what Solver.solve_grid means for the same arguments (and
FAST method); with the same walks-per-task chunking every walk takes the
same steps, so locations and step counts are identical and the statistics
agree to the rounding of the terminal FP64 arithmetic.  The batch runs one classification launch per dimension, one
persistent walk launch per (dimension, equation, method) family over a
device queue of (solve, point, chunk) tasks and one merge launch, captured
once as a CUDA graph when use_graph is set.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .solver import GridResult, Solver, _ptr


class Batch:
    def __init__(self, solver: Solver):
        self.solver = solver
        self._L = solver._L
        b = C.c_void_p()
        solver._check(self._L.wos_batch_create(solver._ctx, C.byref(b)))
        self._b = b
        solver._batches.add(self)
        self._meshes: list[tuple[int, tuple]] = []   # (dim, bbox)
        self._solves: list[tuple[int, tuple]] = []   # (mesh, shape)

    def close(self):
        if getattr(self, "_b", None):
            self._L.wos_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_mesh(self, mesh, leaf_size: int = 0) -> int:
        verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
        prims = np.ascontiguousarray(mesh.prims, dtype=np.int32)
        bids = (np.ascontiguousarray(mesh.boundary_ids, dtype=np.int32)
                if mesh.dim == 2 and getattr(mesh, "boundary_ids", None) is not None else None)
        mid = C.c_int()
        self.solver._check(self._L.wos_batch_add_mesh(self._b, mesh.dim, _ptr(verts),
                                                      verts.shape[0], _ptr(prims),
                                                      prims.shape[0], _ptr(bids), leaf_size,
                                                      C.byref(mid)))
        self._meshes.append((mesh.dim, tuple(mesh.bbox())))
        return mid.value

    def add_solve(self, mesh_id: int, equation="laplace", Nx=32, Ny=32, Nz=1, grid=None,
                  **params) -> int:
        # an unknown mesh id is rejected by the library
        dim, box = (self._meshes[mesh_id] if 0 <= mesh_id < len(self._meshes)
                    else (2, (0.0,) * 6))
        if grid is None:
            grid = _lib.Grid(Nx, Ny, Nz if dim == 3 else 1, *box)
        p = Solver.params(equation, **params)
        sid = C.c_int()
        self.solver._check(self._L.wos_batch_add_solve(self._b, mesh_id, C.byref(p),
                                                       C.byref(grid), C.byref(sid)))
        self._solves.append((mesh_id, (grid.Nx, grid.Ny, grid.Nz if dim == 3 else 1)))
        return sid.value

    def set_tuning(self, chunk: int = 0, blocks: int = 0):
        self.solver._check(self._L.wos_batch_set_tuning(self._b, int(chunk), int(blocks)))

    def prepare(self) -> None:
        """Build and upload new meshes and lay out the solves (else the next run does)."""
        self.solver._check(self._L.wos_batch_prepare(self._b))

    def run(self, use_graph: bool = True) -> float:
        ms = C.c_float()
        self.solver._check(self._L.wos_batch_run(self._b, int(bool(use_graph)), C.byref(ms)))
        return ms.value

    def info(self) -> dict:
        n = C.c_int()
        pts, walks, steps = C.c_longlong(), C.c_longlong(), C.c_longlong()
        self.solver._check(self._L.wos_batch_info(self._b, C.byref(n), C.byref(pts),
                                                  C.byref(walks), C.byref(steps)))
        return {"solves": n.value, "points": pts.value, "walks": walks.value,
                "steps": steps.value}

    def result(self, solve_id: int) -> GridResult:
        shape = self._solves[solve_id][1]
        n = int(np.prod(shape))
        r = GridResult(np.empty(n), np.empty(n), np.empty(n), np.empty(n),
                       np.empty(n, dtype=np.uint8))
        c = _lib.Counters()
        self.solver._check(self._L.wos_batch_result(self._b, solve_id, _ptr(r.mean),
                                                    _ptr(r.variance), _ptr(r.standard_error),
                                                    _ptr(r.mean_steps), _ptr(r.location),
                                                    C.byref(c)))
        for k in ("mean", "variance", "standard_error", "mean_steps", "location"):
            setattr(r, k, getattr(r, k).reshape(shape))
        r.counters = c.as_dict()
        return r
