"""Host API over libwos_b200 mirroring the reference's operator interface.

* :class:`Solver` — one CUDA context with its stream and uploaded mesh; the
  per-grid-point sweep of include/wos/runner.hpp:157-236 (``solve_grid``),
  the point-level ``wos_run`` (``solve_points``, include/wos/wos.hpp:160-191)
  and kernel-level checks (``closest_points``, ``prng_u64``).
* :data:`equation_registry` — the reference registry
  (src/equations/equations.hpp:26-31): entries with ``name``, ``run_2D`` and
  ``run_3D`` taking the reference's arguments (rank, size, mesh_filename,
  output_filename, Nx, Ny, Nz, N_walks, epsilon, max_steps, max_ray_attempts,
  seed, alpha, source_mode) and returning 0 / 1.

All work runs in the CUDA library; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass, field

import numpy as np

from . import _lib

EQUATIONS = ("laplace", "poisson", "screened_poisson", "helmholtz")
METHODS = {"plain": 0, "fast": 1, "fast64": 2}
SOURCE_MODES = {"uniform": 0, "green": 1, "mis": 2}
LOCATION_NAMES = {0: "Outside", 1: "Inside", 2: "Boundary", 3: "Indeterminate"}


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class GridResult:
    """Fields of one sweep in row-major (i, j, k) order, shaped (Nx, Ny, Nz).
    A grid sweep also records what it ran (`equation`, `dim`, `grid`,
    `params`), so `write_hdf5` can write the reference's result file."""
    mean: np.ndarray
    variance: np.ndarray
    standard_error: np.ndarray
    mean_steps: np.ndarray
    location: np.ndarray
    counters: dict = field(default_factory=dict)
    equation: str | None = None
    dim: int = 0
    grid: object = None
    params: object = None

    def write_hdf5(self, path) -> None:
        """Write the result file a registry run of the same sweep writes
        (include/wos/hdf5_io.hpp layout, the run's /metadata)."""
        from . import results
        if self.grid is None or self.params is None or self.equation is None:
            raise ValueError("write_hdf5 needs a grid sweep's result (Solver.solve_grid)")
        p = self.params
        meta = results.run_meta(self.equation, self.dim, p.N_walks,
                                self.counters["effective_epsilon"], p.max_steps, p.seed,
                                alpha=p.alpha, source_mode=p.source_mode,
                                max_ray_attempts=p.max_ray_attempts, counters=self.counters)
        results.write(path, self.grid, {k: getattr(self, k) for k in results.FIELDS}, meta)


def _enum(value, table, what):
    if isinstance(value, str):
        if value not in table:
            raise ValueError(f"unknown {what} {value!r}; expected one of {sorted(table)}")
        return table[value]
    return int(value)


class Solver:
    """A libwos_b200 context on one CUDA device."""

    def __init__(self, device: int = 0):
        self._L = _lib.lib()
        ctx = C.c_void_p()
        _lib.check(self._L.wos_context_create(device, C.byref(ctx)))
        self._ctx = ctx
        self._batches = weakref.WeakSet()
        self.device = device
        self.dim = 0
        self.n_prims = 0
        self.bbox = (0.0,) * 6

    def close(self):
        if self._ctx:
            for b in list(self._batches):
                b.close()
            self._L.wos_context_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status):
        _lib.check(status, self._ctx)

    def _refresh_mesh_info(self):
        d, n = C.c_int(), C.c_int()
        box = np.zeros(6)
        self._check(self._L.wos_mesh_info(self._ctx, C.byref(d), C.byref(n), _ptr(box)))
        self.dim, self.n_prims, self.bbox = d.value, n.value, tuple(box.tolist())

    # ------------------------------------------------------------- mesh
    def set_mesh(self, mesh, leaf_size: int = 0) -> "Solver":
        """Upload a :class:`walk_on_spheres_b200.meshes.Mesh` (or any object with dim,
        verts, prims, boundary_ids) and build its BVHs on the host."""
        verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
        prims = np.ascontiguousarray(mesh.prims, dtype=np.int32)
        bids = np.ascontiguousarray(mesh.boundary_ids, dtype=np.int32)
        self._check(self._L.wos_set_mesh(self._ctx, int(mesh.dim), _ptr(verts), verts.shape[0],
                                         _ptr(prims), prims.shape[0],
                                         _ptr(bids) if mesh.dim == 2 else None, leaf_size))
        self._refresh_mesh_info()
        return self

    def load_obj(self, path: str, leaf_size: int = 0) -> "Solver":
        """Read an OBJ file with the reference's loader semantics and upload it."""
        self._check(self._L.wos_load_obj(self._ctx, str(path).encode(), leaf_size))
        self._refresh_mesh_info()
        return self

    def grid_over_mesh(self, Nx: int, Ny: int, Nz: int = 1) -> _lib.Grid:
        g = _lib.Grid()
        self._check(self._L.wos_grid_over_mesh(self._ctx, Nx, Ny, Nz, C.byref(g)))
        return g

    # ------------------------------------------------------------- solve
    @staticmethod
    def params(equation="laplace", N_walks=10000, epsilon=1e-2, max_steps=1000,
               max_ray_attempts=12, seed=0, alpha=5.0, source_mode="uniform",
               method="plain") -> _lib.Params:
        p = _lib.Params()
        p.equation = EQUATIONS.index(equation) if isinstance(equation, str) else int(equation)
        p.source_mode = _enum(source_mode, SOURCE_MODES, "source mode")
        p.alpha = float(alpha)
        p.N_walks = int(N_walks)
        p.epsilon = float(epsilon)
        p.max_steps = int(max_steps)
        p.max_ray_attempts = int(max_ray_attempts)
        p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        p.method = _enum(method, METHODS, "method")
        return p

    def solve_grid(self, equation="laplace", Nx=32, Ny=32, Nz=1, grid: _lib.Grid | None = None,
                   **kw) -> GridResult:
        """Sweep a grid (default: Nx x Ny x Nz over the mesh bounding box)."""
        g = grid if grid is not None else self.grid_over_mesh(Nx, Ny, Nz)
        shape = (g.Nx, g.Ny, g.Nz if self.dim == 3 else 1)
        n = int(np.prod(shape))
        res = GridResult(np.empty(n), np.empty(n), np.empty(n), np.empty(n),
                         np.empty(n, dtype=np.uint8))
        c = _lib.Counters()
        p = self.params(equation, **kw)
        self._check(self._L.wos_solve_grid(self._ctx, C.byref(p), C.byref(g), _ptr(res.mean),
                                           _ptr(res.variance), _ptr(res.standard_error),
                                           _ptr(res.mean_steps), _ptr(res.location), C.byref(c)))
        for k in ("mean", "variance", "standard_error", "mean_steps", "location"):
            setattr(res, k, getattr(res, k).reshape(shape))
        res.counters = c.as_dict()
        res.equation = EQUATIONS[p.equation]
        res.dim = self.dim
        res.grid = _lib.Grid(g.Nx, g.Ny, shape[2], g.xmin, g.xmax, g.ymin, g.ymax,
                             g.zmin, g.zmax)
        res.params = p
        return res

    def solve_grid_device(self, equation, grid: _lib.Grid, mean=0, variance=0,
                          standard_error=0, mean_steps=0, location=0, **kw) -> dict:
        """Sweep with DEVICE output pointers (integers, e.g. torch.Tensor.data_ptr());
        0 skips a field.  Returns the counters."""
        c = _lib.Counters()
        p = self.params(equation, **kw)
        ptrs = [C.c_void_p(int(x)) if x else None for x in
                (mean, variance, standard_error, mean_steps, location)]
        self._check(self._L.wos_solve_grid_device(self._ctx, C.byref(p), C.byref(grid), *ptrs,
                                                  C.byref(c)))
        return c.as_dict()

    def solve_points(self, equation, points, point_index=None, **kw) -> GridResult:
        """wos_run at arbitrary start points (n x dim); point_index seeds each point like the
        grid's linear index (default: 0..n-1)."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, self.dim)
        n = pts.shape[0]
        idx = None if point_index is None else np.ascontiguousarray(point_index, dtype=np.uint64)
        res = GridResult(np.empty(n), np.empty(n), np.empty(n), np.empty(n),
                         np.empty(n, dtype=np.uint8))
        c = _lib.Counters()
        p = self.params(equation, **kw)
        self._check(self._L.wos_solve_points(self._ctx, C.byref(p), _ptr(pts), _ptr(idx), n,
                                             _ptr(res.mean), _ptr(res.variance),
                                             _ptr(res.standard_error), _ptr(res.mean_steps),
                                             _ptr(res.location), C.byref(c)))
        res.counters = c.as_dict()
        return res

    def set_tuning(self, chunk: int = 0, blocks: int = 0):
        self._check(self._L.wos_set_tuning(self._ctx, int(chunk), int(blocks)))

    # ------------------------------------------------------------- checks
    def closest_points(self, points, precision: int = 64):
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, self.dim)
        n = pts.shape[0]
        dist, near = np.empty(n), np.empty((n, self.dim))
        bid = np.empty(n, dtype=np.int32)
        self._check(self._L.wos_closest_points(self._ctx, precision, _ptr(pts), n, _ptr(dist),
                                               _ptr(near), _ptr(bid)))
        return dist, near, bid

    def distance_bounds(self, points) -> np.ndarray:
        """Lattice lower bounds of the boundary distance used by FAST_FP32 walks."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, self.dim)
        out = np.empty(pts.shape[0])
        self._check(self._L.wos_distance_bounds(self._ctx, _ptr(pts), pts.shape[0], _ptr(out)))
        return out

    def special_functions(self, x, precision: int = 64) -> tuple[np.ndarray, np.ndarray]:
        """(ln I0(x), ln K0(x)) as the walk kernels of `precision` evaluate them."""
        xs = np.ascontiguousarray(x, dtype=np.float64).ravel()
        li, lk = np.empty_like(xs), np.empty_like(xs)
        self._check(self._L.wos_special_functions(self._ctx, precision, _ptr(xs), xs.size,
                                                  _ptr(li), _ptr(lk)))
        return li, lk

    def prng_u64(self, seeds, count: int) -> np.ndarray:
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        out = np.empty((s.shape[0], count), dtype=np.uint64)
        self._check(self._L.wos_prng_u64(self._ctx, _ptr(s), s.shape[0], count, _ptr(out)))
        return out


@dataclass
class Equation:
    """A registry entry with the reference's run signature (src/equations/equations.hpp:7-17)."""
    name: str
    _entry: object

    def run_2D(self, rank, size, mesh_filename, output_filename, Nx, Ny, Nz, N_walks, epsilon,
               max_steps, max_ray_attempts, seed, alpha, source_mode) -> int:
        return self._entry.run_2D(rank, size, str(mesh_filename).encode(),
                                  str(output_filename).encode(), Nx, Ny, Nz, N_walks, epsilon,
                                  max_steps, max_ray_attempts, seed, alpha,
                                  _enum(source_mode, SOURCE_MODES, "source mode"))

    def run_3D(self, rank, size, mesh_filename, output_filename, Nx, Ny, Nz, N_walks, epsilon,
               max_steps, max_ray_attempts, seed, alpha, source_mode) -> int:
        return self._entry.run_3D(rank, size, str(mesh_filename).encode(),
                                  str(output_filename).encode(), Nx, Ny, Nz, N_walks, epsilon,
                                  max_steps, max_ray_attempts, seed, alpha,
                                  _enum(source_mode, SOURCE_MODES, "source mode"))


def registry() -> list[Equation]:
    """The equation registry exported by libwos_b200 (laplace, poisson, screened_poisson,
    helmholtz)."""
    L = _lib.lib()
    n = C.c_int()
    entries = L.wos_equation_registry(C.byref(n))
    return [Equation(entries[i].name.decode(), entries[i]) for i in range(n.value)]


def peek_mesh_dim(path: str) -> int:
    """Mesh dimension from the first `l` / `f` record (src/mesh.cpp:51-74); 0 on error."""
    return int(_lib.lib().wos_peek_mesh_dim(str(path).encode()))
