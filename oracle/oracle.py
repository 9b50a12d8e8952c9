"""ctypes bindings for the two CPU oracles.  TEST INFRASTRUCTURE ONLY.

* :class:`Reference` — ``oracle/_ref/libwos_ref.so``: the reference's own
  sources compiled where they lie (oracle/Makefile) plus the thin C entry
  points of oracle/ref_core.cpp and oracle/ref_driver.hpp.
* :class:`Oracle` — ``oracle/_build/libwos_oracle.so``: the plain C
  restatement in oracle/wos_oracle.c.

Both expose the same methods with the same argument meaning, so tests compare
them one to one and compare the CUDA library against either.  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libwos_ref.so"
ORACLE_LIB = HERE / "_build" / "libwos_oracle.so"

EQUATIONS = ("laplace", "poisson", "screened_poisson", "helmholtz")
LOCATION_NAMES = {0: "Outside", 1: "Inside", 2: "Boundary", 3: "Indeterminate"}


class _Problem(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("verts", C.c_void_p), ("n_verts", C.c_int),
        ("prims", C.c_void_p), ("n_prims", C.c_int), ("boundary_ids", C.c_void_p),
        ("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int), ("use_mesh_bbox", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
        ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double),
        ("N_walks", C.c_int), ("epsilon", C.c_double), ("max_steps", C.c_int),
        ("max_ray_attempts", C.c_int), ("seed", C.c_uint64), ("alpha", C.c_double),
        ("source_mode", C.c_int), ("n_threads", C.c_int), ("points", C.c_void_p),
        ("n_points", C.c_longlong),
    ]


class _Outputs(C.Structure):
    _fields_ = [
        ("mean", C.c_void_p), ("variance", C.c_void_p), ("standard_error", C.c_void_p),
        ("mean_steps", C.c_void_p), ("location", C.c_void_p),
        ("inside_points", C.c_longlong), ("max_steps_hits", C.c_longlong),
        ("ambiguous_ray_retries", C.c_longlong), ("indeterminate_points", C.c_longlong),
        ("sum_variance", C.c_double), ("sum_standard_error", C.c_double),
        ("sum_mean_steps", C.c_double), ("seconds", C.c_double),
    ]


@dataclass
class Solve:
    """Inputs of one grid sweep (the arguments of the reference registry's run_2D/run_3D)."""
    mesh: object                      # walk_on_spheres_b200.meshes.Mesh
    Nx: int
    Ny: int
    Nz: int = 1
    N_walks: int = 10000
    epsilon: float = 1e-2
    max_steps: int = 1000
    max_ray_attempts: int = 12
    seed: int = 0
    alpha: float = 5.0
    source_mode: int = 0
    bounds: tuple | None = None       # None: the mesh bounding box (runner.hpp:83-85)
    points: np.ndarray | None = None  # optional subset of global linear indices
    n_threads: int = 0


@dataclass
class GridResult:
    mean: np.ndarray
    variance: np.ndarray
    standard_error: np.ndarray
    mean_steps: np.ndarray
    location: np.ndarray
    counters: dict = field(default_factory=dict)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class _Lib:
    prefix = ""

    def __init__(self, path: Path):
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (run `make -C oracle`)")
        self.lib = C.CDLL(str(path))
        self._keep = []

    def _fn(self, name, restype, argtypes):
        f = getattr(self.lib, self.prefix + name)
        f.restype = restype
        f.argtypes = argtypes
        return f

    # ---- problem marshalling
    def _problem(self, mesh, solve: Solve | None = None, max_ray_attempts: int = 12):
        verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
        prims = np.ascontiguousarray(mesh.prims, dtype=np.int32)
        bids = np.ascontiguousarray(mesh.boundary_ids, dtype=np.int32)
        keep = [verts, prims, bids]
        pb = _Problem()
        pb.dim = mesh.dim
        pb.verts, pb.n_verts = _ptr(verts), verts.shape[0]
        pb.prims, pb.n_prims = _ptr(prims), prims.shape[0]
        pb.boundary_ids = _ptr(bids)
        pb.use_mesh_bbox = 1
        pb.max_ray_attempts = max_ray_attempts
        pb.Nx = pb.Ny = pb.Nz = 1
        if solve is not None:
            pb.Nx, pb.Ny, pb.Nz = solve.Nx, solve.Ny, (solve.Nz if mesh.dim == 3 else 1)
            if solve.bounds is not None:
                pb.use_mesh_bbox = 0
                (pb.xmin, pb.xmax, pb.ymin, pb.ymax, pb.zmin, pb.zmax) = solve.bounds
            pb.N_walks, pb.epsilon, pb.max_steps = solve.N_walks, solve.epsilon, solve.max_steps
            pb.max_ray_attempts = solve.max_ray_attempts
            pb.seed, pb.alpha, pb.source_mode = solve.seed, solve.alpha, solve.source_mode
            pb.n_threads = solve.n_threads if solve.n_threads > 0 else (os.cpu_count() or 1)
            if solve.points is not None:
                pts = np.ascontiguousarray(solve.points, dtype=np.int64)
                keep.append(pts)
                pb.points, pb.n_points = _ptr(pts), pts.shape[0]
        return pb, keep

    # ---- entry points shared by both oracles
    def solve_grid(self, equation: str, solve: Solve) -> GridResult:
        pb, keep = self._problem(solve.mesh, solve)
        n = pb.Nx * pb.Ny * pb.Nz
        res = GridResult(np.full(n, np.nan), np.full(n, np.nan), np.full(n, np.nan),
                         np.full(n, np.nan), np.full(n, 255, dtype=np.uint8))
        out = _Outputs()
        out.mean, out.variance = _ptr(res.mean), _ptr(res.variance)
        out.standard_error, out.mean_steps = _ptr(res.standard_error), _ptr(res.mean_steps)
        out.location = _ptr(res.location)
        rc = self._solve(equation, pb, out)
        if rc != 0:
            raise RuntimeError(f"{self.prefix}solve {equation} failed ({rc})")
        res.counters = {k: getattr(out, k) for k, _ in _Outputs._fields_[5:]}
        return res

    def prng_u64(self, seed: int, n: int) -> np.ndarray:
        out = np.zeros(n, dtype=np.uint64)
        self._fn("prng_u64", None, [C.c_uint64, C.c_longlong, C.c_void_p])(seed, n, _ptr(out))
        return out

    def prng_unit(self, seed: int, n: int, open_: bool = False) -> np.ndarray:
        out = np.zeros(n)
        self._fn("prng_unit", None, [C.c_uint64, C.c_longlong, C.c_int, C.c_void_p])(
            seed, n, int(open_), _ptr(out))
        return out

    def splitmix64(self, x: int) -> int:
        return int(self._fn("splitmix64", C.c_uint64, [C.c_uint64])(x))

    def build_bvh(self, mesh):
        pb, keep = self._problem(mesh)
        n = max(1, 2 * mesh.n_prims - 1)
        boxes = np.zeros((n, 2 * mesh.dim))
        counts = np.zeros(n, dtype=np.int32)
        idx = np.zeros(n, dtype=np.int32)
        prims = np.zeros(mesh.n_prims, dtype=np.int32)
        nn = self._fn("build_bvh", C.c_int, [C.POINTER(_Problem)] + [C.c_void_p] * 4)(
            C.byref(pb), _ptr(boxes), _ptr(counts), _ptr(idx), _ptr(prims))
        return boxes[:nn], counts[:nn], idx[:nn], prims

    def npq(self, mesh, points):
        pb, keep = self._problem(mesh)
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, mesh.dim)
        n = pts.shape[0]
        dist = np.zeros(n)
        near = np.zeros((n, mesh.dim))
        prim = np.zeros(n, dtype=np.int32)
        bid = np.zeros(n, dtype=np.int32)
        self._npq(pb, pts, n, dist, near, prim, bid)
        return dist, near, prim, bid

    def winding_numbers(self, mesh, points):
        pb, keep = self._problem(mesh)
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
        wn = np.zeros(pts.shape[0], dtype=np.int32)
        self._fn("winding_numbers", None, [C.POINTER(_Problem), C.c_void_p, C.c_longlong,
                                           C.c_void_p])(C.byref(pb), _ptr(pts), pts.shape[0],
                                                        _ptr(wn))
        return wn

    def classify_3d(self, mesh, points, seeds, tolerance, max_ray_attempts=12):
        pb, keep = self._problem(mesh, max_ray_attempts=max_ray_attempts)
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        sd = np.ascontiguousarray(seeds, dtype=np.uint64)
        n = pts.shape[0]
        loc = np.zeros(n, dtype=np.uint8)
        ret = np.zeros(n, dtype=np.int32)
        self._fn("classify_3d", None, [C.POINTER(_Problem), C.c_void_p, C.c_void_p,
                                       C.c_longlong, C.c_double, C.c_void_p, C.c_void_p])(
            C.byref(pb), _ptr(pts), _ptr(sd), n, tolerance, _ptr(loc), _ptr(ret))
        return loc, ret

    def bessel(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros((x.shape[0], 4))
        self._fn("bessel", None, [C.c_void_p, C.c_longlong, C.c_void_p])(_ptr(x), x.shape[0],
                                                                          _ptr(out))
        return out

    def j0y0(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        j0, y0 = np.zeros_like(x), np.zeros_like(x)
        self._fn("j0y0", None, [C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p])(
            _ptr(x), x.shape[0], _ptr(j0), _ptr(y0))
        return j0, y0

    def screened_kernels(self, alpha, R, r):
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        Rr = np.ascontiguousarray(R, dtype=np.float64)
        rr = np.ascontiguousarray(r, dtype=np.float64)
        out = np.zeros((a.shape[0], 6))
        self._fn("screened_kernels", None, [C.c_void_p] * 3 + [C.c_longlong, C.c_void_p])(
            _ptr(a), _ptr(Rr), _ptr(rr), a.shape[0], _ptr(out))
        return out

    def screened_samples(self, dim, alpha, R, seed, n):
        out = np.zeros(n)
        self._fn("screened_samples", None, [C.c_int, C.c_double, C.c_double, C.c_uint64,
                                            C.c_longlong, C.c_void_p])(
            dim, alpha, R, seed, n, _ptr(out))
        return out

    def poisson_green(self, dim, R, r, seed):
        rr = np.ascontiguousarray(r, dtype=np.float64)
        n = rr.shape[0]
        g, m, s = np.zeros(n), np.zeros(n), np.zeros(n)
        self._fn("poisson_green", None, [C.c_int, C.c_double, C.c_void_p, C.c_longlong,
                                         C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p])(
            dim, R, _ptr(rr), n, seed, _ptr(g), _ptr(m), _ptr(s))
        return g, m, s

    def steps(self, dim, centre, radius, seed, n):
        c = np.ascontiguousarray(centre, dtype=np.float64)
        st, bl = np.zeros((n, dim)), np.zeros((n, dim))
        self._fn("steps", None, [C.c_int, C.c_void_p, C.c_double, C.c_uint64, C.c_longlong,
                                 C.c_void_p, C.c_void_p])(dim, _ptr(c), radius, seed, n,
                                                          _ptr(st), _ptr(bl))
        return st, bl


class Reference(_Lib):
    """The reference's own code (oracle/_ref/libwos_ref.so)."""
    prefix = "ref_"

    def __init__(self, path: Path = REF_LIB):
        super().__init__(path)

    def _solve(self, equation, pb, out):
        f = self._fn(f"grid_{equation}", C.c_int, [C.POINTER(_Problem), C.POINTER(_Outputs)])
        return f(C.byref(pb), C.byref(out))

    def _npq(self, pb, pts, n, dist, near, prim, bid):
        self._fn("npq", None, [C.POINTER(_Problem), C.c_void_p, C.c_longlong] + [C.c_void_p] * 4)(
            C.byref(pb), _ptr(pts), n, _ptr(dist), _ptr(near), _ptr(prim), _ptr(bid))

    def run_registry(self, equation: str, dim: int, mesh_path: str, Nx: int, Ny: int, Nz: int,
                     N_walks: int, epsilon: float, max_steps: int, max_ray_attempts: int,
                     seed: int, alpha: float, source_mode: int) -> dict:
        """Run the reference's registry entry (src/equations/<eq>.cpp run_2D/run_3D, i.e. the
        full runner.hpp pipeline on one rank) and return the datasets it wrote."""
        f = self._fn(f"registry_{equation}", C.c_int,
                     [C.c_int, C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int,
                      C.c_double, C.c_int, C.c_int, C.c_uint64, C.c_double, C.c_int])
        rc = f(dim, str(mesh_path).encode(), b"captured.h5", Nx, Ny, Nz, N_walks, epsilon,
               max_steps, max_ray_attempts, seed, alpha, source_mode)
        if rc != 0:
            raise RuntimeError(f"reference run_{dim}D for {equation} returned {rc}")
        names = C.create_string_buffer(1 << 14)
        self.lib.refshim_dataset_names.restype = C.c_longlong
        self.lib.refshim_dataset_names(names, C.c_longlong(1 << 14))
        get = self.lib.refshim_dataset
        get.restype = C.c_longlong
        get.argtypes = [C.c_char_p, C.c_void_p, C.c_longlong]
        out = {}
        for name in names.value.decode().split():
            nbytes = get(name.encode(), None, 0)
            buf = np.zeros(nbytes, dtype=np.uint8)
            get(name.encode(), _ptr(buf), nbytes)
            out[name] = buf
        return out

    def load_mesh(self, path: str):
        """The reference OBJ loader (src/mesh.cpp:51-270): (dim, verts, prims, bids) or raises."""
        f = self._fn("load_mesh", C.c_int, [C.c_char_p] + [C.POINTER(C.c_int)] * 3 +
                     [C.c_void_p] * 3 + [C.c_char_p, C.c_int])
        dim, nv, npr = C.c_int(), C.c_int(), C.c_int()
        err = C.create_string_buffer(512)
        if f(str(path).encode(), C.byref(dim), C.byref(nv), C.byref(npr), None, None, None,
             err, 512):
            raise ValueError(err.value.decode())
        d = dim.value
        verts = np.zeros((nv.value, d))
        prims = np.zeros((npr.value, d), dtype=np.int32)
        bids = np.zeros(npr.value, dtype=np.int32)
        f(str(path).encode(), C.byref(dim), C.byref(nv), C.byref(npr), _ptr(verts), _ptr(prims),
          _ptr(bids), err, 512)
        return d, verts, prims, bids


class Oracle(_Lib):
    """The plain-C restatement (oracle/_build/libwos_oracle.so)."""
    prefix = "wo_"

    def __init__(self, path: Path = ORACLE_LIB):
        super().__init__(path)

    def _solve(self, equation, pb, out):
        f = self._fn("solve_grid", C.c_int, [C.c_int, C.POINTER(_Problem), C.POINTER(_Outputs)])
        return f(EQUATIONS.index(equation), C.byref(pb), C.byref(out))

    def _npq(self, pb, pts, n, dist, near, prim, bid):
        self._fn("npq", None, [C.POINTER(_Problem), C.c_void_p, C.c_longlong] + [C.c_void_p] * 5)(
            C.byref(pb), _ptr(pts), n, _ptr(dist), _ptr(near), _ptr(prim), _ptr(bid), None)

    def npq_visits(self, mesh, points):
        """Per query (node pops, primitive tests) of the reference traversal order."""
        pb, keep = self._problem(mesh)
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, mesh.dim)
        n = pts.shape[0]
        dist, near = np.zeros(n), np.zeros((n, mesh.dim))
        prim, bid = np.zeros(n, dtype=np.int32), np.zeros(n, dtype=np.int32)
        visits = np.zeros((n, 2), dtype=np.int64)
        self._fn("npq", None, [C.POINTER(_Problem), C.c_void_p, C.c_longlong] + [C.c_void_p] * 5)(
            C.byref(pb), _ptr(pts), n, _ptr(dist), _ptr(near), _ptr(prim), _ptr(bid),
            _ptr(visits))
        return visits

    def walk_visit_counts(self, equation: str, solve: Solve, walks: int) -> dict:
        """Totals of walk-step closest-point queries, node pops and primitive tests of the
        reference traversal along the first `walks` walks of each (subset) point."""
        pb, keep = self._problem(solve.mesh, solve)
        q, pops, tests, steps = (C.c_longlong() for _ in range(4))
        self._fn("walk_visit_counts", C.c_int,
                 [C.c_int, C.POINTER(_Problem), C.c_int] + [C.POINTER(C.c_longlong)] * 4)(
            EQUATIONS.index(equation), C.byref(pb), walks, C.byref(q), C.byref(pops),
            C.byref(tests), C.byref(steps))
        return {"queries": q.value, "node_pops": pops.value, "prim_tests": tests.value}

    def screened_epsilon(self, eps, alpha):
        return self._fn("screened_epsilon", C.c_double, [C.c_double, C.c_double])(eps, alpha)

    def heat_solve(self, mesh, probes, Q: float, x0, sigma: float, vertex_values=None,
                   weights=None, N_walks: int = 256, epsilon: float = 1e-3,
                   max_steps: int = 10000, max_ray_attempts: int = 12, seed: int = 0,
                   source_mode: int = 1, point_index=None, n_threads: int = 0,
                   mis_green_probability: float = 0.5, proposal=None) -> dict:
        """FP64 Gaussian heat-source walks (wo_heat_solve; source_mode 0 uniform, 1 Green, 2
        Green-source MIS with probability `mis_green_probability` of a Green sample and the
        proposal (x0, sigma) given or the source's own): per-probe mean, standard error,
        derivative means / standard errors du/d(Q, x0.x, x0.y, x0.z, sigma), locations and
        grad_vertex = sum_i weights[i] du_i/dg_v."""
        pts = np.ascontiguousarray(probes, dtype=np.float64).reshape(-1, mesh.dim)
        n = pts.shape[0]
        solve = Solve(mesh, 1, 1, 1, N_walks=N_walks, epsilon=epsilon, max_steps=max_steps,
                      max_ray_attempts=max_ray_attempts, seed=seed, source_mode=source_mode,
                      n_threads=n_threads,
                      points=None if point_index is None else np.asarray(point_index))
        pb, keep = self._problem(mesh, solve)
        src = _Gaussian()
        src.Q, src.sigma = float(Q), float(sigma)
        xs = list(np.asarray(x0, dtype=np.float64).ravel()) + [0.0, 0.0, 0.0]
        src.x0 = (C.c_double * 3)(*xs[:3])
        src.mis_green_probability = float(mis_green_probability)
        if proposal is not None:
            pxs = list(np.asarray(proposal[0], dtype=np.float64).ravel()) + [0.0, 0.0, 0.0]
            src.proposal_x0 = (C.c_double * 3)(*pxs[:3])
            src.proposal_sigma = float(proposal[1])
        g = None if vertex_values is None else np.ascontiguousarray(vertex_values, np.float64)
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        out = {"mean": np.zeros(n), "standard_error": np.zeros(n),
               "jacobian": np.zeros((n, 5)), "jacobian_se": np.zeros((n, 5)),
               "location": np.zeros(n, dtype=np.uint8),
               "grad_vertex": np.zeros(mesh.verts.shape[0])}
        rc = self._fn("heat_solve", C.c_int, [C.POINTER(_Problem), C.POINTER(_Gaussian)] +
                      [C.c_void_p] * 2 + [C.c_longlong] + [C.c_void_p] * 7)(
            C.byref(pb), C.byref(src), _ptr(g), _ptr(pts), n, _ptr(w), _ptr(out["mean"]),
            _ptr(out["standard_error"]), _ptr(out["jacobian"]), _ptr(out["jacobian_se"]),
            _ptr(out["location"]), _ptr(out["grad_vertex"]))
        if rc != 0:
            raise RuntimeError(f"wo_heat_solve failed ({rc})")
        return out


class _Gaussian(C.Structure):
    _fields_ = [("Q", C.c_double), ("x0", C.c_double * 3), ("sigma", C.c_double),
                ("mis_green_probability", C.c_double), ("proposal_x0", C.c_double * 3),
                ("proposal_sigma", C.c_double)]
