"""Synthetic boundary meshes in the reference's OBJ conventions.

The reference reads 2D polylines (`l` records; each record is its own
``boundary_id``, numbered from 0 in file order, and an open record is closed
automatically, src/mesh.cpp:156-213) and 3D triangle meshes (`f` records,
src/mesh.cpp:215-231).  Its meshes/ directory is not distributed, so the
benchmark and test inputs are generated here:

* :func:`annulus` — two circles, outer loop written first (boundary_id 0),
  inner loop clockwise so the hole has winding number 0;
* :func:`circle` — one counter-clockwise loop;
* :func:`uv_sphere` — a latitude/longitude sphere (128 x 64 bands gives the
  16 128 triangles of the 3D screened-Poisson benchmark);
* :func:`star_polygon` / :func:`perturbed_sphere` — the randomly perturbed
  shapes of the batched benchmark;
* :func:`slab_box` — the triangulated 0.10 x 0.05 x 0.01 m slab of the
  differentiation benchmark.

Each generator returns a :class:`Mesh` (numpy arrays: float64 vertices,
int32 0-based primitive vertex indices, int32 boundary ids for 2D) and
:func:`write_obj` writes it in the reference's OBJ dialect.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np


@dataclass
class Mesh:
    dim: int
    verts: np.ndarray          # (n_verts, dim) float64
    prims: np.ndarray          # (n_prims, dim) int32, 0-based
    boundary_ids: np.ndarray   # (n_prims,) int32 (all zero in 3D)

    @property
    def n_verts(self) -> int:
        return int(self.verts.shape[0])

    @property
    def n_prims(self) -> int:
        return int(self.prims.shape[0])

    def bbox(self) -> tuple[float, float, float, float, float, float]:
        """Bounding box (xmin, xmax, ymin, ymax, zmin, zmax), src/mesh.cpp:297-322."""
        lo = self.verts.min(axis=0)
        hi = self.verts.max(axis=0)
        if self.dim == 2:
            return float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]), 0.0, 0.0
        return float(lo[0]), float(hi[0]), float(lo[1]), float(hi[1]), float(lo[2]), float(hi[2])


def _loops_to_mesh(loops: list[np.ndarray]) -> Mesh:
    verts, prims, bids = [], [], []
    offset = 0
    for bid, pts in enumerate(loops):
        n = pts.shape[0]
        verts.append(pts)
        idx = np.arange(n, dtype=np.int32) + offset
        prims.append(np.stack([idx, np.roll(idx, -1)], axis=1))
        bids.append(np.full(n, bid, dtype=np.int32))
        offset += n
    return Mesh(2, np.ascontiguousarray(np.concatenate(verts), dtype=np.float64),
                np.ascontiguousarray(np.concatenate(prims), dtype=np.int32),
                np.ascontiguousarray(np.concatenate(bids), dtype=np.int32))


def _circle_points(radius: float, n: int, clockwise: bool = False) -> np.ndarray:
    k = np.arange(n, dtype=np.float64)
    theta = 2.0 * math.pi * k / n
    if clockwise:
        theta = -theta
    return np.stack([radius * np.cos(theta), radius * np.sin(theta)], axis=1)


def annulus(inner: float = 0.5, outer: float = 1.0, segments: int = 128) -> Mesh:
    """Annulus: outer circle first (boundary_id 0, counter-clockwise), then the
    inner circle (boundary_id 1, clockwise), `segments` uniform edges each."""
    return _loops_to_mesh([_circle_points(outer, segments),
                           _circle_points(inner, segments, clockwise=True)])


def circle(radius: float = 1.0, segments: int = 1024) -> Mesh:
    """Counter-clockwise circle polyline with `segments` uniform edges."""
    return _loops_to_mesh([_circle_points(radius, segments)])


def star_polygon(rng: np.random.Generator, edges: int, harmonics: int = 6,
                 amplitude: float = 0.3, coeff_max: float = 0.15) -> Mesh:
    """r(theta) = 1 + amplitude * sum_k a_k cos(k theta + phi_k), a_k ~ U[0, coeff_max],
    phi_k ~ U[0, 2 pi), sampled at `edges` uniform angles (counter-clockwise)."""
    a = rng.uniform(0.0, coeff_max, harmonics)
    phi = rng.uniform(0.0, 2.0 * math.pi, harmonics)
    theta = 2.0 * math.pi * np.arange(edges) / edges
    r = 1.0 + amplitude * sum(a[k] * np.cos((k + 1) * theta + phi[k]) for k in range(harmonics))
    return _loops_to_mesh([np.stack([r * np.cos(theta), r * np.sin(theta)], axis=1)])


def _uv_grid(lon: int, lat: int):
    """Vertices of a lat/long sphere: north pole, lat-1 rings of `lon`, south pole;
    and its triangles (pole fans plus two triangles per quad), outward facing."""
    verts = [(0.0, 0.0, 1.0)]
    for i in range(1, lat):
        th = math.pi * i / lat
        for j in range(lon):
            ph = 2.0 * math.pi * j / lon
            verts.append((math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)))
    verts.append((0.0, 0.0, -1.0))
    v = np.asarray(verts, dtype=np.float64)
    south = v.shape[0] - 1

    def ring(i, j):
        return 1 + (i - 1) * lon + (j % lon)

    tris = []
    for j in range(lon):
        tris.append((0, ring(1, j), ring(1, j + 1)))
    for i in range(1, lat - 1):
        for j in range(lon):
            a, b = ring(i, j), ring(i, j + 1)
            c, d = ring(i + 1, j), ring(i + 1, j + 1)
            tris.append((a, c, d))
            tris.append((a, d, b))
    for j in range(lon):
        tris.append((south, ring(lat - 1, j + 1), ring(lat - 1, j)))
    return v, np.asarray(tris, dtype=np.int32)


def uv_sphere(radius: float = 1.0, lon: int = 128, lat: int = 64) -> Mesh:
    """Latitude/longitude triangle sphere: 2*lon pole triangles plus
    2*lon*(lat-2) quad triangles (128 x 64 bands -> 16 128 triangles)."""
    v, t = _uv_grid(lon, lat)
    v = v * radius
    return Mesh(3, np.ascontiguousarray(v), np.ascontiguousarray(t),
                np.zeros(t.shape[0], dtype=np.int32))


def _real_sph_harm_basis(theta: np.ndarray, phi: np.ndarray, degree: int) -> list[np.ndarray]:
    """Unnormalised real spherical harmonics (associated Legendre x cos/sin) up to `degree`."""
    from scipy.special import lpmv
    x = np.cos(theta)
    basis = []
    for l in range(1, degree + 1):
        for m in range(0, l + 1):
            p = lpmv(m, l, x)
            p = p / max(1e-12, np.abs(p).max())
            basis.append(p * np.cos(m * phi))
            if m > 0:
                basis.append(p * np.sin(m * phi))
    return basis


def perturbed_sphere(rng: np.random.Generator, lon: int, lat: int, degree: int = 4,
                     amplitude: float = 0.3, coeff_max: float = 0.15) -> Mesh:
    """UV sphere whose radius is 1 + amplitude * sum c_i Y_i(theta, phi) over real
    spherical harmonics of degree 1..`degree`, c_i ~ U[0, coeff_max]."""
    v, t = _uv_grid(lon, lat)
    theta = np.arccos(np.clip(v[:, 2], -1.0, 1.0))
    phi = np.arctan2(v[:, 1], v[:, 0])
    basis = _real_sph_harm_basis(theta, phi, degree)
    c = rng.uniform(0.0, coeff_max, len(basis))
    r = 1.0 + amplitude * sum(ci * b for ci, b in zip(c, basis))
    r = np.maximum(r, 0.2)
    return Mesh(3, np.ascontiguousarray(v * r[:, None]), np.ascontiguousarray(t),
                np.zeros(t.shape[0], dtype=np.int32))


def slab_box(lx: float = 0.10, ly: float = 0.05, lz: float = 0.01,
             target_triangles: int = 20000) -> Mesh:
    """Closed axis-aligned box [0,lx]x[0,ly]x[0,lz] with every face split into a
    uniform grid of right triangles (outward normals), about `target_triangles`
    triangles in total at roughly equal edge length."""
    area = 2.0 * (lx * ly + lx * lz + ly * lz)
    h = math.sqrt(2.0 * area / target_triangles)
    nx, ny, nz = (max(1, round(s / h)) for s in (lx, ly, lz))
    verts: dict[tuple[int, int, int], int] = {}
    pts: list[tuple[float, float, float]] = []

    def vid(i, j, k):
        key = (i, j, k)
        if key not in verts:
            verts[key] = len(pts)
            pts.append((lx * i / nx, ly * j / ny, lz * k / nz))
        return verts[key]

    tris = []

    def face(fixed_axis, fixed_val, flip):
        axes = [a for a in range(3) if a != fixed_axis]
        n = (nx, ny, nz)
        na, nb = n[axes[0]], n[axes[1]]
        for a in range(na):
            for b in range(nb):
                def at(da, db):
                    idx = [0, 0, 0]
                    idx[fixed_axis] = fixed_val
                    idx[axes[0]] = a + da
                    idx[axes[1]] = b + db
                    return vid(*idx)
                q = (at(0, 0), at(1, 0), at(1, 1), at(0, 1))
                t1, t2 = (q[0], q[1], q[2]), (q[0], q[2], q[3])
                if flip:
                    t1, t2 = t1[::-1], t2[::-1]
                tris.extend([t1, t2])

    face(0, 0, False); face(0, nx, True)
    face(1, 0, True); face(1, ny, False)
    face(2, 0, False); face(2, nz, True)
    return Mesh(3, np.asarray(pts, dtype=np.float64), np.asarray(tris, dtype=np.int32),
                np.zeros(len(tris), dtype=np.int32))


def write_obj(mesh: Mesh, path: str | Path) -> Path:
    """Write `mesh` in the reference's OBJ dialect: `v x y [z]`, one closed `l`
    record per 2D boundary loop (boundary_id order), `f a b c` per triangle."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    lines = []
    if mesh.dim == 2:
        lines.extend(f"v {x:.17g} {y:.17g}" for x, y in mesh.verts)
        # rebuild each loop from consecutive segments of the same boundary id
        for bid in range(int(mesh.boundary_ids.max()) + 1 if mesh.n_prims else 0):
            segs = mesh.prims[mesh.boundary_ids == bid]
            chain = [int(segs[0, 0])] + [int(s[1]) for s in segs]
            lines.append("l " + " ".join(str(v + 1) for v in chain))
    else:
        lines.extend(f"v {x:.17g} {y:.17g} {z:.17g}" for x, y, z in mesh.verts)
        lines.extend(f"f {a + 1} {b + 1} {c + 1}" for a, b, c in mesh.prims)
    path.write_text("\n".join(lines) + "\n")
    return path
