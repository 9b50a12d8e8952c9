"""The FAST_FP32 distance lattice (wos_distance_bounds): its bounds never
exceed the exact FP64 boundary distance (so every lattice radius keeps the
ball inside the domain) and, inside the domain, are within half a lattice
diagonal of it.  Nodes outside the mesh whose neighbours are all outside are
not queried and hold 0."""
from __future__ import annotations

import numpy as np
import pytest

from walk_on_spheres_b200 import meshes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mname,G", [("circle1024", 2048), ("annulus", 2048), ("sphere", 256),
                                     ("star", 2048), ("slab", 256)])
def test_bounds_are_valid_and_tight(solver, mname, G):
    rng = np.random.default_rng(5)
    m = {"circle1024": meshes.circle(segments=1024), "annulus": meshes.annulus(),
         "sphere": meshes.uv_sphere(), "star": meshes.star_polygon(rng, 3000),
         # thin and anisotropic: 0.10 x 0.05 x 0.01 m, cells of 0.4 mm
         "slab": meshes.slab_box(target_triangles=20000)}[mname]
    solver.set_mesh(m)
    lo, hi = np.asarray(solver.bbox[0::2][:m.dim]), np.asarray(solver.bbox[1::2][:m.dim])
    pts = lo + (hi - lo) * rng.random((20000, m.dim))
    bound = solver.distance_bounds(pts)
    exact, _, _ = solver.closest_points(pts, precision=64)
    assert np.all(np.isfinite(bound))
    assert np.all(bound <= exact), np.max(bound - exact)
    h = np.max(hi - lo) / (G - 1)
    loc = solver.solve_points("laplace", pts, N_walks=1, method="fast").location
    ins = loc == 1
    assert ins.sum() > 1000
    # node values are the conservatively pruned query: within 1 - 2^-10 of
    # the node distance
    slack = h * np.sqrt(m.dim) * 1.0001 + 2.0 ** -10 * exact + 1e-5 * max(1.0, np.max(np.abs(hi)))
    assert np.all((exact - bound)[ins] <= slack[ins]), np.max(((exact - bound) / slack)[ins])
    # well outside the mesh the nodes were skipped: their bound is 0 - r.  2D
    # rows are classified exactly; a 3D row passing within 1e-5 of a
    # projected edge stays unclassified (a few per cent of rows)
    far = (loc == 0) & (exact > 2.5 * h * np.sqrt(m.dim))
    if far.sum() > 50:
        frac = (bound[far] <= 0.0).mean()
        assert frac >= (0.99 if m.dim == 2 else 0.9), frac


def test_small_meshes_have_no_lattice(solver):
    solver.set_mesh(meshes.circle(segments=32))
    b = solver.distance_bounds(np.zeros((3, 2)))
    assert np.all(np.isnan(b))
