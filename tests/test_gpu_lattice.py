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


@pytest.mark.parametrize("mname", ["sphere", "slab"])
def test_cut_lists_keep_every_walk(solver, monkeypatch, mname):
    """3D near-boundary lists are scanned only up to the entries that can be
    nearest for the query's distance from its node (list_prefix).  The
    minimum over that prefix is the minimum over the whole list, so every
    walk takes the same steps as with whole lists (WOS_LIST_CUT=0): the
    screened grid solve (walk kernel) and the heat forward pass (heat
    kernel) match bit for bit."""
    from walk_on_spheres_b200.heat import HeatProblem

    m = meshes.uv_sphere() if mname == "sphere" else meshes.slab_box(target_triangles=20000)

    def run():
        solver.set_mesh(m)  # each upload rebuilds the lists on the first solve
        if mname == "sphere":
            r = solver.solve_grid("screened_poisson", 20, 20, 20, N_walks=256, seed=7,
                                  alpha=10.0, method="fast")
            return r.mean.ravel(), r.mean_steps.ravel(), r.counters
        rng = np.random.default_rng(11)
        probes = np.array([0.10, 0.05, 0.01]) * rng.uniform(0.001, 0.999, size=(512, 3))
        heat = HeatProblem(solver, probes, N_walks=256, epsilon=1e-5, seed=3,
                           source_mode="green", method="fast")
        f = heat.forward(1e3, (0.05, 0.025, 0.01), 2e-3)
        return f.mean, f.mean_steps, f.counters

    cut = run()
    monkeypatch.setenv("WOS_LIST_CUT", "0")
    whole = run()
    monkeypatch.delenv("WOS_LIST_CUT")
    assert cut[2]["exact_queries"] > 0
    assert cut[2]["total_steps"] == whole[2]["total_steps"]
    assert cut[2]["exact_queries"] == whole[2]["exact_queries"]
    assert np.array_equal(cut[1], whole[1], equal_nan=True)
    assert np.array_equal(cut[0], whole[0], equal_nan=True)


def test_tile_lattice_stores_the_node_queries_values(solver, monkeypatch):
    """3D lattices are built by warp tiles, each lane taking its node's
    minimum over candidates shared by the tile; WOS_LATTICE_TILES=0 builds
    them node by node with the conservative cooperative query.  The tile
    value is the unpruned minimum, so it is never above the node query's,
    and it equals it at almost every node."""
    m = meshes.uv_sphere()
    rng = np.random.default_rng(9)
    solver.set_mesh(m)
    lo = np.asarray(solver.bbox[0::2][:3])
    hi = np.asarray(solver.bbox[1::2][:3])
    step = np.max(hi - lo) / 255.0
    n = np.ceil((hi - lo) / step).astype(int) + 1
    idx = rng.integers(0, n, size=(20000, 3))
    # the nodes' FP32 positions glo + i h, where the bound is the node value
    pts = (lo.astype(np.float32)[None, :] + idx.astype(np.float32) * np.float32(step))
    pts = pts.astype(np.float64)
    tiles = solver.distance_bounds(pts)
    monkeypatch.setenv("WOS_LATTICE_TILES", "0")
    solver.set_mesh(m)
    nodes = solver.distance_bounds(pts)
    monkeypatch.delenv("WOS_LATTICE_TILES")
    solver.set_mesh(m)
    assert np.all(tiles <= nodes), np.max(tiles - nodes)
    queried = nodes > 0
    assert queried.sum() > 5000
    assert (tiles[queried] == nodes[queried]).mean() >= 0.95
