"""The device tree build (the default of wos_set_mesh and the batches)
against the host build (WOS_TREE_BUILD=host): the scene arena, every tree
and primitive array the walks read (binary FP64 tree boxes, leaf-slot
records, 32-wide tree boxes and slabs, primitive blocks, slot maps), must be
byte-identical, for 2D and 3D meshes of one to four wide heights, every leaf
size, and coordinates of -0.0.  The walks on the two scenes are then the
same walks: a FAST_FP32 sweep gives identical fields."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from walk_on_spheres_b200 import _lib, meshes

pytestmark = pytest.mark.gpu


def _arena(solver):
    L = _lib.lib()
    n = C.c_longlong()
    _lib.check(L.wos_scene_arena(solver._ctx, None, 0, C.byref(n)), solver._ctx)
    buf = np.empty(n.value, dtype=np.uint8)
    _lib.check(L.wos_scene_arena(solver._ctx, buf.ctypes.data_as(C.c_void_p), n.value,
                                 C.byref(n)), solver._ctx)
    return buf


def _signed_zero_square():
    # the unit square, 4 x 64 segments, its left side at x = -0.0
    t = np.linspace(0.0, 1.0, 65)[:-1]
    pts = np.concatenate([np.stack([t, np.zeros_like(t)], 1),
                          np.stack([np.ones_like(t), t], 1),
                          np.stack([1.0 - t, np.ones_like(t)], 1),
                          np.stack([np.full_like(t, -0.0), 1.0 - t], 1)])
    n = len(pts)
    prims = np.stack([np.arange(n), (np.arange(n) + 1) % n], 1).astype(np.int32)
    return meshes.Mesh(2, pts, prims, np.zeros(n, dtype=np.int32))


def _tetra():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
    f = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], dtype=np.int32)
    return meshes.Mesh(3, v, f, np.zeros(4, dtype=np.int32))


MESHES = {
    "annulus": lambda: meshes.annulus(),
    "circle1024": lambda: meshes.circle(segments=1024),
    "star3000": lambda: meshes.star_polygon(np.random.default_rng(3), 3000),
    "signed_zero_square": _signed_zero_square,
    "tetra": _tetra,
    "sphere16128": lambda: meshes.uv_sphere(),
    "perturbed_sphere": lambda: meshes.perturbed_sphere(np.random.default_rng(4), 200, 100),
    "slab20k": lambda: meshes.slab_box(target_triangles=20000),
}


PARTS = ("box64", "seg64", "segid", "tri64", "wbox", "wprim", "wide2bin", "offsets",
         "slot_verts")


def _parts(mesh, leaf):
    """(name, start, end) of each array in the scene arena (arena_layout)."""
    n, dim = mesh.n_prims, mesh.dim
    leaf = leaf or 4
    D = 0
    while -(-n // (1 << D)) > leaf:
        D += 1
    H, span = 1, 32
    while span < n:
        span, H = span * 32, H + 1
    cnt = [n]
    for _ in range(H):
        cnt.append(-(-cnt[-1] // 32))
    nbox = 3 * dim + 2
    total = sum(cnt[h + 1] * nbox * 32 for h in range(1, H))
    npad = -(-n // 32) * 32
    sizes = [(1 << (D + 1)) * 2 * dim * 8, n * 32 if dim == 2 else 0, n * 8 if dim == 2 else 0,
             n * 112 if dim == 3 else 0, max(total, nbox * 32) * 4,
             npad * (5 if dim == 2 else 16) * 4, npad * 4, 32, n * dim * 4]
    out, at = [], 0
    for name, b in zip(PARTS, sizes):
        out.append((name, at, at + b))
        at += -(-max(b, 16) // 256) * 256
    return out


@pytest.fixture
def host_build():
    def set_host(flag: bool):
        if flag:
            os.environ["WOS_TREE_BUILD"] = "host"
        else:
            os.environ.pop("WOS_TREE_BUILD", None)
    yield set_host
    os.environ.pop("WOS_TREE_BUILD", None)


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("leaf", [0, 2, 8])
def test_device_build_is_byte_identical(solver, host_build, name, leaf):
    mesh = MESHES[name]()
    host_build(True)
    solver.set_mesh(mesh, leaf_size=leaf)
    host = _arena(solver)
    host_build(False)
    solver.set_mesh(mesh, leaf_size=leaf)
    dev = _arena(solver)
    assert host.size == dev.size
    diff = np.flatnonzero(host != dev)
    where = {name: int(((diff >= a) & (diff < b)).sum()) for name, a, b in _parts(mesh, leaf)}
    assert diff.size == 0, f"{diff.size} bytes differ: {where}"


@pytest.mark.parametrize("name", ["circle1024", "sphere16128"])
def test_walks_on_the_device_built_scene_are_the_host_built_ones(solver, host_build, name):
    mesh = MESHES[name]()
    shape = (48, 48, 1) if mesh.dim == 2 else (16, 16, 16)
    eq = "poisson" if mesh.dim == 2 else "screened_poisson"
    out = []
    for on_host in (True, False):
        host_build(on_host)
        solver.set_mesh(mesh)
        out.append(solver.solve_grid(eq, *shape, N_walks=256, seed=9, alpha=10.0,
                                     method="fast"))
    assert np.array_equal(out[0].location, out[1].location)
    assert np.array_equal(out[0].mean, out[1].mean, equal_nan=True)
    assert np.array_equal(out[0].mean_steps, out[1].mean_steps, equal_nan=True)
