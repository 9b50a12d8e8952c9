"""CPU tests of libwos_b200's C ABI and host logic (no GPU needed): symbol
exports, the OBJ reader against the reference loader (src/mesh.cpp), the host
BVH build, and the HDF5 result writer against the pure-Python reader (itself
checked on a libhdf5-written file)."""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

import numpy as np
import pytest

from walk_on_spheres_b200 import _lib, h5lite, meshes

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "wos_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(wos_[a-z0-9_]+)\s*\(", text))
    return sorted(n for n in names if not n.endswith("_fn"))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.wos_abi_version() == 2
    assert set(_lib.SIGNATURES) <= set(names)


def test_registry_names():
    from walk_on_spheres_b200.solver import registry
    assert [e.name for e in registry()] == ["laplace", "poisson", "screened_poisson", "helmholtz"]


def test_registry_entry_rejects_several_ranks_without_collectives(tmp_path):
    """With no collectives installed (wos_set_collectives) a multi-rank call
    fails with 1, the reference's failure code, before touching the mesh, the
    output or a GPU."""
    from walk_on_spheres_b200.solver import registry
    out = tmp_path / "never.h5"
    for e in registry():
        for run in (e.run_2D, e.run_3D):
            assert run(1, 2, b"missing.obj", str(out).encode(), 4, 4, 1, 10, 1e-2, 1000, 12, 1,
                       5.0, 0) == 1
            assert run(0, 2, b"missing.obj", str(out).encode(), 4, 4, 1, 10, 1e-2, 1000, 12, 1,
                       5.0, 0) == 1
    assert not out.exists()


def read_obj(path):
    L = _lib.lib()
    f = L.wos_read_obj
    f.restype = C.c_int
    dim, nv, npr = C.c_int(), C.c_int(), C.c_int()
    err = C.create_string_buffer(512)
    rc = f(str(path).encode(), C.byref(dim), C.byref(nv), C.byref(npr), None, None, None, err, 512)
    if rc:
        return rc, err.value.decode()
    verts = np.zeros((nv.value, dim.value))
    prims = np.zeros((npr.value, dim.value), dtype=np.int32)
    bids = np.zeros(npr.value, dtype=np.int32)
    f(str(path).encode(), C.byref(dim), C.byref(nv), C.byref(npr),
      verts.ctypes.data_as(C.c_void_p), prims.ctypes.data_as(C.c_void_p),
      bids.ctypes.data_as(C.c_void_p), err, 512)
    return 0, (dim.value, verts, prims, bids)


BAD_OBJS = {
    "no_vertices.obj": "l 1 2\n",
    "short_polyline.obj": "v 0 0\nv 1 0\nl 1\n",
    "quad.obj": "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n",
    "index_range.obj": "v 0 0\nv 1 0\nv 1 1\nl 1 2 9\n",
    "zero_index.obj": "v 0 0\nv 1 0\nl 0 1\n",
    "bad_index.obj": "v 0 0\nv 1 0\nl 1 x2\n",
    "zero_length.obj": "v 0 0\nv 0 0\nv 1 0\nl 1 2 3\n",
    "degenerate.obj": "v 0 0 0\nv 1 0 0\nv 2 0 0\nv 0 1 0\nf 1 2 3\nf 1 2 4\n",
    "malformed_vertex.obj": "v 0\nv 1 0\nl 1 2\n",
    "nonfinite.obj": "v 0 0 inf\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
    "no_prims.obj": "v 0 0\nv 1 1\n",
    "bad_face.obj": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 #c\n",
}

GOOD_OBJS = {
    # open polyline auto-closed, comments, slash references, second loop
    "open.obj": "# c\nv 0 0\nv 1 0\nv 1 1 # z-less\nl 1 2/5 3\nv 3 3\nv 4 3\nv 4 4\nl 4 5 6 4\n",
    "tri.obj": "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nf 1 3 2\nf 1 2 4\nf 2 3 4\nf 1 4 3\n",
}


@pytest.mark.parametrize("name", sorted(BAD_OBJS))
def test_obj_errors_match_reference(tmp_path, reference, name):
    p = tmp_path / name
    p.write_text(BAD_OBJS[name])
    rc, msg = read_obj(p)
    assert rc == 3
    with pytest.raises(ValueError) as e:
        reference.load_mesh(str(p))
    assert msg == str(e.value)


@pytest.mark.parametrize("name", sorted(GOOD_OBJS))
def test_obj_reader_matches_reference(tmp_path, reference, name):
    p = tmp_path / name
    p.write_text(GOOD_OBJS[name])
    rc, (dim, verts, prims, bids) = read_obj(p)
    assert rc == 0
    rdim, rv, rp, rb = reference.load_mesh(str(p))
    assert dim == rdim
    assert np.array_equal(verts, rv)
    assert np.array_equal(prims, rp)
    if dim == 2:
        assert np.array_equal(bids, rb)


def test_generated_meshes_round_trip(tmp_path):
    for m in (meshes.annulus(), meshes.uv_sphere(lon=16, lat=8)):
        p = meshes.write_obj(m, tmp_path / f"m{m.dim}.obj")
        rc, (dim, verts, prims, bids) = read_obj(p)
        assert rc == 0 and dim == m.dim
        assert np.array_equal(verts, m.verts)
        assert np.array_equal(prims, m.prims)
        if dim == 2:
            assert np.array_equal(bids, m.boundary_ids)


def build_bvh(m, leaf):
    L = _lib.lib()
    f = L.wos_build_bvh
    f.restype = C.c_int
    verts = np.ascontiguousarray(m.verts)
    prims = np.ascontiguousarray(m.prims, dtype=np.int32)
    d = C.c_int()
    assert f(m.dim, verts.ctypes.data_as(C.c_void_p), verts.shape[0],
             prims.ctypes.data_as(C.c_void_p), prims.shape[0], leaf, C.byref(d), None, None) == 0
    D = d.value
    boxes = np.zeros((2 ** (D + 1), 2 * m.dim))
    order = np.zeros(m.n_prims, dtype=np.int32)
    f(m.dim, verts.ctypes.data_as(C.c_void_p), verts.shape[0], prims.ctypes.data_as(C.c_void_p),
      prims.shape[0], leaf, C.byref(d), boxes.ctypes.data_as(C.c_void_p),
      order.ctypes.data_as(C.c_void_p))
    return D, boxes, order


@pytest.mark.parametrize("leaf", [2, 3, 4, 6, 8])
@pytest.mark.parametrize("mname", ["annulus", "sphere", "circle1000"])
def test_host_bvh_invariants(leaf, mname):
    m = {"annulus": meshes.annulus(), "sphere": meshes.uv_sphere(lon=20, lat=11),
         "circle1000": meshes.circle(segments=1000)}[mname]
    D, boxes, order = build_bvh(m, leaf)
    n, d = m.n_prims, m.dim
    assert sorted(order.tolist()) == list(range(n))          # every primitive once
    assert -(-n // 2 ** D) <= leaf                            # ceil(n / 2^D) fits a leaf
    assert D == 0 or -(-n // 2 ** (D - 1)) > leaf             # and D is the smallest such depth
    lo_p = m.verts[m.prims].min(axis=1)
    hi_p = m.verts[m.prims].max(axis=1)
    for j in range(2 ** D):
        b, e = (j * n) >> D, ((j + 1) * n) >> D
        node = 2 ** D + j
        sl = order[b:e]
        assert e > b
        assert np.array_equal(boxes[node, :d], lo_p[sl].min(axis=0))
        assert np.array_equal(boxes[node, d:], hi_p[sl].max(axis=0))
    for i in range(1, 2 ** D):                                # parents bound children
        assert np.array_equal(boxes[i, :d], np.minimum(boxes[2 * i, :d], boxes[2 * i + 1, :d]))
        assert np.array_equal(boxes[i, d:], np.maximum(boxes[2 * i, d:], boxes[2 * i + 1, d:]))


def test_mesh_validation_rejects_degenerate():
    L = _lib.lib()
    verts = np.array([[0.0, 0.0], [0.0, 0.0], [1.0, 0.0]])
    prims = np.array([[0, 1], [1, 2], [2, 0]], dtype=np.int32)
    L.wos_build_bvh.restype = C.c_int
    rc = L.wos_build_bvh(2, verts.ctypes.data_as(C.c_void_p), 3, prims.ctypes.data_as(C.c_void_p),
                         3, 0, None, None, None)
    assert rc == 3


SPECIMEN = Path(np.__file__).resolve().parents[1] / "scipy" / "io" / "matlab" / "tests" / \
    "data" / "testhdf5_7.4_GLNX86.mat"


@pytest.mark.skipif(not SPECIMEN.exists(), reason="libhdf5-written specimen not available")
def test_h5lite_reads_libhdf5_file():
    f = h5lite.read(SPECIMEN)
    assert list(f) == ["/testdouble"]
    assert np.allclose(f["/testdouble"].ravel(), np.arange(9) * np.pi / 4)


def write_result(path, grid, fields, meta):
    L = _lib.lib()
    f = L.wos_write_hdf5
    f.restype = C.c_int
    f.argtypes = [C.c_char_p, C.POINTER(_lib.Grid)] + [C.c_void_p] * 5 + [
        C.c_int, C.c_double, C.c_int, C.c_longlong, C.c_int, C.c_int, C.c_longlong,
        C.c_longlong, C.c_uint64, C.c_int, C.c_double, C.c_int]
    return f(str(path).encode(), C.byref(grid),
             *[a.ctypes.data_as(C.c_void_p) for a in fields], *meta)


@pytest.mark.parametrize("dim", [2, 3])
def test_hdf5_result_layout(tmp_path, dim):
    nx, ny, nz = 5, 4, (3 if dim == 3 else 1)
    g = _lib.Grid(nx, ny, nz, -1.0, 1.0, -0.5, 0.5, (-2.0 if dim == 3 else 0.0),
                  (2.0 if dim == 3 else 0.0))
    rng = np.random.default_rng(dim)
    n = nx * ny * nz
    fields = [rng.standard_normal(n) for _ in range(4)] + [rng.integers(0, 4, n).astype(np.uint8)]
    meta = (1234, 0.005, 1000, 17, int(dim == 3), 12, 5, 2, 2**64 - 5, 1, 10.0, 1)
    assert write_result(tmp_path / "r.h5", g, fields, meta) == 0
    f = h5lite.read(tmp_path / "r.h5")
    names = ["mean", "variance", "standard_error", "mean_steps", "location"]
    for k, a in zip(names, fields):
        assert f["/" + k].shape == (nx, ny, nz)
        assert np.array_equal(f["/" + k].ravel(), a)
    assert f["/location"].dtype == np.uint8 and f["/mean"].dtype == np.float64
    assert np.array_equal(f["/x"], [-1.0 + 2.0 * i / 4 for i in range(nx)])
    assert f["/z"].shape == (nz,)
    m = {k.split("/")[-1]: v for k, v in f.items() if k.startswith("/metadata/")}
    assert m["N_walks"] == 1234 and m["N_walks"].dtype == np.int32
    assert m["epsilon"] == 0.005 and m["max_steps"] == 1000
    assert m["max_steps_hits"] == 17 and m["max_steps_hits"].dtype == np.int64
    assert m["seed"] == 2**64 - 5 and m["seed"].dtype == np.uint64
    assert m["alpha"] == 10.0 and m["source_mode"] == 1
    assert ("ambiguous_ray_retries" in m) == (dim == 3)
    if dim == 3:
        assert m["max_ray_attempts"] == 12 and m["indeterminate_points"] == 2


def build_wide(m):
    L = _lib.lib()
    verts = np.ascontiguousarray(m.verts)
    prims = np.ascontiguousarray(m.prims, dtype=np.int32)
    H, E = C.c_int(), C.c_int()
    offs = np.zeros(8, dtype=np.int32)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    assert L.wos_build_wide_bvh(m.dim, vp(verts), verts.shape[0], vp(prims), prims.shape[0],
                                C.byref(H), C.byref(E), vp(offs), None, None) == 0
    nodes = np.zeros(E.value, dtype=np.float32)
    order = np.zeros(m.n_prims, dtype=np.int32)
    L.wos_build_wide_bvh(m.dim, vp(verts), verts.shape[0], vp(prims), prims.shape[0],
                         C.byref(H), C.byref(E), vp(offs), vp(nodes), vp(order))
    return H.value, offs, nodes, order


@pytest.mark.parametrize("mname", ["annulus", "circle1024", "sphere", "star", "pert"])
def test_wide_bvh_bounds_contain_primitives(mname):
    rng = np.random.default_rng(3)
    m = {"annulus": meshes.annulus(), "circle1024": meshes.circle(segments=1024),
         "sphere": meshes.uv_sphere(lon=48, lat=24),
         "star": meshes.star_polygon(rng, 3000),
         "pert": meshes.perturbed_sphere(rng, 40, 20)}[mname]
    H, offs, nodes, order = build_wide(m)
    n, d = m.n_prims, m.dim
    assert sorted(order.tolist()) == list(range(n))
    assert 32 ** H >= n and (H == 1 or 32 ** (H - 1) < n)
    V = m.verts[m.prims[order]].astype(np.float64)          # (n, dim, dim) in wide-slot order
    for h in range(1, H):
        span = 32 ** h
        count = -(-n // span)
        for i in range(count):
            pts = V[i * span:min(n, (i + 1) * span)].reshape(-1, d)
            nb = 3 * d + 2
            blk = offs[h] + (i // 32) * nb * 32
            col = nodes[blk + np.arange(nb) * 32 + i % 32].astype(np.float64)
            lo, hi = col[:d], col[d:2 * d]
            nrm, c, th = col[2 * d:3 * d], col[3 * d], col[3 * d + 1]
            assert (pts >= lo).all() and (pts <= hi).all()
            # the slab test as the device evaluates it, in float32
            t = np.abs((pts.astype(np.float32) * nrm.astype(np.float32)).sum(axis=1,
                       dtype=np.float32) - np.float32(c))
            assert (t <= np.float32(th)).all(), (h, i, t.max(), th)
            assert abs(np.linalg.norm(nrm) - 1.0) < 1e-5


def _tree_arrays(threads: int) -> dict:
    """Binary and wide trees of a 57 120-triangle mesh built with `threads` host
    threads (WOS_HOST_THREADS), in a fresh process."""
    import json
    import os
    import subprocess
    import sys
    code = (
        "import json, sys, numpy as np, ctypes as C\n"
        "sys.path.insert(0, %r)\n"
        "from walk_on_spheres_b200 import meshes\n"
        "from tests.test_host_abi import build_wide\n"
        "from walk_on_spheres_b200 import _lib\n"
        "m = meshes.perturbed_sphere(np.random.default_rng(11), 240, 120)\n"
        "H, offs, nodes, order = build_wide(m)\n"
        "L = _lib.lib(); vp = lambda a: a.ctypes.data_as(C.c_void_p)\n"
        "v = np.ascontiguousarray(m.verts); p = np.ascontiguousarray(m.prims, dtype=np.int32)\n"
        "D = C.c_int(); L.wos_build_bvh.restype = C.c_int\n"
        "L.wos_build_bvh(3, vp(v), v.shape[0], vp(p), p.shape[0], 4, C.byref(D), None, None)\n"
        "boxes = np.zeros((2 ** (D.value + 1)) * 6); border = np.zeros(p.shape[0], dtype=np.int32)\n"
        "L.wos_build_bvh(3, vp(v), v.shape[0], vp(p), p.shape[0], 4, C.byref(D), vp(boxes), vp(border))\n"
        "np.savez(sys.argv[1], H=H, offs=offs, nodes=nodes, order=order, boxes=boxes, border=border)\n"
    ) % str(Path(__file__).resolve().parents[1])
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "t.npz")
        env = dict(os.environ, WOS_HOST_THREADS=str(threads))
        subprocess.run([sys.executable, "-c", code, out], check=True, env=env)
        return dict(np.load(out))


def test_threaded_build_is_bit_identical_to_a_serial_build():
    serial, threaded = _tree_arrays(1), _tree_arrays(8)
    assert serial["nodes"].size > 0 and serial["order"].size == 57120
    for k in serial:
        assert np.array_equal(serial[k], threaded[k]), k


# OBJ dialect edge cases: whatever the reference's loader does (load, or fail
# with a message), wos_read_obj must do the same
EDGE_OBJS = {
    "crlf.obj": "v 0 0\r\nv 1 0\r\nv 1 1\r\nl 1 2 3 1\r\n",
    "tabs.obj": "v\t0\t0\nv  1   0\nv 1 1\t\nl\t1 2  3\n",
    "leading_space.obj": "  v 0 0\n v 1 0\nv 1 1\n  l 1 2 3\n",
    "scientific.obj": "v 1e-3 -2.5E+1\nv 1.5e0 0\nv +2 .5\nl 1 2 3\n",
    "no_final_newline.obj": "v 0 0\nv 1 0\nv 1 1\nl 1 2 3",
    "blank_lines.obj": "\n\nv 0 0\n   \nv 1 0\nv 1 1\n\nl 1 2 3\n\n",
    "negative_index.obj": "v 0 0\nv 1 0\nv 1 1\nl -3 -2 -1\n",
    "other_records.obj": "mtllib a.mtl\no obj\ng grp\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\n"
                         "vn 0 0 1\nvt 0 0\ns off\nusemtl m\nf 1 3 2\nf 1 2 4\nf 2 3 4\nf 1 4 3\n",
    "face_slashes.obj": "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nf 1/1/1 3//3 2/2\nf 1 2 4\n"
                        "f 2 3 4\nf 1 4 3\n",
    "line_in_3d.obj": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\nl 1 2\n",
    "face_in_2d.obj": "v 0 0\nv 1 0\nv 1 1\nl 1 2 3\nf 1 2 3\n",
    "vertex_w.obj": "v 0 0 0 1\nv 1 0 0 1\nv 0 1 0 1\nv 0 0 1 1\nf 1 3 2\nf 1 2 4\n"
                    "f 2 3 4\nf 1 4 3\n",
    "z_in_2d.obj": "v 0 0 0\nv 1 0 0\nv 1 1 0\nl 1 2 3\n",
    "two_loops_closed.obj": "v 0 0\nv 4 0\nv 4 4\nv 0 4\nl 1 2 3 4 1\nv 1 1\nv 2 1\nv 2 2\n"
                            "l 5 6 7 5\n",
    "comment_only_line.obj": "# header\n#\nv 0 0 # a\nv 1 0\nv 1 1\nl 1 2 3 # closing\n",
    "uppercase_record.obj": "V 0 0\nV 1 0\nV 1 1\nL 1 2 3\n",
    "long_polyline.obj": "".join(f"v {np.cos(t):.17g} {np.sin(t):.17g}\n"
                                 for t in np.linspace(0, 2 * np.pi, 200, endpoint=False))
                         + "l " + " ".join(str(i) for i in range(1, 201)) + " 1\n",
}


@pytest.mark.parametrize("name", sorted(EDGE_OBJS))
def test_obj_edge_cases_match_reference(tmp_path, reference, name):
    p = tmp_path / name
    p.write_bytes(EDGE_OBJS[name].encode())
    rc, got = read_obj(p)
    try:
        rdim, rv, rp, rb = reference.load_mesh(str(p))
    except ValueError as e:
        assert rc == 3, f"reference rejects ({e}); ours loads"
        assert got == str(e)
        return
    assert rc == 0, f"reference loads; ours rejects: {got}"
    dim, verts, prims, bids = got
    assert dim == rdim
    assert np.array_equal(verts, rv)
    assert np.array_equal(prims, rp)
    if dim == 2:
        assert np.array_equal(bids, rb)


def test_missing_library_fails_loudly(tmp_path):
    """Without the built CUDA library the package raises: there is no CPU
    fallback for any solve."""
    import subprocess
    import sys
    code = ("from walk_on_spheres_b200 import Solver\n"
            "try:\n    Solver(0)\nexcept ImportError as e:\n    print('ImportError:', e)\n")
    env = dict(os.environ, WOS_B200_LIB=str(tmp_path / "absent.so"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       cwd=ROOT, env=env, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "ImportError:" in r.stdout and "no CPU fallback" in r.stdout


def test_no_device_is_an_error_not_a_fallback():
    """On a machine without a CUDA device, creating a context fails with the
    CUDA status instead of computing anything on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from walk_on_spheres_b200 import Solver
    with pytest.raises(RuntimeError):
        Solver(0)
