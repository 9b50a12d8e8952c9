"""Parallel write path of the result file (the reference's collective
hyperslab writes, include/wos/hdf5_io.hpp:51-171, over the rank blocks of
include/wos/runner.hpp:90-134): one process creates the file, ranks write
their parts of the fields.  The result must be byte-identical to the serial
writer's file of the whole fields, whatever the split.  CPU only: these are
host entry points of libwos_b200.so."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from walk_on_spheres_b200 import _lib, h5lite, meshes, parallel, results

META2 = results.ResultMeta(N_walks=4096, epsilon=1e-2, max_steps=1000, max_steps_hits=3,
                           seed=12345, write_source_metadata=True, alpha=5.0, source_mode=1)
META3 = results.ResultMeta(N_walks=1024, epsilon=5e-3, max_steps=1000, max_steps_hits=0,
                           write_ray_metadata=True, max_ray_attempts=12,
                           ambiguous_ray_retries=7, indeterminate_points=1, seed=2**64 - 3,
                           write_source_metadata=True, alpha=10.0, source_mode=0)


def _grid(nx, ny, nz):
    return _lib.Grid(nx, ny, nz, -1.0, 1.0, -0.75, 0.5, (-2.0 if nz > 1 else 0.0),
                     (2.0 if nz > 1 else 0.0))


def _fields(n, seed):
    rng = np.random.default_rng(seed)
    f = {k: rng.standard_normal(n) for k in results.FIELDS[:4]}
    f["mean"][rng.random(n) < 0.2] = np.nan        # outside points
    f["location"] = rng.integers(0, 4, n).astype(np.uint8)
    return f


def _serial_bytes(tmp_path, grid, fields, meta):
    p = tmp_path / "serial.h5"
    results.write(p, grid, fields, meta)
    return p.read_bytes()


# the last shape's f64 fields (128 KB each) are written from the caller's
# arrays, the smaller ones through the file image
SHAPES = [((7, 5, 1), META2), ((1, 1, 1), META2), ((6, 5, 4), META3), ((3, 1, 9), META3),
          ((40, 40, 10), META3)]


@pytest.mark.parametrize("shape,meta", SHAPES)
def test_range_shards_equal_the_serial_file(tmp_path, shape, meta):
    grid = _grid(*shape)
    n = int(np.prod(shape))
    fields = _fields(n, n)
    want = _serial_bytes(tmp_path, grid, fields, meta)
    p = tmp_path / "sharded.h5"
    lay = results.create(p, grid, meta)
    cuts = sorted({0, n, n // 3, (2 * n) // 3})
    spans = list(zip(cuts[:-1], cuts[1:])) + [(n, n)]        # includes an empty range
    for s, e in reversed(spans):                               # any order
        results.write_range(p, lay, grid, s, {k: v[s:e] for k, v in fields.items()})
    assert p.read_bytes() == want
    f = h5lite.read(tmp_path / "serial.h5")
    for k in results.FIELDS:
        np.testing.assert_array_equal(f["/" + k].ravel(), fields[k])


def _reference_blocks(shape, dims):
    """The reference's rank blocks: x_start = Nx*cx/dims[0] ... (runner.hpp:116-128)."""
    out = []
    for cx in range(dims[0]):
        for cy in range(dims[1]):
            for cz in range(dims[2]):
                lo = [shape[d] * c // dims[d] for d, c in enumerate((cx, cy, cz))]
                hi = [shape[d] * (c + 1) // dims[d] for d, c in enumerate((cx, cy, cz))]
                out.append((lo, hi))
    return out


@pytest.mark.parametrize("shape,dims,meta", [((7, 5, 1), (2, 2, 1), META2),
                                             ((6, 5, 4), (1, 3, 2), META3),
                                             ((6, 5, 4), (3, 1, 1), META3),
                                             ((5, 4, 7), (2, 2, 2), META3)])
def test_reference_rank_blocks_equal_the_serial_file(tmp_path, shape, dims, meta):
    grid = _grid(*shape)
    n = int(np.prod(shape))
    fields = _fields(n, 7 * n)
    want = _serial_bytes(tmp_path, grid, fields, meta)
    p = tmp_path / "blocks.h5"
    results.create(p, grid, meta)
    lay = results.layout(grid, meta.write_ray_metadata, meta.write_source_metadata)
    full = {k: v.reshape(shape) for k, v in fields.items()}
    for lo, hi in _reference_blocks(shape, dims):
        block = {k: np.ascontiguousarray(v[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]])
                 for k, v in full.items()}
        results.write_block(p, lay, grid, lo, block)
    assert p.read_bytes() == want
    f = h5lite.read(p)
    np.testing.assert_array_equal(f["/location"], full["location"])
    np.testing.assert_array_equal(f["/variance"], full["variance"])


def test_layout_depends_only_on_shape_and_switches(tmp_path):
    grid = _grid(6, 5, 4)
    for ray in (False, True):
        for source in (False, True):
            meta = results.ResultMeta(N_walks=1, epsilon=0.1, max_steps=5, seed=9,
                                      write_ray_metadata=ray, write_source_metadata=source)
            lay = results.layout(grid, ray, source)
            made = results.create(tmp_path / f"l{ray}{source}.h5", grid, meta)
            assert list(lay.field_offset) == list(made.field_offset)
            assert lay.file_size == made.file_size == (tmp_path / f"l{ray}{source}.h5").stat().st_size
            offs = list(lay.field_offset)
            # five disjoint value regions: four f64 fields, then the u8 one
            sizes = [8 * 120] * 4 + [120]
            assert all(offs[i] + sizes[i] <= offs[i + 1] for i in range(4))
            assert offs[4] + sizes[4] <= lay.file_size


def test_created_file_reads_before_the_fields_are_written(tmp_path):
    grid = _grid(4, 3, 1)
    p = tmp_path / "empty.h5"
    results.create(p, grid, META2)
    f = h5lite.read(p)
    assert f["/mean"].shape == (4, 3, 1) and np.all(f["/mean"] == 0.0)
    assert np.array_equal(f["/x"], [-1.0 + 2.0 * i / 3 for i in range(4)])
    m = {k.split("/")[-1]: v for k, v in f.items() if k.startswith("/metadata/")}
    assert m["max_steps_hits"] == 3 and m["alpha"] == 5.0 and m["seed"] == 12345


def test_write_errors(tmp_path):
    grid = _grid(4, 3, 2)
    p = tmp_path / "r.h5"
    lay = results.create(p, grid, META3)
    blk = {k: (np.zeros((2, 2, 2), np.uint8) if k == "location" else np.zeros((2, 2, 2)))
           for k in results.FIELDS}
    with pytest.raises(RuntimeError, match="leaves the grid"):
        results.write_block(p, lay, grid, (3, 0, 0), blk)        # x 3..4 of 4
    with pytest.raises(RuntimeError, match="leaves the grid"):
        results.write_block(p, lay, grid, (0, -1, 0), blk)
    rng = {k: v.reshape(-1)[:5] for k, v in blk.items()}
    with pytest.raises(RuntimeError, match="leaves the grid"):
        results.write_range(p, lay, grid, 20, rng)               # points 20..24 of 24
    with pytest.raises(RuntimeError, match="cannot open"):
        results.write_range(p.with_name("missing.h5"), lay, grid, 0, rng)
    junk = tmp_path / "junk.h5"
    junk.write_bytes(b"\0" * lay.file_size)
    with pytest.raises(RuntimeError, match="not a created result file"):
        results.write_range(junk, lay, grid, 0, rng)
    other = results.layout(_grid(4, 3, 3), True, True)
    with pytest.raises(RuntimeError, match="layout is not this grid's"):
        results.write_range(p, other, grid, 0, rng)
    with pytest.raises(ValueError):
        results.write_range(p, lay, grid, 0, {**rng, "variance": np.zeros(4)})


# --------------------------------------------------------------- two ranks

def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_shard_solver(mesh, eq, shape, kw):
    from oracle.oracle import Oracle, Solve
    o = Oracle()

    def solve(start, end):
        pts = np.arange(start, end, dtype=np.int64)
        r = o.solve_grid(eq, Solve(mesh, *shape, points=pts, n_threads=1, **kw))
        out = {k: getattr(r, k)[start:end] for k in parallel.FIELDS}
        out["counters"] = r.counters
        return out

    return solve


def _worker(rank, world, port, case, path, results_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mesh, eq, shape, kw, meta = case
        grid = _grid_over(mesh, shape)
        total = parallel.solve_grid_sharded_to_file(_oracle_shard_solver(mesh, eq, shape, kw),
                                                    grid, path, meta)
        results_q.put((rank, total))
    finally:
        dist.destroy_process_group()


def _grid_over(mesh, shape):
    b = mesh.bbox()
    return _lib.Grid(*shape, *b)


CASES = {
    "annulus_laplace": (meshes.annulus(), "laplace", (13, 11, 1), dict(N_walks=40, seed=5),
                        results.ResultMeta(N_walks=40, epsilon=1e-2, max_steps=1000, seed=5)),
    "sphere_screened": (meshes.uv_sphere(lon=16, lat=8), "screened_poisson", (5, 6, 7),
                        dict(N_walks=20, seed=9, alpha=10.0),
                        results.ResultMeta(N_walks=20, epsilon=5e-3, max_steps=1000, seed=9,
                                           write_ray_metadata=True, max_ray_attempts=12,
                                           write_source_metadata=True, alpha=10.0)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_two_ranks_write_the_single_process_file(tmp_path, oracle, name):
    from oracle.oracle import Solve
    mesh, eq, shape, kw, meta = CASES[name]
    path = str(tmp_path / "two_ranks.h5")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, CASES[name], path, q))
             for r in range(2)]
    for p in procs:
        p.start()
    totals = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = oracle.solve_grid(eq, Solve(mesh, *shape, n_threads=1, **kw))
    c = ref.counters
    assert totals[0]["inside_points"] == totals[1]["inside_points"] == c["inside_points"]
    import dataclasses
    full = dataclasses.replace(meta, max_steps_hits=c["max_steps_hits"],
                               ambiguous_ray_retries=c.get("ambiguous_ray_retries", 0),
                               indeterminate_points=c.get("indeterminate_points", 0))
    want = _serial_bytes(tmp_path, _grid_over(mesh, shape),
                         {k: getattr(ref, k) for k in results.FIELDS}, full)
    assert open(path, "rb").read() == want


def _failing_worker(rank, world, port, path, results_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        grid = _grid(4, 3, 1)

        def solve(start, end):
            f = _fields(end - start, start)
            f["counters"] = {"inside_points": end - start}
            return f

        try:
            parallel.solve_grid_sharded_to_file(solve, grid, path, META2)
            results_q.put((rank, "no error"))
        except RuntimeError as e:
            results_q.put((rank, str(e)))
    finally:
        dist.destroy_process_group()


def test_failed_create_raises_on_every_rank(tmp_path):
    """Rank 0 cannot create the file (its directory does not exist): every
    rank raises after the same collective steps instead of waiting."""
    path = str(tmp_path / "no_such_dir" / "r.h5")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, path, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all("creating the file failed" in got[r] for r in range(2)), got


def test_serial_write_error_is_reported(tmp_path):
    grid = _grid(2, 2, 1)
    with pytest.raises(RuntimeError, match="could not create"):
        results.write(tmp_path / "no_such_dir" / "r.h5", grid, _fields(4, 1), META2)


# --------------------------------------------- a registry run's metadata

RUNS = [("laplace", "annulus", (9, 8, 1), 40, 1e-2, 3, 5.0, 0),
        ("poisson", "circle", (8, 8, 1), 40, 2e-2, 4, 5.0, 1),
        ("screened_poisson", "sphere", (5, 5, 5), 20, 1e-2, 7, 10.0, 0),
        ("helmholtz", "sphere", (5, 4, 5), 20, 1e-2, 9, 5.0, 0)]


@pytest.mark.parametrize("run", RUNS, ids=[r[0] for r in RUNS])
def test_writer_reproduces_reference_registry_file(tmp_path, reference, run):
    """Our writer, given a reference registry run's fields and the metadata
    rules of results.run_meta, writes exactly the datasets that run wrote."""
    eq, mname, shape, walks, eps, seed, alpha, mode = run
    mesh = {"annulus": meshes.annulus(segments=32), "circle": meshes.circle(segments=64),
            "sphere": meshes.uv_sphere(lon=12, lat=6)}[mname]
    obj = meshes.write_obj(mesh, tmp_path / "m.obj")
    ref = reference.run_registry(eq, mesh.dim, str(obj), *shape, walks, eps, 1000, 12, seed,
                                 alpha, mode)
    eff = min(eps, 0.05 / alpha) if eq == "screened_poisson" else eps
    counters = {k: int(ref["/metadata/" + k].view(np.int64)[0])
                for k in ("max_steps_hits", "ambiguous_ray_retries", "indeterminate_points")
                if "/metadata/" + k in ref}
    meta = results.run_meta(eq, mesh.dim, walks, eff, 1000, seed, alpha=alpha, source_mode=mode,
                            max_ray_attempts=12, counters=counters)
    x, y, z = (ref[a].view(np.float64) for a in ("/x", "/y", "/z"))
    grid = _lib.Grid(*shape, x[0], x[-1], y[0], y[-1], z[0], z[-1])
    fields = {k: ref["/" + k].view(np.uint8 if k == "location" else np.float64)
              for k in results.FIELDS}
    results.write(tmp_path / "ours.h5", grid, fields, meta)
    ours = h5lite.read(tmp_path / "ours.h5")
    assert set(ours) == set(ref)
    for name, raw in ref.items():
        assert ours[name].tobytes() == raw.tobytes(), name


def test_grid_result_writes_its_run(tmp_path):
    """GridResult.write_hdf5 (a Solver.solve_grid result) writes the file of
    results.run_meta for its equation, parameters and counters."""
    from walk_on_spheres_b200.solver import GridResult
    grid = _grid(4, 3, 2)
    f = _fields(24, 3)
    p = _lib.Params(2, 1, 10.0, 64, 1e-2, 1000, 12, 77, 1)      # screened_poisson, Green
    c = {"max_steps_hits": 2, "ambiguous_ray_retries": 5, "indeterminate_points": 1,
         "effective_epsilon": 0.005}
    r = GridResult(*[f[k].reshape(4, 3, 2) for k in results.FIELDS], counters=c,
                   equation="screened_poisson", dim=3, grid=grid, params=p)
    r.write_hdf5(tmp_path / "r.h5")
    want = results.run_meta("screened_poisson", 3, 64, 0.005, 1000, 77, alpha=10.0,
                            source_mode=1, counters=c)
    results.write(tmp_path / "w.h5", grid, f, want)
    assert (tmp_path / "r.h5").read_bytes() == (tmp_path / "w.h5").read_bytes()
    m = h5lite.read(tmp_path / "r.h5")
    assert m["/metadata/epsilon"] == 0.005 and m["/metadata/alpha"] == 10.0
    assert m["/metadata/ambiguous_ray_retries"] == 5
    with pytest.raises(ValueError):
        GridResult(*[f[k] for k in results.FIELDS]).write_hdf5(tmp_path / "x.h5")
