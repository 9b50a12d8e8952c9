"""Autotuner for the FAST walks: walks per task (queue chunking, i.e. walks
per lane = chunk / 32), persistent grid size and BVH leaf size.

    from walk_on_spheres_b200.autotune import Tuner
    t = Tuner(solver)
    best = t.tune(mesh, "screened_poisson", (64, 64, 64), N_walks=1024, alpha=10.0, seed=7)
    # solver now holds best.leaf_size's mesh and best.chunk / best.blocks tuning

Each candidate runs a probe solve through the C ABI and is scored by device
walks per second from the library's CUDA events.  By default the probe is
the full grid sweep (the schedule's best point depends on how many tasks
the grid makes per wave of resident warps, so a small sample would favour
short chunks); with `probe_points` set it is wos_solve_points on a seeded
sample of that many grid points, enlarged so the longest chunk still gives
eight waves of tasks.  The leaf size is
scored by the whole probe solve (classification and FP64 queries use the
binary tree it shapes; the FP32 32-wide tree's clusters are always one warp
wide).  Candidates that fail are skipped.  Results are cached per problem
key (dimension, primitive-count octave, equation, method, walk count) in
memory and, when `cache_path` is given, in a JSON file.  Tuning only changes
the schedule and the tree shape: the estimator, streams and results per walk
stay those of the FAST method.
"""
from __future__ import annotations

import json
import math
from dataclasses import asdict, dataclass, field
from pathlib import Path

import numpy as np

CHUNKS = (256, 512, 1024, 2048)
LEAF_SIZES = (2, 4, 8)
BLOCK_FACTORS = (0,)        # 0: every block that can be resident; k: k blocks per SM
WAVE_WARPS = 148 * 24       # resident warps of the FP32 walk kernel on a B200


@dataclass
class TuneResult:
    chunk: int
    blocks: int
    leaf_size: int
    walks_per_s: float
    key: str
    table: list = field(default_factory=list)


def problem_key(dim: int, n_prims: int, equation: str, method: str, n_walks: int) -> str:
    octave = int(math.floor(math.log2(max(1, n_prims))))
    return f"d{dim}-p{octave}-{equation}-{method}-w{n_walks}"


def pick(table: list[dict], score: str = "walks_per_s") -> dict:
    """Best row of a candidate table (highest score; ties keep the first)."""
    ok = [r for r in table if r.get(score) is not None and np.isfinite(r[score])]
    if not ok:
        raise RuntimeError("no tuning candidate ran")
    return max(ok, key=lambda r: r[score])


def sample_points(grid, dim: int, n: int, seed: int = 0):
    """(coordinates, global linear indices) of a seeded sample of a grid."""
    from .parallel import grid_coords
    total = int(grid.Nx) * int(grid.Ny) * (int(grid.Nz) if dim == 3 else 1)
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(total, size=min(n, total), replace=False))
    return grid_coords(grid, dim, idx), idx.astype(np.uint64)


class Tuner:
    def __init__(self, solver, cache_path: str | None = None, probe_points: int | None = None,
                 chunks=CHUNKS, leaf_sizes=LEAF_SIZES, block_factors=BLOCK_FACTORS):
        self.solver = solver
        self.cache_path = Path(cache_path) if cache_path else None
        self.probe_points = probe_points
        self.chunks = chunks
        self.leaf_sizes = leaf_sizes
        self.block_factors = block_factors
        self.cache: dict[str, dict] = {}
        if self.cache_path and self.cache_path.exists():
            self.cache = json.loads(self.cache_path.read_text())

    def _save(self):
        if self.cache_path:
            self.cache_path.write_text(json.dumps(self.cache, indent=1, sort_keys=True))

    def _probe(self, pts, idx, equation, kw) -> dict | None:
        from ._lib import WosError
        try:
            if pts is None:
                r = self.solver.solve_grid(equation, grid=self._grid, **kw)
            else:
                r = self.solver.solve_points(equation, pts, point_index=idx, **kw)
        except WosError:
            return None
        c = r.counters
        if c["walk_ms"] <= 0 or c["total_walks"] == 0:
            return None
        return {"walks_per_s": c["total_walks"] / (c["walk_ms"] / 1000.0),
                "total_ms": c["total_ms"], "walk_ms": c["walk_ms"]}

    def tune(self, mesh, equation: str, grid_shape, use_cache: bool = True, **kw) -> TuneResult:
        s = self.solver
        method = kw.get("method", "fast")
        n_walks = int(kw.get("N_walks", 10000))
        key = problem_key(mesh.dim, mesh.prims.shape[0], equation, method, n_walks)
        if use_cache and key in self.cache:
            r = TuneResult(**self.cache[key])
            self.apply(mesh, r)
            return r
        table = []
        # leaf size: whole probe solve at the default schedule
        s.set_tuning(0, 0)
        leaf_rows = []
        pts = idx = None
        for leaf in self.leaf_sizes:
            s.set_mesh(mesh, leaf_size=leaf)
            self._grid = s.grid_over_mesh(*grid_shape)
            if self.probe_points and pts is None:
                longest = max(c for c in self.chunks if c <= max(n_walks, self.chunks[0]))
                per_point = -(-n_walks // longest)
                n = max(self.probe_points, -(-8 * WAVE_WARPS // per_point))
                pts, idx = sample_points(self._grid, mesh.dim, n)
            row = self._probe(pts, idx, equation, kw)
            if row is not None:
                row = {"leaf_size": leaf, "chunk": 0, "blocks": 0, **row,
                       "inv_total_ms": 1.0 / row["total_ms"]}
                leaf_rows.append(row)
                table.append(row)
        leaf = pick(leaf_rows, "inv_total_ms")["leaf_size"]
        s.set_mesh(mesh, leaf_size=leaf)
        # schedule: walks per task x persistent grid size
        sms = _sm_count(s)
        sched_rows = []
        for chunk in self.chunks:
            if chunk > max(32, n_walks) and chunk != self.chunks[0]:
                continue
            for f in self.block_factors:
                blocks = 0 if f == 0 else f * sms
                s.set_tuning(chunk, blocks)
                row = self._probe(pts, idx, equation, kw)
                if row is not None:
                    row = {"leaf_size": leaf, "chunk": chunk, "blocks": blocks, **row}
                    sched_rows.append(row)
                    table.append(row)
        s.set_tuning(0, 0)
        best = pick(sched_rows)
        r = TuneResult(best["chunk"], best["blocks"], leaf, best["walks_per_s"], key, table)
        self.cache[key] = asdict(r)
        self._save()
        self.apply(mesh, r)
        return r

    def apply(self, mesh, r: TuneResult):
        self.solver.set_mesh(mesh, leaf_size=r.leaf_size)
        self.solver.set_tuning(r.chunk, r.blocks)

    def tune_batch(self, batch, chunks=None) -> dict:
        """Walks per task for a whole batch (scored by its total device time)."""
        rows = []
        for chunk in chunks or self.chunks:
            batch.set_tuning(chunk, 0)
            ms = batch.run(use_graph=True)
            ms = batch.run(use_graph=True)
            rows.append({"chunk": chunk, "batch_ms": ms, "inv_ms": 1.0 / ms})
        best = pick(rows, "inv_ms")
        batch.set_tuning(best["chunk"], 0)
        return {"chunk": best["chunk"], "batch_ms": best["batch_ms"], "table": rows}


def _sm_count(solver) -> int:
    try:
        import torch
        return torch.cuda.get_device_properties(solver.device).multi_processor_count
    except Exception:
        return 148
