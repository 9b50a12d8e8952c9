"""Benchmark: walk-on-spheres walks/s on B200 at matched standard error.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--scaling weak|strong]

Workload (one "step"): the 2D `poisson` equation on a unit-circle polyline of
1024 uniform segments, a 256 x 256 grid over its bounding box, 4096 walks per
inside point, epsilon 0.01, seed 12345, solved once with uniform-ball and once
with Green-function source sampling (the two source modes of the workload).
Synthetic mesh, generated in-process.

`value` is the whole-job walks/s of the FAST_FP32 path (FP32 walk and
closest-point arithmetic with an FP64 epsilon shell), scaled to matched
standard error against the FP64 estimator: walks/s * var_fp64 / var_fast
(per-walk variances averaged over inside points; the time to reach a given
standard error is proportional to var / throughput).  Device time is taken
with CUDA events on the library's stream around each solve; the L2 cache is
flushed (256 MiB write) between steps, outside the events.  `e2e` is the same
metric through the C ABI with host buffers (mesh upload + BVH build on the
device + solve + copy of the five result fields into pinned host memory,
both modes), wall-clocked.

`closest_point_queries_per_s` counts the walk steps that ran a BVH
closest-point query; the other steps took their radius from the distance
lattice (`lattice_step_share`).  `roofline` is the walk kernel's issue-slot
bound: warp instructions issued per second (the issued-instruction count per
walk step of an ncu capture of this workload, times the steps counted live,
over the kernel's live CUDA-event time) against 4 issue slots per SM per
cycle at the SM clock sampled during the run; its `memory` part gives the L2
and DRAM bytes of the same capture per step, scaled the same way, against
ncu's L2 peak and the measured HBM copy peak.

With N GPUs (one process per GPU over NCCL; `--gpus N` without torchrun
re-launches itself under torch.distributed.run): `--scaling weak` (default)
gives every rank its own copy of the workload on a disjoint range of grid
indices; `--scaling strong` splits the one grid across the ranks by
linear-index ranges (walk_on_spheres_b200.parallel, the library's sharded
solve).  The job time is the maximum over ranks.

On one GPU the line also carries single-GPU legs: `adjoint` (backward passes
per second of the differentiable heat-source workload: 3D Gaussian source on
a 0.10 x 0.05 x 0.01 m slab of ~20k triangles, 4096 interior probes, 2048
walks), `annulus` (laplace, 2 x 128 segments, 64 x 64, 10 000 walks),
`sphere` (screened_poisson alpha 10 on the 16 128-triangle UV sphere, 64^3,
1024 walks, with the autotuner's tuned-versus-default gain) and `batch` (the
64-solve mixed batch in one CUDA graph, with and without its set-up time).

`--impl reference` times the reference's own CPU code (oracle/_ref, the
reference sources compiled with one-rank stand-ins) on all host threads on
the same workload; each step is one stratified slice of the grid (every
128th point, a different offset per step, both source modes, full walks).
Under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import signal
import socket
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "poisson2d_circle1024_256sq"
NX = NY = 256
N_WALKS = 4096
EPSILON = 1e-2
SEED = 12345
MODES = ("uniform", "green")
METRIC = "WoS walks/sec on 1 B200 at matched std error vs FP64 oracle"
UNIT = "walks/s"
CONFIG = {"workload": WORKLOAD,
          "equation": "poisson (2D, f = 0.1 on r <= 0.15, g = 0)",
          "mesh": "unit circle polyline, 1024 uniform segments",
          "grid": [NX, NY, 1], "N_walks": N_WALKS, "epsilon": EPSILON, "seed": SEED,
          "source_modes": list(MODES),
          "l2": "GPU arm: flushed between steps (256 MiB write); reference arm: CPU, n/a"}
METHOD_NAMES = {"fast": "FAST_FP32 (FP32 walk + FP64 epsilon shell, FP64 sums)",
                "fast64": "FAST_FP64", "plain": "PLAIN_FP64"}
# The reference arm's slices: step s solves the grid points whose linear
# index is congruent to s modulo REF_STRIDE.
REF_STRIDE = 128
# walk_fast_kernel on this workload (FAST_FP32), from one ncu capture of each
# source mode's launch (`python -m walk_on_spheres_b200.benchmarks --profile
# disk_uniform` / `disk_green`, 2048 walks: tasks of 2048 walks, as in the
# timed steps): warp instructions issued (sm__inst_issued.sum) and L2 bytes
# (lts__t_bytes.sum) per walk step, DRAM bytes (dram__bytes_read.sum +
# dram__bytes_write.sum) per launch (the distance lattice read once and the
# fields written: the same at any walk count), and the L2 peak the capture
# implies (lts__t_bytes.sum.per_second over
# lts__t_sectors.sum.pct_of_peak_sustained_elapsed).
NCU_PER_STEP = {"uniform": {"issued": 9703405858 / 595884179, "l2_bytes": 28.752065e9 / 595884179},
                "green": {"issued": 9536526621 / 595900507, "l2_bytes": 28.762581e9 / 595900507}}
NCU_DRAM_BYTES_PER_LAUNCH = 17.6e6
NCU_L2_PEAK_GBS = 2527.816 / 0.07299269
ISSUE_SLOTS_PER_SM_CYCLE = 4   # one warp instruction per SM sub-partition per cycle
# Adjoint workload: 3D Gaussian heat source Q exp(-|x - x0|^2 / sigma^2) on a
# 0.10 x 0.05 x 0.01 m slab of ~20k triangles, g = 0, 4096 probes uniform in
# the interior, 2048 FP32 walks each; one "gradient" is one full backward
# pass (the vector-Jacobian product of the 4096 probe values with respect to
# Q, x0, sigma and every vertex value).
ADJ_WORKLOAD = "heat3d_slab20k_4096probes"
ADJ_PROBES = 4096
ADJ_WALKS = 2048
ADJ_EPSILON = 1e-5
ADJ_THETA = (1e3, (0.05, 0.025, 0.01), 2e-3)
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"])
    ap.add_argument("--method", default="fast", choices=["fast", "fast64", "plain"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="CPU budget of the baseline sample")
    ap.add_argument("--walks", type=int, default=N_WALKS,
                    help="walks per point (profiling of smaller cases; the headline uses 4096)")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the single-GPU legs (adjoint, annulus, sphere, batch)")
    ap.add_argument("--kernels-only", action="store_true",
                    help="time the device solves only (no matched-SE, e2e, legs or CPU baseline)")
    return ap.parse_args(argv)


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch_command(argv: list[str], gpus: int, port: int) -> list[str]:
    """torch.distributed.run command that runs this script on `gpus` local ranks."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
            f"--nproc-per-node={gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
            str(ROOT / "bench.py")] + list(argv)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.send_signal(signal.SIGTERM)
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- helpers
def workload_mesh():
    from walk_on_spheres_b200 import meshes
    return meshes.circle(segments=1024)


def mesh_upload_bytes(mesh) -> int:
    """Bytes wos_set_mesh copies host->device: the vertices, primitives and
    boundary ids, from which the trees and the distance lattice are built on
    the device (plus the wide tree's split plan, a few hundred bytes, and
    the 8 height offsets, not counted)."""
    return int(mesh.verts.nbytes + np.asarray(mesh.prims, dtype=np.int32).nbytes +
               np.asarray(mesh.boundary_ids, dtype=np.int32).nbytes)


def hbm_peak():
    try:
        p = json.loads(PEAKS_FILE.read_text())
        return float(p["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (burst copy), of measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s, of fallback"


def reduce_over_ranks(dist, device, seconds: float, counts: list[float]):
    """(max of `seconds`, elementwise sum of `counts`) over the ranks; the
    inputs themselves on one process."""
    if dist is None:
        return seconds, list(counts)
    import torch
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(x) for x in counts], dtype=torch.float64, device=device)
    dist.all_reduce(c)
    return float(t.item()), [float(x) for x in c.cpu().tolist()]


def roofline(per_mode: dict, clock_mhz: float | None, sms: int, launches: int) -> dict:
    """Issue-slot roofline of the walk kernel from its `launches` live
    launches.  per_mode[mode] = (summed walk-kernel seconds, summed walk
    steps)."""
    peak_hbm, hbm_src = hbm_peak()
    measured = all(NCU_PER_STEP[m]["issued"] for m in per_mode)
    secs = sum(s for s, _ in per_mode.values())
    out = {"bound": "issue", "unit": "Gwarp-inst/s", "kernel": "walk_fast_kernel",
           "achieved": None, "peak": None, "frac": None, "traffic": None}
    if clock_mhz:
        out["peak"] = sms * ISSUE_SLOTS_PER_SM_CYCLE * clock_mhz * 1e6 / 1e9
        out["peak_source"] = (f"{sms} SMs x {ISSUE_SLOTS_PER_SM_CYCLE} issue slots per cycle x "
                              f"{clock_mhz:.0f} MHz (median SM clock sampled during the run)")
    if not measured:
        out["note"] = "no ncu per-step figures recorded for this build"
        return out
    issued = sum(NCU_PER_STEP[m]["issued"] * st for m, (_, st) in per_mode.items())
    l2 = sum(NCU_PER_STEP[m]["l2_bytes"] * st for m, (_, st) in per_mode.items())
    dram = NCU_DRAM_BYTES_PER_LAUNCH * launches
    out["achieved"] = issued / secs / 1e9
    if out["peak"]:
        out["frac"] = out["achieved"] / out["peak"]
    out["traffic"] = NCU_DRAM_BYTES_PER_LAUNCH
    out["per_step"] = {m: dict(NCU_PER_STEP[m]) for m in per_mode}
    out["memory"] = {
        "l2_gbs": l2 / secs / 1e9, "l2_peak_gbs": NCU_L2_PEAK_GBS,
        "l2_frac": (l2 / secs / 1e9 / NCU_L2_PEAK_GBS) if NCU_L2_PEAK_GBS else None,
        "l2_peak_source": "ncu lts__t_bytes peak of the part, of ncu",
        "dram_gbs": dram / secs / 1e9, "hbm_peak_gbs": peak_hbm,
        "hbm_frac": dram / secs / 1e9 / peak_hbm, "hbm_peak_source": hbm_src}
    return out


# ---------------------------------------------------------------- CPU reference
def _ref_slice(step: int) -> np.ndarray:
    return np.arange(step % REF_STRIDE, NX * NY, REF_STRIDE, dtype=np.int64)


def reference_slices(steps: list[int], threads: int | None = None):
    """The reference's own code (oracle/_ref) on all host threads, one
    stratified slice of the workload grid per step (both source modes, full
    walks).  Returns per step (walks, reference-timed seconds, wall seconds)."""
    from oracle.oracle import Reference, Solve
    ref = Reference()
    mesh = workload_mesh()
    threads = threads or os.cpu_count() or 1
    rows = []
    for step in steps:
        pts = _ref_slice(step)
        walks, secs = 0, 0.0
        t0 = time.perf_counter()
        for mode in MODES:
            s = Solve(mesh, NX, NY, 1, N_walks=N_WALKS, epsilon=EPSILON, seed=SEED,
                      source_mode=MODES.index(mode), points=pts, n_threads=threads)
            r = ref.solve_grid("poisson", s)
            walks += r.counters["inside_points"] * N_WALKS
            secs += r.counters["seconds"]
        rows.append((walks, secs, time.perf_counter() - t0))
    return rows, threads


def reference_rate(budget_s: float):
    """Walks/s of the reference's code on as many grid slices as fit about
    budget_s seconds (at least one).  Returns (rate, description, threads)."""
    rows, threads = reference_slices([0])
    per_slice = max(rows[0][2], 1e-3)
    k = int(max(1, min(REF_STRIDE, budget_s // per_slice)))
    if k > 1:
        more, _ = reference_slices(list(range(1, k)), threads)
        rows += more
    walks = sum(r[0] for r in rows)
    secs = sum(r[1] for r in rows)
    desc = (f"{k} of the {REF_STRIDE} stratified slices of the {NX}x{NY} grid (every "
            f"{REF_STRIDE}th grid point; {k * NX * NY // REF_STRIDE} points), {N_WALKS} walks each, "
            f"uniform and green source modes")
    return walks / secs, desc, threads


# ---------------------------------------------------------------- GPU legs
def _device_fields(torch, n, dev):
    return ([torch.empty(n, dtype=torch.float64, device=dev) for _ in range(4)] +
            [torch.empty(n, dtype=torch.uint8, device=dev)])


def single_leg(solver, torch, dev, flush, name, mesh, equation, shape, walks, kw, steps,
               plain_walks, tune=False):
    """One single-solve configuration: FAST_FP32 device walks/s over `steps`
    timed solves (L2 flushed between them), the matched-SE factor against
    PLAIN_FP64 at `plain_walks` walks, exact queries and lattice steps."""
    solver.set_mesh(mesh)
    grid = solver.grid_over_mesh(*shape)
    n = int(np.prod(shape))
    out_t = _device_fields(torch, n, dev)
    ptrs = [t.data_ptr() for t in out_t]
    out = {"workload": name, "grid": list(shape), "N_walks": walks, "method": METHOD_NAMES["fast"]}
    tuned = None
    if tune:
        from walk_on_spheres_b200.autotune import Tuner
        solver.set_tuning(0, 0)
        tuned = Tuner(solver).tune(mesh, equation, shape, N_walks=walks, method="fast", **kw)
        solver.set_tuning(0, 0)
        solver.set_mesh(mesh)

    def timed(k):
        ms = walk_ms = 0.0
        tw = ts = tq = 0
        for _ in range(k):
            flush.zero_()
            torch.cuda.synchronize()
            c = solver.solve_grid_device(equation, grid, *ptrs, N_walks=walks, method="fast",
                                         **kw)
            ms += c["total_ms"]
            walk_ms += c["walk_ms"]
            tw += c["total_walks"]
            ts += c["total_steps"]
            tq += c["exact_queries"]
        return ms / 1000.0, walk_ms / 1000.0, tw, ts, tq

    solver.solve_grid_device(equation, grid, *ptrs, N_walks=walks, method="fast", **kw)
    secs, wsecs, tw, ts, tq = timed(steps)
    loc = out_t[4].cpu().numpy()
    ins = loc == 1
    var_fast = float(out_t[1].cpu().numpy()[ins].mean())
    p = solver.solve_grid(equation, *shape, N_walks=plain_walks, method="plain", **kw)
    var_plain = float(np.mean(p.variance.ravel()[ins]))
    plain_rate = p.counters["total_walks"] / (p.counters["total_ms"] / 1000.0)
    ratio = var_plain / var_fast
    out.update({
        "walks_per_s": tw / secs, "matched_se_walks_per_s": tw / secs * ratio,
        "variance_ratio_fp64_over_fast": ratio, "ms_per_solve": secs * 1000.0 / steps,
        "walk_kernel_ms": wsecs * 1000.0 / steps,
        "mean_steps": ts / max(tw, 1), "closest_point_queries_per_s": tq / secs,
        "lattice_step_share": 1.0 - tq / max(ts, 1),
        "plain_fp64_walks_per_s": plain_rate, "plain_walks": plain_walks,
        "speedup_vs_plain_fp64_matched_se": tw / secs * ratio / plain_rate})
    if tuned is not None:
        solver.set_mesh(mesh, leaf_size=tuned.leaf_size)
        grid = solver.grid_over_mesh(*shape)
        solver.set_tuning(tuned.chunk, tuned.blocks)
        solver.solve_grid_device(equation, grid, *ptrs, N_walks=walks, method="fast", **kw)
        t_secs = timed(steps)[0]
        solver.set_tuning(0, 0)
        out["autotune"] = {"leaf_size": tuned.leaf_size, "chunk": tuned.chunk,
                           "blocks": tuned.blocks, "default": {"leaf_size": 4, "chunk": 1024},
                           "tuned_ms_per_solve": t_secs * 1000.0 / steps,
                           "gain_vs_default": secs / t_secs}
    return out


def batch_leg(solver, runs):
    """The 64-solve mixed batch (benchmarks.mixed_batch_specs, generator seed
    2024) in one captured CUDA graph: walks/s of the graph replays, with and
    without the one-time set-up (tree builds, uploads, lattices), and the
    batch autotuner's walks-per-task choice (tuned on the same batch at a
    quarter of the walks) against the default."""
    from walk_on_spheres_b200.autotune import Tuner
    from walk_on_spheres_b200.batch import Batch
    from walk_on_spheres_b200.benchmarks import build_mesh, mixed_batch_specs

    def make(scale):
        specs = mixed_batch_specs(2024, scale)
        b = Batch(solver)
        t0 = time.perf_counter()
        for sp, m in zip(specs, meshes_built):
            mid = b.add_mesh(m)
            b.add_solve(mid, sp["equation"], *sp["grid"], **sp["params"])
        b.prepare()
        return b, time.perf_counter() - t0

    specs = mixed_batch_specs(2024, 1.0)
    meshes_built = [build_mesh(sp["mesh"]) for sp in specs]
    b, setup_s = make(1.0)
    t0 = time.perf_counter()
    first_ms = b.run(use_graph=True)          # capture and first replay
    first_wall = time.perf_counter() - t0
    ms = [b.run(use_graph=True) for _ in range(runs)]
    info = b.info()
    secs = float(np.mean(ms)) / 1000.0
    out = {"workload": "mixed_batch_64", "solves": info["solves"], "points": info["points"],
           "walks": info["walks"], "steps": info["steps"],
           "prims_total": int(sum(m.prims.shape[0] for m in meshes_built)),
           "setup_s": setup_s, "graph_ms": float(np.mean(ms)), "runs": runs,
           "walks_per_s": info["walks"] / secs,
           "walks_per_s_with_setup": info["walks"] / (setup_s + first_wall),
           "first_run_ms": first_ms}
    q, qsetup = make(0.25)
    tuned = Tuner(solver).tune_batch(q)
    q.close()
    b.set_tuning(tuned["chunk"], 0)
    b.run(use_graph=True)
    t_ms = float(np.mean([b.run(use_graph=True) for _ in range(max(1, runs // 2))]))
    b.close()
    out["autotune"] = {"chunk": tuned["chunk"], "default_chunk": 1024,
                       "tuned_graph_ms": t_ms, "gain_vs_default": float(np.mean(ms)) / t_ms,
                       "probe": "the same batch at a quarter of the walks",
                       "candidates": [{k: r[k] for k in ("chunk", "batch_ms")}
                                      for r in tuned["table"]]}
    return out


def adjoint_leg(solver, args, rank, world, dist, dev):
    """Backward passes (adjoint replay) of the heat-source workload per second,
    device time from the library's CUDA events, max over ranks."""
    from walk_on_spheres_b200 import meshes
    from walk_on_spheres_b200.heat import HeatProblem
    slab = meshes.slab_box(target_triangles=20000)
    solver.set_mesh(slab)
    rng = np.random.default_rng(20240 + rank)
    lo, hi = np.zeros(3), np.array([0.10, 0.05, 0.01])
    probes = lo + (hi - lo) * rng.uniform(0.001, 0.999, size=(ADJ_PROBES, 3))
    heat = HeatProblem(solver, probes, N_walks=ADJ_WALKS, epsilon=ADJ_EPSILON,
                       seed=SEED + rank * 1000003, source_mode="green", method="fast")
    g = np.zeros(heat.n_verts)
    Q, x0, sigma = ADJ_THETA
    fwd = heat.forward(Q, x0, sigma, g)
    for _ in range(args.warmup):
        heat.adjoint(Q, x0, sigma, g)
    ms, walks, steps, queries = [], 0, 0, 0
    for _ in range(args.steps):
        r = heat.adjoint(Q, x0, sigma, g)
        ms.append(r.counters["total_ms"])
        walks += r.counters["total_walks"]
        steps += r.counters["total_steps"]
        queries += r.counters["exact_queries"]
    dev_s, (walks, steps, queries) = reduce_over_ranks(dist, dev, sum(ms) / 1000.0,
                                                       [walks, steps, queries])
    return {"workload": ADJ_WORKLOAD, "metric": "adjoint gradients/s",
            "value": world * args.steps / dev_s, "unit": "gradients/s",
            "gradient": f"VJP of {ADJ_PROBES} probe values w.r.t. Q, x0 (3), sigma and "
                        f"{heat.n_verts} vertex values",
            "backward_ms": dev_s * 1000.0 / args.steps, "forward_ms": fwd.counters["total_ms"],
            "walks_per_s": walks / dev_s, "closest_point_queries_per_s": queries / dev_s,
            "lattice_step_share": 1.0 - queries / max(steps, 1),
            "N_walks": ADJ_WALKS, "epsilon": ADJ_EPSILON, "method": "FAST_FP32",
            "triangles": int(slab.prims.shape[0]), "gpu_launches_per_gradient": 3}


# ---------------------------------------------------------------- GPU arm
def gpu_arm(args, rank, world, local):
    import torch
    from walk_on_spheres_b200 import Solver, parallel

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    strong = args.scaling == "strong" and world > 1
    mesh = workload_mesh()
    solver = Solver(local)
    solver.set_mesh(mesh)
    grid = solver.grid_over_mesh(NX, NY, 1)
    n = NX * NY
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    # weak scaling: each rank owns a copy of the workload on a disjoint seeding
    # range; strong scaling: each rank owns a linear-index range of the grid
    seed = SEED + (0 if strong else rank * 1000003)
    start, end = parallel.shard_bounds(n, rank, world) if strong else (0, n)
    if strong:
        shard_pts = parallel.grid_points(grid, 2, start, end)
        shard_idx = np.arange(start, end, dtype=np.uint64)
        fields = None
    else:
        fields = _device_fields(torch, n, dev)

    def solve(mode):
        kw = dict(N_walks=args.walks, epsilon=EPSILON, seed=seed, source_mode=mode,
                  method=args.method)
        if strong:
            return solver.solve_points("poisson", shard_pts, point_index=shard_idx,
                                       **kw).counters
        return solver.solve_grid_device("poisson", grid, *[f.data_ptr() for f in fields], **kw)

    for _ in range(args.warmup):
        for mode in MODES:
            solve(mode)
    barrier()
    step_ms = []
    per_mode = {m: [0.0, 0] for m in MODES}
    walks = steps_total = queries = 0
    launches = 0
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ms = 0.0
            for mode in MODES:
                c = solve(mode)
                ms += c["total_ms"]
                per_mode[mode][0] += c["walk_ms"] / 1000.0
                per_mode[mode][1] += c["total_steps"]
                walks += c["total_walks"]
                steps_total += c["total_steps"]
                queries += c["exact_queries"]
                launches += 3  # classification, walk, merge
            step_ms.append(ms)
        barrier()
        wall = time.perf_counter() - t0
    clock = clocks.summary()
    job_s, (job_walks, job_steps, job_queries) = reduce_over_ranks(
        dist, dev, sum(step_ms) / 1000.0, [walks, steps_total, queries])
    raw_rate = job_walks / job_s

    if args.kernels_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "raw_walks_per_s": raw_rate, "n_gpus": world,
                              "walks": args.walks, "ms_per_step": job_s * 1000.0 / args.steps,
                              "exact_queries": job_queries, "steps": job_steps,
                              "clocks": clock}), flush=True)
        if dist:
            dist.destroy_process_group()
        solver.close()
        return

    # matched standard error: per-walk variance of the fast path against the
    # FP64 estimator (PLAIN_FP64, the reference's streams) on the same grid
    fast_var, ref_var = {}, {}
    plain_rate = None
    for mode in MODES:
        r = solver.solve_grid("poisson", NX, NY, N_walks=N_WALKS, epsilon=EPSILON, seed=seed,
                              source_mode=mode, method=args.method)
        ins = r.location == 1
        fast_var[mode] = float(np.mean(r.variance[ins]))
        p = solver.solve_grid("poisson", NX, NY, N_walks=256, epsilon=EPSILON, seed=seed,
                              source_mode=mode, method="plain")
        ref_var[mode] = float(np.mean(p.variance[ins]))
        pr = p.counters["total_walks"] / (p.counters["total_ms"] / 1000.0)
        plain_rate = pr if plain_rate is None else 2.0 / (1.0 / plain_rate + 1.0 / pr)
    var_ratio = sum(ref_var.values()) / sum(fast_var.values())
    value = raw_rate * var_ratio

    # end to end through the C ABI with host buffers
    import ctypes as C
    from walk_on_spheres_b200 import _lib
    L = _lib.lib()
    m_loc = end - start
    # the step's results land in pinned host memory
    host = ([torch.empty(m_loc, dtype=torch.float64, pin_memory=True).numpy() for _ in range(4)]
            + [torch.empty(m_loc, dtype=torch.uint8, pin_memory=True).numpy()])

    def host_step():
        solver.set_mesh(mesh)
        w = 0
        for mode in MODES:
            if strong:
                r = solver.solve_points("poisson", shard_pts, point_index=shard_idx,
                                        N_walks=N_WALKS, epsilon=EPSILON, seed=seed,
                                        source_mode=mode, method=args.method)
                w += r.counters["total_walks"]
                continue
            p = solver.params("poisson", N_walks=N_WALKS, epsilon=EPSILON, seed=seed,
                              source_mode=mode, method=args.method)
            cnt = _lib.Counters()
            _lib.check(L.wos_solve_grid(solver._ctx, C.byref(p), C.byref(grid),
                                        *[a.ctypes.data_as(C.c_void_p) for a in host],
                                        C.byref(cnt)), solver._ctx)
            w += cnt.total_walks
        return w

    for _ in range(max(1, args.warmup // 2)):
        host_step()
    e2e_walks = 0
    e2e_s = 0.0
    barrier()
    for _ in range(args.steps):
        t = time.perf_counter()
        e2e_walks += host_step()
        e2e_s += time.perf_counter() - t
    e2e_s, (e2e_walks,) = reduce_over_ranks(dist, dev, e2e_s, [e2e_walks])
    e2e_value = e2e_walks / e2e_s * var_ratio
    pts_bytes = (m_loc * 2 * 8 + m_loc * 8) if strong else 0
    h2d = mesh_upload_bytes(mesh) + pts_bytes
    d2h = len(MODES) * m_loc * (4 * 8 + 1)

    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    roof = roofline({m: tuple(v) for m, v in per_mode.items()},
                    clock["sm_mhz"] if clock else None, sms, args.steps * len(MODES))

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": job_s * 1000.0 / args.steps,
        "higher_is_better": True, "scaling": "strong" if strong else "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(CONFIG),
        "method": METHOD_NAMES[args.method],
        "parallelism": (f"dp{world} (grid split by linear-index ranges)" if strong
                        else f"dp{world} (independent grid shards)"),
        "global_batch_points": n if strong else n * world,
        "raw_walks_per_s": raw_rate,
        "variance_ratio_fp64_over_fast": var_ratio,
        # one GPU's PLAIN_FP64 rate (the reference's estimator and streams)
        "plain_fp64_walks_per_s": plain_rate,
        "speedup_vs_plain_fp64_matched_se": value / world / plain_rate,
        # walk steps that ran a BVH closest-point query; the rest took their
        # radius from the distance lattice
        "closest_point_queries_per_s": job_queries / job_s,
        "walk_steps_per_s": job_steps / job_s,
        "lattice_step_share": 1.0 - job_queries / max(job_steps, 1.0),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": launches,
        "roofline": roof,
        "clocks": clock,
        "wall_s_timed_region": wall,
    }
    if world == 1 and not args.no_legs:
        from walk_on_spheres_b200 import meshes
        line["adjoint"] = adjoint_leg(solver, args, rank, world, dist, dev)
        k = max(3, min(args.steps, 10))
        line["annulus"] = single_leg(solver, torch, dev, flush, "laplace2d_annulus256_64sq",
                                     meshes.annulus(), "laplace", (64, 64, 1), 10000,
                                     dict(seed=12345, epsilon=1e-2), k, plain_walks=1000)
        line["sphere"] = single_leg(solver, torch, dev, flush, "screened3d_sphere16128_64cube",
                                    meshes.uv_sphere(), "screened_poisson", (64, 64, 64), 1024,
                                    dict(seed=7, alpha=10.0, epsilon=1e-2), k, plain_walks=64,
                                    tune=True)
        line["batch"] = batch_leg(solver, runs=3)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, desc, threads = reference_rate(args.cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                                "sample": desc}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    solver.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def reference_arm(args, rank, world):
    """The reference's CPU code on the workload: each step is one stratified
    slice of the grid; `value` = walks / the reference's own timer over the
    timed steps, `ms_per_step` = their mean wall time."""
    if rank != 0:
        return
    steps = list(range(args.warmup + args.steps))
    rows, threads = reference_slices(steps)
    timed = rows[args.warmup:]
    walks = sum(r[0] for r in timed)
    secs = sum(r[1] for r in timed)
    wall = sum(r[2] for r in timed)
    value = walks / secs
    k = len(timed)
    desc = (f"{k} timed steps, each one stratified slice of the {NX}x{NY} grid (every "
            f"{REF_STRIDE}th grid point, offset = step; {NX * NY // REF_STRIDE} points), "
            f"together {k * NX * NY // REF_STRIDE} points ({100.0 * k / REF_STRIDE:.1f}% of the "
            f"grid), {N_WALKS} walks each, uniform and green source modes")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": wall * 1000.0 / max(k, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": dict(CONFIG),
        "method": "reference CPU code (FP64, xoshiro256++ streams)",
        "parallelism": f"{threads} host threads",
        "global_batch_points": NX * NY // REF_STRIDE,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    args = parse(argv)
    rank, world, local = dist_info()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: re-launch under torch.distributed.run
        return subprocess.call(launch_command(argv, args.gpus, free_port()))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return 0
    gpu_arm(args, rank, world, local)
    return 0


if __name__ == "__main__":
    sys.exit(main())
