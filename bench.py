"""Benchmark: walk-on-spheres walks/s on B200 at matched standard error.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

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
metric through the C ABI with host buffers (mesh upload + BVH build + solve +
copy of the five result fields to the host, both modes), wall-clocked.

With N GPUs (torchrun, one process per GPU over NCCL) every rank solves its
own copy of the workload on a disjoint range of grid indices (weak scaling);
the job time is the maximum over ranks.

The line also carries `adjoint`: backward passes per second of the
differentiable heat-source workload (3D Gaussian source on a 0.10 x 0.05 x
0.01 m slab of ~20k triangles, 4096 interior probes, 2048 walks; each pass
replays the forward walks from their seeds and returns the gradient with
respect to Q, x0, sigma and every vertex value), timed the same way.

`--impl reference` times the reference's own CPU code (oracle/_ref, the
reference sources compiled with one-rank stand-ins) on all host threads on a
bounded sample of the same workload; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import signal
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
# Algorithmic bytes of one closest-point query of this workload: node pops and
# primitive tests of the reference BVH traversal (src/bvh.cpp:295-387) along
# the workload's walks, times the reference record sizes (40 B node, 40 B
# segment); measured by `python -m oracle.measure_traversal`.
BYTES_PER_QUERY = 1863.4
# DRAM bytes (read + write) of one walk-kernel launch of this workload, from a
# one-pass ncu capture of the full launch (profiles/walk_fast_kernel_poisson2d_
# circle1024.md): 17.8 MB and 19.2 MB for the two source modes, most of it
# the 16 MB distance lattice read once.
TRAFFIC_BYTES_PER_LAUNCH = 18.5e6
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


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--method", default="fast", choices=["fast", "fast64", "plain"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="CPU budget of the baseline sample")
    ap.add_argument("--walks", type=int, default=N_WALKS,
                    help="walks per point (profiling of smaller cases; the headline uses 4096)")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint-gradient leg")
    ap.add_argument("--kernels-only", action="store_true",
                    help="time the device solves only (no matched-SE, e2e or CPU legs)")
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


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


def scene_upload_bytes(mesh) -> int:
    """Bytes wos_set_mesh copies host->device for a 2D mesh: binary-tree boxes
    (2^(D+1) x 4 doubles), FP64 segments (4 doubles) and {boundary id,
    primitive} per slot, the 32-wide tree's child blocks, its primitive
    blocks (5 floats per slot), wide-to-binary slot map, height offsets and
    vertex ids per slot.  The distance lattice is built on the device."""
    from walk_on_spheres_b200 import _lib
    import ctypes as C
    L = _lib.lib()
    d, H, E = C.c_int(), C.c_int(), C.c_int()
    verts = np.ascontiguousarray(mesh.verts)
    prims = np.ascontiguousarray(mesh.prims, dtype=np.int32)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    L.wos_build_bvh.restype = C.c_int
    L.wos_build_bvh(2, vp(verts), verts.shape[0], vp(prims), prims.shape[0], 0, C.byref(d),
                    None, None)
    L.wos_build_wide_bvh(2, vp(verts), verts.shape[0], vp(prims), prims.shape[0], C.byref(H),
                         C.byref(E), None, None, None)
    n, D = mesh.n_prims, d.value
    npad = (n + 31) // 32 * 32
    return ((2 ** (D + 1)) * 32 + n * 32 + n * 8 + E.value * 4 + npad * 20 + npad * 4 + 32
            + n * 8)


def hbm_peak():
    try:
        p = json.loads(PEAKS_FILE.read_text())
        return float(p["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (burst copy), of measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s, of fallback"


# ---------------------------------------------------------------- CPU reference
def reference_rate(budget_s: float, threads: int | None = None):
    """The reference's own code (oracle/_ref) on all host threads, on a strided
    sample of the workload's grid points sized to ~budget_s seconds.
    Returns (walks/s, sample description, threads, mean variance)."""
    from oracle.oracle import Reference, Solve
    ref = Reference()
    mesh = workload_mesh()
    threads = threads or os.cpu_count() or 1
    n_grid = NX * NY

    def run(points):
        walks = 0
        secs = 0.0
        var = []
        for mode in MODES:
            s = Solve(mesh, NX, NY, 1, N_walks=N_WALKS, epsilon=EPSILON, seed=SEED,
                      source_mode=MODES.index(mode), points=points, n_threads=threads)
            r = ref.solve_grid("poisson", s)
            walks += r.counters["inside_points"] * N_WALKS
            secs += r.counters["seconds"]
            ins = r.location[points] == 1
            if ins.any():
                var.append(float(np.mean(r.variance[points][ins])))
        return walks, secs, float(np.mean(var)) if var else float("nan")

    # calibrate on a small random sample, then size the sample to the budget
    order = np.random.default_rng(2024).permutation(n_grid)
    probe = np.sort(order[:max(8, 2 * threads)])
    w, s, _ = run(probe)
    rate = w / max(s, 1e-9)
    inside_frac = max(w / (len(MODES) * N_WALKS * probe.size), 1e-3)
    want_points = int(rate * budget_s / (len(MODES) * N_WALKS * inside_frac))
    pts = np.sort(order[:min(n_grid, max(probe.size, want_points))])
    w, s, var = run(pts)
    desc = (f"{pts.size} of {n_grid} grid points (seeded random subset), {N_WALKS} walks each, "
            f"uniform and green source modes")
    return w / s, desc, threads, var


# ---------------------------------------------------------------- GPU arm
def adjoint_leg(solver, args, rank, world, dist, dev):
    """Backward passes (adjoint replay) of the heat-source workload per second,
    device time from the library's CUDA events, max over ranks."""
    import torch
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
    ms, walks, steps = [], 0, 0
    for _ in range(args.steps):
        r = heat.adjoint(Q, x0, sigma, g)
        ms.append(r.counters["total_ms"])
        walks += r.counters["total_walks"]
        steps += r.counters["total_steps"]
    dev_s = sum(ms) / 1000.0
    if dist:
        t = torch.tensor([dev_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_s = float(t.item())
        tw = torch.tensor([float(walks), float(steps)], dtype=torch.float64, device=dev)
        dist.all_reduce(tw)
        walks, steps = int(tw[0].item()), int(tw[1].item())
    return {"workload": ADJ_WORKLOAD, "metric": "adjoint gradients/s",
            "value": world * args.steps / dev_s, "unit": "gradients/s",
            "gradient": f"VJP of {ADJ_PROBES} probe values w.r.t. Q, x0 (3), sigma and "
                        f"{heat.n_verts} vertex values",
            "backward_ms": dev_s * 1000.0 / args.steps, "forward_ms": fwd.counters["total_ms"],
            "walks_per_s": walks / dev_s, "closest_point_queries_per_s": steps / dev_s,
            "N_walks": ADJ_WALKS, "epsilon": ADJ_EPSILON, "method": "FAST_FP32",
            "triangles": int(slab.prims.shape[0]), "gpu_launches_per_gradient": 3}


def gpu_arm(args, rank, world, local):
    import torch
    from walk_on_spheres_b200 import Solver

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    mesh = workload_mesh()
    solver = Solver(local)
    solver.set_mesh(mesh)
    grid = solver.grid_over_mesh(NX, NY, 1)
    n = NX * NY
    dev = torch.device("cuda", local)
    fields = [torch.empty(n, dtype=torch.float64, device=dev) for _ in range(4)]
    loc = torch.empty(n, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    # each rank owns its own copy of the workload: a disjoint seeding range
    seed = SEED + rank * 1000003

    def solve(mode):
        return solver.solve_grid_device("poisson", grid, *[f.data_ptr() for f in fields],
                                        loc.data_ptr(), N_walks=args.walks, epsilon=EPSILON,
                                        seed=seed, source_mode=mode, method=args.method)

    for _ in range(args.warmup):
        for mode in MODES:
            solve(mode)
    barrier()
    step_ms, kernel_ms, walks, steps_total = [], [], 0, 0
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
                kernel_ms.append(c["walk_ms"])
                walks += c["total_walks"]
                steps_total += c["total_steps"]
                launches += 3  # classification, walk, merge
            step_ms.append(ms)
        barrier()
        wall = time.perf_counter() - t0
    clock = clocks.summary()
    dev_s = sum(step_ms) / 1000.0
    if dist:
        t = torch.tensor([dev_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        job_s = float(t.item())
        tw = torch.tensor([float(walks)], dtype=torch.float64, device=dev)
        dist.all_reduce(tw)
        job_walks = float(tw.item())
    else:
        job_s, job_walks = dev_s, float(walks)
    raw_rate = job_walks / job_s

    if args.kernels_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "raw_walks_per_s": raw_rate, "n_gpus": world,
                              "walks": args.walks, "ms_per_step": job_s * 1000.0 / args.steps,
                              "walk_kernel_ms": kernel_ms, "clocks": clock}), flush=True)
        if dist:
            dist.destroy_process_group()
        solver.close()
        return

    # matched standard error: per-walk variance of the fast path against the
    # FP64 estimator (PLAIN_FP64, the reference's streams) on the same grid
    fast_var = {}
    ref_var = {}
    plain_rate = None
    for mode in MODES:
        r = solver.solve_grid("poisson", NX, NY, N_walks=N_WALKS, epsilon=EPSILON, seed=seed,
                              source_mode=mode, method=args.method)
        ins = r.location == 1
        fast_var[mode] = float(np.mean(r.variance[ins]))
        p_walks = 256
        p = solver.solve_grid("poisson", NX, NY, N_walks=p_walks, epsilon=EPSILON, seed=seed,
                              source_mode=mode, method="plain")
        ref_var[mode] = float(np.mean(p.variance[ins]))
        pr = p.counters["total_walks"] / (p.counters["total_ms"] / 1000.0)
        plain_rate = pr if plain_rate is None else 2.0 / (1.0 / plain_rate + 1.0 / pr)
    var_ratio = sum(ref_var.values()) / sum(fast_var.values())
    value = raw_rate * var_ratio

    # end to end through the C ABI with host buffers
    e2e_times = []
    mean_h = np.empty(n)
    var_h, se_h, st_h = np.empty(n), np.empty(n), np.empty(n)
    loc_h = np.empty(n, dtype=np.uint8)
    import ctypes as C
    from walk_on_spheres_b200 import _lib
    L = _lib.lib()

    def host_step():
        solver.set_mesh(mesh)
        w = 0
        for mode in MODES:
            p = solver.params("poisson", N_walks=N_WALKS, epsilon=EPSILON, seed=seed,
                              source_mode=mode, method=args.method)
            cnt = _lib.Counters()
            _lib.check(L.wos_solve_grid(solver._ctx, C.byref(p), C.byref(grid),
                                        *[a.ctypes.data_as(C.c_void_p) for a in
                                          (mean_h, var_h, se_h, st_h, loc_h)], C.byref(cnt)),
                       solver._ctx)
            w += cnt.total_walks
        return w

    for _ in range(max(1, args.warmup // 2)):
        host_step()
    e2e_walks = 0
    barrier()
    for _ in range(args.steps):
        t = time.perf_counter()
        e2e_walks += host_step()
        e2e_times.append(time.perf_counter() - t)
    e2e_s = sum(e2e_times)
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
        tw = torch.tensor([float(e2e_walks)], dtype=torch.float64, device=dev)
        dist.all_reduce(tw)
        e2e_walks = int(tw.item())
    e2e_value = e2e_walks / e2e_s * var_ratio
    h2d = scene_upload_bytes(mesh) + mesh.verts.nbytes + mesh.prims.nbytes
    d2h = len(MODES) * n * (4 * 8 + 1)

    # roofline of the dominant kernel (the walk kernel)
    peak, peak_src = hbm_peak()
    avg_kernel_s = (sum(kernel_ms) / len(kernel_ms)) / 1000.0
    queries_per_launch = steps_total / len(kernel_ms)
    achieved = BYTES_PER_QUERY * queries_per_launch / avg_kernel_s / 1e9
    traffic = TRAFFIC_BYTES_PER_LAUNCH if args.method == "fast" and args.walks == N_WALKS else None

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": job_s * 1000.0 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD,
                   "equation": "poisson (2D, f = 0.1 on r <= 0.15, g = 0)",
                   "mesh": "unit circle polyline, 1024 uniform segments",
                   "grid": [NX, NY, 1], "N_walks": N_WALKS, "epsilon": EPSILON, "seed": SEED,
                   "source_modes": list(MODES),
                   "method": {"fast": "FAST_FP32 (FP32 walk + FP64 epsilon shell, FP64 sums)",
                              "fast64": "FAST_FP64", "plain": "PLAIN_FP64"}[args.method],
                   "global_batch_points": NX * NY * world, "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"dp{world} (independent grid shards)"},
        "raw_walks_per_s": raw_rate,
        "variance_ratio_fp64_over_fast": var_ratio,
        "plain_fp64_walks_per_s": plain_rate,
        "speedup_vs_plain_fp64_matched_se": value / plain_rate if plain_rate else None,
        # walk steps: each is one closest-point query of the reference's
        # algorithm; FAST_FP32 answers most of them with a distance-lattice
        # bound instead of a BVH query
        "closest_point_queries_per_s": (steps_total / job_s) * (world if dist else 1),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_src,
                     "algorithmic_bytes": f"{BYTES_PER_QUERY} B per closest-point query x "
                                          f"{queries_per_launch:.0f} queries per launch",
                     "note": "algorithmic bytes of the reference traversal per walk step; "
                             "the mesh is staged in shared memory and most steps take "
                             "their radius from the L2-resident distance lattice, so the "
                             "kernel is issue-bound and frac > 1 is expected"},
        "clocks": clock,
        "wall_s_timed_region": wall,
    }
    if not args.no_adjoint:
        line["adjoint"] = adjoint_leg(solver, args, rank, world, dist, dev)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, desc, threads, _ = reference_rate(args.cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                                "sample": desc}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    solver.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def reference_arm(args, rank, world):
    if rank != 0:
        return
    per_step = max(1.0, min(6.0, 150.0 / max(1, args.steps + args.warmup)))
    rates = []
    desc = threads = None
    for i in range(args.warmup + args.steps):
        rate, desc, threads, _ = reference_rate(per_step)
        if i >= args.warmup:
            rates.append(rate)
    value = float(np.mean(rates))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step * 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "grid": [NX, NY, 1], "N_walks": N_WALKS,
                   "epsilon": EPSILON, "seed": SEED, "source_modes": list(MODES)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_info()
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return 0
    gpu_arm(args, rank, world, local)
    return 0


if __name__ == "__main__":
    sys.exit(main())
