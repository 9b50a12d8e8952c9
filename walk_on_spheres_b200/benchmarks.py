"""Throughput and accuracy of the single-solve workloads, per walk method.

    python -m walk_on_spheres_b200.benchmarks [--workloads a,b] [--scale 1.0] [--tune]
    python -m walk_on_spheres_b200.benchmarks --batch [--scale 1.0]
    python -m walk_on_spheres_b200.benchmarks --batch-setup [--reps 3]
    python -m walk_on_spheres_b200.benchmarks --heat [--scale 1.0]
    python -m walk_on_spheres_b200.benchmarks --transient [--scale 1.0]
    python -m walk_on_spheres_b200.benchmarks --stationary [--scale 1.0]
    python -m walk_on_spheres_b200.benchmarks --profile sphere [--walks 512]

Workloads (synthetic meshes from walk_on_spheres_b200.meshes):

* laplace2d_annulus256_64sq — `laplace` on the annulus 0.5 < r < 1
  (2 x 128 segments), 64 x 64 grid, 10 000 walks, eps 0.01, seed 12345;
  analytic u = (16/15 r^2 - 1/(15 r^2)) cos 2 theta.
* poisson2d_circle1024_256sq_{uniform,green} — `poisson` on the unit circle
  (1024 segments), 256 x 256 grid, 4096 walks; analytic piecewise solution of
  the f = 0.1 disk load.
* screened3d_sphere16128_64cube — `screened_poisson`, alpha 10, on the UV
  sphere with 128 x 64 bands (16 128 triangles), 64^3 grid, 1024 walks,
  seed 7 (eps clamped to 0.005).

`--batch` runs the 64-solve mixed batch (mixed_batch_specs) as one
graph-captured launch sequence and, for comparison, solve by solve.
`--batch-setup` times the same batch's set-up alone (mesh checks, tree
builds, uploads, lattices, near-boundary lists) at 1/250 of the walks, the
launches an ncu launch list of the set-up selects.
`--heat`, `--transient` and `--stationary` run the Gaussian heat-source
forward/adjoint workload and the reference's welding levels 2 and 1.

For each workload and method it prints device walks/s, closest-point
queries/s, mean steps and, against PLAIN_FP64 (the reference estimator and
streams), the mean |difference| / combined standard error and the variance
ratio; where an analytic solution exists, the largest |mean - u| and the
fraction of points within 5 SE + eps max|grad u|.  `--scale` multiplies the
walk counts (e.g. 0.25 for a quick look); PLAIN_FP64 runs with at most 256
walks per point on the 3D workload to keep it within a minute.
"""
from __future__ import annotations

import argparse
import json
import time
import sys

import numpy as np

from . import meshes
from .solver import Solver


def _annulus_u(X, Y, Z):
    r2 = X * X + Y * Y
    return (16.0 / 15.0 * r2 - 1.0 / (15.0 * r2)) * (X * X - Y * Y) / r2


def _disk_u(X, Y, Z, f=0.1, a=0.15):
    r = np.hypot(X, Y)
    return np.where(r <= a, f / 4 * (a * a - r * r) + f * a * a / 2 * np.log(1 / a),
                    f * a * a / 2 * np.log(1 / np.maximum(r, 1e-300)))


WORKLOADS = {
    "laplace2d_annulus256_64sq": dict(mesh=meshes.annulus, eq="laplace", grid=(64, 64, 1),
                                      walks=10000, kw=dict(seed=12345), analytic=_annulus_u,
                                      grad=2.2),
    "poisson2d_circle1024_256sq_uniform": dict(
        mesh=lambda: meshes.circle(segments=1024), eq="poisson", grid=(256, 256, 1), walks=4096,
        kw=dict(seed=12345, source_mode="uniform"), analytic=_disk_u, grad=0.0075),
    "poisson2d_circle1024_256sq_green": dict(
        mesh=lambda: meshes.circle(segments=1024), eq="poisson", grid=(256, 256, 1), walks=4096,
        kw=dict(seed=12345, source_mode="green"), analytic=_disk_u, grad=0.0075),
    "screened3d_sphere16128_64cube": dict(mesh=meshes.uv_sphere, eq="screened_poisson",
                                          grid=(64, 64, 64), walks=1024,
                                          kw=dict(seed=7, alpha=10.0), analytic=None, grad=None,
                                          plain_walks=256),
}


def _coords(s: Solver, nx, ny, nz):
    b = s.bbox
    ax = [np.array([lo + (hi - lo) * i / (n - 1) if n > 1 else lo for i in range(n)])
          for lo, hi, n in ((b[0], b[1], nx), (b[2], b[3], ny), (b[4], b[5], nz))]
    return np.meshgrid(*ax, indexing="ij")


def run(name: str, scale: float = 1.0, device: int = 0, tune: bool = False) -> dict:
    w = WORKLOADS[name]
    mesh = w["mesh"]()
    s = Solver(device).set_mesh(mesh)
    nx, ny, nz = w["grid"]
    walks = max(16, int(round(w["walks"] * scale)))
    out = {"workload": name, "walks": walks, "methods": {}}
    tuned = None
    if tune:
        from .autotune import Tuner
        tuned = Tuner(s).tune(mesh, w["eq"], (nx, ny, nz), N_walks=walks, method="fast",
                              **w["kw"])
        out["tuning"] = {"chunk": tuned.chunk, "blocks": tuned.blocks,
                         "leaf_size": tuned.leaf_size,
                         "probe_walks_per_s": tuned.walks_per_s,
                         "candidates": [{k: r[k] for k in ("leaf_size", "chunk", "blocks",
                                                             "walks_per_s")}
                                        for r in tuned.table]}
    res = {}
    for method in ("fast", "fast64", "plain"):
        n = walks if method != "plain" else min(walks, w.get("plain_walks", walks))
        if tuned is not None and method != "fast":
            s.set_tuning(0, 0)
        # an untimed short solve first: module loading and first-launch set-up
        # stay out of the timed one
        s.solve_grid(w["eq"], nx, ny, nz, N_walks=min(n, 16), method=method, **w["kw"])
        r = s.solve_grid(w["eq"], nx, ny, nz, N_walks=n, method=method, **w["kw"])
        c = r.counters
        secs = c["walk_ms"] / 1000.0
        res[method] = r
        ins = r.location == 1
        out["methods"][method] = {
            "walks": n,
            "walks_per_s": c["total_walks"] / secs,
            "queries_per_s": c["exact_queries"] / secs,
            "lattice_step_share": 1.0 - c["exact_queries"] / max(1, c["total_steps"]),
            "walk_ms": c["walk_ms"], "classify_ms": c["classify_ms"],
            "mean_steps": float(np.mean(r.mean_steps[ins])),
            "variance_per_walk": float(np.mean(r.variance[ins])),
        }
    ins = res["plain"].location == 1
    for method in ("fast", "fast64"):
        a, b = res[method], res["plain"]
        se = np.sqrt(a.standard_error[ins] ** 2 + b.standard_error[ins] ** 2)
        live = se > 0
        z = np.abs(a.mean[ins] - b.mean[ins])[live] / se[live]
        m = out["methods"][method]
        m["vs_plain_mean_abs_z"] = float(z.mean())
        m["vs_plain_frac_within_3se"] = float((z <= 3).mean())
        m["variance_ratio_plain_over_method"] = (
            out["methods"]["plain"]["variance_per_walk"] / m["variance_per_walk"])
        m["matched_se_speedup_vs_plain"] = (
            m["walks_per_s"] / out["methods"]["plain"]["walks_per_s"]
            * m["variance_ratio_plain_over_method"])
    if w["analytic"] is not None:
        X, Y, Z = _coords(s, nx, ny, nz)
        u = w["analytic"](X, Y, Z)
        eps = res["plain"].counters["effective_epsilon"]
        for method, r in res.items():
            ins_m = r.location == 1
            err = np.abs(r.mean - u)[ins_m]
            bound = 5 * r.standard_error[ins_m] + eps * w["grad"] + 1e-6
            out["methods"][method]["analytic_max_abs_err"] = float(err.max())
            out["methods"][method]["analytic_frac_within_bound"] = float((err <= bound).mean())
    s.close()
    return out


EQUATIONS3 = ("laplace", "poisson", "screened_poisson")


def mixed_batch_specs(seed: int = 2024, scale: float = 1.0) -> list[dict]:
    """The mixed batch of 64 independent solves: 32 star polygons
    r = 1 + 0.3 sum_{k<=6} a_k cos(k theta + phi_k) (a_k ~ U[0, 0.15]) with
    64..4096 edges (log-uniform) on square grids of side 32..512, and 32 UV
    spheres radially perturbed by real spherical harmonics up to degree 4 with
    2k..200k triangles on cubic grids of side 16..64; N_walks from
    {256, 1024, 4096}, equation from laplace / poisson / screened_poisson
    (alpha ~ U[1, 20]), source mode uniform or Green, one seed per solve.
    `scale` multiplies the walk counts."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(64):
        dim = 2 if k < 32 else 3
        if dim == 2:
            edges = int(round(np.exp(rng.uniform(np.log(64), np.log(4096)))))
            side = int(round(np.exp(rng.uniform(np.log(32), np.log(512)))))
            mesh = dict(kind="star", edges=edges, seed=int(rng.integers(1 << 31)))
            grid = (side, side, 1)
        else:
            tris = np.exp(rng.uniform(np.log(2000), np.log(200000)))
            lon = max(8, int(round(np.sqrt(tris))))
            mesh = dict(kind="sphere", lon=lon, lat=max(4, lon // 2),
                        seed=int(rng.integers(1 << 31)))
            side = int(round(np.exp(rng.uniform(np.log(16), np.log(64)))))
            grid = (side, side, side)
        walks = int(rng.choice([256, 1024, 4096]))
        eq = EQUATIONS3[int(rng.integers(3))]
        alpha = float(rng.uniform(1.0, 20.0))
        mode = ("uniform", "green")[int(rng.integers(2))]
        specs.append(dict(dim=dim, mesh=mesh, grid=grid, equation=eq,
                          params=dict(N_walks=max(1, int(round(walks * scale))), alpha=alpha,
                                      source_mode=mode, seed=int(rng.integers(1 << 62)),
                                      method="fast")))
    return specs


def build_mesh(m: dict):
    rng = np.random.default_rng(m["seed"])
    if m["kind"] == "star":
        return meshes.star_polygon(rng, m["edges"])
    return meshes.perturbed_sphere(rng, m["lon"], m["lat"])


def run_batch(scale: float = 1.0, device: int = 0, sequential: bool = True,
              seed: int = 2024) -> dict:
    """Device time of the mixed batch as one graph-captured launch sequence,
    against the same solves run one after another (sum of their device
    times)."""
    from .batch import Batch
    specs = mixed_batch_specs(seed, scale)
    s = Solver(device)
    b = Batch(s)
    built = []
    host_build_s = 0.0
    for sp in specs:
        mesh = build_mesh(sp["mesh"])
        built.append(mesh)
        t0 = time.perf_counter()
        mid = b.add_mesh(mesh)          # checks only
        host_build_s += time.perf_counter() - t0
        b.add_solve(mid, sp["equation"], *sp["grid"], **sp["params"])
    t0 = time.perf_counter()
    b.prepare()                      # parallel BVH builds, uploads, lattices
    host_build_s += time.perf_counter() - t0
    b.run(use_graph=True)            # capture, warm
    ms = b.run(use_graph=True)
    info = b.info()
    out = {"workload": "mixed_batch_64", "scale": scale, "solves": info["solves"],
           "points": info["points"], "walks": info["walks"], "steps": info["steps"],
           "prims": [int(m.prims.shape[0]) for m in built],
           "host_build_and_upload_s": host_build_s,
           "batch_graph_ms": ms, "batch_walks_per_s": info["walks"] / (ms / 1000.0),
           "batch_walk_steps_per_s": info["steps"] / (ms / 1000.0)}
    ms_stream = b.run(use_graph=False)
    out["batch_stream_ms"] = ms_stream
    b.close()
    if sequential:
        total = 0.0
        for sp, mesh in zip(specs, built):
            s.set_mesh(mesh)
            r = s.solve_grid(sp["equation"], *sp["grid"], **sp["params"])
            total += r.counters["total_ms"]
        out["sequential_ms"] = total
        out["sequential_walks_per_s"] = info["walks"] / (total / 1000.0)
        out["batch_speedup"] = total / ms
    s.close()
    return out


def run_batch_setup(reps: int = 3, device: int = 0, seed: int = 2024) -> dict:
    """Wall time of the mixed batch's one-time set-up: add_mesh / add_solve
    for the 64 solves, prepare (tree builds on the host threads, uploads,
    lattices) and the first run's plan (near-boundary lists), with the walk
    counts scaled by 1/250 so the run itself is short.  Repeated `reps` times
    on one context after a warm-up solve."""
    from .batch import Batch
    specs = mixed_batch_specs(seed, 0.004)
    built = [build_mesh(sp["mesh"]) for sp in specs]
    s = Solver(device)
    s.set_mesh(built[0])
    s.solve_grid(specs[0]["equation"], 8, 8, N_walks=64, method="fast")
    runs = []
    for _ in range(reps):
        b = Batch(s)
        t0 = time.perf_counter()
        for sp, m in zip(specs, built):
            mid = b.add_mesh(m)
            b.add_solve(mid, sp["equation"], *sp["grid"], **sp["params"])
        t1 = time.perf_counter()
        b.prepare()
        t2 = time.perf_counter()
        ms = b.run(use_graph=False)
        t3 = time.perf_counter()
        runs.append({"add_s": t1 - t0, "prepare_s": t2 - t1,
                     "plan_s": (t3 - t2) - ms / 1000.0, "run_ms": ms})
        b.close()
    s.close()
    return {"workload": "mixed_batch_64_setup", "meshes": len(built),
            "prims_total": int(sum(m.prims.shape[0] for m in built)), "runs": runs}


def run_heat(scale: float = 1.0, device: int = 0, seed: int = 7) -> dict:
    """The differentiable heat-source workload: 3D Gaussian source Q = 1e3,
    sigma = 2 mm, x0 at the centre of the top face of a 0.10 x 0.05 x 0.01 m
    slab of ~20k triangles, g = 0, 4096 probes uniform in the interior,
    2048 FP32 walks (times `scale`), epsilon 1e-5 m.  For Green and MIS source
    sampling: forward and backward device times, walks and queries per
    second, and the median relative standard error of the probe values and
    of du/dQ over probes where the source is felt (|u| > 1e-6 max|u|)."""
    from .heat import HeatProblem
    slab = meshes.slab_box(target_triangles=20000)
    s = Solver(device).set_mesh(slab)
    rng = np.random.default_rng(20240)
    hi = np.array([0.10, 0.05, 0.01])
    probes = hi * rng.uniform(0.001, 0.999, size=(4096, 3))
    walks = max(32, int(round(2048 * scale)))
    theta = (1e3, (0.05, 0.025, 0.01), 2e-3)
    out = {"workload": "heat3d_slab20k_4096probes", "walks": walks,
           "triangles": int(slab.prims.shape[0]), "modes": {}}
    for mode in ("green", "mis"):
        heat = HeatProblem(s, probes, N_walks=walks, epsilon=1e-5, seed=seed, source_mode=mode,
                           method="fast", proposal=(theta[1], theta[2]))
        g = np.zeros(heat.n_verts)
        heat.forward(*theta, g)
        f = heat.forward(*theta, g)
        a = heat.adjoint(*theta, g)
        felt = np.abs(f.mean) > 1e-6 * np.nanmax(np.abs(f.mean))
        rel = f.standard_error[felt] / np.abs(f.mean[felt])
        jrel = a.jacobian_se[felt, 0] / np.abs(a.jacobian[felt, 0])
        c, ca = f.counters, a.counters
        out["modes"][mode] = {
            "forward_ms": c["total_ms"], "backward_ms": ca["total_ms"],
            "gradients_per_s": 1000.0 / ca["total_ms"],
            "walks_per_s": c["total_walks"] / (c["walk_ms"] / 1000.0),
            "queries_per_s": c["exact_queries"] / (c["walk_ms"] / 1000.0),
            "mean_steps": c["total_steps"] / max(1, c["total_walks"]),
            "probes_felt": int(felt.sum()),
            "median_rel_se_u": float(np.median(rel)),
            "median_rel_se_dudQ": float(np.median(jrel)),
            "grad_source": a.grad_source.tolist()}
    s.close()
    return out


def run_transient(scale: float = 1.0, device: int = 0) -> dict:
    """The reference's level-2 transient welding baseline at its defaults
    (49 x 33 grid, 100 steps of 0.1 s, 500 walks, epsilon 8e-6 m; walks
    times `scale`), one CUDA graph per run, for each walk method."""
    from .transient import solve_transient
    s = Solver(device)
    walks = max(8, int(round(500 * scale)))
    out = {"workload": "level2_plate_49x33_100steps", "walks": walks, "methods": {}}
    for method in ("fast", "fast64", "plain"):
        solve_transient(s, method=method, walks=walks, total_time=0.2, heat_on_time=0.1)  # warm-up
        r = solve_transient(s, method=method, walks=walks)
        inner = r.fields[:, 1:-1, 1:-1]
        n_walks = (r.fields.shape[1] - 2) * (r.fields.shape[2] - 2) * walks * r.steps
        out["methods"][method] = {
            "device_ms": r.device_ms, "walks_per_s": n_walks / (r.device_ms / 1000.0),
            "centre_rise_final": float(r.fields[-1, r.fields.shape[1] // 2,
                                                r.fields.shape[2] // 2]),
            "peak_rise": float(inner.max()),
            "mean_se_final": float(r.standard_error[-1, 1:-1, 1:-1].mean()),
            "max_steps_hits": r.max_steps_hits}
    s.close()
    return out


def run_stationary(scale: float = 1.0, device: int = 0) -> dict:
    """The reference's level-1 stationary welding program (49 x 33 grid, 6000
    walks, epsilon 8e-6 m; walks times `scale`): its three solves for each
    walk method, with the reference's gates against the finite-difference
    solution for the Gaussian cases."""
    from .stationary import LEVEL1_CASES, gaussian_summary, manufactured_summary, solve_stationary
    s = Solver(device)
    walks = max(8, int(round(6000 * scale)))
    out = {"workload": "level1_plate_49x33", "walks": walks, "cases": {}}
    for case, spec in LEVEL1_CASES.items():
        res = {}
        for method in ("fast", "fast64", "plain"):
            solve_stationary(s, method=method, walks=16, **spec)  # warm-up
            r = solve_stationary(s, method=method, walks=walks, **spec)
            n_walks = (r.mean.shape[0] - 2) * (r.mean.shape[1] - 2) * walks
            summ = (manufactured_summary(r) if spec["source"] == "manufactured"
                    else gaussian_summary(r))
            res[method] = {"device_ms": r.device_ms,
                           "walks_per_s": n_walks / (r.device_ms / 1000.0),
                           "mean_standard_error": summ["mean_standard_error"],
                           "mean_steps": summ["mean_steps"],
                           "max_steps_hits": r.max_steps_hits}
            if spec["source"] == "manufactured":
                res[method]["field_rmse"] = summ["field_rmse"]
            else:
                res[method]["peak_temperature_rise"] = summ["peak_temperature_rise"]
        out["cases"][case] = res
    s.close()
    return out


PROFILE_CASES = ("annulus", "disk_uniform", "disk_green", "sphere", "heat")


def run_profile(case: str, walks: int, device: int = 0) -> dict:
    """One small warm-up solve, then ONE FAST_FP32 solve of a workload at
    `walks` walks per point: the launch an ncu capture selects with
    `-k regex:<kernel> -s 1 -c 1` (the lattice build and the warm-up solve's
    launches come first).  Prints the launch's walk counters, so its
    per-step figures can be formed."""
    s = Solver(device)
    if case == "heat":
        from .heat import HeatProblem
        s.set_mesh(meshes.slab_box(target_triangles=20000))
        rng = np.random.default_rng(20240)
        probes = np.array([0.10, 0.05, 0.01]) * rng.uniform(0.001, 0.999, size=(4096, 3))
        theta = (1e3, (0.05, 0.025, 0.01), 2e-3)
        heat = HeatProblem(s, probes[:64], N_walks=16, epsilon=1e-5, seed=12345,
                           source_mode="green", method="fast")
        heat.adjoint(*theta)
        heat = HeatProblem(s, probes, N_walks=walks, epsilon=1e-5, seed=12345,
                           source_mode="green", method="fast")
        c = heat.adjoint(*theta).counters
    else:
        name = {"annulus": "laplace2d_annulus256_64sq",
                "disk_uniform": "poisson2d_circle1024_256sq_uniform",
                "disk_green": "poisson2d_circle1024_256sq_green",
                "sphere": "screened3d_sphere16128_64cube"}[case]
        w = WORKLOADS[name]
        s.set_mesh(w["mesh"]())
        s.solve_grid(w["eq"], 8, 8, 8, N_walks=16, method="fast", **w["kw"])
        c = s.solve_grid(w["eq"], *w["grid"], N_walks=walks, method="fast", **w["kw"]).counters
    s.close()
    keys = ("total_walks", "total_steps", "exact_queries", "walk_ms", "total_ms")
    return {"case": case, "walks": walks, **{k: c[k] for k in keys}}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--workloads", default=",".join(WORKLOADS))
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--tune", action="store_true",
                    help="autotune the FAST_FP32 schedule and leaf size first")
    ap.add_argument("--batch", action="store_true",
                    help="run the 64-solve mixed batch instead of the single solves")
    ap.add_argument("--batch-setup", action="store_true",
                    help="time the mixed batch's set-up alone (1/250 of the walks)")
    ap.add_argument("--reps", type=int, default=3, help="repetitions of --batch-setup")
    ap.add_argument("--heat", action="store_true",
                    help="run the differentiable heat-source workload (Green and MIS)")
    ap.add_argument("--transient", action="store_true",
                    help="run the transient plate heating workload (reference level 2)")
    ap.add_argument("--stationary", action="store_true",
                    help="run the stationary plate heating workload (reference level 1)")
    ap.add_argument("--profile", choices=PROFILE_CASES,
                    help="one FAST_FP32 solve of a workload for an ncu capture (walks: --walks)")
    ap.add_argument("--walks", type=int, default=512, help="walks per point of --profile")
    a = ap.parse_args(argv)
    if a.profile:
        print(json.dumps(run_profile(a.profile, a.walks, a.device)), flush=True)
        return 0
    if a.stationary:
        print(json.dumps(run_stationary(a.scale, a.device)), flush=True)
        return 0
    if a.transient:
        print(json.dumps(run_transient(a.scale, a.device)), flush=True)
        return 0
    if a.heat:
        print(json.dumps(run_heat(a.scale, a.device)), flush=True)
        return 0
    if a.batch_setup:
        print(json.dumps(run_batch_setup(a.reps, a.device)), flush=True)
        return 0
    if a.batch:
        print(json.dumps(run_batch(a.scale, a.device)), flush=True)
        return 0
    for name in a.workloads.split(","):
        print(json.dumps(run(name.strip(), a.scale, a.device, a.tune)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
