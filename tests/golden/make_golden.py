"""Generate the golden fixtures from the REFERENCE's own code.

    make -C oracle ref        # compiles the reference sources ($WOS_REFERENCE_DIR)
    python tests/golden/make_golden.py

Every array here is computed by oracle/_ref/libwos_ref.so, i.e. the
reference's src/{prng,bvh,npq,inside,wos,mesh}.cpp and src/equations/*.cpp
compiled where they lie, on synthetic inputs made by
walk_on_spheres_b200.meshes.  The fixtures pin the plain-C oracle
(tests/test_oracle_golden.py) and, through it, the CUDA library.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[0] = str(ROOT)

from oracle.oracle import Reference, Solve  # noqa: E402
from walk_on_spheres_b200 import meshes  # noqa: E402

OUT = Path(__file__).resolve().parent

# (name, equation, mesh, grid, walks, seed, extra)
GRID_CASES = [
    ("annulus_laplace", "laplace", "annulus", (16, 16, 1), 400, 12345, {}),
    ("circle_poisson_uniform", "poisson", "circle256", (14, 14, 1), 300, 99, {"source_mode": 0}),
    ("circle_poisson_green", "poisson", "circle256", (14, 14, 1), 300, 99, {"source_mode": 1}),
    ("annulus_screened_uniform", "screened_poisson", "annulus", (12, 12, 1), 200, 5,
     {"source_mode": 0, "alpha": 5.0}),
    ("annulus_screened_green", "screened_poisson", "annulus", (12, 12, 1), 200, 5,
     {"source_mode": 1, "alpha": 5.0}),
    ("circle_screened_green_x", "screened_poisson", "circle256", (10, 10, 1), 200, 8,
     {"source_mode": 1, "alpha": 40.0}),
    ("circle_helmholtz", "helmholtz", "circle256", (12, 12, 1), 300, 3, {}),
    ("sphere_laplace", "laplace", "sphere", (8, 8, 8), 100, 7, {}),
    ("sphere_poisson", "poisson", "sphere", (7, 7, 7), 100, 11, {"source_mode": 1}),
    ("sphere_screened", "screened_poisson", "sphere", (8, 8, 8), 100, 7, {"alpha": 10.0}),
    ("sphere_helmholtz", "helmholtz", "sphere", (7, 7, 7), 100, 2, {}),
    # edge cases: walks cut at max_steps (value g at the last nearest point,
    # counted in max_steps_hits), one walk per point (variance 0), a grid row
    # (Ny = 1: y = ymin, one point on the boundary), a wide epsilon shell, the
    # 3D classification with its minimum of three rays
    ("annulus_laplace_max_steps", "laplace", "annulus", (10, 10, 1), 60, 21, {"max_steps": 3}),
    ("sphere_laplace_max_steps", "laplace", "sphere", (5, 5, 5), 30, 17, {"max_steps": 2}),
    ("circle_poisson_one_walk", "poisson", "circle256", (9, 9, 1), 1, 4, {"source_mode": 1}),
    ("annulus_laplace_row", "laplace", "annulus", (17, 1, 1), 50, 8, {}),
    ("circle_helmholtz_wide_shell", "helmholtz", "circle256", (10, 10, 1), 100, 6,
     {"epsilon": 0.2}),
    ("sphere_poisson_three_rays", "poisson", "sphere", (6, 6, 6), 40, 13,
     {"max_ray_attempts": 3, "source_mode": 0}),
]


def mesh_by_name(name):
    return {
        "annulus": meshes.annulus(),
        "circle256": meshes.circle(segments=256),
        "sphere": meshes.uv_sphere(lon=32, lat=16),
    }[name]


def main() -> int:
    ref = Reference()
    rng = np.random.default_rng(20261203)
    g: dict[str, np.ndarray] = {}

    # PRNG streams (include/wos/prng.hpp, src/prng.cpp, include/wos/hash.hpp)
    seeds = np.array([0, 1, 7, 12345, 2**63, 2**64 - 1] +
                     [int(x) for x in rng.integers(0, 2**63, 10, dtype=np.int64)], dtype=np.uint64)
    g["prng_seeds"] = seeds
    g["prng_u64"] = np.stack([ref.prng_u64(int(s), 64) for s in seeds])
    g["prng_unit"] = np.stack([ref.prng_unit(int(s), 16) for s in seeds])
    g["prng_unit_open"] = np.stack([ref.prng_unit(int(s), 16, open_=True) for s in seeds])
    g["splitmix64"] = np.array([ref.splitmix64(int(s)) for s in seeds], dtype=np.uint64)

    for mname in ("annulus", "sphere"):
        m = mesh_by_name(mname)
        boxes, counts, idx, prims = ref.build_bvh(m)
        g[f"bvh_{mname}_boxes"], g[f"bvh_{mname}_counts"] = boxes, counts
        g[f"bvh_{mname}_idx"], g[f"bvh_{mname}_prims"] = idx, prims
        pts = rng.uniform(-1.2, 1.2, (3000, m.dim))
        d, near, prim, bid = ref.npq(m, pts)
        g[f"npq_{mname}_points"], g[f"npq_{mname}_dist"] = pts, d
        g[f"npq_{mname}_nearest"], g[f"npq_{mname}_bid"] = near, bid
    ann = mesh_by_name("annulus")
    wpts = rng.uniform(-1.1, 1.1, (4000, 2))
    g["winding_points"], g["winding_numbers"] = wpts, ref.winding_numbers(ann, wpts)
    sph = mesh_by_name("sphere")
    cpts = rng.uniform(-1.1, 1.1, (1500, 3))
    cseeds = rng.integers(0, 2**63, 1500, dtype=np.int64).astype(np.uint64)
    loc, ret = ref.classify_3d(sph, cpts, cseeds, 1e-10 * 2.0)
    g["classify_points"], g["classify_seeds"] = cpts, cseeds
    g["classify_location"], g["classify_retries"] = loc, ret

    x = np.concatenate([np.geomspace(1e-8, 2.0, 60), np.linspace(2.0, 49.9, 120),
                        np.linspace(50.0, 300.0, 40)])
    g["bessel_x"], g["bessel"] = x, ref.bessel(x)
    jx = np.linspace(1e-6, 2.3, 100)
    g["j0y0_x"] = jx
    g["j0"], g["y0"] = ref.j0y0(jx)
    a = rng.uniform(0.5, 40.0, 400)
    R = rng.uniform(1e-4, 1.0, 400)
    r = R * rng.uniform(0.01, 0.999, 400)
    g["screened_alpha"], g["screened_R"], g["screened_r"] = a, R, r
    g["screened_kernels"] = ref.screened_kernels(a, R, r)
    for dim in (2, 3):
        for alpha, Rv in ((5.0, 0.3), (20.0, 0.5)):
            g[f"screened_samples_{dim}d_{int(alpha)}"] = ref.screened_samples(dim, alpha, Rv, 42, 200)
        gr, ms, sm = ref.poisson_green(dim, 0.7, np.linspace(0.01, 0.7, 50), 9)
        g[f"poisson_green_{dim}d"], g[f"poisson_mass_{dim}d"] = gr, ms
        g[f"poisson_samples_{dim}d"] = sm
        st, bl = ref.steps(dim, np.array([0.1, -0.2, 0.3][:dim]), 0.25, 77, 100)
        g[f"steps_{dim}d"], g[f"balls_{dim}d"] = st, bl

    for name, eq, mname, (nx, ny, nz), walks, seed, extra in GRID_CASES:
        s = Solve(mesh_by_name(mname), nx, ny, nz, N_walks=walks, seed=seed, **extra)
        res = ref.solve_grid(eq, s)
        for k in ("mean", "variance", "standard_error", "mean_steps", "location"):
            g[f"grid_{name}_{k}"] = getattr(res, k)
        g[f"grid_{name}_counters"] = np.array([res.counters["inside_points"],
                                               res.counters["max_steps_hits"],
                                               res.counters["ambiguous_ray_retries"],
                                               res.counters["indeterminate_points"]],
                                              dtype=np.int64)

    np.savez_compressed(OUT / "reference_golden.npz", **g)
    size = (OUT / "reference_golden.npz").stat().st_size
    print(f"wrote {OUT / 'reference_golden.npz'} ({size / 1024:.0f} KiB, {len(g)} arrays)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
