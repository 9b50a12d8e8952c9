"""Algorithmic bytes per closest-point query of the benchmark workloads.
TEST / MEASUREMENT INFRASTRUCTURE ONLY.

The roofline's algorithmic byte count of a walk-on-spheres step is the data
the reference's BVH traversal (src/bvh.cpp:295-387) has to touch for one
closest-point query:

    B_npq = V_node * S_node + V_prim * S_prim

with V the node pops and primitive tests of that traversal, replayed by the
oracle along real walk queries (oracle/wos_oracle.c, wo_walk_visit_counts),
and S the reference's record sizes: BVHNode<2> 40 B, BVHNode<3> 56 B
(include/wos/bvh.hpp:10-15), a 2D segment 2 x 16 B vertices + 2 x 4 B
indices = 40 B, an EberlyCache 112 B (include/wos/npq.hpp:6-10).

    python -m oracle.measure_traversal            # prints the table used by bench.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path[0] = str(ROOT)

from oracle.oracle import Oracle, Solve  # noqa: E402
from walk_on_spheres_b200 import meshes  # noqa: E402

NODE_BYTES = {2: 40, 3: 56}
PRIM_BYTES = {2: 40, 3: 112}

WORKLOADS = {
    # 2D poisson, unit circle 1024 segments, 256^2 grid (the headline workload)
    "poisson2d_circle1024_256sq": dict(eq="poisson", mesh=lambda: meshes.circle(segments=1024),
                                       grid=(256, 256, 1), stride=97, walks=256, extra={}),
    # 2D laplace, annulus 2 x 128 segments, 64^2 grid
    "laplace2d_annulus256_64sq": dict(eq="laplace", mesh=lambda: meshes.annulus(),
                                      grid=(64, 64, 1), stride=7, walks=256, extra={}),
    # 3D screened poisson alpha 10, UV sphere 16 128 triangles, 64^3 grid
    "screened3d_sphere16128_64cube": dict(eq="screened_poisson", mesh=lambda: meshes.uv_sphere(),
                                          grid=(64, 64, 64), stride=1009, walks=64,
                                          extra={"alpha": 10.0}),
}


def measure(name: str) -> dict:
    w = WORKLOADS[name]
    m = w["mesh"]()
    nx, ny, nz = w["grid"]
    pts = np.arange(0, nx * ny * nz, w["stride"], dtype=np.int64)
    o = Oracle()
    s = Solve(m, nx, ny, nz, N_walks=w["walks"], seed=12345, points=pts, **w["extra"])
    v = o.walk_visit_counts(w["eq"], s, w["walks"])
    q = max(1, v["queries"])
    vn, vp = v["node_pops"] / q, v["prim_tests"] / q
    return {"workload": name, "queries": q, "node_pops_per_query": vn,
            "prim_tests_per_query": vp,
            "bytes_per_query": vn * NODE_BYTES[m.dim] + vp * PRIM_BYTES[m.dim]}


def main() -> int:
    for name in WORKLOADS:
        r = measure(name)
        print(f"{r['workload']:34s} queries={r['queries']:9d} nodes/q={r['node_pops_per_query']:8.2f} "
              f"prims/q={r['prim_tests_per_query']:8.2f} bytes/q={r['bytes_per_query']:9.1f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
