// Threaded per-grid-point driver around the REFERENCE's own walk-on-spheres
// functions.  TEST INFRASTRUCTURE ONLY: it is compiled into oracle/_ref
// together with the reference sources (oracle/Makefile) and is used by the
// tests, by the golden-fixture generator and by bench.py's CPU baseline.
//
// The per-point body restates include/wos/runner.hpp:157-236: the global
// linear index (i*Ny + j)*Nz + k, the point seed
// splitmix64(seed ^ splitmix64(linear)) (runner.hpp:163-168), the start
// point (wos.hpp:42-52), classification (runner.hpp:177-193, 3D with the
// INSIDE stream), the boundary value for boundary points (runner.hpp:196-206)
// and wos_run on the WOS (+ 2D SOURCE) streams (runner.hpp:207-222).  The
// reference's seeding depends only on global indices, so running the points
// on any number of threads gives the same fields as `mpirun -np P`
// (README.md:87-90).
#pragma once

#include <algorithm>
#include <atomic>
#include <chrono>
#include <exception>
#include <memory>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "wos/bvh.hpp"
#include "wos/grid.hpp"
#include "wos/hash.hpp"
#include "wos/inside.hpp"
#include "wos/mesh.hpp"
#include "wos/prng.hpp"
#include "wos/wos.hpp"

extern "C" {

// Problem description shared by every oracle/_ref entry point (plain C).
struct ref_problem {
    int dim;                  // 2 or 3
    const double *verts;      // n_verts * dim
    int n_verts;
    const int *prims;         // n_prims * dim vertex indices (0-based)
    int n_prims;
    const int *boundary_ids;  // 2D only: per segment; may be null (all 0)
    int Nx, Ny, Nz;
    int use_mesh_bbox;        // 1: grid spans the mesh bounding box (runner.hpp:83-85)
    double xmin, xmax, ymin, ymax, zmin, zmax;
    int N_walks;
    double epsilon;
    int max_steps;
    int max_ray_attempts;
    uint64_t seed;
    double alpha;
    int source_mode;          // 0 uniform, 1 green
    int n_threads;            // <= 0: all hardware threads
    const long long *points;  // optional subset of global linear indices
    long long n_points;       // number of entries in `points` (ignored when null)
};

struct ref_outputs {
    double *mean;             // full grid (Nx*Ny*Nz), row-major (i, j, k)
    double *variance;
    double *standard_error;
    double *mean_steps;
    unsigned char *location;
    long long inside_points;
    long long max_steps_hits;
    long long ambiguous_ray_retries;
    long long indeterminate_points;
    double sum_variance;
    double sum_standard_error;
    double sum_mean_steps;
    double seconds;           // wall time of the point loop
};

}  // extern "C"

namespace wos_ref {

template <int N>
wos::Mesh<N> mesh_from_arrays(const ref_problem &pb) {
    wos::Mesh<N> m;
    m.verts.resize(pb.n_verts);
    for (int v = 0; v < pb.n_verts; ++v) {
        if constexpr (N == 2) {
            m.verts[v] = wos::Point2D{pb.verts[2 * v], pb.verts[2 * v + 1]};
        } else {
            m.verts[v] = wos::Point3D{pb.verts[3 * v], pb.verts[3 * v + 1], pb.verts[3 * v + 2]};
        }
    }
    m.prims.assign(pb.prims, pb.prims + static_cast<size_t>(N) * pb.n_prims);
    if constexpr (N == 2) {
        m.boundary_ids.assign(pb.n_prims, 0);
        if (pb.boundary_ids) {
            m.boundary_ids.assign(pb.boundary_ids, pb.boundary_ids + pb.n_prims);
        }
    }
    return m;
}

inline double now_seconds() {
    return std::chrono::duration<double>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

template <int N, typename Eq>
int solve_grid(const ref_problem &pb, const Eq &eq, double epsilon, ref_outputs &out) {
    using namespace wos;
    Mesh<N> domain = mesh_from_arrays<N>(pb);
    std::unique_ptr<BVH<N>> bvh = build_bvh(domain);

    const int Nx = pb.Nx, Ny = pb.Ny, Nz = (N == 2) ? 1 : pb.Nz;
    Grid grid{Nx, Ny, Nz, pb.xmin, pb.xmax, pb.ymin, pb.ymax, pb.zmin, pb.zmax};
    if (pb.use_mesh_bbox) {
        mesh_bbox(domain, &grid.xmin, &grid.xmax, &grid.ymin, &grid.ymax, &grid.zmin,
                  &grid.zmax);
    }
    const double mesh_scale = std::max({1.0, grid.xmax - grid.xmin, grid.ymax - grid.ymin,
                                        grid.zmax - grid.zmin});
    const double boundary_tolerance = 1e-10 * mesh_scale;

    const long long total = static_cast<long long>(Nx) * Ny * Nz;
    const long long n_work = pb.points ? pb.n_points : total;
    int threads = pb.n_threads > 0 ? pb.n_threads
                                   : static_cast<int>(std::thread::hardware_concurrency());
    threads = std::max(1, threads);

    std::atomic<long long> cursor{0};
    struct Tally {
        long long inside = 0, hits = 0, retries = 0, indeterminate = 0;
        double sums[3] = {0.0, 0.0, 0.0};
    };
    std::vector<Tally> tallies(threads);

    auto worker = [&](int tid) {
        Tally &t = tallies[tid];
        for (;;) {
            const long long w = cursor.fetch_add(1, std::memory_order_relaxed);
            if (w >= n_work) break;
            const long long linear = pb.points ? pb.points[w] : w;
            const int i = static_cast<int>(linear / (static_cast<long long>(Ny) * Nz));
            const int j = static_cast<int>((linear / Nz) % Ny);
            const int k = static_cast<int>(linear % Nz);
            const double x = grid_coordinate(grid.xmin, grid.xmax, i, grid.Nx);
            const double y = grid_coordinate(grid.ymin, grid.ymax, j, grid.Ny);
            const double z = grid_coordinate(grid.zmin, grid.zmax, k, grid.Nz);
            const uint64_t point_seed =
                splitmix64(pb.seed ^ splitmix64(static_cast<uint64_t>(linear)));

            Point<N> p0;
            if constexpr (N == 2) {
                p0 = Point2D{x, y};
            } else {
                p0 = Point3D{x, y, z};
            }
            auto start = get_start_point(*bvh, p0);

            PointLocation where;
            if constexpr (N == 2) {
                where = classify_point(domain, p0, start.radius, boundary_tolerance);
            } else {
                PRNG inside_rng(splitmix64(point_seed ^ 0x243F6A8885A308D3ULL));
                const PointClassification c = classify_point(
                    *bvh, p0, start.radius, boundary_tolerance, pb.max_ray_attempts, inside_rng);
                where = c.location;
                t.retries += c.ambiguous_ray_retries;
                if (where == PointLocation::Indeterminate) ++t.indeterminate;
            }

            WoSResult r{NAN, NAN, NAN, NAN, 0};
            if (where == PointLocation::Boundary) {
                double g;
                if constexpr (N == 2) {
                    g = eq.boundary(start.nearest, start.boundary_id);
                } else {
                    g = eq.boundary(start.nearest);
                }
                r = WoSResult{g, 0.0, 0.0, 0.0, 0};
            } else if (where == PointLocation::Inside) {
                PRNG walk_rng(splitmix64(point_seed ^ 0x13198A2E03707344ULL));
                if constexpr (N == 2) {
                    PRNG source_rng(splitmix64(point_seed ^ 0xA4093822299F31D0ULL));
                    r = wos_run(*bvh, p0, start, eq, pb.N_walks, epsilon, walk_rng, source_rng,
                                pb.max_steps);
                } else {
                    r = wos_run(*bvh, p0, start, eq, pb.N_walks, epsilon, walk_rng, walk_rng,
                                pb.max_steps);
                }
                ++t.inside;
                t.hits += r.max_steps_hits;
                t.sums[0] += r.variance;
                t.sums[1] += r.standard_error;
                t.sums[2] += r.mean_steps;
            }
            if (out.mean) out.mean[linear] = r.mean;
            if (out.variance) out.variance[linear] = r.variance;
            if (out.standard_error) out.standard_error[linear] = r.standard_error;
            if (out.mean_steps) out.mean_steps[linear] = r.mean_steps;
            if (out.location) out.location[linear] = static_cast<unsigned char>(where);
        }
    };

    const double t0 = now_seconds();
    if (threads == 1) {
        worker(0);
    } else {
        std::vector<std::thread> pool;
        for (int tid = 0; tid < threads; ++tid) pool.emplace_back(worker, tid);
        for (auto &th : pool) th.join();
    }
    out.seconds = now_seconds() - t0;

    out.inside_points = out.max_steps_hits = 0;
    out.ambiguous_ray_retries = out.indeterminate_points = 0;
    out.sum_variance = out.sum_standard_error = out.sum_mean_steps = 0.0;
    for (const Tally &t : tallies) {
        out.inside_points += t.inside;
        out.max_steps_hits += t.hits;
        out.ambiguous_ray_retries += t.retries;
        out.indeterminate_points += t.indeterminate;
        out.sum_variance += t.sums[0];
        out.sum_standard_error += t.sums[1];
        out.sum_mean_steps += t.sums[2];
    }
    return 0;
}

}  // namespace wos_ref

// Defines `extern "C" int ref_grid_<name>(const ref_problem*, ref_outputs*)`
// and `extern "C" int ref_registry_<name>(...)` for one equation translation
// unit of the reference.  MAKE2D/MAKE3D build the reference's equation value
// from the problem (alpha, source mode); EPS maps the requested epsilon to the
// one the reference's run_2D/run_3D pass on.
#define WOS_REF_ENTRY(NAME, MAKE2D, MAKE3D, EPS)                                         \
    extern "C" int ref_grid_##NAME(const ref_problem *pb, ref_outputs *out) {            \
        using namespace wos;                                                             \
        const double eps = EPS;                                                          \
        try {                                                                            \
            if (pb->dim == 2) return wos_ref::solve_grid<2>(*pb, MAKE2D, eps, *out);     \
            return wos_ref::solve_grid<3>(*pb, MAKE3D, eps, *out);                       \
        } catch (const std::exception &) {                                               \
            return 1;                                                                    \
        }                                                                                \
    }                                                                                    \
    extern "C" int ref_registry_##NAME(int dim, const char *mesh, const char *output,    \
                                       int Nx, int Ny, int Nz, int N_walks, double eps,  \
                                       int max_steps, int max_ray_attempts,              \
                                       uint64_t seed, double alpha, int source_mode) {   \
        const wos::Equation &e = wos::NAME;                                              \
        auto fn = dim == 2 ? e.run_2D : e.run_3D;                                        \
        return fn(0, 1, mesh, output, Nx, Ny, Nz, N_walks, eps, max_steps,               \
                  max_ray_attempts, seed, alpha,                                         \
                  static_cast<wos::SourceMode>(source_mode));                            \
    }
