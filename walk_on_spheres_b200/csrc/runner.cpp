// Equation registry with the reference's run signature
// (src/equations/equations.hpp:7-31) on top of the C ABI: mesh load, GPU
// sweep, the reference's console diagnostics (include/wos/runner.hpp:28-300)
// and the HDF5 result layout (include/wos/hdf5_io.hpp:15-338).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wos_b200.h"
#include "obj_reader.h"

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int method_from_env() {
    const char *m = std::getenv("WOS_B200_METHOD");
    if (!m) return WOS_METHOD_PLAIN_FP64;
    if (std::strcmp(m, "fast") == 0) return WOS_METHOD_FAST_FP32;
    if (std::strcmp(m, "fast64") == 0) return WOS_METHOD_FAST_FP64;
    return WOS_METHOD_PLAIN_FP64;
}

int device_from_env() {
    const char *d = std::getenv("WOS_B200_DEVICE");
    return d ? std::atoi(d) : 0;
}

// include/wos/runner.hpp:22-308 for one process (size == 1).
int run_equation(int equation, int dim, int rank, int size, const char *mesh_filename,
                 const char *output_filename, int Nx, int Ny, int Nz, int N_walks,
                 double epsilon, int max_steps, int max_ray_attempts, uint64_t seed, double alpha,
                 int source_mode) {
    if (size != 1 || rank != 0) {
        std::fprintf(stderr,
                     "libwos_b200 runs one process per solve; shard grids across GPUs with "
                     "walk_on_spheres_b200.parallel\n");
        return 1;
    }
    // screened_poisson reduces epsilon before the run (src/equations/screened_poisson.cpp:22-38)
    double eps = epsilon;
    if (equation == WOS_EQ_SCREENED_POISSON) {
        const double limited = 0.05 / alpha;
        const double effective = std::min(epsilon, limited);
        if (effective < epsilon) {
            std::printf("Screened stopping distance reduced:\n"
                        "  requested epsilon:       %.12g\n"
                        "  effective epsilon:       %.12g\n"
                        "  alpha * effective eps:   %.12g\n",
                        epsilon, effective, alpha * effective);
        }
        eps = effective;
    }

    std::printf("Reading mesh from disk (%s)...\n", mesh_filename);
    wosb::ObjMesh mesh;
    const std::string err = wosb::read_obj(mesh_filename, mesh);
    if (!err.empty()) {
        std::fprintf(stderr, "%s\n", err.c_str());
        return 1;
    }
    if (mesh.dim != dim) {
        std::fprintf(stderr, "Mesh %s: expected a %dD mesh\n", mesh_filename, dim);
        return 1;
    }
    std::printf("Finished reading. Broadcasting mesh...\n");
    std::printf("Finished broadcasting.\n");

    wos_context *ctx = nullptr;
    if (wos_context_create(device_from_env(), &ctx) != WOS_OK) {
        std::fprintf(stderr, "%s\n", wos_last_global_error());
        return 1;
    }
    struct Guard {
        wos_context *c;
        ~Guard() { wos_context_destroy(c); }
    } guard{ctx};

    std::printf("Building BVH...\n");
    const double t0 = now_s();
    if (wos_set_mesh(ctx, dim, mesh.verts.data(), mesh.n_verts(), mesh.prims.data(),
                     mesh.n_prims(), dim == 2 ? mesh.boundary_ids.data() : nullptr, 0) != WOS_OK) {
        std::fprintf(stderr, "BVH build failed: %s\n", wos_last_error(ctx));
        return 1;
    }
    std::printf("Finished BVH build in %.6f s.\n", now_s() - t0);

    if (dim == 2) Nz = 1;
    wos_grid grid;
    wos_grid_over_mesh(ctx, Nx, Ny, Nz, &grid);
    std::printf("Parallelisation: %d x %d x %d ranks across (Nx=%d, Ny=%d, Nz=%d)\n", 1, 1, 1,
                grid.Nx, grid.Ny, grid.Nz);

    const size_t n = static_cast<size_t>(grid.Nx) * grid.Ny * grid.Nz;
    std::vector<double> mean(n), variance(n), se(n), steps(n);
    std::vector<uint8_t> location(n);
    wos_params p{};
    p.equation = equation;
    p.source_mode = source_mode;
    p.alpha = alpha;
    p.N_walks = N_walks;
    p.epsilon = eps;
    p.max_steps = max_steps;
    p.max_ray_attempts = max_ray_attempts;
    p.seed = seed;
    p.method = method_from_env();
    wos_counters c{};
    std::printf("Beginning walk-on-spheres...\n");
    std::fflush(stdout);
    const double w0 = now_s();
    if (wos_solve_grid(ctx, &p, &grid, mean.data(), variance.data(), se.data(), steps.data(),
                       location.data(), &c) != WOS_OK) {
        std::fprintf(stderr, "walk-on-spheres failed: %s\n", wos_last_error(ctx));
        return 1;
    }
    const double seconds = now_s() - w0;

    if (c.inside_points > 0) {
        const double count = static_cast<double>(c.inside_points);
        std::printf("\nWoS inside-grid averages:\n");
        std::printf("  number of inside points:       %lld\n", c.inside_points);
        std::printf("  average variance:              %.12g\n", c.sum_variance / count);
        std::printf("  average standard error:        %.12g\n", c.sum_standard_error / count);
        std::printf("  average steps per walk:        %.12g\n", c.sum_mean_steps / count);
        std::printf("  paths reaching max steps:      %lld\n", c.max_steps_hits);
        std::printf("\n");
    }
    if (dim == 3) {
        std::printf("3D ray-classification diagnostics:\n");
        std::printf("  ambiguous ray retries:         %lld\n", c.ambiguous_ray_retries);
        std::printf("  indeterminate grid points:     %lld\n\n", c.indeterminate_points);
    }
    std::printf("Finished walk-on-spheres in %.6f s. Writing results...\n", seconds);

    // result file (include/wos/hdf5_io.hpp:15-338); poisson records alpha 0
    // (src/equations/poisson.cpp:126-134)
    const bool source_meta = equation == WOS_EQ_POISSON || equation == WOS_EQ_SCREENED_POISSON;
    const double alpha_meta = equation == WOS_EQ_SCREENED_POISSON ? alpha : 0.0;
    if (wos_write_hdf5(output_filename, &grid, mean.data(), variance.data(), se.data(),
                       steps.data(), location.data(), N_walks, eps, max_steps, c.max_steps_hits,
                       dim == 3, max_ray_attempts, c.ambiguous_ray_retries,
                       c.indeterminate_points, seed, source_meta, alpha_meta,
                       source_mode) != WOS_OK) {
        std::fprintf(stderr, "Failed writing results to %s.\n", output_filename);
        return 1;
    }
    std::printf("Finished writing to %s.\n", output_filename);
    return 0;
}

#define WOS_RUNNERS(NAME, KIND)                                                                  \
    int NAME##_2d(int rank, int size, const char *mesh, const char *out, int Nx, int Ny, int Nz, \
                  int N_walks, double eps, int max_steps, int rays, uint64_t seed, double alpha, \
                  int mode) {                                                                    \
        return run_equation(KIND, 2, rank, size, mesh, out, Nx, Ny, Nz, N_walks, eps,            \
                            max_steps, rays, seed, alpha, mode);                                 \
    }                                                                                            \
    int NAME##_3d(int rank, int size, const char *mesh, const char *out, int Nx, int Ny, int Nz, \
                  int N_walks, double eps, int max_steps, int rays, uint64_t seed, double alpha, \
                  int mode) {                                                                    \
        return run_equation(KIND, 3, rank, size, mesh, out, Nx, Ny, Nz, N_walks, eps,            \
                            max_steps, rays, seed, alpha, mode);                                 \
    }

WOS_RUNNERS(laplace, WOS_EQ_LAPLACE)
WOS_RUNNERS(poisson, WOS_EQ_POISSON)
WOS_RUNNERS(screened_poisson, WOS_EQ_SCREENED_POISSON)
WOS_RUNNERS(helmholtz, WOS_EQ_HELMHOLTZ)

const wos_equation_entry kRegistry[] = {
    {"laplace", laplace_2d, laplace_3d},
    {"poisson", poisson_2d, poisson_3d},
    {"screened_poisson", screened_poisson_2d, screened_poisson_3d},
    {"helmholtz", helmholtz_2d, helmholtz_3d},
};

}  // namespace

extern "C" const wos_equation_entry *wos_equation_registry(int *count) {
    if (count) *count = static_cast<int>(sizeof(kRegistry) / sizeof(kRegistry[0]));
    return kRegistry;
}

extern "C" int wos_peek_mesh_dim(const char *path) {
    std::string err;
    const int d = wosb::peek_obj_dim(path, err);
    if (d == 0) std::fprintf(stderr, "%s\n", err.c_str());
    return d;
}
