// Equation registry with the reference's run signature
// (src/equations/equations.hpp:7-31) on top of the C ABI: mesh load, GPU
// sweep, the reference's console diagnostics (include/wos/runner.hpp:28-300)
// and the HDF5 result layout (include/wos/hdf5_io.hpp:15-338).  With
// size > 1 every rank solves the reference's Cartesian block of the grid
// (runner.hpp:90-134) on its own GPU and the ranks meet only through the
// caller's collectives (wos_set_collectives): counter reductions
// (runner.hpp:240-263) and the parallel result write (hdf5_io.hpp:51-171).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

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

// GPU of a rank: WOS_B200_DEVICE when set, else rank modulo the device count.
int device_for_rank(int rank) {
    if (const char *d = std::getenv("WOS_B200_DEVICE")) return std::atoi(d);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) return 0;
    return rank % count;
}

std::mutex g_coll_lock;
wos_collectives g_coll{};
bool g_coll_set = false;

wos_collectives collectives() {
    std::lock_guard<std::mutex> lock(g_coll_lock);
    return g_coll_set ? g_coll : wos_collectives{};
}

// MPI_Dims_create for 3 dimensions: the free (zero) entries of dims get a
// factorisation of size / (product of the fixed entries) that is as balanced
// as possible (smallest largest-to-smallest spread, then the smallest
// largest factor), in non-increasing order.  Returns false if the fixed
// entries do not divide size.
bool dims_create(int size, int dims[3]) {
    int fixed = 1, nfree = 0;
    for (int k = 0; k < 3; ++k) {
        if (dims[k] < 0) return false;
        if (dims[k] > 0) fixed *= dims[k];
        else ++nfree;
    }
    if (fixed <= 0 || size % fixed != 0) return false;
    const int rest = size / fixed;
    if (nfree == 0) return rest == 1;
    int best[3] = {rest, 1, 1};
    long long best_spread = -1, best_max = 0;
    // factorisations a >= b >= c with a * b * c = rest (unused slots stay 1)
    for (int a = 1; a <= rest; ++a) {
        if (rest % a) continue;
        const int ra = rest / a;
        for (int b = 1; b <= a && b <= ra; ++b) {
            if (ra % b) continue;
            const int c = ra / b;
            if (c > b) continue;
            if (nfree < 3 && c != 1) continue;
            if (nfree < 2 && b != 1) continue;
            int f[3] = {a, b, c};
            const int lo = f[nfree - 1];
            const long long spread = static_cast<long long>(a) - lo;
            if (best_spread < 0 || spread < best_spread ||
                (spread == best_spread && a < best_max)) {
                best_spread = spread;
                best_max = a;
                best[0] = a;
                best[1] = b;
                best[2] = c;
            }
        }
    }
    int next = 0;
    for (int k = 0; k < 3; ++k) {
        if (dims[k] == 0) dims[k] = best[next++];
    }
    return true;
}

// The reference's rank block (include/wos/runner.hpp:90-134); on failure
// returns the reference's message (empty on success).
std::string rank_block(int dim, int Nx, int Ny, int Nz, int rank, int size, int dims[3],
                       int offset[3], int count[3]) {
    if (dim == 2) Nz = 1;
    const long long points = static_cast<long long>(Nx) * Ny * Nz;
    char msg[256];
    if (size > points) {
        std::snprintf(msg, sizeof msg,
                      "Cannot assign %d MPI ranks to only %lld grid points; "
                      "use fewer ranks or a larger grid", size, points);
        return msg;
    }
    dims[0] = Nx == 1 ? 1 : 0;
    dims[1] = Ny == 1 ? 1 : 0;
    dims[2] = (dim == 2 || Nz == 1) ? 1 : 0;
    const wos_collectives c = collectives();
    bool ok;
    if (c.dims_create) {
        ok = c.dims_create(size, dims, c.user) == 0;
    } else {
        ok = dims_create(size, dims);
    }
    if (!ok) return "MPI_Dims_create failed";
    if (dims[0] > Nx || dims[1] > Ny || dims[2] > Nz) {
        std::snprintf(msg, sizeof msg,
                      "MPI decomposition %d x %d x %d exceeds grid %d x %d x %d; "
                      "use fewer ranks or a larger grid", dims[0], dims[1], dims[2], Nx, Ny, Nz);
        return msg;
    }
    const int c3[3] = {rank / (dims[1] * dims[2]), (rank / dims[2]) % dims[1], rank % dims[2]};
    const int n3[3] = {Nx, Ny, Nz};
    for (int k = 0; k < 3; ++k) {
        offset[k] = static_cast<int>((static_cast<long long>(n3[k]) * c3[k]) / dims[k]);
        count[k] = static_cast<int>((static_cast<long long>(n3[k]) * (c3[k] + 1)) / dims[k]) -
                   offset[k];
    }
    return std::string();
}

// Every rank's flag: true if any rank passed true (an all-reduce max).
bool any_rank(const wos_collectives &c, bool mine) {
    double v = mine ? 1.0 : 0.0;
    if (c.allreduce(&v, 1, WOS_REDUCE_MAX, c.user) != 0) return true;
    return v != 0.0;
}

// include/wos/runner.hpp:22-308.  size == 1: the whole grid on one GPU.
// size > 1: this rank's block of the grid (runner.hpp:90-134) on its GPU,
// the counters reduced over the ranks with the caller's collectives, rank 0
// creating the result file and every rank writing its block into it.
int run_equation(int equation, int dim, int rank, int size, const char *mesh_filename,
                 const char *output_filename, int Nx, int Ny, int Nz, int N_walks,
                 double epsilon, int max_steps, int max_ray_attempts, uint64_t seed, double alpha,
                 int source_mode) {
    const bool multi = size > 1;
    const wos_collectives coll = collectives();
    if (size < 1 || rank < 0 || rank >= size) {
        std::fprintf(stderr, "invalid MPI rank %d of %d\n", rank, size);
        return 1;
    }
    if (multi && (!coll.barrier || !coll.allreduce)) {
        if (rank == 0) {
            std::fprintf(stderr,
                         "libwos_b200: %d ranks need the caller's collectives "
                         "(wos_set_collectives)\n", size);
        }
        return 1;
    }
    const bool root = rank == 0;
    // screened_poisson reduces epsilon before the run (src/equations/screened_poisson.cpp:22-38)
    double eps = epsilon;
    if (equation == WOS_EQ_SCREENED_POISSON) {
        const double limited = 0.05 / alpha;
        const double effective = std::min(epsilon, limited);
        if (effective < epsilon && root) {
            std::printf("Screened stopping distance reduced:\n"
                        "  requested epsilon:       %.12g\n"
                        "  effective epsilon:       %.12g\n"
                        "  alpha * effective eps:   %.12g\n",
                        epsilon, effective, alpha * effective);
        }
        eps = effective;
    }

    // every rank reads the mesh (the reference reads on rank 0 and broadcasts)
    if (root) std::printf("Reading mesh from disk (%s)...\n", mesh_filename);
    wosb::ObjMesh mesh;
    std::string err = wosb::read_obj(mesh_filename, mesh);
    if (err.empty() && mesh.dim != dim) {
        err = std::string("Mesh ") + mesh_filename + ": expected a " + std::to_string(dim) +
              "D mesh";
    }
    if (!err.empty() && (root || multi)) std::fprintf(stderr, "%s\n", err.c_str());
    if (multi ? any_rank(coll, !err.empty()) : !err.empty()) return 1;
    if (root) {
        std::printf("Finished reading. Broadcasting mesh...\n");
        std::printf("Finished broadcasting.\n");
    }

    // the rank's block, checked before any GPU work
    if (dim == 2) Nz = 1;
    int dims[3] = {1, 1, 1}, off[3] = {0, 0, 0}, cnt[3] = {Nx, Ny, Nz};
    if (multi) {
        err = rank_block(dim, Nx, Ny, Nz, rank, size, dims, off, cnt);
        if (!err.empty()) {
            if (root) std::fprintf(stderr, "%s\n", err.c_str());
            return 1;  // every rank computes the same verdict
        }
    }

    wos_context *ctx = nullptr;
    const int device = multi ? device_for_rank(rank) : device_for_rank(0);
    const bool ctx_failed = wos_context_create(device, &ctx) != WOS_OK;
    if (ctx_failed) std::fprintf(stderr, "%s\n", wos_last_global_error());
    struct Guard {
        wos_context *c;
        ~Guard() {
            if (c) wos_context_destroy(c);
        }
    } guard{ctx};
    if (multi ? any_rank(coll, ctx_failed) : ctx_failed) return 1;

    if (root) std::printf("Building BVH...\n");
    const double t0 = now_s();
    const bool bvh_failed =
        wos_set_mesh(ctx, dim, mesh.verts.data(), mesh.n_verts(), mesh.prims.data(),
                     mesh.n_prims(), dim == 2 ? mesh.boundary_ids.data() : nullptr, 0) != WOS_OK;
    if (bvh_failed) std::fprintf(stderr, "BVH build failed: %s\n", wos_last_error(ctx));
    if (multi ? any_rank(coll, bvh_failed) : bvh_failed) return 1;
    if (root) {
        if (multi) {
            std::printf("Finished BVH build in %.6f s. Broadcasting BVH...\n", now_s() - t0);
        } else {
            std::printf("Finished BVH build in %.6f s.\n", now_s() - t0);
        }
    }
    if (multi) {
        // every rank built its own trees; the "broadcast" is the wait for all
        const double b0 = now_s();
        coll.barrier(coll.user);
        if (root) std::printf("Finished BVH broadcast in %.6f s.\n", now_s() - b0);
    }

    wos_grid grid;
    wos_grid_over_mesh(ctx, Nx, Ny, Nz, &grid);
    if (root) {
        std::printf("Parallelisation: %d x %d x %d ranks across (Nx=%d, Ny=%d, Nz=%d)\n",
                    dims[0], dims[1], dims[2], grid.Nx, grid.Ny, grid.Nz);
    }

    const size_t n = static_cast<size_t>(cnt[0]) * cnt[1] * cnt[2];
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
    if (root) std::printf("Beginning walk-on-spheres...\n");
    std::fflush(stdout);
    if (multi) coll.barrier(coll.user);
    const double w0 = now_s();
    bool solve_failed;
    if (!multi) {
        solve_failed = wos_solve_grid(ctx, &p, &grid, mean.data(), variance.data(), se.data(),
                                      steps.data(), location.data(), &c) != WOS_OK;
    } else {
        // the block's points in C order, seeded by their global linear index
        // (runner.hpp:157-168)
        std::vector<double> pts(n * dim);
        std::vector<uint64_t> idx(n);
        const double lo[3] = {grid.xmin, grid.ymin, grid.zmin};
        const double hi[3] = {grid.xmax, grid.ymax, grid.zmax};
        const int N3[3] = {grid.Nx, grid.Ny, grid.Nz};
        size_t t = 0;
        for (int i = 0; i < cnt[0]; ++i) {
            for (int j = 0; j < cnt[1]; ++j) {
                for (int k = 0; k < cnt[2]; ++k, ++t) {
                    const int g3[3] = {off[0] + i, off[1] + j, off[2] + k};
                    for (int d = 0; d < dim; ++d) {
                        pts[t * dim + d] =
                            N3[d] > 1 ? lo[d] + (hi[d] - lo[d]) * static_cast<double>(g3[d]) /
                                                    static_cast<double>(N3[d] - 1)
                                      : lo[d];
                    }
                    idx[t] = (static_cast<uint64_t>(g3[0]) * static_cast<uint64_t>(grid.Ny) +
                              static_cast<uint64_t>(g3[1])) *
                                 static_cast<uint64_t>(grid.Nz) +
                             static_cast<uint64_t>(g3[2]);
                }
            }
        }
        solve_failed = wos_solve_points(ctx, &p, pts.data(), idx.data(),
                                        static_cast<long long>(n), mean.data(), variance.data(),
                                        se.data(), steps.data(), location.data(), &c) != WOS_OK;
        // the block's diagnostics in the reference's loop order
        c.inside_points = 0;
        c.sum_variance = c.sum_standard_error = c.sum_mean_steps = 0.0;
        for (size_t q = 0; q < n && !solve_failed; ++q) {
            if (location[q] != WOS_INSIDE) continue;
            ++c.inside_points;
            c.sum_variance += variance[q];
            c.sum_standard_error += se[q];
            c.sum_mean_steps += steps[q];
        }
    }
    if (solve_failed) std::fprintf(stderr, "walk-on-spheres failed: %s\n", wos_last_error(ctx));
    if (multi ? any_rank(coll, solve_failed) : solve_failed) return 1;
    double seconds = now_s() - w0;
    if (multi) {
        // runner.hpp:240-263: maximum time, summed counters
        double sums[7] = {static_cast<double>(c.inside_points),
                          static_cast<double>(c.max_steps_hits),
                          static_cast<double>(c.ambiguous_ray_retries),
                          static_cast<double>(c.indeterminate_points),
                          c.sum_variance, c.sum_standard_error, c.sum_mean_steps};
        if (coll.allreduce(&seconds, 1, WOS_REDUCE_MAX, coll.user) != 0 ||
            coll.allreduce(sums, 7, WOS_REDUCE_SUM, coll.user) != 0) {
            std::fprintf(stderr, "libwos_b200: a collective failed\n");
            return 1;
        }
        c.inside_points = static_cast<long long>(sums[0]);
        c.max_steps_hits = static_cast<long long>(sums[1]);
        c.ambiguous_ray_retries = static_cast<long long>(sums[2]);
        c.indeterminate_points = static_cast<long long>(sums[3]);
        c.sum_variance = sums[4];
        c.sum_standard_error = sums[5];
        c.sum_mean_steps = sums[6];
    }

    if (root && c.inside_points > 0) {
        const double count = static_cast<double>(c.inside_points);
        std::printf("\nWoS inside-grid averages:\n");
        std::printf("  number of inside points:       %lld\n", c.inside_points);
        std::printf("  average variance:              %.12g\n", c.sum_variance / count);
        std::printf("  average standard error:        %.12g\n", c.sum_standard_error / count);
        std::printf("  average steps per walk:        %.12g\n", c.sum_mean_steps / count);
        std::printf("  paths reaching max steps:      %lld\n", c.max_steps_hits);
        std::printf("\n");
    }
    if (root && dim == 3) {
        std::printf("3D ray-classification diagnostics:\n");
        std::printf("  ambiguous ray retries:         %lld\n", c.ambiguous_ray_retries);
        std::printf("  indeterminate grid points:     %lld\n\n", c.indeterminate_points);
    }
    if (root) std::printf("Finished walk-on-spheres in %.6f s. Writing results...\n", seconds);

    // result file (include/wos/hdf5_io.hpp:15-338); poisson records alpha 0
    // (src/equations/poisson.cpp:126-134)
    const bool source_meta = equation == WOS_EQ_POISSON || equation == WOS_EQ_SCREENED_POISSON;
    const double alpha_meta = equation == WOS_EQ_SCREENED_POISSON ? alpha : 0.0;
    bool write_failed;
    if (!multi) {
        write_failed = wos_write_hdf5(output_filename, &grid, mean.data(), variance.data(),
                                      se.data(), steps.data(), location.data(), N_walks, eps,
                                      max_steps, c.max_steps_hits, dim == 3, max_ray_attempts,
                                      c.ambiguous_ray_retries, c.indeterminate_points, seed,
                                      source_meta, alpha_meta, source_mode) != WOS_OK;
    } else {
        // rank 0 writes coordinates and metadata; every rank its block of the
        // five fields (hdf5_io.hpp:51-171)
        wos_h5_layout lay{};
        bool created = true;
        if (root) {
            created = wos_hdf5_create(output_filename, &grid, N_walks, eps, max_steps,
                                      c.max_steps_hits, dim == 3, max_ray_attempts,
                                      c.ambiguous_ray_retries, c.indeterminate_points, seed,
                                      source_meta, alpha_meta, source_mode, &lay) == WOS_OK;
        }
        write_failed = any_rank(coll, !created);
        if (!write_failed) {
            const bool ok =
                wos_hdf5_layout(&grid, dim == 3, source_meta, &lay) == WOS_OK &&
                wos_hdf5_write_block(output_filename, &lay, &grid, off, cnt, mean.data(),
                                     variance.data(), se.data(), steps.data(),
                                     location.data()) == WOS_OK;
            write_failed = any_rank(coll, !ok);
        }
    }
    if (write_failed) {
        if (root) std::fprintf(stderr, "Failed writing results to %s.\n", output_filename);
        return 1;
    }
    if (root) std::printf("Finished writing to %s.\n", output_filename);
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

extern "C" int wos_set_collectives(const wos_collectives *c) {
    std::lock_guard<std::mutex> lock(g_coll_lock);
    if (!c) {
        g_coll = wos_collectives{};
        g_coll_set = false;
        return WOS_OK;
    }
    if (!c->barrier || !c->allreduce) return WOS_ERR_INVALID;
    g_coll = *c;
    g_coll_set = true;
    return WOS_OK;
}

extern "C" int wos_rank_block(int dim, int Nx, int Ny, int Nz, int rank, int size, int dims[3],
                              int offset[3], int count[3], char *error, int error_capacity) {
    if ((dim != 2 && dim != 3) || Nx < 1 || Ny < 1 || (dim == 3 && Nz < 1) || size < 1 ||
        rank < 0 || rank >= size || !dims || !offset || !count) {
        return WOS_ERR_INVALID;
    }
    const std::string err = rank_block(dim, Nx, Ny, Nz, rank, size, dims, offset, count);
    if (error && error_capacity > 0) {
        std::snprintf(error, static_cast<size_t>(error_capacity), "%s", err.c_str());
    }
    return err.empty() ? WOS_OK : WOS_ERR_INVALID;
}

extern "C" int wos_peek_mesh_dim(const char *path) {
    std::string err;
    const int d = wosb::peek_obj_dim(path, err);
    if (d == 0) std::fprintf(stderr, "%s\n", err.c_str());
    return d;
}
