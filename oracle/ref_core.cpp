// oracle/_ref entry points around the reference's core functions.
// TEST INFRASTRUCTURE ONLY: compiled with the reference sources
// (src/{bvh,npq,inside,prng,wos,mesh}.cpp, where they lie) by oracle/Makefile.
// Each function calls the reference code and copies its answers out through
// plain C arrays, so golden vectors and parity checks come from the reference
// itself rather than from a restatement.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <type_traits>

#include "ref_driver.hpp"
#include "wos/bessel.hpp"
#include "wos/bvh.hpp"
#include "wos/fastmath.hpp"
#include "wos/hash.hpp"
#include "wos/inside.hpp"
#include "wos/mesh.hpp"
#include "wos/npq.hpp"
#include "wos/poisson.hpp"
#include "wos/prng.hpp"
#include "wos/screened.hpp"
#include "wos/wos.hpp"

using namespace wos;

extern "C" {

// splitmix64 (include/wos/hash.hpp:7-12)
uint64_t ref_splitmix64(uint64_t x) { return splitmix64(x); }

// First n raw outputs of PRNG(seed) (include/wos/prng.hpp:14-24, src/prng.cpp:6-15).
void ref_prng_u64(uint64_t seed, long long n, uint64_t *out) {
    PRNG rng(seed);
    for (long long i = 0; i < n; ++i) out[i] = rng.u64();
}

// First n unit() / unit_open() values (include/wos/prng.hpp:27-37).
void ref_prng_unit(uint64_t seed, long long n, int open, double *out) {
    PRNG rng(seed);
    for (long long i = 0; i < n; ++i) out[i] = open ? rng.unit_open() : rng.unit();
}

// Reference BVH (src/bvh.cpp:174-253) flattened: per node
// {pmin.x, pmin.y, [pmin.z], pmax.x, pmax.y, [pmax.z]} doubles plus
// {prim_count, idx} ints; `prims` is the leaf-order primitive permutation.
// Returns the node count; arrays must hold 2*n_prims-1 nodes.
int ref_build_bvh(const ref_problem *pb, double *node_boxes, int *node_counts, int *node_idx,
                  int *prims) {
    auto export_bvh = [&](auto &bvh, int dim) {
        const int n = static_cast<int>(bvh.nodes.size());
        for (int i = 0; i < n; ++i) {
            const auto &nd = bvh.nodes[i];
            double *b = node_boxes + static_cast<size_t>(2 * dim) * i;
            if constexpr (std::is_same_v<std::decay_t<decltype(nd.bbox.pmin)>, Point3D>) {
                const double v[6] = {nd.bbox.pmin.x, nd.bbox.pmin.y, nd.bbox.pmin.z,
                                     nd.bbox.pmax.x, nd.bbox.pmax.y, nd.bbox.pmax.z};
                std::memcpy(b, v, sizeof(v));
            } else {
                const double v[4] = {nd.bbox.pmin.x, nd.bbox.pmin.y, nd.bbox.pmax.x,
                                     nd.bbox.pmax.y};
                std::memcpy(b, v, sizeof(v));
            }
            node_counts[i] = nd.prim_count;
            node_idx[i] = nd.idx;
        }
        std::memcpy(prims, bvh.prims.data(), bvh.prims.size() * sizeof(int));
        return n;
    };
    if (pb->dim == 2) {
        Mesh<2> m = wos_ref::mesh_from_arrays<2>(*pb);
        auto bvh = build_bvh(m);
        return export_bvh(*bvh, 2);
    }
    Mesh<3> m = wos_ref::mesh_from_arrays<3>(*pb);
    auto bvh = build_bvh(m);
    return export_bvh(*bvh, 3);
}

// Closest-point queries through the reference BVH (src/bvh.cpp:295-387).
// 2D also returns the primitive and boundary ids; 3D writes -1 for both.
void ref_npq(const ref_problem *pb, const double *points, long long n, double *dist,
             double *nearest, int *prim_id, int *boundary_id) {
    if (pb->dim == 2) {
        Mesh<2> m = wos_ref::mesh_from_arrays<2>(*pb);
        auto bvh = build_bvh(m);
        for (long long q = 0; q < n; ++q) {
            const auto r = bvh_npq(*bvh, Point2D{points[2 * q], points[2 * q + 1]});
            dist[q] = r.distance;
            nearest[2 * q] = r.point.x;
            nearest[2 * q + 1] = r.point.y;
            prim_id[q] = r.primitive_id;
            boundary_id[q] = r.boundary_id;
        }
        return;
    }
    Mesh<3> m = wos_ref::mesh_from_arrays<3>(*pb);
    auto bvh = build_bvh(m);
    for (long long q = 0; q < n; ++q) {
        Point3D np{};
        dist[q] = bvh_npq(*bvh, Point3D{points[3 * q], points[3 * q + 1], points[3 * q + 2]}, &np);
        nearest[3 * q] = np.x;
        nearest[3 * q + 1] = np.y;
        nearest[3 * q + 2] = np.z;
        prim_id[q] = -1;
        boundary_id[q] = -1;
    }
}

// 2D winding numbers over every segment (src/inside.cpp:122-137).
void ref_winding_numbers(const ref_problem *pb, const double *points, long long n, int *wn) {
    Mesh<2> m = wos_ref::mesh_from_arrays<2>(*pb);
    for (long long q = 0; q < n; ++q) wn[q] = winding_number(m, Point2D{points[2 * q], points[2 * q + 1]});
}

// 3D classification with explicit per-query INSIDE-stream seeds
// (src/inside.cpp:228-260); returns location codes and ambiguous retries.
void ref_classify_3d(const ref_problem *pb, const double *points, const uint64_t *seeds,
                     long long n, double boundary_distance_tolerance, unsigned char *location,
                     int *retries) {
    Mesh<3> m = wos_ref::mesh_from_arrays<3>(*pb);
    auto bvh = build_bvh(m);
    for (long long q = 0; q < n; ++q) {
        const Point3D p{points[3 * q], points[3 * q + 1], points[3 * q + 2]};
        Point3D np{};
        const double d = bvh_npq(*bvh, p, &np);
        PRNG rng(seeds[q]);
        const PointClassification c =
            classify_point(*bvh, p, d, boundary_distance_tolerance, pb->max_ray_attempts, rng);
        location[q] = static_cast<unsigned char>(c.location);
        retries[q] = c.ambiguous_ray_retries;
    }
}

// Scaled Bessel functions and their logs (include/wos/bessel.hpp:39-87):
// out[4*i + {0,1,2,3}] = i0_scaled, k0_scaled, log_i0, log_k0 of x[i].
void ref_bessel(const double *x, long long n, double *out) {
    for (long long i = 0; i < n; ++i) {
        out[4 * i + 0] = i0_scaled(x[i]);
        out[4 * i + 1] = k0_scaled(x[i]);
        out[4 * i + 2] = log_i0(x[i]);
        out[4 * i + 3] = log_k0(x[i]);
    }
}

// Series J0 / Y0 (include/wos/fastmath.hpp:15-50).
void ref_j0y0(const double *x, long long n, double *j0, double *y0) {
    for (long long i = 0; i < n; ++i) {
        j0[i] = bessel_J0(x[i]);
        y0[i] = bessel_Y0(x[i]);
    }
}

// Screened-Poisson kernels (include/wos/screened.hpp:14-97):
// out[6*i + ...] = weight_2d, green_2d(r), mass_2d, weight_3d, green_3d(r), mass_3d
// for (alpha, radius R, distance r).
void ref_screened_kernels(const double *alpha, const double *R, const double *r, long long n,
                          double *out) {
    for (long long i = 0; i < n; ++i) {
        out[6 * i + 0] = screened::weight_2d(alpha[i], R[i]);
        out[6 * i + 1] = screened::green_2d(alpha[i], R[i], r[i]);
        out[6 * i + 2] = screened::mass_2d(alpha[i], R[i]);
        out[6 * i + 3] = screened::weight_3d(alpha[i], R[i]);
        out[6 * i + 4] = screened::green_3d(alpha[i], R[i], r[i]);
        out[6 * i + 5] = screened::mass_3d(alpha[i], R[i]);
    }
}

// Screened radius samplers (include/wos/screened.hpp:105-156): n draws from
// one PRNG(seed); also returns the raw u64 count consumed per draw.
void ref_screened_samples(int dim, double alpha, double R, uint64_t seed, long long n,
                          double *out) {
    PRNG rng(seed);
    for (long long i = 0; i < n; ++i) {
        out[i] = dim == 2 ? screened::sample_radius_2d(alpha, R, rng)
                          : screened::sample_radius_3d(alpha, R, rng);
    }
}

// Poisson Green kernels and radius samplers (include/wos/poisson.hpp:12-51).
void ref_poisson_green(int dim, double R, const double *r, long long n, uint64_t seed,
                       double *green, double *mass, double *samples) {
    PRNG rng(seed);
    for (long long i = 0; i < n; ++i) {
        green[i] = dim == 2 ? poisson_green::green_2d(R, r[i]) : poisson_green::green_3d(R, r[i]);
        mass[i] = dim == 2 ? poisson_green::mass_2d(R) : poisson_green::mass_3d(R);
        samples[i] = dim == 2 ? poisson_green::sample_radius_2d(R, rng)
                              : poisson_green::sample_radius_3d(R, rng);
    }
}

// Sphere steps and ball samples (src/wos.cpp:9-56) from one PRNG(seed).
void ref_steps(int dim, const double *centre, double radius, uint64_t seed, long long n,
               double *steps, double *balls) {
    PRNG rng(seed);
    for (long long i = 0; i < n; ++i) {
        if (dim == 2) {
            Sphere2D s{Point2D{centre[0], centre[1]}, radius};
            const Point2D a = step(s, rng);
            const Point2D b = sphere_sample(s, rng);
            steps[2 * i] = a.x;
            steps[2 * i + 1] = a.y;
            balls[2 * i] = b.x;
            balls[2 * i + 1] = b.y;
        } else {
            Sphere3D s{Point3D{centre[0], centre[1], centre[2]}, radius};
            const Point3D a = step(s, rng);
            const Point3D b = sphere_sample(s, rng);
            steps[3 * i] = a.x;
            steps[3 * i + 1] = a.y;
            steps[3 * i + 2] = a.z;
            balls[3 * i] = b.x;
            balls[3 * i + 1] = b.y;
            balls[3 * i + 2] = b.z;
        }
    }
}

// OBJ loader (src/mesh.cpp:51-270): dimension, counts, then arrays.
// Returns 0 on success and 1 on a reference mesh error (message copied).
int ref_load_mesh(const char *path, int *dim, int *n_verts, int *n_prims, double *verts,
                  int *prims, int *boundary_ids, char *error, int error_capacity) {
    try {
        const int d = peek_mesh_dim(path);
        *dim = d;
        if (d == 2) {
            Mesh<2> m = load_mesh<2>(path);
            *n_verts = m.n_verts();
            *n_prims = m.n_prims();
            if (verts) {
                for (int v = 0; v < m.n_verts(); ++v) {
                    verts[2 * v] = m.verts[v].x;
                    verts[2 * v + 1] = m.verts[v].y;
                }
                std::memcpy(prims, m.prims.data(), m.prims.size() * sizeof(int));
                std::memcpy(boundary_ids, m.boundary_ids.data(),
                            m.boundary_ids.size() * sizeof(int));
            }
        } else {
            Mesh<3> m = load_mesh<3>(path);
            *n_verts = m.n_verts();
            *n_prims = m.n_prims();
            if (verts) {
                for (int v = 0; v < m.n_verts(); ++v) {
                    verts[3 * v] = m.verts[v].x;
                    verts[3 * v + 1] = m.verts[v].y;
                    verts[3 * v + 2] = m.verts[v].z;
                }
                std::memcpy(prims, m.prims.data(), m.prims.size() * sizeof(int));
            }
        }
        return 0;
    } catch (const std::exception &e) {
        if (error && error_capacity > 0) {
            std::strncpy(error, e.what(), static_cast<size_t>(error_capacity) - 1);
            error[error_capacity - 1] = '\0';
        }
        return 1;
    }
}

}  // extern "C"
