// Shared device-side types of the walk-on-spheres kernels.
#pragma once
#include <cstdint>

#include "equations.cuh"
#include "prng.cuh"
#include "scene.cuh"
#include "wide.cuh"

namespace wosb {

// Where the query points come from: a Cartesian grid (include/wos/grid.hpp,
// coordinates min + (max-min)*i/(N-1)) or an explicit list of points.
struct PointSet {
    int dim;
    int Nx, Ny, Nz;
    double lo[3], hi[3];
    const double *coords;         // explicit points (n * dim) or null for the grid
    const uint64_t *index;        // seeding index per point (null: the point's position)
    long long n;
};

__device__ __forceinline__ double grid_coordinate(double lo, double hi, int i, int n) {
    return n > 1 ? lo + (hi - lo) * static_cast<double>(i) / static_cast<double>(n - 1) : lo;
}

// Coordinates and seeding index of point t (include/wos/runner.hpp:157-168).
__device__ __forceinline__ void point_at(const PointSet &ps, long long t, double &x, double &y,
                                         double &z, uint64_t &linear) {
    if (ps.coords) {
        x = ps.coords[ps.dim * t];
        y = ps.coords[ps.dim * t + 1];
        z = ps.dim == 3 ? ps.coords[ps.dim * t + 2] : 0.0;
        linear = ps.index ? ps.index[t] : static_cast<uint64_t>(t);
        return;
    }
    const long long plane = static_cast<long long>(ps.Ny) * ps.Nz;
    const int i = static_cast<int>(t / plane);
    const int j = static_cast<int>((t / ps.Nz) % ps.Ny);
    const int k = static_cast<int>(t % ps.Nz);
    x = grid_coordinate(ps.lo[0], ps.hi[0], i, ps.Nx);
    y = grid_coordinate(ps.lo[1], ps.hi[1], j, ps.Ny);
    z = ps.dim == 3 ? grid_coordinate(ps.lo[2], ps.hi[2], k, ps.Nz) : 0.0;
    linear = ps.index ? ps.index[t] : static_cast<uint64_t>(t);
}

// Start point of a point (include/wos/wos.hpp:35-52): nearest boundary point,
// its distance and (2D) boundary id, plus the binary-tree slot of the nearest
// primitive (for per-vertex boundary data).  Written by the classification
// kernel.
struct StartRecord {
    double radius;
    double nx, ny, nz;
    int boundary_id;
    int slot;
};

// Equation selection for runtime dispatch.
struct EqDesc {
    int kind;    // kLaplace ... kHelmholtz, kTransient, kPlate (2D only)
    int mode;    // kUniform / kGreen / kMis (kPlate only)
    double alpha;
    const TransientDesc *tr;  // kTransient: the step's descriptor (device memory)
    const PlateDesc *pl;      // kPlate: the plate's descriptor (HOST memory, copied
                              // into the kernel's equation at launch)
};

// Per-solve device counters (include/wos/runner.hpp:147-151).
struct DeviceCounters {
    unsigned long long max_steps_hits;
    unsigned long long ambiguous_ray_retries;
    unsigned long long indeterminate_points;
    unsigned long long total_steps;
    unsigned long long total_walks;
    unsigned int error_flags;   // bit 0: a rejection sampler hit its cap
    unsigned int pad;
    // closest-point queries that traversed the BVH (FAST_FP32 lattice steps
    // take their radius without one; every PLAIN_FP64 / FAST_FP64 step is one)
    unsigned long long exact_queries;
};

// error_flags bits: a bounded rejection loop ran out; a walk reached a state
// the kernels must not act on (a closest-point query without a primitive)
enum : unsigned { kErrRejectionCap = 1u, kErrBadState = 2u };

// Output fields (any may be null).
struct Fields {
    double *mean;
    double *variance;
    double *standard_error;
    double *mean_steps;
    uint8_t *location;
};

// Boundary value g(p) of an equation at a boundary point (runtime dispatch),
// used for boundary grid points (include/wos/runner.hpp:196-206).
template <int DIM>
__device__ __forceinline__ double boundary_value(const EqDesc &e, V3<double> p, int bid) {
    switch (e.kind) {
        case kLaplace: return Laplace<DIM>{}.boundary(p, bid);
        case kPoisson: return Poisson<DIM>{e.mode, e.alpha}.boundary(p, bid);
        case kScreened: return Screened<DIM>{e.mode, e.alpha}.boundary(p, bid);
        case kTransient:
        case kPlate: return 0.0;
        default: return Helmholtz<DIM>{}.boundary(p, bid);
    }
}

}  // namespace wosb
