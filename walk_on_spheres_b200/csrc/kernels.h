// Host-side launchers of the walk-on-spheres kernels (internal to
// libwos_b200.so; the public boundary is include/wos_b200.h).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "device/common.cuh"

namespace wosb {

// Start points, classification and boundary values for every point of `ps`
// (include/wos/runner.hpp:170-206).  Writes location, start records and the
// fields of non-inside points.
cudaError_t launch_classify(const SceneView &s, const PointSet &ps, uint64_t seed,
                            int max_ray_attempts, double boundary_tolerance, EqDesc eq,
                            Fields out, uint8_t *location, StartRecord *start,
                            DeviceCounters *counters, cudaStream_t stream);

// PLAIN_FP64: every walk of every inside point on the point's reference
// xoshiro256++ streams, in the reference order (include/wos/wos.hpp:54-191).
cudaError_t launch_walk_plain(const SceneView &s, const PointSet &ps, uint64_t seed, EqDesc eq,
                              int n_walks, double epsilon, int max_steps,
                              const uint8_t *location, const StartRecord *start, Fields out,
                              DeviceCounters *counters, cudaStream_t stream);

// Work decomposition of the fast walks: task t covers walks
// [c*chunk, min(N, (c+1)*chunk)) of point p, t = p*chunks + c.
struct FastPlan {
    int chunk;            // walks per task
    int chunks;           // tasks per point
    long long n_tasks;    // points * chunks
    int blocks;           // persistent grid size
    int threads;          // block size
    bool stage_scene;     // copy the wide FP32 boxes into shared memory
    bool stage_prims;     // ... and the wide FP32 primitives
    int smem_bytes;
};

// Per-task partial statistics written by the fast kernel.
struct TaskPartial {
    double n;        // walks
    double mean;     // Welford mean
    double m2;       // Welford M2
    double steps;    // sum of steps
    unsigned int hits;
    unsigned int pad;
};

// FAST_FP32 (precision 32) / FAST_FP64 (precision 64) walks over all tasks,
// then the per-point merge into the output fields.
cudaError_t launch_walk_fast(const SceneView &s, const WideView &w, const PointSet &ps,
                             uint64_t seed, EqDesc eq,
                             int n_walks, double epsilon, int max_steps, double shell_delta,
                             int precision, const FastPlan &plan, const uint8_t *location,
                             const StartRecord *start, TaskPartial *partials,
                             unsigned long long *queue, Fields out, DeviceCounters *counters,
                             cudaStream_t stream, cudaEvent_t after_walk = nullptr);

FastPlan plan_fast(const SceneView &s, const WideView &w, long long n_points, int n_walks,
                   int precision, int device_sms, size_t smem_optin);

// Gaussian heat source -Δu = Q exp(-|x - x0|^2 / sigma^2) with per-vertex
// Dirichlet data (kernels_adjoint.cu).
struct HeatDesc {
    int mode;               // kUniform / kGreen source sampling
    double Q, x0[3], sigma;
    const double *g;        // per-vertex boundary values (null: all zero)
    const int *slot_verts;  // per binary-tree slot: the primitive's dim vertex ids
    int adjoint;            // 0: forward walks; 1: replay accumulating derivatives
    const double *grad_u;   // adjoint: weight of each point's value (dL/du_p)
    double *grad_g;         // adjoint: dL/dg_v accumulators (zeroed by the caller)
};

// Per-task partial of the heat walks: value statistics as TaskPartial plus
// sums and sums of squares of the five source-parameter derivatives
// (Q, x0.x, x0.y, x0.z, sigma) in adjoint mode.
struct HeatPartial {
    double n, mean, m2, steps;
    double jsum[5];
    double jsq[5];
    unsigned int hits;
    unsigned int pad;
};

struct HeatOut {
    Fields f;
    double *jac;          // adjoint: n * 5 walk means of du_p/dtheta (optional)
    double *jac_se;       // adjoint: their standard errors (optional)
    double *grad_source;  // adjoint: 5 accumulators of sum_p grad_u[p] du_p/dtheta (zeroed)
};

cudaError_t launch_heat(const SceneView &s, const WideView &w, const PointSet &ps,
                        uint64_t seed, const HeatDesc &h, int n_walks, double epsilon,
                        int max_steps, double shell_delta, int precision, const FastPlan &plan,
                        const uint8_t *location, const StartRecord *start, HeatPartial *partials,
                        unsigned long long *queue, HeatOut out, DeviceCounters *counters,
                        cudaStream_t stream, cudaEvent_t after_walk = nullptr);

// Kernel-level checks.
cudaError_t launch_prng(const uint64_t *seeds, long long n, int count, uint64_t *out,
                        cudaStream_t stream);
cudaError_t launch_closest64(const SceneView &s, const double *pts, long long n, double *dist,
                             double *nearest, int *boundary_id, cudaStream_t stream);
cudaError_t launch_closest32(const SceneView &s, const WideView &w, const double *pts,
                             long long n, double *dist, double *nearest, int *boundary_id,
                             cudaStream_t stream);

}  // namespace wosb
