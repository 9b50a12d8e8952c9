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

// Kernel-level checks.
cudaError_t launch_prng(const uint64_t *seeds, long long n, int count, uint64_t *out,
                        cudaStream_t stream);
cudaError_t launch_closest64(const SceneView &s, const double *pts, long long n, double *dist,
                             double *nearest, int *boundary_id, cudaStream_t stream);
cudaError_t launch_closest32(const SceneView &s, const WideView &w, const double *pts,
                             long long n, double *dist, double *nearest, int *boundary_id,
                             cudaStream_t stream);

}  // namespace wosb
