// Host-side launchers of the walk-on-spheres kernels (internal to
// libwos_b200.so; the public boundary is include/wos_b200.h).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "device/common.cuh"

namespace wosb {

// Absolute error margin of FP32 primitive distances in a scene with this
// bounding box: a few ulps of its largest coordinate or extent.
inline float fp32_distance_margin(const double bbox[6], int dim) {
    double ext = 0.0, mag = 0.0;
    for (int k = 0; k < dim; ++k) {
        const double lo = bbox[2 * k], hi = bbox[2 * k + 1];
        ext = ext > hi - lo ? ext : hi - lo;
        mag = mag > (lo < 0 ? -lo : lo) ? mag : (lo < 0 ? -lo : lo);
        mag = mag > (hi < 0 ? -hi : hi) ? mag : (hi < 0 ? -hi : hi);
    }
    return static_cast<float>(4e-6 * (mag > ext ? mag : ext));
}

// FAST_FP32 start radii.  A walk only needs its start radius to be a lower
// bound of the boundary distance; the exact FP64 distance matters only where
// it decides something: the boundary class (radius <= boundary tolerance)
// and a start inside the epsilon shell.  With `fast` set, each point first
// gets a conservative FP32 bound from the wide tree (the lattice build's
// query, shrunk by 2^-10 and `margin`); points whose bound exceeds
// `exact_below` (the larger of epsilon and the boundary tolerance) keep it
// as their start radius and skip the exact query, whose cost on
// sphere-like meshes grows with the number of nearly equidistant
// primitives.  Locations and which walks start inside the shell are the
// same as with exact radii.
struct FastStart {
    bool on = false;
    WideView w{};
    double exact_below = 0.0;
    float margin = 0.0f;
};

// Start points, classification and boundary values for every point of `ps`
// (include/wos/runner.hpp:170-206).  Writes location, start records and the
// fields of non-inside points.
cudaError_t launch_classify(const SceneView &s, const PointSet &ps, uint64_t seed,
                            int max_ray_attempts, double boundary_tolerance, EqDesc eq,
                            Fields out, uint8_t *location, StartRecord *start,
                            DeviceCounters *counters, cudaStream_t stream,
                            const FastStart &fast = FastStart{});

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
    double queries;  // closest-point queries that traversed the BVH
    unsigned int hits;
    unsigned int pad;
};

// Arguments of the fast walk kernel for one solve.
struct FastArgs {
    SceneView s;
    WideView w;
    PointSet ps;
    uint64_t seed;
    int n_walks;
    double eps;
    int max_steps;
    double shell_delta;
    float keep;     // (1 - tau)^2: approximate pruning bound of the FP32 query
    float shrink;   // 1 - tau: conservative radius factor
    float exact2;   // below this squared distance the FP32 query prunes exactly
    float shell2;   // (eps + shell_delta)^2: FP32 radius inside the epsilon shell
    float list_t;   // nodes with lattice value <= list_t answer queries from their
                    // candidate list (near_list_threshold; -1: no lists)
    int chunk;
    int chunks;
    long long n_tasks;
    int stage;
    int stage_box;   // floats of the wide box arrays staged in shared memory
    int stage_prim;  // floats of the wide primitive arrays staged (0: read from global)
    const uint8_t *location;
    const StartRecord *start;
    TaskPartial *partials;
    unsigned long long *queue;
    DeviceCounters *ctr;
};

// Fills the walk arguments of one solve (pruning bounds from epsilon and the
// shell margin); the scene is never staged.
FastArgs make_fast_args(const SceneView &s, const WideView &w, const PointSet &ps, uint64_t seed,
                        int n_walks, double epsilon, int max_steps, double shell_delta,
                        const FastPlan &plan, const uint8_t *location, const StartRecord *start,
                        TaskPartial *partials, unsigned long long *queue, DeviceCounters *ctr);

// One solve of a batch (many solves of different meshes, grids, equations
// and walk counts run by one launch per walk family).  Point arrays are the
// solve's own slices of the batch buffers.
struct BatchItem {
    FastArgs a;              // walk arguments (a.queue unused: one queue per family)
    EqDesc eq;
    Fields out;
    double btol;             // boundary tolerance of the classification
    double exact_below;      // FastStart::exact_below, or < 0: exact start radii
    float start_margin;      // FastStart::margin
    int max_ray_attempts;
    int precision;           // 32 / 64
    long long point_begin;   // first point of the solve in the batch's point order
    long long task_begin;    // first task of the solve in its family's queue
};

// Classification of the points [point_base, point_base + n_points) of the
// batch items [0, n_items) (all of one dimension, sorted by point_begin).
cudaError_t launch_classify_batch(int dim, const BatchItem *items, int n_items,
                                  long long point_base, long long n_points, cudaStream_t stream);

// Fast walks of one family (all items share dim, equation kind, precision
// and, for precision 32, the wide tree's height class `hc`; tasks numbered
// by task_begin from 0) on a persistent grid of `blocks` blocks
// (batch_walk_blocks: every block that can be resident).
cudaError_t launch_walk_batch(int dim, int kind, int precision, int hc, const BatchItem *items,
                              int n_items, long long n_tasks, unsigned long long *queue,
                              int blocks, cudaStream_t stream);
cudaError_t batch_walk_blocks(int dim, int kind, int precision, int hc, int *blocks);

// Per-point merge of every item of the batch.
cudaError_t launch_merge_batch(const BatchItem *items, int n_items, long long n_points,
                               cudaStream_t stream);

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

// Sets the walks per task of `plan` to `chunk` (clamped to [1, n_walks]) and
// recomputes its task counts.  A task counts its closest-point queries, at
// most chunk * max_steps, in 32 bits, and each lane sums the steps of its
// ceil(chunk/32) walks in 32 bits, so the chunk is also capped at
// floor((2^32 - 1) / max_steps), which keeps both below 2^32 and 2^31.
inline void set_chunk(FastPlan &plan, long long chunk, int n_walks, int max_steps,
                      long long n_points) {
    const long long per_task = 4294967295LL / (max_steps > 0 ? max_steps : 1);
    const long long cap = per_task < (1LL << 30) ? per_task : (1LL << 30);
    if (chunk > cap) chunk = cap;
    if (chunk > n_walks) chunk = n_walks;
    if (chunk < 1) chunk = 1;
    plan.chunk = static_cast<int>(chunk);
    plan.chunks = static_cast<int>((n_walks + chunk - 1) / chunk);
    plan.n_tasks = n_points * plan.chunks;
}

// Gaussian heat source -Δu = Q exp(-|x - x0|^2 / sigma^2) with per-vertex
// Dirichlet data (kernels_adjoint.cu).
struct HeatDesc {
    int mode;               // kUniform / kGreen / kMis source sampling
    double Q, x0[3], sigma;
    double beta;            // kMis: probability of a Green sample
    double px0[3], psigma;  // kMis: proposal N(px0, psigma^2 / 2 I)
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
    double n, mean, m2, steps, queries;
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

// Distance lattice of a scene (w's lattice geometry gn / glo / gh set, gd
// unused): out[(i*gn[1] + j)*gn[2] + k] = the exact FP32 cooperative query's
// boundary distance at the FP32 node glo + (i, j, k) * gh, minus `margin`,
// rounded down (0 if negative).  FP64 per-thread queries took 240 ms for a
// 173k-triangle mesh at 160^3 nodes.  With `scratch` (lattice_skip_bytes(w)
// bytes of device memory, else null) the nodes whose own and neighbours'
// centres lie outside the mesh, by the crossing parity of their lattice row
// (rows within `tol` of an edge or vertex stay unclassified), store 0 without
// a query.
size_t lattice_skip_bytes(const WideView &w);

// Lattice value below which a walk step of a solve with this epsilon may run
// a closest-point query: above it, for any point whose nearest node has that
// value, the lattice step is taken (D >= gratio r and (D - r)(1 - tau) beyond
// the shell for every r <= r_max).  Near-boundary lists are needed below it.
inline float near_list_threshold(const WideView &w, double epsilon, double shell_delta) {
    const double tau = 1.0 / 1024.0;
    const double rmax = 0.5 * w.gh * (w.dim == 3 ? 1.7320508075688772 : 1.4142135623730951) *
                        (1.0 + 1e-3);
    const double shell = epsilon + shell_delta;
    const double a = w.gratio * rmax, b = shell / (1.0 - tau) + rmax;
    return static_cast<float>((a > b ? a : b) * (1.0 + 1e-3));
}

// Capacity of a near-boundary list (wide slots).
// (16 in 2D and 3D: on the B200 16, 24 and 32 ran within 1% of each other,
// 8 cost the heat walks 1.7x)
inline int near_list_capacity(int) { return 16; }

// Near-boundary candidate lists of a lattice (w's lattice built): every node
// with 0 <= value <= t gets the wide slots of all primitives within its exact
// FP32 distance plus `extra` (2 r_max and a rounding margin), if there are
// at most near_list_capacity of them.  `count` (device) receives the number
// of such nodes first (band pass); the lists are then written end to end into
// the pool's `pool_slots` slots, `counter` counting the slots used.
cudaError_t launch_near_band(const WideView &w, float t, unsigned *count, cudaStream_t stream);
// The primitive records one slot after another (WideView::aos) for the list
// scans: prim_aos_bytes(w) bytes.
size_t prim_aos_bytes(const WideView &w);
cudaError_t launch_prim_aos(const WideView &w, float *aos, cudaStream_t stream);
cudaError_t launch_near_lists(const WideView &w, float t, float extra, float rmax, float slack,
                              int2 *gl, int *pool, int pool_slots, unsigned *counter, int sms,
                              cudaStream_t stream);
cudaError_t launch_lattice32(const SceneView &s, const WideView &w, float margin, float *out,
                             int sms, void *scratch, double tol, cudaStream_t stream);
// lattice_bound at each point (FP32), NaN where the scene has no lattice.
cudaError_t launch_lattice_bounds(const WideView &w, const double *pts, long long n, double *out,
                                  cudaStream_t stream);

// Kernel-level checks.
// ln I0(x) and ln K0(x) as the walk kernels of `precision` evaluate them
// (64: the exact path's translation unit, 32: the fast path's).
cudaError_t launch_special(int precision, const double *x, long long n, double *log_i0,
                           double *log_k0, cudaStream_t stream);
cudaError_t launch_special64(const double *x, long long n, double *log_i0, double *log_k0,
                             cudaStream_t stream);
cudaError_t launch_prng(const uint64_t *seeds, long long n, int count, uint64_t *out,
                        cudaStream_t stream);
cudaError_t launch_closest64(const SceneView &s, const double *pts, long long n, double *dist,
                             double *nearest, int *boundary_id, cudaStream_t stream);
cudaError_t launch_closest32(const SceneView &s, const WideView &w, const double *pts,
                             long long n, double *dist, double *nearest, int *boundary_id,
                             cudaStream_t stream);

}  // namespace wosb
