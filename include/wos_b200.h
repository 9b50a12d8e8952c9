/*
 * wos_b200.h — C ABI of the B200 walk-on-spheres library (libwos_b200.so).
 *
 * Plain C types only: host or device pointers and sizes, int status codes,
 * no exceptions across the boundary.  One CUDA stream per context.  Each
 * entry point names the reference interface it replaces (paths inside the
 * zhouzh721/walk-on-spheres sources).
 *
 * Status: every function returning int returns WOS_OK (0) on success; on
 * failure the message is available from wos_last_error(ctx) (or
 * wos_last_global_error() when no context exists).
 */
#ifndef WOS_B200_H
#define WOS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WOS_B200_ABI_VERSION 2

/* status codes */
enum {
    WOS_OK = 0,
    WOS_ERR_INVALID = 1,   /* bad argument or state */
    WOS_ERR_CUDA = 2,      /* CUDA runtime error */
    WOS_ERR_MESH = 3,      /* mesh file or mesh content rejected (src/mesh.cpp:17-22) */
    WOS_ERR_DEVICE = 4,    /* a kernel raised its error word (bounded loop ran out) */
    WOS_ERR_IO = 5         /* output file could not be written */
};

/* Equation kinds in the order of the reference registry
 * (src/equations/equations.hpp:26-31). */
enum {
    WOS_EQ_LAPLACE = 0,
    WOS_EQ_POISSON = 1,
    WOS_EQ_SCREENED_POISSON = 2,
    WOS_EQ_HELMHOLTZ = 3
};

/* Source sampling modes (include/wos/source_mode.hpp:5-9).  WOS_SOURCE_MIS is
 * the reference's GreenSourceMIS (include/wos/source_sampling.hpp:35-78): it
 * needs a source proposal, which only the Gaussian heat source below
 * provides; the registry equations reject it, as the reference's walk does
 * (include/wos/wos.hpp:83-92). */
enum { WOS_SOURCE_UNIFORM = 0, WOS_SOURCE_GREEN = 1, WOS_SOURCE_MIS = 2 };

/* Walk methods.
 *  PLAIN_FP64: the reference estimator (include/wos/wos.hpp:54-191) in FP64,
 *    every walk of a point on the point's own xoshiro256++ streams in the
 *    reference's order (include/wos/runner.hpp:208-222); matches the
 *    reference run to rounding of the transcendental functions.
 *  FAST_FP32: FP32 distance / closest-point / sphere-step arithmetic with an
 *    FP64 re-projection inside the epsilon shell, FP64 estimator sums, and
 *    counter-based Philox streams per (grid point, walk); statistically
 *    equivalent, not bitwise equal, to PLAIN_FP64.
 *  FAST_FP64: the FAST_FP32 scheduling with FP64 arithmetic throughout
 *    (the same counter-based streams). */
enum { WOS_METHOD_PLAIN_FP64 = 0, WOS_METHOD_FAST_FP32 = 1, WOS_METHOD_FAST_FP64 = 2 };

/* Location codes (include/wos/inside.hpp:8-13). */
enum { WOS_OUTSIDE = 0, WOS_INSIDE = 1, WOS_BOUNDARY = 2, WOS_INDETERMINATE = 3 };

typedef struct wos_context wos_context;

/* Cartesian grid (include/wos/grid.hpp:5-10); coordinate i is
 * min + (max-min)*i/(N-1) (grid.hpp:12-18).  2D grids use Nz = 1. */
typedef struct {
    int Nx, Ny, Nz;
    double xmin, xmax, ymin, ymax, zmin, zmax;
} wos_grid;

/* Solver arguments: the scalars of the reference registry entry
 * (src/equations/equations.hpp:8-16) plus the walk method. */
typedef struct {
    int equation;          /* WOS_EQ_* */
    int source_mode;       /* WOS_SOURCE_* (poisson, screened_poisson) */
    double alpha;          /* screened_poisson coefficient */
    int N_walks;           /* walks per inside point (>= 1) */
    double epsilon;        /* requested stopping distance; screened_poisson clamps it to
                              min(epsilon, 0.05/alpha) (src/equations/screened_poisson.cpp:22-38) */
    int max_steps;         /* walk step cap (>= 1) */
    int max_ray_attempts;  /* 3D inside-test ray budget (>= 3) */
    uint64_t seed;         /* --seed: per-point streams are splitmix64(seed ^ splitmix64(index)) */
    int method;            /* WOS_METHOD_* */
} wos_params;

/* Run diagnostics (include/wos/runner.hpp:240-283 plus timings). */
typedef struct {
    long long inside_points;
    long long max_steps_hits;
    long long ambiguous_ray_retries;
    long long indeterminate_points;
    long long total_walks;
    long long total_steps;          /* sum of steps over all walks */
    double sum_variance;            /* over inside points, grid order */
    double sum_standard_error;
    double sum_mean_steps;
    double effective_epsilon;
    float classify_ms;              /* device time of the classification kernel */
    float walk_ms;                  /* device time of the walk kernel(s) */
    float total_ms;                 /* device time of the whole solve */
    long long exact_queries;        /* walk steps that ran a BVH closest-point query
                                       (bvh_npq, src/bvh.cpp:295-387): every step of
                                       PLAIN_FP64 / FAST_FP64; FAST_FP32 steps that take
                                       their radius from the distance lattice run none */
} wos_counters;

/* ---------------------------------------------------------------- context */

/* Create a context on CUDA device `device` with its own stream. */
int wos_context_create(int device, wos_context **out);
void wos_context_destroy(wos_context *ctx);
const char *wos_last_error(const wos_context *ctx);
const char *wos_last_global_error(void);
int wos_abi_version(void);

/* ------------------------------------------------------------------- mesh */

/* Upload a boundary mesh and build its device BVHs.  Replaces the mesh
 * broadcast and BVH build/broadcast of include/wos/runner.hpp:28-77
 * (load_mesh src/mesh.cpp:76-270, build_bvh src/bvh.cpp:234-253).
 *  dim 2: prims = n_prims segments (2 vertex indices each, 0-based),
 *         boundary_ids = the `l` record of each segment (may be NULL: all 0);
 *  dim 3: prims = n_prims triangles (3 vertex indices each).
 *  leaf_size: maximum primitives per BVH leaf, 2..8 (0 selects the default 4,
 *  the reference's LEAF_SIZE, src/bvh.cpp:15).
 * Rejects zero-length segments and degenerate triangles like
 * src/mesh.cpp:239-267. */
int wos_set_mesh(wos_context *ctx, int dim, const double *verts, int n_verts, const int *prims,
                 int n_prims, const int *boundary_ids, int leaf_size);

/* Load an OBJ file with the reference's reader semantics (src/mesh.cpp:51-270:
 * `v`, `l` polylines auto-closed with one boundary_id per record, `f`
 * triangles only) and upload it as wos_set_mesh does. */
int wos_load_obj(wos_context *ctx, const char *path, int leaf_size);

/* Mesh bounding box {xmin, xmax, ymin, ymax, zmin, zmax} (src/mesh.cpp:297-322)
 * and dimension of the current mesh. */
int wos_mesh_info(const wos_context *ctx, int *dim, int *n_prims, double bbox[6]);

/* Fill `grid` with Nx x Ny x Nz points over the mesh bounding box, as
 * include/wos/runner.hpp:83-85 does. */
int wos_grid_over_mesh(const wos_context *ctx, int Nx, int Ny, int Nz, wos_grid *grid);

/* ------------------------------------------------------------------ solve */

/* Per-grid-point WoS sweep: the loop body of include/wos/runner.hpp:157-236
 * for every point of `grid` (start point, inside/outside/boundary
 * classification, boundary value, wos_run).  Output arrays are HOST arrays of
 * Nx*Ny*Nz elements in row-major (i, j, k) order (include/wos/field_3D.hpp:
 * 9-31); any of them may be NULL.  Values of outside / indeterminate points
 * are NaN, boundary points get {g(nearest), 0, 0, 0} (runner.hpp:196-206).
 * Blocks until the results are on the host. */
int wos_solve_grid(wos_context *ctx, const wos_params *params, const wos_grid *grid,
                   double *mean, double *variance, double *standard_error, double *mean_steps,
                   uint8_t *location, wos_counters *counters);

/* As wos_solve_grid, but the output pointers are DEVICE pointers on the
 * context's device (any may be NULL) and nothing is copied to the host;
 * counters (if given) are filled after the solve completes. */
int wos_solve_grid_device(wos_context *ctx, const wos_params *params, const wos_grid *grid,
                          double *mean, double *variance, double *standard_error,
                          double *mean_steps, uint8_t *location, wos_counters *counters);

/* As wos_solve_grid_device, but allocating no device memory; it has no
 * counterpart in the reference.  For callers that cannot call cudaMalloc
 * while they solve (an allocator or pool that owns the device budget, code
 * that must not take the device-wide synchronisation cudaMalloc / cudaFree
 * can cause, hosts that forbid allocation after start-up).  Temporaries live
 * in one static 8 MiB device array inside the library, reserved on a device
 * when a context is created there (wos_context_create takes its address) and
 * held until the process exits, so grids are limited to about 94 000 points
 * (WOS_ERR_INVALID beyond).  Arguments are checked by the same rules as
 * wos_solve_grid_device.  The call still blocks until the solve has finished
 * on the context's stream.  Calls that overlap on the GPU share the array and
 * race, so serialise them.  The context (mesh upload) is set up by the
 * allocating entry points beforehand. */
int wos_solve_grid_device_noalloc(wos_context *ctx, const wos_params *params,
                                  const wos_grid *grid, double *mean, double *variance,
                                  double *standard_error, double *mean_steps, uint8_t *location,
                                  wos_counters *counters);

/* The point-level operator: wos_run (include/wos/wos.hpp:160-191) with
 * get_start_point (wos.hpp:42-52) and classification for `n` arbitrary start
 * points (host array n*dim).  point_index[i] plays the role of the grid
 * linear index in the seeding (runner.hpp:163-168); NULL uses i. */
int wos_solve_points(wos_context *ctx, const wos_params *params, const double *points,
                     const uint64_t *point_index, long long n, double *mean, double *variance,
                     double *standard_error, double *mean_steps, uint8_t *location,
                     wos_counters *counters);

/* ----------------------------------------------------------------- batches */

/* Many independent grid sweeps, each with its own mesh, grid, equation,
 * walk count and seed, run together (no reference counterpart: the reference
 * runs one registry entry per process).  Each solve means exactly what
 * wos_solve_grid means for the same arguments and FAST method: under the
 * same chunking (wos_set_tuning / wos_batch_set_tuning) every walk draws the
 * same numbers and takes the same steps, so locations, step counts and
 * counters are identical and the statistics differ at most by the rounding
 * of the terminal FP64 arithmetic (the batch kernel is compiled apart from
 * the single-solve kernel).  The batch runs one classification launch per
 * dimension, one persistent walk launch per (dimension, equation, method)
 * family over a device work queue of (solve, point, chunk-of-walks) tasks,
 * and one merge launch; wos_batch_run can capture that sequence once as a
 * CUDA graph and replay it. */
typedef struct wos_batch wos_batch;

/* A batch on the context's device and stream.  The context's own mesh and
 * buffers are untouched. */
int wos_batch_create(wos_context *ctx, wos_batch **out);
void wos_batch_destroy(wos_batch *batch);

/* Add a mesh (arguments as wos_set_mesh); *mesh_id indexes it.  The mesh is
 * checked now (wos_set_mesh's errors and messages); its trees are built with
 * the batch's other new meshes, in parallel on the host threads, by
 * wos_batch_prepare or the next wos_batch_run. */
int wos_batch_add_mesh(wos_batch *batch, int dim, const double *verts, int n_verts,
                       const int *prims, int n_prims, const int *boundary_ids, int leaf_size,
                       int *mesh_id);

/* Add a sweep of `grid` over mesh `mesh_id` (params as wos_solve_grid; the
 * method must be FAST_FP32 or FAST_FP64).  *solve_id indexes it. */
int wos_batch_add_solve(wos_batch *batch, int mesh_id, const wos_params *params,
                        const wos_grid *grid, int *solve_id);

/* Walks per task (<= 0: min(N_walks, 1024) per solve) and persistent grid
 * size of every walk launch (<= 0: every block that can be resident). */
int wos_batch_set_tuning(wos_batch *batch, int chunk, int blocks);

/* Build and upload the meshes added since the last run and lay out every
 * solve (what the first wos_batch_run does before launching), so that set-up
 * can be timed or overlapped apart from the runs. */
int wos_batch_prepare(wos_batch *batch);

/* Run every solve.  use_graph != 0 captures the launch sequence as a CUDA
 * graph on the first run (and after any change to the batch) and replays
 * it.  *device_ms (may be NULL) is the device time of the whole batch. */
int wos_batch_run(wos_batch *batch, int use_graph, float *device_ms);

/* Totals of the batch: solves, grid points, walks of the last run. */
int wos_batch_info(const wos_batch *batch, int *n_solves, long long *n_points,
                   long long *total_walks, long long *total_steps);

/* Fields (host arrays of the solve's Nx*Ny*Nz points, any may be NULL) and
 * counters of solve `solve_id` from the last run. */
int wos_batch_result(wos_batch *batch, int solve_id, double *mean, double *variance,
                     double *standard_error, double *mean_steps, uint8_t *location,
                     wos_counters *counters);

/* ------------------------------------------------- transient plate heating */

/* The reference's transient welding programs (apps/welding/src/
 * level{0_cooling,2_transient_heat,3_moving_heat}.cpp): a rectangular plate
 * [plate_x0, plate_x0 + length_x] x [plate_y0, plate_y0 + length_y] with zero
 * temperature rise on its edges and implicit Euler steps of dt up to
 * total_time, each solved by screened walk on spheres with
 * alpha = 1/sqrt(kappa dt), kappa = conductivity / (density specific_heat),
 * and a source built from the previous step's grid field u_prev (sampled
 * bilinearly or by cubic Lagrange weights, FieldSampler2D):
 *   scenario 0  alpha^2 u_prev                          (level 0, cooling)
 *   scenario 2  alpha^2 max(0, u_prev) + f q/k, a stationary Gaussian at the
 *               plate centre normalised on the finite plate
 *               (gaussian_heat_source.hpp), f the share of the step before
 *               heat_on_time                           (level 2)
 *   scenario 3  alpha^2 max(0, u_prev) + q/k, a Gaussian moving along
 *               y = weld_y from source_start_x at weld_speed until
 *               heat_on_time, two Gauss-Legendre components per step
 *               (moving_gaussian_heat_source.hpp)      (level 3)
 * Seeds per step and point as the reference: splitmix64(seed ^
 * splitmix64(step) ^ splitmix64(i*ny + j)); PLAIN_FP64 follows the
 * reference's streams. */
typedef struct {
    int nx, ny;                /* odd, >= 3 */
    double dt, total_time, heat_on_time;
    int walks, max_steps;
    double epsilon;
    uint64_t seed;
    int cubic;                 /* history interpolation: 1 cubic, 0 bilinear */
    double length_x, length_y, thickness;
    double conductivity, density, specific_heat;
    double electrical_power, efficiency, sigma_x, sigma_y;
    int method;                /* WOS_METHOD_* */
    int scenario;              /* 0, 2 or 3 (above) */
    double plate_x0, plate_y0; /* lower-left corner of the plate */
    double weld_y, source_start_x, weld_speed;  /* scenario 3 */
} wos_transient_params;

/* The reference's level-2 defaults (Level2Config:46-78), scenario 2. */
void wos_transient_defaults(wos_transient_params *p);

/* Number of time steps of p (total_time / dt), or -1 if p is invalid. */
int wos_transient_steps(const wos_transient_params *p);

/* Run every time step on the context's device (the context's mesh is not
 * used or changed).  initial (host, may be NULL for zeros): the nx x ny
 * field at time 0.  fields / standard_error (host, may be NULL):
 * (steps + 1) x nx x ny doubles, step 0 the initial field.  max_steps_hits
 * (may be NULL): summed over all steps.  use_graph != 0 captures the whole
 * time loop as one CUDA graph before launching it.  device_ms (may be NULL):
 * device time of all steps.  Parameter errors carry the reference's
 * messages (level2_transient_heat.cpp:206-223, moving_gaussian_heat_source.hpp:
 * 21-28, 55-58). */
int wos_transient_solve(wos_context *ctx, const wos_transient_params *p, const double *initial,
                        int use_graph, double *fields, double *standard_error,
                        long long *max_steps_hits, float *device_ms);

/* ------------------------------------------------ stationary plate heating */

/* The reference's stationary welding program (apps/welding/src/
 * level1_stationary_heat.cpp:132-269): -Lap u = f on the plate
 * [0, length_x] x [0, length_y] with u = 0 on its edges, on an nx x ny grid
 * whose edge points are boundary points (value 0) and whose interior points
 * run `walks` walks each.
 *   WOS_PLATE_MANUFACTURED  f = pi^2 (1/Lx^2 + 1/Ly^2) u*, with the exact
 *                           solution u* = peak_rise sin(pi x/Lx) sin(pi y/Ly)
 *                           (ManufacturedPoisson2D, :75-130)
 *   WOS_PLATE_GAUSSIAN      f = q/k, q the Gaussian centred at
 *                           (source_x, source_y) normalised on the finite
 *                           plate (gaussian_heat_source.hpp)
 *                           (StationaryGaussianHeat2D, :132-191)
 * source_mode WOS_SOURCE_GREEN, WOS_SOURCE_UNIFORM or (Gaussian only)
 * WOS_SOURCE_MIS: Green samples with probability mis_green_probability, else
 * samples of the finite-plate Gaussian (include/wos/source_sampling.hpp:
 * 35-78).  Seeds as the reference: splitmix64(seed ^ case_stream ^
 * splitmix64(i*ny + j)); PLAIN_FP64 follows the reference's streams. */
enum { WOS_PLATE_MANUFACTURED = 0, WOS_PLATE_GAUSSIAN = 1 };

typedef struct {
    int nx, ny;                /* >= 3 */
    int walks, max_steps;
    double epsilon;
    uint64_t seed;
    uint64_t case_stream;      /* the reference's per-case stream constant */
    double length_x, length_y, thickness, conductivity;
    double electrical_power, efficiency, sigma_x, sigma_y;
    double source_x, source_y; /* Gaussian centre */
    double peak_rise;          /* manufactured amplitude */
    int source;                /* WOS_PLATE_* */
    int source_mode;           /* WOS_SOURCE_* */
    double mis_green_probability;
    int method;                /* WOS_METHOD_* */
    int max_proposal_attempts; /* rejection cap of the Gaussian proposal */
} wos_stationary_params;

/* The reference's Level1Config (:42-61) for `source`, with that case's
 * stream constant and Green source sampling. */
void wos_stationary_defaults(wos_stationary_params *p, int source);

/* Solve on the context's device (the context's mesh is not used or
 * changed).  mean / variance / standard_error / mean_steps (host, may be
 * NULL): nx x ny doubles, index i*ny + j.  Parameter errors carry the
 * reference's messages (gaussian_heat_source.hpp:28-36,
 * source_sampling.hpp:41-47, wos.hpp:88-91); a proposal that found no plate
 * point in max_proposal_attempts draws returns WOS_ERR_DEVICE with the
 * reference's message (gaussian_heat_source.hpp:70-72). */
int wos_stationary_solve(wos_context *ctx, const wos_stationary_params *p, double *mean,
                         double *variance, double *standard_error, double *mean_steps,
                         long long *max_steps_hits, float *device_ms);

/* ------------------------------------ Gaussian heat source and its adjoint */

/* Source of the differentiable heat problem (no reference counterpart; the
 * reference's only Gaussian source is the 2D welding one of
 * apps/welding/include/welding/gaussian_heat_source.hpp, with another
 * normalisation):
 *     -Δu = f,  f(x) = Q exp(-|x - x0|^2 / sigma^2),
 *     u = g on the boundary, g given per mesh vertex and interpolated at the
 *     nearest boundary point (linearly along a segment in 2D,
 *     barycentrically on a triangle in 3D). */
typedef struct {
    double Q;       /* amplitude */
    double x0[3];   /* centre (x0[2] unused in 2D) */
    double sigma;   /* width (> 0) */
    /* WOS_SOURCE_MIS only: each step draws its source point from the Green
     * density of the ball with this probability, else from the proposal
     * N(proposal_x0, proposal_sigma^2 / 2 I) (the source's own shape), and
     * weighs it by the balance heuristic G f / (beta p_green + (1 - beta)
     * p_proposal), as include/wos/source_sampling.hpp:35-78 does.  The
     * proposal is held fixed under differentiation; proposal_sigma <= 0
     * takes x0 and sigma. */
    double mis_green_probability;
    double proposal_x0[3];
    double proposal_sigma;
} wos_gaussian_source;

/* Number of vertices of the current mesh (the length of the per-vertex
 * boundary data). */
int wos_mesh_vertex_count(const wos_context *ctx, int *n_verts);

/* Forward solve at `n` probe points (host array n*dim) with the reference's
 * Poisson walk estimator (include/wos/wos.hpp:54-138 with the Green kernels
 * of include/wos/poisson.hpp:12-51) for the source above.  vertex_values:
 * host array of n_verts boundary values (NULL: g = 0).  params: N_walks,
 * epsilon (used as given), max_steps, max_ray_attempts, seed, source_mode
 * (uniform, Green or MIS source samples) and method (FAST_FP32 or FAST_FP64;
 * PLAIN_FP64 is rejected); params->equation and alpha are ignored.  Probe i
 * is seeded like grid index point_index[i] (NULL: i).  Outputs as
 * wos_solve_points (host arrays, any may be NULL); boundary probes get
 * g(nearest), outside / indeterminate probes NaN. */
int wos_heat_forward(wos_context *ctx, const wos_params *params,
                     const wos_gaussian_source *source, const double *vertex_values,
                     const double *probes, const uint64_t *point_index, long long n,
                     double *mean, double *variance, double *standard_error,
                     double *mean_steps, uint8_t *location, wos_counters *counters);

/* Adjoint of wos_heat_forward for the same arguments: re-runs every walk
 * from its seed (paths are not stored; the replayed values are bit-identical
 * to the forward ones) and accumulates, for probe weights grad_u (host, n;
 * dL/du_p; NULL: all 1):
 *   grad_source[5]   sum_p grad_u[p] du_p/d(Q, x0.x, x0.y, x0.z, sigma)
 *   grad_vertex_values[n_verts]   sum_p grad_u[p] du_p/dg_v
 *   jacobian[n*5]    per-probe walk means of du_p/d(Q, x0.x, x0.y, x0.z, sigma)
 *   jacobian_se[n*5] their standard errors
 *   replayed_mean[n] the replayed probe values
 * All host arrays; any may be NULL.  Outside / indeterminate probes carry NaN
 * in jacobian and contribute nothing. */
int wos_heat_adjoint(wos_context *ctx, const wos_params *params,
                     const wos_gaussian_source *source, const double *vertex_values,
                     const double *probes, const uint64_t *point_index, long long n,
                     const double *grad_u, double *grad_source, double *grad_vertex_values,
                     double *jacobian, double *jacobian_se, double *replayed_mean,
                     wos_counters *counters);

/* -------------------------------------------------- kernel-level checks */

/* First `count` outputs of the device xoshiro256++ stream PRNG(seeds[s])
 * (include/wos/prng.hpp:14-24, src/prng.cpp:6-15) for every seed:
 * out[s*count + i]. */
int wos_prng_u64(wos_context *ctx, const uint64_t *seeds, long long n_seeds, int count,
                 uint64_t *out);

/* Closest boundary point of each query (bvh_npq, src/bvh.cpp:295-387) on the
 * device.  precision 64: the FP64 traversal used by PLAIN_FP64, the
 * classification and the epsilon shell; 32: the FP32 traversal of FAST_FP32
 * (distances then carry FP32 rounding).  boundary_id may be NULL. */
int wos_closest_points(wos_context *ctx, int precision, const double *points, long long n,
                       double *dist, double *nearest, int *boundary_id);

/* Lower bounds of the boundary distance that FAST_FP32 walks take from the
 * mesh's distance lattice (no reference counterpart).  The lattice is a
 * regular grid of nodes over the bounding box, 2048 along the longest axis
 * in 2D, 256 in 3D.  Each node stores a lower bound of its boundary
 * distance D, in FP32: the pruned FP32 query's distance times 1 - 2^-10,
 * minus an FP32 rounding margin.  The bound at a point is that node value
 * of its nearest node minus r, the distance to that node, so
 * bound <= the exact distance everywhere.
 * A walk step takes the bound times 1 - 2^-10 as its radius, instead of a
 * closest-point query, when three conditions hold: D >= 2 r, that radius is
 * positive, and it stays outside the epsilon shell.  WoS is unbiased for any ball
 * inside the domain.  NaN when the mesh has no lattice (meshes of at most 64
 * segments or 32 triangles, or WOS_BOUND_GRID=0). */
int wos_distance_bounds(wos_context *ctx, const double *points, long long n, double *bound);

/* ln I0(x) and ln K0(x) of the screened kernels as the walks evaluate them on
 * the device (include/wos/bessel.hpp:16-87): precision 64 as PLAIN_FP64 /
 * FAST_FP64 (series, quadrature and Hankel sums to FP64 accuracy), 32 as
 * FAST_FP32 (x rounded to float; Abramowitz & Stegun 9.8.1-9.8.6). */
int wos_special_functions(wos_context *ctx, int precision, const double *x, long long n,
                          double *log_i0, double *log_k0);

/* The current mesh's device scene (every tree and primitive array of
 * wos_set_mesh, not the lattice) copied to a host buffer, for checks that the
 * device tree build (the default; WOS_TREE_BUILD=host builds on the host
 * threads) and the host build give the same bytes.  *bytes receives the size;
 * out may be NULL to ask for it.  No reference counterpart. */
int wos_scene_arena(wos_context *ctx, void *out, long long capacity, long long *bytes);

/* Scheduling overrides of the FAST methods (no reference counterpart):
 * walks per task and persistent grid size; <= 0 restores the automatic
 * choice.  Used by the benchmark's tuner. */
int wos_set_tuning(wos_context *ctx, int chunk, int blocks);

/* ------------------------------------------------------- registry (drop-in) */

/* One entry of the equation registry with the reference's run signature
 * (src/equations/equations.hpp:7-17): load the OBJ mesh, sweep the grid over
 * its bounding box on the GPU, print the reference's diagnostics and write
 * the HDF5 result (include/wos/hdf5_io.hpp layout).  source_mode is the
 * integer value of wos::SourceMode.  Returns 0 on success, 1 on failure, as
 * the reference does.  The walk method is PLAIN_FP64 unless the environment
 * variable WOS_B200_METHOD is "fast" (FAST_FP32) or "fast64" (FAST_FP64). */
typedef int (*wos_run_fn)(int rank, int size, const char *mesh_filename,
                          const char *output_filename, int Nx, int Ny, int Nz, int N_walks,
                          double epsilon, int max_steps, int max_ray_attempts, uint64_t seed,
                          double alpha, int source_mode);

typedef struct {
    const char *name;
    wos_run_fn run_2D;
    wos_run_fn run_3D;
} wos_equation_entry;

/* The registry: laplace, poisson, screened_poisson, helmholtz
 * (src/equations/equations.hpp:26-31).  With size == 1 an entry sweeps the
 * whole grid on the GPU named by WOS_B200_DEVICE (default 0).  With size > 1
 * (the reference's `mpirun -np P wos ...`, README.md:32) rank `rank` solves
 * the reference's Cartesian block of the grid (include/wos/runner.hpp:90-134,
 * rank blocks from MPI_Dims_create) on GPU rank % device count (or
 * WOS_B200_DEVICE), the counters are reduced over the ranks
 * (runner.hpp:240-263), rank 0 creates the result file and every rank writes
 * its block into it (include/wos/hdf5_io.hpp:51-171).  The ranks meet only
 * through the collectives installed with wos_set_collectives; without them a
 * call with size > 1 fails with 1. */
const wos_equation_entry *wos_equation_registry(int *count);

/* The caller's process-group collectives, used by the registry entries when
 * size > 1 in place of the reference's MPI calls (MPI_Barrier, MPI_Reduce /
 * MPI_Allreduce, MPI_Dims_create in include/wos/runner.hpp:90-263 and
 * include/wos/hdf5_io.hpp:51-171).  Every callback returns 0 on success.
 *  barrier:     return once every rank has entered it.
 *  allreduce:   reduce `n` doubles in place over the ranks, every rank
 *               receiving the result; op WOS_REDUCE_SUM or WOS_REDUCE_MAX.
 *  dims_create: optional (NULL: the library's restatement of MPI_Dims_create,
 *               a balanced factorisation in non-increasing order); fill the
 *               zero entries of dims[3] for `size` ranks, as MPI_Dims_create
 *               does. */
enum { WOS_REDUCE_SUM = 0, WOS_REDUCE_MAX = 1 };
typedef struct {
    int (*barrier)(void *user);
    int (*allreduce)(double *values, int n, int op, void *user);
    int (*dims_create)(int size, int dims[3], void *user);
    void *user;
} wos_collectives;

/* Install (or, with NULL, remove) the collectives for this process.
 * WOS_ERR_INVALID if barrier or allreduce is missing. */
int wos_set_collectives(const wos_collectives *collectives);

/* Rank `rank`'s block of an Nx x Ny x Nz grid split over `size` ranks as the
 * reference splits it (include/wos/runner.hpp:90-134): the decomposition
 * dims[3], the block's first grid index offset[3] and extent count[3] along
 * x, y, z.  WOS_ERR_INVALID with the reference's message in `error` (may be
 * NULL) when the ranks do not fit the grid.  Host only. */
int wos_rank_block(int dim, int Nx, int Ny, int Nz, int rank, int size, int dims[3],
                   int offset[3], int count[3], char *error, int error_capacity);

/* ------------------------------------------------ host-only (no GPU needed) */

/* Read an OBJ boundary mesh (load_mesh, src/mesh.cpp:76-270).  Call once with
 * null arrays to get dim / n_verts / n_prims, then with arrays of
 * n_verts*dim doubles, n_prims*dim ints and (2D) n_prims ints.  On failure
 * returns WOS_ERR_MESH and copies the reference-formatted message
 * ("Mesh <path>[:<line>]: <what>") into `error`. */
int wos_read_obj(const char *path, int *dim, int *n_verts, int *n_prims, double *verts,
                 int *prims, int *boundary_ids, char *error, int error_capacity);

/* Host BVH build (the device layout's FP64 part; build_bvh, src/bvh.cpp:234-253):
 * depth D, node boxes (2^(D+1) nodes x 2*dim doubles: lo then hi, node id 0
 * unused, 1-based heap order) and the leaf-slot primitive order (n_prims).
 * Pass null arrays to get the depth only. */
int wos_build_bvh(int dim, const double *verts, int n_verts, const int *prims, int n_prims,
                  int leaf_size, int *depth, double *node_boxes, int *order);

/* Host build of the FP32 32-wide tree used by the FAST_FP32 walks (no
 * counterpart in the reference): root height H (32^H >= n_prims), the float
 * count of the node blocks, the node blocks (the 32 children of a height-(h+1)
 * node form a block of (3*dim+2) x 32 floats starting at offsets[h] + parent
 * * (3*dim+2)*32: box lo[dim], hi[dim], slab normal[dim], slab offset, slab
 * half-thickness, field f of child k at f*32 + k) and the wide-slot primitive
 * order.  Pass null arrays to get the sizes. */
int wos_build_wide_bvh(int dim, const double *verts, int n_verts, const int *prims, int n_prims,
                       int *height, int *entries, int *offsets, float *nodes, int *order);

/* Write a result file with the reference's HDF5 layout (wos_write_hdf5,
 * include/wos/hdf5_io.hpp:15-338): /mean /variance /standard_error
 * /mean_steps (f64 [Nx,Ny,Nz]), /location (u8), /x /y /z and the /metadata
 * scalars (ray counters when write_ray_metadata, alpha and source_mode when
 * write_source_metadata). */
int wos_write_hdf5(const char *path, const wos_grid *grid, const double *mean,
                   const double *variance, const double *standard_error,
                   const double *mean_steps, const uint8_t *location, int N_walks,
                   double epsilon, int max_steps, long long max_steps_hits,
                   int write_ray_metadata, int max_ray_attempts, long long ambiguous_ray_retries,
                   long long indeterminate_points, uint64_t seed, int write_source_metadata,
                   double alpha, int source_mode);

/* Parallel write path: the reference's collective hyperslab writes
 * (include/wos/hdf5_io.hpp:51-171: every rank writes its own block of the
 * five fields, rank 0 writes /x /y /z and the /metadata scalars) without
 * MPI-IO.  The file layout depends only on the grid shape and the two
 * metadata switches, so every rank can compute it (wos_hdf5_layout).
 * One process creates the file (wos_hdf5_create): coordinates and metadata
 * written, the five fields' storage reserved.  Then every rank writes its
 * part of the fields into that storage (wos_hdf5_write_block or
 * wos_hdf5_write_range). Writes to disjoint parts may run from many
 * processes at once. Once every point has been written, the file is
 * byte-identical to wos_write_hdf5 of the whole fields. */
typedef struct {
    /* file offsets of the raw values of mean, variance, standard_error,
     * mean_steps (f64, C order) and location (u8, C order) */
    long long field_offset[5];
    long long file_size;
} wos_h5_layout;

/* The layout of a result file for `grid`, writing nothing. */
int wos_hdf5_layout(const wos_grid *grid, int write_ray_metadata, int write_source_metadata,
                    wos_h5_layout *layout);

/* Create the result file with every dataset but the fields' values
 * (arguments as wos_write_hdf5); `layout` (may be null) receives its layout.
 * The metadata counters are the totals over all ranks (the reference reduces
 * them first, include/wos/runner.hpp:240-263). */
int wos_hdf5_create(const char *path, const wos_grid *grid, int N_walks, double epsilon,
                    int max_steps, long long max_steps_hits, int write_ray_metadata,
                    int max_ray_attempts, long long ambiguous_ray_retries,
                    long long indeterminate_points, uint64_t seed, int write_source_metadata,
                    double alpha, int source_mode, wos_h5_layout *layout);

/* Write one rank's block of the fields into a created file: grid points
 * offset[d] .. offset[d] + count[d] - 1 along x, y, z (the reference's
 * x_start / block_Nx etc., include/wos/runner.hpp:116-128).  The arrays hold
 * the block in C order, count[0] x count[1] x count[2] values, like the
 * reference's per-rank Field3D.  WOS_ERR_INVALID if the block leaves the
 * grid; WOS_ERR_IO if the file is missing, is not a result file with this
 * layout, or a write fails. */
int wos_hdf5_write_block(const char *path, const wos_h5_layout *layout, const wos_grid *grid,
                         const int offset[3], const int count[3], const double *mean,
                         const double *variance, const double *standard_error,
                         const double *mean_steps, const uint8_t *location);

/* Write grid points start .. start + count - 1 in linear (C) order, the shard
 * of a linear-index split; the arrays hold `count` values.  Errors as
 * wos_hdf5_write_block. */
int wos_hdf5_write_range(const char *path, const wos_h5_layout *layout, const wos_grid *grid,
                         long long start, long long count, const double *mean,
                         const double *variance, const double *standard_error,
                         const double *mean_steps, const uint8_t *location);

/* Peek the mesh dimension (2 if the first primitive record is `l`, 3 if `f`),
 * src/mesh.cpp:51-74.  Returns 2, 3, or 0 on error. */
int wos_peek_mesh_dim(const char *path);

#ifdef __cplusplus
}
#endif

#endif /* WOS_B200_H */
