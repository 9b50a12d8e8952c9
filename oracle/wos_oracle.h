/*
 * wos_oracle — plain C, FP64 restatement of the reference walk-on-spheres hot
 * path.  TEST INFRASTRUCTURE ONLY: the oracle for the CUDA library, used by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.  It is
 * never linked into, or called by, the product library.
 *
 * Parity: pinned against the reference compiled from its own sources
 * (oracle/_ref, built by oracle/Makefile) through the golden fixtures in
 * tests/golden/ (generated by tests/golden/make_golden.py).  The only
 * intentional difference is the modified-Bessel evaluation: the reference
 * calls libstdc++'s std::cyl_bessel_i/k (include/wos/bessel.hpp:43,53); this
 * file evaluates I0 by its power series and K0 by its series (x <= 2) or a
 * trapezoidal rule on its integral representation (2 < x < 50), which agree
 * with libstdc++ to a few ulps (tests/test_oracle_golden.py states the bound).
 *
 * Every entry point mirrors an oracle/_ref entry point of the same suffix
 * (ref_* in oracle/ref_core.cpp and oracle/ref_driver.hpp) so the tests can
 * compare them one to one.
 */
#ifndef WOS_ORACLE_H
#define WOS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as `struct ref_problem` in oracle/ref_driver.hpp. */
typedef struct {
    int dim;
    const double *verts;
    int n_verts;
    const int *prims;
    int n_prims;
    const int *boundary_ids;
    int Nx, Ny, Nz;
    int use_mesh_bbox;
    double xmin, xmax, ymin, ymax, zmin, zmax;
    int N_walks;
    double epsilon;
    int max_steps;
    int max_ray_attempts;
    uint64_t seed;
    double alpha;
    int source_mode;
    int n_threads;
    const long long *points;
    long long n_points;
} wo_problem;

/* Same layout as `struct ref_outputs` in oracle/ref_driver.hpp. */
typedef struct {
    double *mean;
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
    double seconds;
} wo_outputs;

/* Equation kinds, in the order of the reference registry
 * (src/equations/equations.hpp:26-31). */
enum { WO_LAPLACE = 0, WO_POISSON = 1, WO_SCREENED_POISSON = 2, WO_HELMHOLTZ = 3 };

uint64_t wo_splitmix64(uint64_t x);
void wo_prng_u64(uint64_t seed, long long n, uint64_t *out);
void wo_prng_unit(uint64_t seed, long long n, int open, double *out);

int wo_build_bvh(const wo_problem *pb, double *node_boxes, int *node_counts, int *node_idx,
                 int *prims);
/* visits (optional): per query {node pops, primitive tests} of the reference
 * traversal order (src/bvh.cpp:295-387). */
void wo_npq(const wo_problem *pb, const double *points, long long n, double *dist,
            double *nearest, int *prim_id, int *boundary_id, long long *visits);
void wo_winding_numbers(const wo_problem *pb, const double *points, long long n, int *wn);
void wo_classify_3d(const wo_problem *pb, const double *points, const uint64_t *seeds,
                    long long n, double boundary_distance_tolerance, unsigned char *location,
                    int *retries);

void wo_bessel(const double *x, long long n, double *out);
void wo_j0y0(const double *x, long long n, double *j0, double *y0);
void wo_screened_kernels(const double *alpha, const double *R, const double *r, long long n,
                         double *out);
void wo_screened_samples(int dim, double alpha, double R, uint64_t seed, long long n,
                         double *out);
void wo_poisson_green(int dim, double R, const double *r, long long n, uint64_t seed,
                      double *green, double *mass, double *samples);
void wo_steps(int dim, const double *centre, double radius, uint64_t seed, long long n,
              double *steps, double *balls);

/* Full per-grid-point sweep (include/wos/runner.hpp:157-236) for one equation.
 * Returns 0 on success. */
int wo_solve_grid(int equation, const wo_problem *pb, wo_outputs *out);

/* Effective epsilon of the screened equation (src/equations/screened_poisson.cpp:22-38). */
double wo_screened_epsilon(double requested, double alpha);

/* Walk statistics of the reference traversal along the walks of the given
 * points (first `walks` walks each): totals of closest-point queries, node
 * pops and primitive tests, for the algorithmic-byte count of a walk. */
int wo_walk_visit_counts(int equation, const wo_problem *pb, int walks, long long *queries,
                         long long *node_pops, long long *prim_tests, long long *steps);

/* Gaussian heat source (same layout as wos_gaussian_source in include/wos_b200.h). */
typedef struct {
    double Q;
    double x0[3];
    double sigma;
    double mis_green_probability;  /* source_mode 2 */
    double proposal_x0[3];         /* proposal N(proposal_x0, proposal_sigma^2/2 I); */
    double proposal_sigma;         /* <= 0: x0 and sigma */
} wo_gaussian;

/* FP64 heat-source walks at `n` probes (host n*dim; probe i seeded like grid
 * index pb->points[i], or i when pb->points is NULL): per probe the mean
 * value and its standard error, the walk means of du/d(Q, x0.x, x0.y, x0.z,
 * sigma) and their standard errors (n*5), the location code, and
 * grad_vertex[v] = sum_i weights[i] du_i/dg_v (weights NULL: all 1).  Uses
 * pb's mesh, N_walks, epsilon, max_steps, max_ray_attempts, seed,
 * source_mode (0 uniform, 1 Green, 2 Green-source MIS) and n_threads.  Any output may be NULL.  Returns 0 on
 * success. */
int wo_heat_solve(const wo_problem *pb, const wo_gaussian *src, const double *vertex_values,
                  const double *probes, long long n, const double *weights, double *mean,
                  double *standard_error, double *jacobian, double *jacobian_se,
                  unsigned char *location, double *grad_vertex);

#ifdef __cplusplus
}
#endif

#endif
