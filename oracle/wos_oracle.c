/*
 * wos_oracle.c — plain C, FP64 restatement of the reference walk-on-spheres
 * hot path.  TEST INFRASTRUCTURE ONLY (see wos_oracle.h): the oracle, never
 * the product.  Compiled with -ffp-contract=off so every expression rounds
 * like the reference's C++17 build on x86-64 (no FMA contraction).
 *
 * Each function names the reference file:line it restates.  Expression
 * shapes (operand order of products and sums) follow the reference so the
 * results round identically; the comments say where this matters.
 */
#define _GNU_SOURCE
#include "wos_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------ PRNG */

/* include/wos/hash.hpp:7-12 */
uint64_t wo_splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

typedef struct {
    uint64_t s[4];
} xoshiro;

/* src/prng.cpp:6-15: the four state words are splitmix64 of the seed plus
 * multiples of the golden-ratio increment; an all-zero state becomes 1. */
static void rng_seed(xoshiro *r, uint64_t seed) {
    r->s[0] = wo_splitmix64(seed);
    r->s[1] = wo_splitmix64(seed + 0x9E3779B97F4A7C15ULL);
    r->s[2] = wo_splitmix64(seed + 0x3C6EF372FE94F82AULL);
    r->s[3] = wo_splitmix64(seed + 0xDAA66D2C7DDF743FULL);
    if (!(r->s[0] | r->s[1] | r->s[2] | r->s[3])) r->s[0] = 1;
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* xoshiro256++ step, include/wos/prng.hpp:14-24 */
static inline uint64_t rng_u64(xoshiro *r) {
    uint64_t *s = r->s;
    const uint64_t out = rotl(s[0] + s[3], 23) + s[0];
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return out;
}

/* include/wos/prng.hpp:27-29: top 53 bits scaled by 2^-53 */
static inline double rng_unit(xoshiro *r) {
    return (double)(rng_u64(r) >> 11) * (1.0 / 9007199254740992.0);
}

/* include/wos/prng.hpp:31-37: rejects an exact zero */
static inline double rng_unit_open(xoshiro *r) {
    double v;
    do {
        v = rng_unit(r);
    } while (v == 0.0);
    return v;
}

void wo_prng_u64(uint64_t seed, long long n, uint64_t *out) {
    xoshiro r;
    rng_seed(&r, seed);
    for (long long i = 0; i < n; ++i) out[i] = rng_u64(&r);
}

void wo_prng_unit(uint64_t seed, long long n, int open, double *out) {
    xoshiro r;
    rng_seed(&r, seed);
    for (long long i = 0; i < n; ++i) out[i] = open ? rng_unit_open(&r) : rng_unit(&r);
}

/* ------------------------------------------------------------------ mesh */

typedef struct {
    double x, y, z;
} vec3;

static inline double dmin_(double a, double b) { return a < b ? a : b; } /* fastmath.hpp:10 */
static inline double dmax_(double a, double b) { return a > b ? a : b; } /* fastmath.hpp:11 */

typedef struct {
    int dim;
    int n_prims;
    const double *verts;
    const int *prims;
    const int *bids;
} mesh_view;

static vec3 vert(const mesh_view *m, int v) {
    vec3 p;
    if (m->dim == 2) {
        p.x = m->verts[2 * v];
        p.y = m->verts[2 * v + 1];
        p.z = 0.0;
    } else {
        p.x = m->verts[3 * v];
        p.y = m->verts[3 * v + 1];
        p.z = m->verts[3 * v + 2];
    }
    return p;
}

/* src/mesh.cpp:297-322 */
static void mesh_bbox(const wo_problem *pb, double b[6]) {
    const int d = pb->dim;
    double xl = pb->verts[0], xu = xl, yl = pb->verts[1], yu = yl;
    double zl = d == 3 ? pb->verts[2] : 0.0, zu = zl;
    for (int i = 1; i < pb->n_verts; ++i) {
        const double *v = pb->verts + (size_t)d * i;
        if (v[0] < xl) xl = v[0]; else if (v[0] > xu) xu = v[0];
        if (v[1] < yl) yl = v[1]; else if (v[1] > yu) yu = v[1];
        if (d == 3) {
            if (v[2] < zl) zl = v[2]; else if (v[2] > zu) zu = v[2];
        }
    }
    b[0] = xl; b[1] = xu; b[2] = yl; b[3] = yu; b[4] = zl; b[5] = zu;
}

/* ------------------------------------------------------------------- BVH */

/* Node of the reference layout (include/wos/bvh.hpp:10-15): DFS order, left
 * child = node + 1, idx = right child (internal) or first leaf slot. */
typedef struct {
    double lo[3], hi[3];
    int count, idx;
} bnode;

/* Eberly cache per leaf slot (include/wos/npq.hpp:6-10, src/bvh.cpp:204-217). */
typedef struct {
    vec3 v0, e1, e2;
    double a, b, c, det, denom;
} ebcache;

typedef struct {
    mesh_view m;
    bnode *nodes;
    int n_nodes;
    int *prims;      /* leaf-order primitive ids */
    ebcache *eb;     /* 3D only, leaf order */
} bvh_t;

typedef struct {
    double lo[3], hi[3], c[3];
    int prim;
} bitem;

static int g_sort_axis; /* axis for the qsort comparator (single-threaded build) */

/* (coordinate, primitive index) order of src/bvh.cpp:143-171 */
static int cmp_item(const void *pa, const void *pb) {
    const bitem *a = (const bitem *)pa, *b = (const bitem *)pb;
    const double ca = a->c[g_sort_axis], cb = b->c[g_sort_axis];
    if (ca < cb) return -1;
    if (ca > cb) return 1;
    return (a->prim > b->prim) - (a->prim < b->prim);
}

/* src/bvh.cpp:174-230.  The reference partitions with nth_element; a full
 * sort by the same strict order puts the same set on each side (the order
 * is total), so node boxes and the tree shape match exactly; only the order
 * of primitives inside a leaf can differ. */
static int build_rec(bvh_t *t, bitem *it, int start, int end, int *node_ptr) {
    const int d = t->m.dim;
    const int node = (*node_ptr)++;
    bnode *nd = &t->nodes[node];
    for (int k = 0; k < 3; ++k) {
        nd->lo[k] = it[start].lo[k];
        nd->hi[k] = it[start].hi[k];
    }
    for (int i = start + 1; i < end; ++i) {
        for (int k = 0; k < d; ++k) {
            nd->lo[k] = dmin_(nd->lo[k], it[i].lo[k]);
            nd->hi[k] = dmax_(nd->hi[k], it[i].hi[k]);
        }
    }
    const int span = end - start;
    if (span <= 4) { /* LEAF_SIZE, src/bvh.cpp:15 */
        nd->count = span;
        nd->idx = start;
        for (int i = 0; i < span; ++i) {
            const int p = it[start + i].prim;
            t->prims[start + i] = p;
            if (d == 3) {
                const vec3 v0 = vert(&t->m, t->m.prims[3 * p]);
                const vec3 v1 = vert(&t->m, t->m.prims[3 * p + 1]);
                const vec3 v2 = vert(&t->m, t->m.prims[3 * p + 2]);
                ebcache *e = &t->eb[start + i];
                e->v0 = v0;
                e->e1.x = v1.x - v0.x; e->e1.y = v1.y - v0.y; e->e1.z = v1.z - v0.z;
                e->e2.x = v2.x - v0.x; e->e2.y = v2.y - v0.y; e->e2.z = v2.z - v0.z;
                e->a = e->e1.x * e->e1.x + e->e1.y * e->e1.y + e->e1.z * e->e1.z;
                e->b = e->e1.x * e->e2.x + e->e1.y * e->e2.y + e->e1.z * e->e2.z;
                e->c = e->e2.x * e->e2.x + e->e2.y * e->e2.y + e->e2.z * e->e2.z;
                e->det = e->a * e->c - e->b * e->b;
                e->denom = e->a - 2 * e->b + e->c;
            }
        }
        return node;
    }
    nd->count = 0;
    const double ex = nd->hi[0] - nd->lo[0];
    const double ey = nd->hi[1] - nd->lo[1];
    int axis;
    if (d == 2) {
        axis = ex >= ey ? 0 : 1;
    } else {
        const double ez = nd->hi[2] - nd->lo[2];
        axis = (ex >= ey) ? (ex >= ez ? 0 : 2) : (ey >= ez ? 1 : 2);
    }
    const int mid = (start + end) / 2;
    g_sort_axis = axis;
    qsort(it + start, (size_t)span, sizeof(bitem), cmp_item);
    build_rec(t, it, start, mid, node_ptr);
    const int right = build_rec(t, it, mid, end, node_ptr);
    t->nodes[node].idx = right;
    return node;
}

static pthread_mutex_t g_build_lock = PTHREAD_MUTEX_INITIALIZER;

/* src/bvh.cpp:234-253 (prim bbox and centroid: src/mesh.cpp:324-366) */
static void bvh_build(bvh_t *t, const wo_problem *pb) {
    const int d = pb->dim, n = pb->n_prims;
    t->m.dim = d;
    t->m.n_prims = n;
    t->m.verts = pb->verts;
    t->m.prims = pb->prims;
    t->m.bids = pb->boundary_ids;
    t->nodes = (bnode *)calloc((size_t)(2 * n), sizeof(bnode));
    t->prims = (int *)calloc((size_t)n, sizeof(int));
    t->eb = d == 3 ? (ebcache *)calloc((size_t)n, sizeof(ebcache)) : NULL;
    bitem *it = (bitem *)calloc((size_t)n, sizeof(bitem));
    for (int p = 0; p < n; ++p) {
        bitem *b = &it[p];
        b->prim = p;
        memset(b->lo, 0, sizeof(b->lo));
        memset(b->hi, 0, sizeof(b->hi));
        memset(b->c, 0, sizeof(b->c));
        if (d == 2) {
            const vec3 s0 = vert(&t->m, pb->prims[2 * p]), s1 = vert(&t->m, pb->prims[2 * p + 1]);
            b->lo[0] = fmin(s0.x, s1.x); b->lo[1] = fmin(s0.y, s1.y);
            b->hi[0] = fmax(s0.x, s1.x); b->hi[1] = fmax(s0.y, s1.y);
            b->c[0] = (s0.x + s1.x) / 2.0;
            b->c[1] = (s0.y + s1.y) / 2.0;
        } else {
            const vec3 v0 = vert(&t->m, pb->prims[3 * p]);
            const vec3 v1 = vert(&t->m, pb->prims[3 * p + 1]);
            const vec3 v2 = vert(&t->m, pb->prims[3 * p + 2]);
            b->lo[0] = fmin(fmin(v0.x, v1.x), v2.x);
            b->lo[1] = fmin(fmin(v0.y, v1.y), v2.y);
            b->lo[2] = fmin(fmin(v0.z, v1.z), v2.z);
            b->hi[0] = fmax(fmax(v0.x, v1.x), v2.x);
            b->hi[1] = fmax(fmax(v0.y, v1.y), v2.y);
            b->hi[2] = fmax(fmax(v0.z, v1.z), v2.z);
            b->c[0] = (v0.x + v1.x + v2.x) / 3.0;
            b->c[1] = (v0.y + v1.y + v2.y) / 3.0;
            b->c[2] = (v0.z + v1.z + v2.z) / 3.0;
        }
    }
    int node_ptr = 0;
    pthread_mutex_lock(&g_build_lock);
    build_rec(t, it, 0, n, &node_ptr);
    pthread_mutex_unlock(&g_build_lock);
    t->n_nodes = node_ptr;
    free(it);
}

static void bvh_free(bvh_t *t) {
    free(t->nodes);
    free(t->prims);
    free(t->eb);
}

int wo_build_bvh(const wo_problem *pb, double *node_boxes, int *node_counts, int *node_idx,
                 int *prims) {
    bvh_t t;
    bvh_build(&t, pb);
    const int d = pb->dim;
    for (int i = 0; i < t.n_nodes; ++i) {
        double *b = node_boxes + (size_t)(2 * d) * i;
        for (int k = 0; k < d; ++k) {
            b[k] = t.nodes[i].lo[k];
            b[d + k] = t.nodes[i].hi[k];
        }
        node_counts[i] = t.nodes[i].count;
        node_idx[i] = t.nodes[i].idx;
    }
    memcpy(prims, t.prims, sizeof(int) * (size_t)pb->n_prims);
    const int n = t.n_nodes;
    bvh_free(&t);
    return n;
}

/* ------------------------------------------------------ closest points */

/* src/bvh.cpp:111-121 */
static inline double aabb_d_sq(const bnode *b, int d, const double p[3]) {
    double s = 0.0;
    const double dx = dmax_(0.0, dmax_(b->lo[0] - p[0], p[0] - b->hi[0]));
    const double dy = dmax_(0.0, dmax_(b->lo[1] - p[1], p[1] - b->hi[1]));
    if (d == 2) return dx * dx + dy * dy;
    const double dz = dmax_(0.0, dmax_(b->lo[2] - p[2], p[2] - b->hi[2]));
    s = dx * dx + dy * dy + dz * dz;
    return s;
}

/* src/npq.cpp:8-29 */
static double npq_seg(vec3 s0, vec3 s1, const double p[3], double nearest[2]) {
    const double vx = s1.x - s0.x, vy = s1.y - s0.y;
    const double wx = p[0] - s0.x, wy = p[1] - s0.y;
    const double vv = vx * vx + vy * vy;
    const double wv = wx * vx + wy * vy;
    double par = (vv > 0.0) ? wv / vv : 0.0;
    if (par < 0.0) par = 0.0;
    if (par > 1.0) par = 1.0;
    nearest[0] = s0.x + par * vx;
    nearest[1] = s0.y + par * vy;
    const double dx = p[0] - nearest[0], dy = p[1] - nearest[1];
    return dx * dx + dy * dy;
}

/* Eberly's seven-region closest point on a triangle, src/npq.cpp:52-189 */
static double eberly(const double p[3], double nearest[3], const ebcache *e) {
    const double a = e->a, b = e->b, c = e->c, det = e->det, denom = e->denom;
    const double bpx = e->v0.x - p[0], bpy = e->v0.y - p[1], bpz = e->v0.z - p[2];
    const double d = e->e1.x * bpx + e->e1.y * bpy + e->e1.z * bpz;
    const double ee = e->e2.x * bpx + e->e2.y * bpy + e->e2.z * bpz;
    double s = b * ee - c * d;
    double t = b * d - a * ee;
    if (s + t <= det) {
        if (s < 0) {
            if (t < 0) { /* region 4 */
                if (d < 0) {
                    t = 0;
                    s = (-d >= a) ? 1 : -d / a;
                } else {
                    s = 0;
                    if (ee >= 0) t = 0;
                    else if (-ee >= c) t = 1;
                    else t = -ee / c;
                }
            } else { /* region 3 */
                s = 0;
                if (ee >= 0) t = 0;
                else if (-ee >= c) t = 1;
                else t = -ee / c;
            }
        } else if (t < 0) { /* region 5 */
            t = 0;
            if (d >= 0) s = 0;
            else if (-d >= a) s = 1;
            else s = -d / a;
        } else { /* region 0 */
            s /= det;
            t /= det;
        }
    } else {
        if (s < 0) { /* region 2 */
            const double bd = b + d, ce = c + ee;
            if (ce > bd) {
                const double numer = ce - bd;
                s = (numer >= denom) ? 1 : numer / denom;
                t = 1 - s;
            } else {
                s = 0;
                if (ce <= 0) t = 1;
                else if (ee >= 0) t = 0;
                else t = -ee / c;
            }
        } else if (t < 0) { /* region 6 */
            const double be = b + ee, ad = a + d;
            if (ad > be) {
                const double numer = ad - be;
                t = (numer >= denom) ? 1 : numer / denom;
                s = 1 - t;
            } else {
                t = 0;
                if (ad <= 0) s = 1;
                else if (d >= 0) s = 0;
                else s = -d / a;
            }
        } else { /* region 1 */
            const double numer = (c + ee) - (b + d);
            if (numer <= 0) s = 0;
            else s = (numer >= denom) ? 1 : numer / denom;
            t = 1 - s;
        }
    }
    nearest[0] = e->v0.x + s * e->e1.x + t * e->e2.x;
    nearest[1] = e->v0.y + s * e->e1.y + t * e->e2.y;
    nearest[2] = e->v0.z + s * e->e1.z + t * e->e2.z;
    const double dx = nearest[0] - p[0], dy = nearest[1] - p[1], dz = nearest[2] - p[2];
    return dx * dx + dy * dy + dz * dz;
}

typedef struct {
    double dist;
    double point[3];
    int prim;
    int bid;
    int tri;    /* nearest primitive id in both dimensions (prim is -1 in 3D, as in
                   the reference, whose 3D query returns no id) */
    long long pops, tests;
} npq_result;

/* src/bvh.cpp:295-387: stack traversal, nearer child popped first, node
 * pruned when its box distance is >= the best squared distance, first
 * strict minimum kept. */
static npq_result bvh_npq(const bvh_t *t, const double p[3]) {
    const int d = t->m.dim;
    npq_result r;
    double best = INFINITY;
    r.point[0] = r.point[1] = r.point[2] = 0.0;
    r.prim = -1;
    r.bid = -1;
    r.tri = -1;
    r.pops = r.tests = 0;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const int cur = stack[--sp];
        const bnode *nd = &t->nodes[cur];
        ++r.pops;
        if (aabb_d_sq(nd, d, p) >= best) continue;
        if (nd->count > 0) {
            for (int i = 0; i < nd->count; ++i) {
                double q[3] = {0.0, 0.0, 0.0};
                double dsq;
                int prim = -1;
                ++r.tests;
                if (d == 2) {
                    prim = t->prims[nd->idx + i];
                    dsq = npq_seg(vert(&t->m, t->m.prims[2 * prim]),
                                  vert(&t->m, t->m.prims[2 * prim + 1]), p, q);
                } else {
                    dsq = eberly(p, q, &t->eb[nd->idx + i]);
                }
                if (dsq < best) {
                    best = dsq;
                    r.point[0] = q[0];
                    r.point[1] = q[1];
                    r.point[2] = q[2];
                    r.tri = t->prims[nd->idx + i];
                    if (d == 2) {
                        r.prim = prim;
                        r.bid = t->m.bids ? t->m.bids[prim] : 0;
                    }
                }
            }
        } else {
            const int l = cur + 1, rr = nd->idx;
            const double ld = aabb_d_sq(&t->nodes[l], d, p);
            const double rd = aabb_d_sq(&t->nodes[rr], d, p);
            if (ld <= rd) {
                stack[sp++] = rr;
                stack[sp++] = l;
            } else {
                stack[sp++] = l;
                stack[sp++] = rr;
            }
        }
    }
    r.dist = sqrt(best);
    return r;
}

void wo_npq(const wo_problem *pb, const double *points, long long n, double *dist,
            double *nearest, int *prim_id, int *boundary_id, long long *visits) {
    bvh_t t;
    bvh_build(&t, pb);
    const int d = pb->dim;
    for (long long q = 0; q < n; ++q) {
        double p[3] = {points[d * q], points[d * q + 1], d == 3 ? points[d * q + 2] : 0.0};
        const npq_result r = bvh_npq(&t, p);
        dist[q] = r.dist;
        for (int k = 0; k < d; ++k) nearest[d * q + k] = r.point[k];
        prim_id[q] = r.prim;
        boundary_id[q] = r.bid;
        if (visits) {
            visits[2 * q] = r.pops;
            visits[2 * q + 1] = r.tests;
        }
    }
    bvh_free(&t);
}

/* --------------------------------------------------- inside / outside */

/* src/inside.cpp:117-137: Sunday's winding number over every segment */
static int winding_number(const mesh_view *m, const double p[2]) {
    int wn = 0;
    for (int s = 0; s < m->n_prims; ++s) {
        const vec3 s0 = vert(m, m->prims[2 * s]), s1 = vert(m, m->prims[2 * s + 1]);
        const double area = (s1.x - s0.x) * (p[1] - s0.y) - (p[0] - s0.x) * (s1.y - s0.y);
        if (s0.y <= p[1]) {
            if (s1.y > p[1] && area > 0) wn++;
        } else {
            if (s1.y <= p[1] && area < 0) wn--;
        }
    }
    return wn;
}

void wo_winding_numbers(const wo_problem *pb, const double *points, long long n, int *wn) {
    mesh_view m = {2, pb->n_prims, pb->verts, pb->prims, pb->boundary_ids};
    for (long long q = 0; q < n; ++q) wn[q] = winding_number(&m, points + 2 * q);
}

#define RAY_EPS 1e-9 /* INTERSECTION_EPSILON, src/inside.cpp:14 */

/* src/inside.cpp:18-25 */
static vec3 random_unit_direction(xoshiro *rng) {
    const double u = rng_unit(rng);
    const double v = rng_unit(rng);
    const double z = 2 * u - 1;
    const double phi = 2 * M_PI * v;
    const double r = sqrt(1 - z * z);
    vec3 o = {r * cos(phi), r * sin(phi), z};
    return o;
}

/* src/inside.cpp:27-51 */
static int update_ray_interval(double origin, double dir, double bmin, double bmax,
                               double *tmin, double *tmax) {
    const double extent_scale = dmax_(1.0, fabs(bmax - bmin));
    double cs = 1.0;
    if (fabs(origin) > cs) cs = fabs(origin);
    if (fabs(bmin) > cs) cs = fabs(bmin);
    if (fabs(bmax) > cs) cs = fabs(bmax);
    const double padding = RAY_EPS * extent_scale + 16.0 * 2.220446049250313e-16 * cs;
    bmin -= padding;
    bmax += padding;
    if (dir == 0.0) return origin >= bmin && origin <= bmax;
    double t0 = (bmin - origin) / dir;
    double t1 = (bmax - origin) / dir;
    if (t0 > t1) {
        const double tmp = t0;
        t0 = t1;
        t1 = tmp;
    }
    /* std::max(t_min, t0) keeps t_min unless t_min < t0; std::min likewise */
    *tmin = (*tmin < t0) ? t0 : *tmin;
    *tmax = (t1 < *tmax) ? t1 : *tmax;
    return *tmin <= *tmax;
}

/* src/inside.cpp:53-62 */
static int ray_hits_box(const double o[3], vec3 r, const bnode *b) {
    double tmin = 0.0, tmax = INFINITY;
    return update_ray_interval(o[0], r.x, b->lo[0], b->hi[0], &tmin, &tmax) &&
           update_ray_interval(o[1], r.y, b->lo[1], b->hi[1], &tmin, &tmax) &&
           update_ray_interval(o[2], r.z, b->lo[2], b->hi[2], &tmin, &tmax);
}

static inline vec3 cross3(vec3 a, vec3 b) {
    vec3 o = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return o;
}
static inline double dot3(vec3 a, vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

enum { HIT_MISS = 0, HIT_HIT = 1, HIT_AMBIGUOUS = 2 };

/* Moller-Trumbore with the reference's ambiguity bands, src/inside.cpp:140-182 */
static int moller_trumbore(const double p[3], vec3 ray, vec3 a, vec3 b, vec3 c) {
    const vec3 e1 = {b.x - a.x, b.y - a.y, b.z - a.z};
    const vec3 e2 = {c.x - a.x, c.y - a.y, c.z - a.z};
    const vec3 s = {p[0] - a.x, p[1] - a.y, p[2] - a.z};
    const vec3 rxe2 = cross3(ray, e2);
    const double det = dot3(e1, rxe2);
    const vec3 normal = cross3(e1, e2);
    const double nlen = sqrt(dot3(normal, normal));
    const double det_tol = RAY_EPS * nlen;
    if (fabs(det) <= det_tol) {
        if (nlen == 0.0) return HIT_MISS;
        double es = 1.0;
        const double l1 = sqrt(dot3(e1, e1)), l2 = sqrt(dot3(e2, e2));
        if (l1 > es) es = l1;
        if (l2 > es) es = l2;
        const double plane = fabs(dot3(normal, s)) / nlen;
        return plane <= RAY_EPS * es ? HIT_AMBIGUOUS : HIT_MISS;
    }
    const double u = dot3(s, rxe2) / det;
    if (u < -RAY_EPS || u - 1.0 > RAY_EPS) return HIT_MISS;
    const vec3 sxe1 = cross3(s, e1);
    const double v = dot3(ray, sxe1) / det;
    if (v < -RAY_EPS || u + v - 1.0 > RAY_EPS) return HIT_MISS;
    const double tt = dot3(e2, sxe1) / det;
    if (tt <= RAY_EPS) return HIT_MISS;
    const double w = 1.0 - u - v;
    if (u <= RAY_EPS || v <= RAY_EPS || w <= RAY_EPS) return HIT_AMBIGUOUS;
    return HIT_HIT;
}

/* src/inside.cpp:78-111: every node whose padded box the ray meets, left
 * subtree first; an ambiguous triangle ends the cast */
static int count_ray_hits(const bvh_t *t, const double p[3], vec3 ray, int *ambiguous) {
    int hits = 0;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    *ambiguous = 0;
    while (sp > 0) {
        const int ni = stack[--sp];
        const bnode *nd = &t->nodes[ni];
        if (!ray_hits_box(p, ray, nd)) continue;
        if (nd->count > 0) {
            for (int i = 0; i < nd->count; ++i) {
                const int tri = t->prims[nd->idx + i];
                const vec3 a = vert(&t->m, t->m.prims[3 * tri]);
                const vec3 b = vert(&t->m, t->m.prims[3 * tri + 1]);
                const vec3 c = vert(&t->m, t->m.prims[3 * tri + 2]);
                const int h = moller_trumbore(p, ray, a, b, c);
                if (h == HIT_AMBIGUOUS) {
                    *ambiguous = 1;
                    return hits;
                }
                if (h == HIT_HIT) ++hits;
            }
        } else {
            stack[sp++] = nd->idx;
            stack[sp++] = ni + 1;
        }
    }
    return hits;
}

/* src/inside.cpp:228-260: up to max_attempts rays, ambiguous rays retried,
 * majority of three valid parities */
static int classify_3d(const bvh_t *t, const double p[3], double bdist, double btol,
                       int max_attempts, xoshiro *rng, int *retries) {
    *retries = 0;
    if (bdist <= btol) return 2;
    int valid = 0, votes = 0;
    for (int a = 0; a < max_attempts && valid < 3; ++a) {
        const vec3 ray = random_unit_direction(rng);
        int amb;
        const int hits = count_ray_hits(t, p, ray, &amb);
        if (amb) {
            ++*retries;
            continue;
        }
        votes += hits & 1;
        ++valid;
    }
    if (valid < 3) return 3;
    return votes > 1 ? 1 : 0;
}

void wo_classify_3d(const wo_problem *pb, const double *points, const uint64_t *seeds,
                    long long n, double btol, unsigned char *location, int *retries) {
    bvh_t t;
    bvh_build(&t, pb);
    for (long long q = 0; q < n; ++q) {
        const double *p = points + 3 * q;
        const npq_result r = bvh_npq(&t, p);
        xoshiro rng;
        rng_seed(&rng, seeds[q]);
        location[q] = (unsigned char)classify_3d(&t, p, r.dist, btol, pb->max_ray_attempts,
                                                 &rng, &retries[q]);
    }
    bvh_free(&t);
}

/* ------------------------------------------------------ Bessel functions */

#define BESSEL_ASYMPTOTIC_START 50.0 /* include/wos/bessel.hpp:13 */

/* Hankel asymptotic series of e^-x I0(x) (alternating=0) and e^x K0(x)
 * (alternating=1) up to the leading factor: terms t_k = t_{k-1} (2k-1)^2/(8kx),
 * stopped when they start to grow or fall below one ulp of the sum
 * (the same truncation rule as include/wos/bessel.hpp:16-36). */
static double hankel_sum(double x, int alternating) {
    double sum = 1.0, term = 1.0, prev = INFINITY;
    for (int k = 1; k <= 24; ++k) {
        const double odd = (double)(2 * k - 1);
        double f = odd * odd / (8.0 * x * (double)k);
        if (alternating) f = -f;
        term *= f;
        const double mag = fabs(term);
        if (mag > prev) break;
        sum += term;
        if (mag <= 2.220446049250313e-16 * fabs(sum)) break;
        prev = mag;
    }
    return sum;
}

/* I0 by its power series sum (x^2/4)^k / (k!)^2: every term is positive, so
 * the sum is well conditioned for all x < 50. */
static double i0_series(double x) {
    const double q = 0.25 * x * x;
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 500; ++k) {
        term *= q / ((double)k * (double)k);
        sum += term;
        if (term <= 1e-17 * sum) break;
    }
    return sum;
}

/* e^x K0(x) for x > 2 from K0(x) = integral_0^inf exp(-x cosh t) dt.  With
 * s = sinh(t/2) and s = w / sqrt(2x):
 *   e^x K0(x) = sqrt(2/x) * integral_0^inf exp(-w^2) / sqrt(1 + w^2/(2x)) dw.
 * The integrand is even and analytic for |Im w| < sqrt(2x) >= 2, so the
 * trapezoidal rule with step 1/4 converges to double precision; 27 nodes
 * reach exp(-w^2) < 1e-18. */
static double k0_scaled_integral(double x) {
    const double h = 0.25;
    const double inv2x = 1.0 / (2.0 * x);
    double sum = 0.5;
    for (int k = 1; k <= 27; ++k) {
        const double w = h * (double)k;
        sum += exp(-w * w) / sqrt(1.0 + w * w * inv2x);
    }
    return sqrt(2.0 / x) * h * sum;
}

/* K0 for 0 < x <= 2 by its series
 *   K0(x) = -(ln(x/2) + gamma) I0(x) + sum_{k>=1} (x^2/4)^k / (k!)^2 H_k. */
static double k0_series(double x) {
    const double gamma = 0.57721566490153286061;
    const double q = 0.25 * x * x;
    double term = 1.0, h = 0.0, sum = 0.0;
    for (int k = 1; k < 60; ++k) {
        term *= q / ((double)k * (double)k);
        h += 1.0 / (double)k;
        sum += term * h;
        if (term * h <= 1e-18 * fabs(sum)) break;
    }
    return -(log(0.5 * x) + gamma) * i0_series(x) + sum;
}

/* include/wos/bessel.hpp:39-47 */
static double i0_scaled(double x) {
    x = fabs(x);
    if (x < BESSEL_ASYMPTOTIC_START) return exp(-x) * i0_series(x);
    return hankel_sum(x, 0) / sqrt(2.0 * M_PI * x);
}

/* include/wos/bessel.hpp:49-57 */
static double k0_scaled(double x) {
    if (x < 0.0) return NAN;
    if (x == 0.0) return INFINITY;
    if (x < BESSEL_ASYMPTOTIC_START) {
        if (x <= 2.0) return exp(x) * k0_series(x);
        return k0_scaled_integral(x);
    }
    return sqrt(M_PI / (2.0 * x)) * hankel_sum(x, 1);
}

/* include/wos/bessel.hpp:59-68 */
static double log_i0(double x) {
    x = fabs(x);
    return x + log(i0_scaled(x));
}
static double log_k0(double x) {
    if (x < 0.0) return NAN;
    if (x == 0.0) return INFINITY;
    return -x + log(k0_scaled(x));
}

void wo_bessel(const double *x, long long n, double *out) {
    for (long long i = 0; i < n; ++i) {
        out[4 * i + 0] = i0_scaled(x[i]);
        out[4 * i + 1] = k0_scaled(x[i]);
        out[4 * i + 2] = log_i0(x[i]);
        out[4 * i + 3] = log_k0(x[i]);
    }
}

/* Series J0 truncated when a term drops below 1e-8, include/wos/fastmath.hpp:15-28 */
static double bessel_j0(double x) {
    const double hx = 0.25 * x * x;
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 200; ++k) {
        term *= hx / (double)(k * k);
        if (term < 1e-8) return sum;
        sum += (k % 2 == 0 ? term : -term);
    }
    return sum;
}

/* include/wos/fastmath.hpp:32-50 */
static double bessel_y0(double x) {
    const double hx = 0.25 * x * x;
    const double j0 = (2.0 / M_PI) * (log(x / 2.0) + 0.577215664901532860606512090082402431) *
                      bessel_j0(x);
    double hk = 0.0, term = 1.0, sum = 0.0;
    for (int k = 1; k < 200; ++k) {
        hk += 1.0 / (double)k;
        term *= hx / (double)(k * k);
        const double prod = hk * term;
        sum += (k % 2 == 0 ? prod : -prod);
        if (prod < 1e-8) break;
    }
    return j0 - (2.0 / M_PI) * sum;
}

void wo_j0y0(const double *x, long long n, double *j0, double *y0) {
    for (long long i = 0; i < n; ++i) {
        j0[i] = bessel_j0(x[i]);
        y0[i] = bessel_y0(x[i]);
    }
}

/* ------------------------------------------------- Green's functions */

/* include/wos/poisson.hpp:14-20 */
static double pg_green_2d(double R, double r) {
    if (!(r > 0.0) || r > R || R <= 0.0) return NAN;
    if (r == R) return 0.0;
    return log(R / r) / (2.0 * M_PI);
}
static double pg_mass_2d(double R) { return R * R / 4.0; } /* poisson.hpp:22-24 */
/* poisson.hpp:29-32: r/R = sqrt(U V) */
static double pg_sample_radius_2d(double R, xoshiro *rng) {
    const double u = rng_unit_open(rng);
    const double v = rng_unit_open(rng);
    return R * sqrt(u * v);
}
/* poisson.hpp:34-41 */
static double pg_green_3d(double R, double r) {
    if (!(r > 0.0) || r > R || R <= 0.0) return NAN;
    if (r == R) return 0.0;
    return (R - r) / (4.0 * M_PI * r * R);
}
static double pg_mass_3d(double R) { return R * R / 6.0; } /* poisson.hpp:43-45 */
/* poisson.hpp:47-51: r/R ~ Beta(2,2) from two Gamma(2) variates */
static double pg_sample_radius_3d(double R, xoshiro *rng) {
    double u = rng_unit_open(rng), v = rng_unit_open(rng);
    const double a = -log(u * v);
    u = rng_unit_open(rng);
    v = rng_unit_open(rng);
    const double b = -log(u * v);
    return R * a / (a + b);
}

/* include/wos/screened.hpp:14-22 */
static double sc_weight_2d(double alpha, double R) {
    const double x = alpha * R;
    if (x == 0.0) return 1.0;
    if (x < 1e-3) {
        const double x2 = x * x;
        return 1.0 - x2 / 4.0 + 3.0 * x2 * x2 / 64.0;
    }
    return exp(-log_i0(x));
}
/* screened.hpp:24-41 */
static double sc_green_2d(double alpha, double R, double r) {
    if (!(r > 0.0) || r > R || R <= 0.0) return NAN;
    if (r == R) return 0.0;
    const double x = alpha * r, X = alpha * R;
    if (X < 1e-5) return pg_green_2d(R, r);
    const double la = log_k0(x);
    const double lb = log_i0(x) + log_k0(X) - log_i0(X);
    double delta = lb - la;
    if (delta > 0.0) delta = 0.0;
    return exp(la) * (-expm1(delta)) / (2.0 * M_PI);
}
/* screened.hpp:43-52 */
static double sc_mass_2d(double alpha, double R) {
    const double x = alpha * R;
    if (x < 1e-3) {
        const double x2 = x * x;
        return R * R * (1.0 / 4.0 - 3.0 * x2 / 64.0 + 19.0 * x2 * x2 / 2304.0);
    }
    return -expm1(-log_i0(x)) / (alpha * alpha);
}
/* screened.hpp:54-62 */
static double sc_weight_3d(double alpha, double R) {
    const double x = alpha * R;
    if (x == 0.0) return 1.0;
    if (x < 1e-3) {
        const double x2 = x * x;
        return 1.0 - x2 / 6.0 + 7.0 * x2 * x2 / 360.0;
    }
    return 2.0 * x * exp(-x) / (-expm1(-2.0 * x));
}
/* screened.hpp:64-78 */
static double sc_green_3d(double alpha, double R, double r) {
    if (!(r > 0.0) || r > R || R <= 0.0) return NAN;
    if (r == R) return 0.0;
    const double x = alpha * r, X = alpha * R;
    if (X < 1e-5) return pg_green_3d(R, r);
    const double ratio = exp(-x) * (-expm1(-2.0 * (X - x))) / (-expm1(-2.0 * X));
    return ratio / (4.0 * M_PI * r);
}
/* screened.hpp:80-89 */
static double sc_mass_3d(double alpha, double R) {
    const double x = alpha * R;
    if (x < 1e-3) {
        const double x2 = x * x;
        return R * R * (1.0 / 6.0 - 7.0 * x2 / 360.0 + 31.0 * x2 * x2 / 15120.0);
    }
    return (1.0 - sc_weight_3d(alpha, R)) / (alpha * alpha);
}
/* screened.hpp:91-93 with std::min/std::max argument order (NaN -> 1) */
static double clamp_probability(double v) {
    const double lo = (v < 1.0) ? v : 1.0;
    return (0.0 < lo) ? lo : 0.0;
}
/* screened.hpp:95-99 */
static double sc_normal(xoshiro *rng) {
    const double radius = sqrt(-2.0 * log(rng_unit_open(rng)));
    const double angle = 2.0 * M_PI * rng_unit(rng);
    return radius * cos(angle);
}
/* screened.hpp:103-129 */
static double sc_sample_radius_2d(double alpha, double R, xoshiro *rng) {
    const double X = alpha * R;
    for (;;) {
        double r, acc;
        if (X < 2.0) {
            r = pg_sample_radius_2d(R, rng);
            const double proposal = pg_green_2d(R, r);
            acc = sc_green_2d(alpha, R, r) / proposal;
        } else {
            const double time = -log(rng_unit_open(rng)) / (alpha * alpha);
            r = sqrt(-4.0 * time * log(rng_unit_open(rng)));
            if (r >= R) continue;
            const double x = alpha * r;
            const double lr = log_i0(x) + log_k0(X) - log_i0(X) - log_k0(x);
            acc = -expm1((lr < 0.0) ? lr : 0.0);
        }
        if (rng_unit(rng) < clamp_probability(acc)) return r;
    }
}
/* screened.hpp:131-156 */
static double sc_sample_radius_3d(double alpha, double R, xoshiro *rng) {
    const double X = alpha * R;
    for (;;) {
        double r, acc;
        if (X < 2.0) {
            r = pg_sample_radius_3d(R, rng);
            const double proposal = pg_green_3d(R, r);
            acc = sc_green_3d(alpha, R, r) / proposal;
        } else {
            const double time = -log(rng_unit_open(rng)) / (alpha * alpha);
            const double scale = sqrt(2.0 * time);
            const double x0 = scale * sc_normal(rng);
            const double x1 = scale * sc_normal(rng);
            const double x2 = scale * sc_normal(rng);
            r = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
            if (r >= R) continue;
            const double x = alpha * r;
            acc = (-expm1(-2.0 * (X - x))) / (-expm1(-2.0 * X));
        }
        if (rng_unit(rng) < clamp_probability(acc)) return r;
    }
}

void wo_screened_kernels(const double *alpha, const double *R, const double *r, long long n,
                         double *out) {
    for (long long i = 0; i < n; ++i) {
        out[6 * i + 0] = sc_weight_2d(alpha[i], R[i]);
        out[6 * i + 1] = sc_green_2d(alpha[i], R[i], r[i]);
        out[6 * i + 2] = sc_mass_2d(alpha[i], R[i]);
        out[6 * i + 3] = sc_weight_3d(alpha[i], R[i]);
        out[6 * i + 4] = sc_green_3d(alpha[i], R[i], r[i]);
        out[6 * i + 5] = sc_mass_3d(alpha[i], R[i]);
    }
}

void wo_screened_samples(int dim, double alpha, double R, uint64_t seed, long long n,
                         double *out) {
    xoshiro rng;
    rng_seed(&rng, seed);
    for (long long i = 0; i < n; ++i) {
        out[i] = dim == 2 ? sc_sample_radius_2d(alpha, R, &rng) : sc_sample_radius_3d(alpha, R, &rng);
    }
}

void wo_poisson_green(int dim, double R, const double *r, long long n, uint64_t seed,
                      double *green, double *mass, double *samples) {
    xoshiro rng;
    rng_seed(&rng, seed);
    for (long long i = 0; i < n; ++i) {
        green[i] = dim == 2 ? pg_green_2d(R, r[i]) : pg_green_3d(R, r[i]);
        mass[i] = dim == 2 ? pg_mass_2d(R) : pg_mass_3d(R);
        samples[i] = dim == 2 ? pg_sample_radius_2d(R, &rng) : pg_sample_radius_3d(R, &rng);
    }
}

double wo_screened_epsilon(double requested, double alpha) {
    const double limit = 0.05 / alpha; /* max_terminal_alpha_radius / alpha */
    return (limit < requested) ? limit : requested;
}

/* --------------------------------------------------- sphere sampling */

/* src/wos.cpp:9-16: exit point uniform on the circle; theta = (U*2)*pi */
static void step_2d(const double c[3], double R, xoshiro *rng, double o[3]) {
    const double theta = rng_unit(rng) * 2 * M_PI;
    o[0] = c[0] + R * cos(theta);
    o[1] = c[1] + R * sin(theta);
    o[2] = 0.0;
}
/* src/wos.cpp:17-30 */
static void step_3d(const double c[3], double R, xoshiro *rng, double o[3]) {
    const double u = rng_unit(rng);
    const double v = rng_unit(rng);
    const double z = 2 * u - 1;
    const double phi = 2 * M_PI * v;
    const double r = sqrt(1 - z * z);
    o[0] = c[0] + R * r * cos(phi);
    o[1] = c[1] + R * r * sin(phi);
    o[2] = c[2] + R * z;
}
/* src/wos.cpp:33-41: uniform in the disk */
static void ball_2d(const double c[3], double R, xoshiro *rng, double o[3]) {
    const double theta = rng_unit(rng) * 2 * M_PI;
    const double r = R * sqrt(rng_unit_open(rng));
    o[0] = c[0] + r * cos(theta);
    o[1] = c[1] + r * sin(theta);
    o[2] = 0.0;
}
/* src/wos.cpp:42-56: uniform in the ball */
static void ball_3d(const double c[3], double R, xoshiro *rng, double o[3]) {
    const double u = rng_unit(rng);
    const double v = rng_unit(rng);
    const double w = rng_unit_open(rng);
    const double z = 2 * u - 1;
    const double phi = 2 * M_PI * v;
    const double surf = sqrt(1 - z * z);
    const double vol = R * cbrt(w);
    o[0] = c[0] + vol * surf * cos(phi);
    o[1] = c[1] + vol * surf * sin(phi);
    o[2] = c[2] + vol * z;
}

void wo_steps(int dim, const double *centre, double radius, uint64_t seed, long long n,
              double *steps, double *balls) {
    xoshiro rng;
    rng_seed(&rng, seed);
    double c[3] = {centre[0], centre[1], dim == 3 ? centre[2] : 0.0};
    for (long long i = 0; i < n; ++i) {
        double a[3], b[3];
        if (dim == 2) {
            step_2d(c, radius, &rng, a);
            ball_2d(c, radius, &rng, b);
        } else {
            step_3d(c, radius, &rng, a);
            ball_3d(c, radius, &rng, b);
        }
        for (int k = 0; k < dim; ++k) {
            steps[dim * i + k] = a[k];
            balls[dim * i + k] = b[k];
        }
    }
}

/* ---------------------------------------------------------- equations */

typedef struct {
    int kind, dim, source_mode;
    double alpha;
} equation;

static int eq_has_source(const equation *e) {
    /* poisson (src/equations/poisson.cpp:16,76); screened 2D only
     * (screened_poisson.cpp:41 vs :94) */
    return e->kind == WO_POISSON || (e->kind == WO_SCREENED_POISSON && e->dim == 2);
}
static int eq_has_screening(const equation *e) {
    return e->kind == WO_SCREENED_POISSON || e->kind == WO_HELMHOLTZ;
}

/* degree-5 harmonic boundary data, src/equations/laplace.cpp:30-36 (and
 * poisson.cpp:93-99, screened_poisson.cpp:103-109) */
static double harmonic_y5(const double p[3]) {
    const double r_sq = p[0] * p[0] + p[1] * p[1];
    const double z = p[2];
    const double y50 = z * (8 * z * z * z * z - 40 * z * z * r_sq + 15 * r_sq * r_sq);
    const double y5m3 = (8 * z * z - r_sq) * p[1] * (3 * p[0] * p[0] - p[1] * p[1]);
    return y50 + 4.0 * y5m3;
}

static double eq_boundary(const equation *e, const double p[3], int bid) {
    switch (e->kind) {
        case WO_LAPLACE: /* laplace.cpp:16-18 */
        case WO_SCREENED_POISSON: /* screened_poisson.cpp:62-64 */
            if (e->dim == 2) return bid == 0 ? p[0] * p[0] - p[1] * p[1] : 0.0;
            return harmonic_y5(p);
        case WO_POISSON: /* poisson.cpp:46-51 */
            return e->dim == 2 ? 0.0 : harmonic_y5(p);
        default: /* helmholtz.cpp:26-30, 59-62 */
            return 1.0;
    }
}

static double eq_source(const equation *e, const double p[3]) {
    if (e->kind == WO_POISSON) {
        if (e->dim == 3) return 0.0; /* poisson.cpp:82-85 */
        /* poisson.cpp:35-44: f = 0.1 on the disk of radius 0.15 at the origin */
        const double dx = p[0] - 0.0, dy = p[1] - 0.0;
        return dx * dx + dy * dy <= 0.15 * 0.15 ? 0.1 : 0.0;
    }
    if (e->kind == WO_SCREENED_POISSON && e->dim == 2) {
        /* screened_poisson.cpp:57-60: f = 5 on the disk of radius 0.5 at (0.45, 0) */
        return sqrt((p[0] - 0.45) * (p[0] - 0.45) + p[1] * p[1]) <= 0.5 ? 5.0 : 0.0;
    }
    return 0.0;
}

/* 2D culling, poisson.cpp:27-33 and screened_poisson.cpp:48-55 */
static int eq_source_may_intersect(const equation *e, const double c[3], double R) {
    double sx = 0.0, sr = 0.15;
    if (e->kind == WO_SCREENED_POISSON) {
        sx = 0.45;
        sr = 0.5;
    }
    const double dx = c[0] - sx, dy = c[1] - 0.0;
    const double reach = R + sr;
    return dx * dx + dy * dy <= reach * reach;
}

static double dist3(const double a[3], const double b[3], int d) {
    if (d == 2) return sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]));
    return sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) +
                (a[2] - b[2]) * (a[2] - b[2]));
}

static double eq_green(const equation *e, double R, const double x[3], const double y[3]) {
    const double r = dist3(x, y, e->dim);
    if (e->kind == WO_POISSON) return e->dim == 2 ? pg_green_2d(R, r) : pg_green_3d(R, r);
    return e->dim == 2 ? sc_green_2d(e->alpha, R, r) : sc_green_3d(e->alpha, R, r);
}

static double eq_green_mass(const equation *e, double R) {
    if (e->kind == WO_POISSON) return e->dim == 2 ? pg_mass_2d(R) : pg_mass_3d(R);
    return e->dim == 2 ? sc_mass_2d(e->alpha, R) : sc_mass_3d(e->alpha, R);
}

/* Green-distributed point in the ball: poisson.cpp:62-72 / :105-117 and
 * screened_poisson.cpp:80-90 / :130-140 */
static void eq_sample_green(const equation *e, const double c[3], double R, xoshiro *rng,
                            double o[3]) {
    double radius;
    if (e->kind == WO_POISSON) {
        radius = e->dim == 2 ? pg_sample_radius_2d(R, rng) : pg_sample_radius_3d(R, rng);
    } else {
        radius = e->dim == 2 ? sc_sample_radius_2d(e->alpha, R, rng)
                             : sc_sample_radius_3d(e->alpha, R, rng);
    }
    if (e->dim == 2) {
        const double angle = 2.0 * M_PI * rng_unit(rng);
        o[0] = c[0] + radius * cos(angle);
        o[1] = c[1] + radius * sin(angle);
        o[2] = 0.0;
    } else {
        const double z = 2.0 * rng_unit(rng) - 1.0;
        const double angle = 2.0 * M_PI * rng_unit(rng);
        const double xy = sqrt(1.0 - z * z);
        o[0] = c[0] + radius * xy * cos(angle);
        o[1] = c[1] + radius * xy * sin(angle);
        o[2] = c[2] + radius * z;
    }
}

static double eq_screening_factor(const equation *e, double R) {
    if (e->kind == WO_SCREENED_POISSON) {
        return e->dim == 2 ? sc_weight_2d(e->alpha, R) : sc_weight_3d(e->alpha, R);
    }
    /* helmholtz.cpp:40-45 (1/J0(kR)) and :71-76 (kR/sin kR), k = 1 */
    const double prod = R * 1.0;
    if (prod < 1e-8) return 1.0;
    return e->dim == 2 ? 1.0 / bessel_j0(prod) : prod / sin(prod);
}

/* --------------------------------------------------------------- walks */

typedef struct {
    double radius;
    double nearest[3];
    int bid;
} start_point;

typedef struct {
    double value;
    int steps;
    int hit;
} sample_result;

/* include/wos/wos.hpp:54-138 */
static sample_result wos_sample(const bvh_t *t, const double p0[3], const start_point *st,
                                const equation *e, double eps, xoshiro *walk, xoshiro *src,
                                int max_steps, long long *visit_tally) {
    const int d = e->dim;
    double p[3] = {p0[0], p0[1], p0[2]};
    double np[3] = {st->nearest[0], st->nearest[1], st->nearest[2]};
    int bid = st->bid;
    double R = st->radius;
    double sample = 0.0, weight = 1.0;
    int steps = 0;
    const int has_source = eq_has_source(e);
    const int has_screening = eq_has_screening(e);
    while (R > eps && steps < max_steps) {
        if (has_source) {
            const int may = d == 2 ? eq_source_may_intersect(e, p, R) : 1;
            if (may) {
                double sp[3];
                if (e->source_mode == 1) { /* Green importance sampling, wos.hpp:75-82 */
                    eq_sample_green(e, p, R, src, sp);
                    const double f = eq_source(e, sp);
                    if (f != 0.0) sample += weight * eq_green_mass(e, R) * f;
                } else { /* uniform ball sample, wos.hpp:93-100 */
                    if (d == 2) ball_2d(p, R, src, sp);
                    else ball_3d(p, R, src, sp);
                    const double f = eq_source(e, sp);
                    if (f != 0.0) {
                        const double vol = d == 2 ? M_PI * R * R
                                                  : 4.0 * M_PI * (R * R * R) / 3.0;
                        sample += weight * vol * f * eq_green(e, R, p, sp);
                    }
                }
            }
        }
        if (has_screening) weight *= eq_screening_factor(e, R);
        double q[3];
        if (d == 2) step_2d(p, R, walk, q);
        else step_3d(p, R, walk, q);
        p[0] = q[0];
        p[1] = q[1];
        p[2] = q[2];
        ++steps;
        const npq_result r = bvh_npq(t, p);
        if (visit_tally) {
            visit_tally[0] += 1;
            visit_tally[1] += r.pops;
            visit_tally[2] += r.tests;
        }
        R = r.dist;
        np[0] = r.point[0];
        np[1] = r.point[1];
        np[2] = r.point[2];
        if (d == 2) bid = r.bid;
    }
    sample_result out;
    out.hit = R > eps;
    sample += weight * eq_boundary(e, np, bid);
    out.value = sample;
    out.steps = steps;
    return out;
}

typedef struct {
    double mean, variance, se, mean_steps;
    int hits;
} run_result;

/* include/wos/wos.hpp:160-191: Welford mean / M2 over N walks */
static run_result wos_run(const bvh_t *t, const double p0[3], const start_point *st,
                          const equation *e, int N, double eps, xoshiro *walk, xoshiro *src,
                          int max_steps, long long *visit_tally) {
    double mean = 0.0, m2 = 0.0, total_steps = 0.0;
    int hits = 0;
    for (int i = 0; i < N; ++i) {
        const sample_result s = wos_sample(t, p0, st, e, eps, walk, src, max_steps, visit_tally);
        const double count = (double)(i + 1);
        const double before = s.value - mean;
        mean += before / count;
        const double after = s.value - mean;
        m2 += before * after;
        total_steps += s.steps;
        if (s.hit) ++hits;
    }
    run_result r;
    r.variance = N > 1 ? m2 / (double)(N - 1) : 0.0;
    r.se = N > 0 ? sqrt(r.variance / (double)N) : 0.0;
    r.mean_steps = N > 0 ? total_steps / (double)N : 0.0;
    r.mean = mean;
    r.hits = hits;
    return r;
}

/* ---------------------------------------------------------- grid sweep */

typedef struct {
    const wo_problem *pb;
    const equation *eq;
    const bvh_t *t;
    double box[6];
    double btol;
    double eps;
    long long n_work;
    long long cursor;
    pthread_mutex_t lock;
    wo_outputs *out;
    long long *visit_tally; /* optional {queries, pops, tests, steps} */
    int walks_override;
} sweep;

typedef struct {
    sweep *sw;
    long long inside, hits, retries, indeterminate;
    double sums[3];
    long long tally[3];
} sweep_worker;

static double grid_coordinate(double lo, double hi, int i, int n) {
    /* include/wos/grid.hpp:12-18 */
    return n > 1 ? lo + (hi - lo) * (double)i / (double)(n - 1) : lo;
}

/* include/wos/runner.hpp:157-236 for one global linear index */
static void sweep_point(sweep_worker *wk, long long linear) {
    sweep *sw = wk->sw;
    const wo_problem *pb = sw->pb;
    const equation *e = sw->eq;
    const int d = pb->dim;
    const int Ny = pb->Ny, Nz = d == 2 ? 1 : pb->Nz;
    const int i = (int)(linear / ((long long)Ny * Nz));
    const int j = (int)((linear / Nz) % Ny);
    const int k = (int)(linear % Nz);
    double p0[3];
    p0[0] = grid_coordinate(sw->box[0], sw->box[1], i, pb->Nx);
    p0[1] = grid_coordinate(sw->box[2], sw->box[3], j, Ny);
    p0[2] = d == 3 ? grid_coordinate(sw->box[4], sw->box[5], k, Nz) : 0.0;
    if (d == 2) p0[2] = 0.0;
    const uint64_t point_seed = wo_splitmix64(pb->seed ^ wo_splitmix64((uint64_t)linear));

    const npq_result s0 = bvh_npq(sw->t, p0);
    start_point st;
    st.radius = s0.dist;
    st.nearest[0] = s0.point[0];
    st.nearest[1] = s0.point[1];
    st.nearest[2] = s0.point[2];
    st.bid = d == 2 ? s0.bid : -1;

    int where;
    if (d == 2) {
        if (st.radius <= sw->btol) {
            where = 2;
        } else {
            mesh_view m = {2, pb->n_prims, pb->verts, pb->prims, pb->boundary_ids};
            where = winding_number(&m, p0) != 0 ? 1 : 0;
        }
    } else {
        xoshiro ins;
        rng_seed(&ins, wo_splitmix64(point_seed ^ 0x243F6A8885A308D3ULL));
        int retries = 0;
        where = classify_3d(sw->t, p0, st.radius, sw->btol, pb->max_ray_attempts, &ins, &retries);
        wk->retries += retries;
        if (where == 3) ++wk->indeterminate;
    }

    run_result r = {NAN, NAN, NAN, NAN, 0};
    if (where == 2) {
        r.mean = eq_boundary(e, st.nearest, st.bid);
        r.variance = r.se = r.mean_steps = 0.0;
    } else if (where == 1) {
        xoshiro walk, src;
        rng_seed(&walk, wo_splitmix64(point_seed ^ 0x13198A2E03707344ULL));
        const int N = sw->walks_override > 0 ? sw->walks_override : pb->N_walks;
        long long *tally = sw->visit_tally ? wk->tally : NULL;
        if (d == 2) {
            rng_seed(&src, wo_splitmix64(point_seed ^ 0xA4093822299F31D0ULL));
            r = wos_run(sw->t, p0, &st, e, N, sw->eps, &walk, &src, pb->max_steps, tally);
        } else {
            r = wos_run(sw->t, p0, &st, e, N, sw->eps, &walk, &walk, pb->max_steps, tally);
        }
        ++wk->inside;
        wk->hits += r.hits;
        wk->sums[0] += r.variance;
        wk->sums[1] += r.se;
        wk->sums[2] += r.mean_steps;
    }
    wo_outputs *o = sw->out;
    if (o) {
        if (o->mean) o->mean[linear] = r.mean;
        if (o->variance) o->variance[linear] = r.variance;
        if (o->standard_error) o->standard_error[linear] = r.se;
        if (o->mean_steps) o->mean_steps[linear] = r.mean_steps;
        if (o->location) o->location[linear] = (unsigned char)where;
    }
}

static void *sweep_thread(void *arg) {
    sweep_worker *wk = (sweep_worker *)arg;
    sweep *sw = wk->sw;
    for (;;) {
        pthread_mutex_lock(&sw->lock);
        const long long w = sw->cursor++;
        pthread_mutex_unlock(&sw->lock);
        if (w >= sw->n_work) break;
        sweep_point(wk, sw->pb->points ? sw->pb->points[w] : w);
    }
    return NULL;
}

static int run_sweep(int equation_kind, const wo_problem *pb, wo_outputs *out, int walks_override,
                     long long *visit_tally) {
    if (pb->dim != 2 && pb->dim != 3) return 1;
    if (equation_kind < 0 || equation_kind > 3) return 1;
    equation e = {equation_kind, pb->dim, pb->source_mode, pb->alpha};
    bvh_t t;
    bvh_build(&t, pb);
    sweep sw;
    memset(&sw, 0, sizeof(sw));
    sw.pb = pb;
    sw.eq = &e;
    sw.t = &t;
    sw.out = out;
    sw.visit_tally = visit_tally;
    sw.walks_override = walks_override;
    if (pb->use_mesh_bbox) {
        mesh_bbox(pb, sw.box);
    } else {
        sw.box[0] = pb->xmin; sw.box[1] = pb->xmax;
        sw.box[2] = pb->ymin; sw.box[3] = pb->ymax;
        sw.box[4] = pb->zmin; sw.box[5] = pb->zmax;
    }
    if (pb->dim == 2) sw.box[4] = sw.box[5] = 0.0;
    /* runner.hpp:86-88 */
    double scale = 1.0;
    for (int k = 0; k < 3; ++k) {
        const double ext = sw.box[2 * k + 1] - sw.box[2 * k];
        if (ext > scale) scale = ext;
    }
    sw.btol = 1e-10 * scale;
    sw.eps = equation_kind == WO_SCREENED_POISSON ? wo_screened_epsilon(pb->epsilon, pb->alpha)
                                                  : pb->epsilon;
    const long long total = (long long)pb->Nx * pb->Ny * (pb->dim == 2 ? 1 : pb->Nz);
    sw.n_work = pb->points ? pb->n_points : total;
    pthread_mutex_init(&sw.lock, NULL);

    int threads = pb->n_threads > 0 ? pb->n_threads : 1;
    sweep_worker *wk = (sweep_worker *)calloc((size_t)threads, sizeof(sweep_worker));
    pthread_t *th = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    struct timespec a, b;
    clock_gettime(CLOCK_MONOTONIC, &a);
    for (int i = 0; i < threads; ++i) {
        wk[i].sw = &sw;
        if (threads == 1) {
            sweep_thread(&wk[i]);
        } else {
            pthread_create(&th[i], NULL, sweep_thread, &wk[i]);
        }
    }
    if (threads > 1) {
        for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
    }
    clock_gettime(CLOCK_MONOTONIC, &b);
    if (out) {
        out->seconds = (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
        out->inside_points = out->max_steps_hits = 0;
        out->ambiguous_ray_retries = out->indeterminate_points = 0;
        out->sum_variance = out->sum_standard_error = out->sum_mean_steps = 0.0;
    }
    for (int i = 0; i < threads; ++i) {
        if (out) {
            out->inside_points += wk[i].inside;
            out->max_steps_hits += wk[i].hits;
            out->ambiguous_ray_retries += wk[i].retries;
            out->indeterminate_points += wk[i].indeterminate;
            out->sum_variance += wk[i].sums[0];
            out->sum_standard_error += wk[i].sums[1];
            out->sum_mean_steps += wk[i].sums[2];
        }
        if (visit_tally) {
            for (int k = 0; k < 3; ++k) visit_tally[k] += wk[i].tally[k];
        }
    }
    pthread_mutex_destroy(&sw.lock);
    free(wk);
    free(th);
    bvh_free(&t);
    return 0;
}

int wo_solve_grid(int equation_kind, const wo_problem *pb, wo_outputs *out) {
    return run_sweep(equation_kind, pb, out, 0, NULL);
}

int wo_walk_visit_counts(int equation_kind, const wo_problem *pb, int walks, long long *queries,
                         long long *node_pops, long long *prim_tests, long long *steps) {
    long long tally[3] = {0, 0, 0};
    wo_outputs out;
    memset(&out, 0, sizeof(out));
    const int rc = run_sweep(equation_kind, pb, &out, walks, tally);
    *queries = tally[0];
    *node_pops = tally[1];
    *prim_tests = tally[2];
    *steps = tally[0];
    return rc;
}

/* ------------------------------------------------- Gaussian heat source */

/* FP64 restatement of the heat-source walks and their derivative sums
 * (walk_on_spheres_b200/csrc/kernels_adjoint.cu states the estimator).  The
 * walk is the reference's Poisson estimator (include/wos/wos.hpp:54-138 with
 * include/wos/poisson.hpp:12-51) on the reference's xoshiro256++ streams,
 * seeded like the grid sweep (include/wos/runner.hpp:163-168, 208-221), with
 * the source sampled at every step (no culling). */

typedef struct {
    const wo_problem *pb;
    const wo_gaussian *src;
    const bvh_t *t;
    const double *g;
    const double *probes;
    long long n;
    const double *weights;
    double btol;
    double *mean, *se, *jac, *jac_se;
    unsigned char *location;
    long long cursor;
    pthread_mutex_t lock;
} heat_job;

typedef struct {
    heat_job *job;
    double *grad;  /* per-worker vertex gradient (n_verts) or NULL */
} heat_worker;

/* interpolation weights of primitive `prim` at its point q */
static void heat_weights(const bvh_t *t, int prim, const double q[3], int v[3], double w[3]) {
    const int d = t->m.dim;
    for (int k = 0; k < 3; ++k) {
        v[k] = k < d ? t->m.prims[d * prim + k] : 0;
        w[k] = 0.0;
    }
    const vec3 a = vert(&t->m, v[0]), b = vert(&t->m, v[1]);
    if (d == 2) {
        const double vx = b.x - a.x, vy = b.y - a.y;
        double s = ((q[0] - a.x) * vx + (q[1] - a.y) * vy) / (vx * vx + vy * vy);
        s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
        w[0] = 1.0 - s;
        w[1] = s;
        return;
    }
    const vec3 c = vert(&t->m, v[2]);
    const double e1[3] = {b.x - a.x, b.y - a.y, b.z - a.z};
    const double e2[3] = {c.x - a.x, c.y - a.y, c.z - a.z};
    const double dd[3] = {q[0] - a.x, q[1] - a.y, q[2] - a.z};
    const double A = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
    const double B = e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2];
    const double C = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
    const double d1 = dd[0] * e1[0] + dd[1] * e1[1] + dd[2] * e1[2];
    const double d2 = dd[0] * e2[0] + dd[1] * e2[1] + dd[2] * e2[2];
    const double det = A * C - B * B;
    double s = (C * d1 - B * d2) / det, u = (A * d2 - B * d1) / det;
    if (s < 0.0) s = 0.0;
    if (u < 0.0) u = 0.0;
    if (s + u > 1.0) {
        const double sum = s + u;
        s /= sum;
        u /= sum;
    }
    w[0] = 1.0 - s - u;
    w[1] = s;
    w[2] = u;
}

static double heat_boundary(const heat_job *job, int prim, const double q[3], double c,
                            double *grad) {
    int v[3];
    double w[3];
    heat_weights(job->t, prim, q, v, w);
    double val = 0.0;
    for (int k = 0; k < job->pb->dim; ++k) {
        if (job->g) val += w[k] * job->g[v[k]];
        if (grad && c != 0.0) grad[v[k]] += c * w[k];
    }
    return val;
}

/* one step's source term and its parameter derivatives (added to j) */
static double heat_source(const heat_job *job, const double p[3], double R, xoshiro *rng,
                          double j[5]) {
    const int d = job->pb->dim;
    const wo_gaussian *s = job->src;
    double y[3] = {0.0, 0.0, 0.0};
    double m;
    if (job->pb->source_mode == 2) {
        /* include/wos/source_sampling.hpp:35-78: random mixture of the Green
         * density and the Gaussian proposal, balance-heuristic weight */
        const double beta = s->mis_green_probability;
        const int own = !(s->proposal_sigma > 0.0);
        const double *c = own ? s->x0 : s->proposal_x0;
        const double ps = own ? s->sigma : s->proposal_sigma;
        if (rng_unit(rng) < beta) {
            const double radius =
                d == 2 ? pg_sample_radius_2d(R, rng) : pg_sample_radius_3d(R, rng);
            if (d == 2) {
                const double angle = 2.0 * M_PI * rng_unit(rng);
                y[0] = p[0] + radius * cos(angle);
                y[1] = p[1] + radius * sin(angle);
            } else {
                const double z = 2.0 * rng_unit(rng) - 1.0;
                const double angle = 2.0 * M_PI * rng_unit(rng);
                const double xy = sqrt(1.0 - z * z);
                y[0] = p[0] + radius * xy * cos(angle);
                y[1] = p[1] + radius * xy * sin(angle);
                y[2] = p[2] + radius * z;
            }
        } else {
            const double sc = ps / sqrt(2.0);
            const double rho0 = sqrt(-2.0 * log(rng_unit_open(rng)));
            const double a0 = 2.0 * M_PI * rng_unit(rng);
            y[0] = c[0] + sc * rho0 * cos(a0);
            y[1] = c[1] + sc * rho0 * sin(a0);
            if (d == 3) {
                const double rho1 = sqrt(-2.0 * log(rng_unit_open(rng)));
                y[2] = c[2] + sc * rho1 * cos(2.0 * M_PI * rng_unit(rng));
            }
        }
        const double r = dist3(p, y, d);
        if (!(r > 0.0 && r < R)) return 0.0;
        const double G = d == 2 ? pg_green_2d(R, r) : pg_green_3d(R, r);
        const double mass = d == 2 ? pg_mass_2d(R) : pg_mass_3d(R);
        double qq = 0.0;
        for (int k = 0; k < d; ++k) qq += (y[k] - c[k]) * (y[k] - c[k]);
        const double norm = 1.0 / (pow(M_PI, 0.5 * d) * pow(ps, d));
        const double src_pdf = norm * exp(-qq / (ps * ps));
        const double mix = beta * (G / mass) + (1.0 - beta) * src_pdf;
        if (!(mix > 0.0)) return 0.0;
        m = G / mix;
    } else if (job->pb->source_mode == 1) {
        const double radius = d == 2 ? pg_sample_radius_2d(R, rng) : pg_sample_radius_3d(R, rng);
        if (d == 2) {
            const double angle = 2.0 * M_PI * rng_unit(rng);
            y[0] = p[0] + radius * cos(angle);
            y[1] = p[1] + radius * sin(angle);
        } else {
            const double z = 2.0 * rng_unit(rng) - 1.0;
            const double angle = 2.0 * M_PI * rng_unit(rng);
            const double xy = sqrt(1.0 - z * z);
            y[0] = p[0] + radius * xy * cos(angle);
            y[1] = p[1] + radius * xy * sin(angle);
            y[2] = p[2] + radius * z;
        }
        m = d == 2 ? pg_mass_2d(R) : pg_mass_3d(R);
    } else {
        if (d == 2) ball_2d(p, R, rng, y);
        else ball_3d(p, R, rng, y);
        double r = dist3(p, y, d);
        if (r > R) r = R;
        if (!(r > 0.0)) return 0.0;
        const double vol = d == 2 ? M_PI * R * R : 4.0 * M_PI * (R * R * R) / 3.0;
        m = vol * (d == 2 ? pg_green_2d(R, r) : pg_green_3d(R, r));
    }
    const double dx = y[0] - s->x0[0], dy = y[1] - s->x0[1];
    const double dz = d == 3 ? y[2] - s->x0[2] : 0.0;
    const double inv_s2 = 1.0 / (s->sigma * s->sigma);
    const double q = (dx * dx + dy * dy + dz * dz) * inv_s2;
    const double e = exp(-q);
    const double mf = m * s->Q * e;
    j[0] += m * e;
    j[1] += 2.0 * mf * inv_s2 * dx;
    j[2] += 2.0 * mf * inv_s2 * dy;
    j[3] += 2.0 * mf * inv_s2 * dz;
    j[4] += 2.0 * mf * q / s->sigma;
    return mf;
}

static void heat_probe(heat_worker *wk, long long i) {
    heat_job *job = wk->job;
    const wo_problem *pb = job->pb;
    const int d = pb->dim;
    double p0[3] = {job->probes[d * i], job->probes[d * i + 1],
                    d == 3 ? job->probes[d * i + 2] : 0.0};
    const uint64_t linear = pb->points ? (uint64_t)pb->points[i] : (uint64_t)i;
    const uint64_t point_seed = wo_splitmix64(pb->seed ^ wo_splitmix64(linear));
    const npq_result s0 = bvh_npq(job->t, p0);
    int where;
    if (d == 2) {
        if (s0.dist <= job->btol) {
            where = 2;
        } else {
            mesh_view m = {2, pb->n_prims, pb->verts, pb->prims, pb->boundary_ids};
            where = winding_number(&m, p0) != 0 ? 1 : 0;
        }
    } else {
        xoshiro ins;
        rng_seed(&ins, wo_splitmix64(point_seed ^ 0x243F6A8885A308D3ULL));
        int retries = 0;
        where = classify_3d(job->t, p0, s0.dist, job->btol, pb->max_ray_attempts, &ins, &retries);
    }
    double mean = NAN, se = NAN, jm[5], js[5];
    for (int k = 0; k < 5; ++k) jm[k] = js[k] = NAN;
    const double wgt = job->weights ? job->weights[i] : 1.0;
    if (where == 2) {
        mean = heat_boundary(job, s0.tri, s0.point, wgt, wk->grad);
        se = 0.0;
        for (int k = 0; k < 5; ++k) jm[k] = js[k] = 0.0;
    } else if (where == 1) {
        xoshiro walk, srcr;
        rng_seed(&walk, wo_splitmix64(point_seed ^ 0x13198A2E03707344ULL));
        rng_seed(&srcr, wo_splitmix64(point_seed ^ 0xA4093822299F31D0ULL));
        xoshiro *src = d == 2 ? &srcr : &walk;
        const int N = pb->N_walks;
        const double c = wgt / (double)N;
        double m = 0.0, m2 = 0.0, sum[5] = {0, 0, 0, 0, 0}, sq[5] = {0, 0, 0, 0, 0};
        for (int w = 0; w < N; ++w) {
            double p[3] = {p0[0], p0[1], p0[2]};
            double np[3] = {s0.point[0], s0.point[1], s0.point[2]};
            int tri = s0.tri;
            double R = s0.dist, sample = 0.0, j[5] = {0, 0, 0, 0, 0};
            int steps = 0;
            while (R > pb->epsilon && steps < pb->max_steps) {
                sample += heat_source(job, p, R, src, j);
                double q[3];
                if (d == 2) step_2d(p, R, &walk, q);
                else step_3d(p, R, &walk, q);
                p[0] = q[0];
                p[1] = q[1];
                p[2] = q[2];
                ++steps;
                const npq_result r = bvh_npq(job->t, p);
                R = r.dist;
                np[0] = r.point[0];
                np[1] = r.point[1];
                np[2] = r.point[2];
                tri = r.tri;
            }
            const double value = sample + heat_boundary(job, tri, np, c, wk->grad);
            const double before = value - m;
            m += before / (double)(w + 1);
            m2 += before * (value - m);
            for (int k = 0; k < 5; ++k) {
                sum[k] += j[k];
                sq[k] += j[k] * j[k];
            }
        }
        mean = m;
        const double var = N > 1 ? m2 / (double)(N - 1) : 0.0;
        se = sqrt(var / (double)N);
        for (int k = 0; k < 5; ++k) {
            jm[k] = sum[k] / (double)N;
            double v = N > 1 ? (sq[k] - sum[k] * jm[k]) / (double)(N - 1) : 0.0;
            if (v < 0.0) v = 0.0;
            js[k] = sqrt(v / (double)N);
        }
    }
    if (job->mean) job->mean[i] = mean;
    if (job->se) job->se[i] = se;
    if (job->location) job->location[i] = (unsigned char)where;
    for (int k = 0; k < 5; ++k) {
        if (job->jac) job->jac[5 * i + k] = jm[k];
        if (job->jac_se) job->jac_se[5 * i + k] = js[k];
    }
}

static void *heat_thread(void *arg) {
    heat_worker *wk = (heat_worker *)arg;
    heat_job *job = wk->job;
    for (;;) {
        pthread_mutex_lock(&job->lock);
        const long long i = job->cursor++;
        pthread_mutex_unlock(&job->lock);
        if (i >= job->n) break;
        heat_probe(wk, i);
    }
    return NULL;
}

int wo_heat_solve(const wo_problem *pb, const wo_gaussian *src, const double *vertex_values,
                  const double *probes, long long n, const double *weights, double *mean,
                  double *standard_error, double *jacobian, double *jacobian_se,
                  unsigned char *location, double *grad_vertex) {
    if (pb->dim != 2 && pb->dim != 3) return 1;
    if (!(src->sigma > 0.0)) return 1;
    if (pb->source_mode == 2 &&
        !(src->mis_green_probability > 0.0 && src->mis_green_probability < 1.0)) {
        return 1;
    }
    bvh_t t;
    bvh_build(&t, pb);
    heat_job job;
    memset(&job, 0, sizeof(job));
    job.pb = pb;
    job.src = src;
    job.t = &t;
    job.g = vertex_values;
    job.probes = probes;
    job.n = n;
    job.weights = weights;
    job.mean = mean;
    job.se = standard_error;
    job.jac = jacobian;
    job.jac_se = jacobian_se;
    job.location = location;
    double box[6];
    mesh_bbox(pb, box);
    double scale = 1.0; /* runner.hpp:86-88 */
    for (int k = 0; k < pb->dim; ++k) {
        const double ext = box[2 * k + 1] - box[2 * k];
        if (ext > scale) scale = ext;
    }
    job.btol = 1e-10 * scale;
    pthread_mutex_init(&job.lock, NULL);
    const int threads = pb->n_threads > 0 ? pb->n_threads : 1;
    heat_worker *wk = (heat_worker *)calloc((size_t)threads, sizeof(heat_worker));
    pthread_t *th = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    for (int i = 0; i < threads; ++i) {
        wk[i].job = &job;
        wk[i].grad = grad_vertex ? (double *)calloc((size_t)pb->n_verts, sizeof(double)) : NULL;
    }
    if (threads == 1) {
        heat_thread(&wk[0]);
    } else {
        for (int i = 0; i < threads; ++i) pthread_create(&th[i], NULL, heat_thread, &wk[i]);
        for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
    }
    if (grad_vertex) {
        for (int v = 0; v < pb->n_verts; ++v) grad_vertex[v] = 0.0;
        for (int i = 0; i < threads; ++i) {
            for (int v = 0; v < pb->n_verts; ++v) grad_vertex[v] += wk[i].grad[v];
            free(wk[i].grad);
        }
    }
    pthread_mutex_destroy(&job.lock);
    free(wk);
    free(th);
    bvh_free(&t);
    return 0;
}
