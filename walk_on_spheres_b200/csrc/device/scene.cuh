// Device scene: the boundary mesh laid out for closest-point and ray queries.
//
// BVH shape.  An implicit, perfectly balanced binary tree of depth D over the
// primitives in leaf order: node ids are 1-based heap indices (children of i
// are 2i and 2i+1, parent i>>1, sibling i^1), leaves are the ids
// [2^D, 2^(D+1)), and leaf j holds the primitive slots
// [floor(j*n/2^D), floor((j+1)*n/2^D)).  Every internal split is a median
// split along the longest axis of the node box by (centroid, primitive id),
// the rule of the reference build (src/bvh.cpp:143-230); only the split
// positions are fixed by the formula above instead of by (start+end)/2, so
// no child pointers, leaf offsets or parent pointers are stored.
//
// Traversal.  Stackless: a 32-bit "bitstack" records, per level of the
// current path, whether the far child is still pending; backtracking moves
// up by shifting the node id and across with id^1, and re-tests the pending
// sibling against the best distance found so far.  Nearer child first, a
// node is entered only while its box distance is < best, ties go to the left
// child (the reference order of src/bvh.cpp:327-339), and a primitive
// replaces the best only when strictly closer.
//
// Records (all 16-byte aligned, one array per kind):
//   box64  FP64 node boxes by node id, lo[dim] then hi[dim]      (plain, shell)
//   seg64  2D FP64 segments per slot as 2 double2 {(x0,y0),(x1,y1)}
//   segid  2D per slot {boundary_id, primitive id}
//   tri64  3D FP64 Eberly records per slot, 7 double2: v0, e1, e2, a, b, c,
//          det, denom (values of src/bvh.cpp:204-217)
// The FP32 fast path queries the 32-wide tree of wide.cuh instead, whose
// primitive blocks hold FP32 records (eberly32 below reads the 3D one).
#pragma once
#include <cstdint>

namespace wosb {

struct WideView;

struct SceneView {
    int dim;
    int n_prims;
    int depth;            // D; leaves are ids [2^D, 2^(D+1))
    const double *box64;  // (2^(D+1)) * 2*dim doubles, id 0 unused
    const double2 *seg64;
    const int2 *segid;
    const double2 *tri64;
};

__host__ __device__ __forceinline__ int leaf_first(int j, int n, int depth) {
    return static_cast<int>((static_cast<uint64_t>(j) * static_cast<uint64_t>(n)) >> depth);
}

template <typename T>
struct Pt3 {
    T x, y, z;
};

// --------------------------------------------------------------------------
// FP64 primitive tests (reference arithmetic; compiled without FMA contraction
// in the exact-path translation unit).

// src/npq.cpp:8-29
__device__ __forceinline__ double npq_seg64(double s0x, double s0y, double s1x, double s1y,
                                            double px, double py, double &nx, double &ny) {
    const double vx = s1x - s0x;
    const double vy = s1y - s0y;
    const double wx = px - s0x;
    const double wy = py - s0y;
    const double vv = vx * vx + vy * vy;
    const double wv = wx * vx + wy * vy;
    double par = (vv > 0.0) ? wv / vv : 0.0;
    if (par < 0.0) par = 0.0;
    if (par > 1.0) par = 1.0;
    nx = s0x + par * vx;
    ny = s0y + par * vy;
    const double dx = px - nx;
    const double dy = py - ny;
    return dx * dx + dy * dy;
}

// Eberly seven-region closest point, src/npq.cpp:52-189 (T = double: exact
// reference arithmetic; T = float: the FP32 fast path, same regions).
template <typename T>
__device__ __forceinline__ T eberly(T px, T py, T pz, T v0x, T v0y, T v0z, T e1x, T e1y, T e1z,
                                    T e2x, T e2y, T e2z, T a, T b, T c, T det, T denom,
                                    T &nx, T &ny, T &nz) {
    const T bpx = v0x - px, bpy = v0y - py, bpz = v0z - pz;
    const T d = e1x * bpx + e1y * bpy + e1z * bpz;
    const T e = e2x * bpx + e2y * bpy + e2z * bpz;
    T s = b * e - c * d;
    T t = b * d - a * e;
    if (s + t <= det) {
        if (s < T(0)) {
            if (t < T(0)) {  // region 4
                if (d < T(0)) {
                    t = T(0);
                    s = (-d >= a) ? T(1) : -d / a;
                } else {
                    s = T(0);
                    t = (e >= T(0)) ? T(0) : ((-e >= c) ? T(1) : -e / c);
                }
            } else {  // region 3
                s = T(0);
                t = (e >= T(0)) ? T(0) : ((-e >= c) ? T(1) : -e / c);
            }
        } else if (t < T(0)) {  // region 5
            t = T(0);
            s = (d >= T(0)) ? T(0) : ((-d >= a) ? T(1) : -d / a);
        } else {  // region 0
            s /= det;
            t /= det;
        }
    } else {
        if (s < T(0)) {  // region 2
            const T bd = b + d, ce = c + e;
            if (ce > bd) {
                const T numer = ce - bd;
                s = (numer >= denom) ? T(1) : numer / denom;
                t = T(1) - s;
            } else {
                s = T(0);
                t = (ce <= T(0)) ? T(1) : ((e >= T(0)) ? T(0) : -e / c);
            }
        } else if (t < T(0)) {  // region 6
            const T be = b + e, ad = a + d;
            if (ad > be) {
                const T numer = ad - be;
                t = (numer >= denom) ? T(1) : numer / denom;
                s = T(1) - t;
            } else {
                t = T(0);
                s = (ad <= T(0)) ? T(1) : ((d >= T(0)) ? T(0) : -d / a);
            }
        } else {  // region 1
            const T numer = (c + e) - (b + d);
            s = (numer <= T(0)) ? T(0) : ((numer >= denom) ? T(1) : numer / denom);
            t = T(1) - s;
        }
    }
    nx = v0x + s * e1x + t * e2x;
    ny = v0y + s * e1y + t * e2y;
    nz = v0z + s * e1z + t * e2z;
    const T dx = nx - px, dy = ny - py, dz = nz - pz;
    return dx * dx + dy * dy + dz * dz;
}

__device__ __forceinline__ double dmax_(double a, double b) { return a > b ? a : b; }

// src/bvh.cpp:111-121
template <int DIM>
__device__ __forceinline__ double box_dist64(const double *box, const double *p) {
    const double dx = dmax_(0.0, dmax_(box[0] - p[0], p[0] - box[DIM + 0]));
    const double dy = dmax_(0.0, dmax_(box[1] - p[1], p[1] - box[DIM + 1]));
    if (DIM == 2) return dx * dx + dy * dy;
    const double dz = dmax_(0.0, dmax_(box[2] - p[2], p[2] - box[DIM + 2]));
    return dx * dx + dy * dy + dz * dz;
}

// Result of a closest-point query.
template <typename T>
struct Nearest {
    T best;      // squared distance (the query's bound until a primitive beats it)
    T limit;     // nodes are entered only while their box distance is below this
    T x, y, z;   // closest point
    int slot;    // leaf slot of the closest primitive (-1: none beat the bound)
};

// Stackless near-first traversal.  Policy provides child_dists(id, dl, dr),
// node_dist(id) and test_leaf(j, Q&); Q has `limit` (the pruning bound the
// leaf tests maintain).
template <typename T, class Policy, class Q>
__device__ __forceinline__ void traverse_nearest(const Policy &P, int depth, Q &q) {
    if (depth == 0) {
        P.test_leaf(0, q);
        return;
    }
    const unsigned leaf_base = 1u << depth;
    const unsigned last_internal = leaf_base >> 1;  // ids >= this have leaf children
    unsigned cur = 1, bits = 0;
    for (;;) {
        T dl, dr;
        P.child_dists(cur, dl, dr);
        const bool left_near = dl <= dr;
        const unsigned nearc = 2 * cur + (left_near ? 0u : 1u);
        const T dn = left_near ? dl : dr;
        const T df = left_near ? dr : dl;
        bool descended = false;
        if (cur >= last_internal) {
            if (dn < q.limit) P.test_leaf(static_cast<int>(nearc - leaf_base), q);
            if (df < q.limit) P.test_leaf(static_cast<int>((nearc ^ 1u) - leaf_base), q);
        } else if (dn < q.limit) {
            bits = (bits << 1) | (df < q.limit ? 1u : 0u);
            cur = nearc;
            descended = true;
        }
        if (descended) continue;
        // backtrack to the deepest pending far sibling that can still win
        for (;;) {
            if (bits == 0) return;
            while ((bits & 1u) == 0u) {
                bits >>= 1;
                cur >>= 1;
            }
            bits ^= 1u;
            cur ^= 1u;
            if (P.node_dist(cur) < q.limit) break;
        }
    }
}

// ---- FP64 policies ----------------------------------------------------------

struct Seg64Policy {
    const SceneView &s;
    double p[2];
    __device__ Seg64Policy(const SceneView &sv, double px, double py) : s(sv) {
        p[0] = px;
        p[1] = py;
    }
    __device__ __forceinline__ double node_dist(unsigned id) const {
        return box_dist64<2>(s.box64 + 4 * id, p);
    }
    __device__ __forceinline__ void child_dists(unsigned id, double &dl, double &dr) const {
        dl = node_dist(2 * id);
        dr = node_dist(2 * id + 1);
    }
    __device__ __forceinline__ void test_leaf(int j, Nearest<double> &q) const {
        const int b = leaf_first(j, s.n_prims, s.depth);
        const int e = leaf_first(j + 1, s.n_prims, s.depth);
        for (int k = b; k < e; ++k) {
            const double2 a = s.seg64[2 * k], c = s.seg64[2 * k + 1];
            double nx, ny;
            const double d2 = npq_seg64(a.x, a.y, c.x, c.y, p[0], p[1], nx, ny);
            if (d2 < q.best) {
                q.best = d2;
                q.limit = d2;
                q.x = nx;
                q.y = ny;
                q.slot = k;
            }
        }
    }
};

struct Tri64Policy {
    const SceneView &s;
    double p[3];
    __device__ Tri64Policy(const SceneView &sv, double px, double py, double pz) : s(sv) {
        p[0] = px;
        p[1] = py;
        p[2] = pz;
    }
    __device__ __forceinline__ double node_dist(unsigned id) const {
        return box_dist64<3>(s.box64 + 6 * id, p);
    }
    __device__ __forceinline__ void child_dists(unsigned id, double &dl, double &dr) const {
        dl = node_dist(2 * id);
        dr = node_dist(2 * id + 1);
    }
    __device__ __forceinline__ void test_leaf(int j, Nearest<double> &q) const {
        const int b = leaf_first(j, s.n_prims, s.depth);
        const int e = leaf_first(j + 1, s.n_prims, s.depth);
        for (int k = b; k < e; ++k) {
            const double2 *r = s.tri64 + 7 * k;
            const double2 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4], r5 = r[5],
                          r6 = r[6];
            double nx, ny, nz;
            const double d2 = eberly<double>(p[0], p[1], p[2], r0.x, r0.y, r1.x, r1.y, r2.x,
                                             r2.y, r3.x, r3.y, r4.x, r4.y, r5.x, r5.y, r6.x,
                                             r6.y, nx, ny, nz);
            if (d2 < q.best) {
                q.best = d2;
                q.limit = d2;
                q.x = nx;
                q.y = ny;
                q.z = nz;
                q.slot = k;
            }
        }
    }
};

// Exact FP64 closest point (bvh_npq, src/bvh.cpp:295-387).  `bound2` limits
// the search to primitives closer than sqrt(bound2) (INFINITY: unbounded).
template <int DIM>
__device__ __forceinline__ Nearest<double> nearest64(const SceneView &s, double px, double py,
                                                     double pz, double bound2) {
    Nearest<double> q;
    q.best = bound2;
    q.limit = bound2;
    q.x = q.y = q.z = 0.0;
    q.slot = -1;
    if (DIM == 2) {
        Seg64Policy P(s, px, py);
        traverse_nearest<double>(P, s.depth, q);
    } else {
        Tri64Policy P(s, px, py, pz);
        traverse_nearest<double>(P, s.depth, q);
    }
    return q;
}

// ---- FP32 primitive test ----------------------------------------------------

// Eberly's regions in FP32 with precomputed reciprocals; returns the squared
// distance only.  Record: {v0, a} {e1, b} {e2, c} {det, 1/det, 1/a, 1/c}.
__device__ __forceinline__ float eberly32(float px, float py, float pz, const float4 *r) {
    const float4 A = r[0], B = r[1], C = r[2], D = r[3];
    const float a = A.w, b = B.w, c = C.w, det = D.x;
    const float bpx = A.x - px, bpy = A.y - py, bpz = A.z - pz;
    const float d = B.x * bpx + B.y * bpy + B.z * bpz;
    const float e = C.x * bpx + C.y * bpy + C.z * bpz;
    float s = b * e - c * d;
    float t = b * d - a * e;
    if (s + t <= det) {
        if (s < 0.0f) {
            if (t < 0.0f && d < 0.0f) {  // region 4, edge t = 0
                t = 0.0f;
                s = (-d >= a) ? 1.0f : -d * D.z;
            } else {  // regions 3 and 4, edge s = 0
                s = 0.0f;
                t = (e >= 0.0f) ? 0.0f : ((-e >= c) ? 1.0f : -e * D.w);
            }
        } else if (t < 0.0f) {  // region 5
            t = 0.0f;
            s = (d >= 0.0f) ? 0.0f : ((-d >= a) ? 1.0f : -d * D.z);
        } else {  // region 0
            s *= D.y;
            t *= D.y;
        }
    } else {
        const float denom = a - 2.0f * b + c;
        if (s < 0.0f) {  // region 2
            const float bd = b + d, ce = c + e;
            if (ce > bd) {
                const float numer = ce - bd;
                s = (numer >= denom) ? 1.0f : __fdividef(numer, denom);
                t = 1.0f - s;
            } else {
                s = 0.0f;
                t = (ce <= 0.0f) ? 1.0f : ((e >= 0.0f) ? 0.0f : -e * D.w);
            }
        } else if (t < 0.0f) {  // region 6
            const float be = b + e, ad = a + d;
            if (ad > be) {
                const float numer = ad - be;
                t = (numer >= denom) ? 1.0f : __fdividef(numer, denom);
                s = 1.0f - t;
            } else {
                t = 0.0f;
                s = (ad <= 0.0f) ? 1.0f : ((d >= 0.0f) ? 0.0f : -d * D.z);
            }
        } else {  // region 1
            const float numer = (c + e) - (b + d);
            s = (numer <= 0.0f) ? 0.0f : ((numer >= denom) ? 1.0f : __fdividef(numer, denom));
            t = 1.0f - s;
        }
    }
    const float dx = bpx + s * B.x + t * C.x;
    const float dy = bpy + s * B.y + t * C.y;
    const float dz = bpz + s * B.z + t * C.z;
    return dx * dx + dy * dy + dz * dz;
}

// --------------------------------------------------------------------------
// Inside / outside (FP64, reference arithmetic).

// Sunday's winding number over every segment, src/inside.cpp:117-137.
__device__ __forceinline__ int winding_number(const SceneView &s, double px, double py) {
    int wn = 0;
    for (int k = 0; k < s.n_prims; ++k) {
        const double2 a = s.seg64[2 * k], c = s.seg64[2 * k + 1];
        const double area = (c.x - a.x) * (py - a.y) - (px - a.x) * (c.y - a.y);
        if (a.y <= py) {
            if (c.y > py && area > 0) ++wn;
        } else {
            if (c.y <= py && area < 0) --wn;
        }
    }
    return wn;
}

constexpr double kRayEps = 1e-9;  // INTERSECTION_EPSILON, src/inside.cpp:14

// src/inside.cpp:27-51
__device__ __forceinline__ bool update_ray_interval(double origin, double dir, double bmin,
                                                    double bmax, double &tmin, double &tmax) {
    const double ext = fabs(bmax - bmin);
    const double extent_scale = (1.0 < ext) ? ext : 1.0;
    double cs = 1.0;
    if (cs < fabs(origin)) cs = fabs(origin);
    if (cs < fabs(bmin)) cs = fabs(bmin);
    if (cs < fabs(bmax)) cs = fabs(bmax);
    const double padding = kRayEps * extent_scale + 16.0 * 2.220446049250313e-16 * cs;
    bmin -= padding;
    bmax += padding;
    if (dir == 0.0) return origin >= bmin && origin <= bmax;
    double t0 = (bmin - origin) / dir;
    double t1 = (bmax - origin) / dir;
    if (t0 > t1) {
        const double tt = t0;
        t0 = t1;
        t1 = tt;
    }
    tmin = (tmin < t0) ? t0 : tmin;
    tmax = (t1 < tmax) ? t1 : tmax;
    return tmin <= tmax;
}

// src/inside.cpp:53-62
__device__ __forceinline__ bool ray_box(const double *box, const double *o, const double *r) {
    double tmin = 0.0, tmax = __longlong_as_double(0x7ff0000000000000LL);
    return update_ray_interval(o[0], r[0], box[0], box[3], tmin, tmax) &&
           update_ray_interval(o[1], r[1], box[1], box[4], tmin, tmax) &&
           update_ray_interval(o[2], r[2], box[2], box[5], tmin, tmax);
}

enum : int { kMiss = 0, kHit = 1, kAmbiguous = 2 };

// Moller-Trumbore with the reference's ambiguity bands, src/inside.cpp:140-182.
// a = v0, edge1 = e1, edge2 = e2 of the Eberly record (equal to b-a, c-a).
__device__ __forceinline__ int moller_trumbore(const double *p, const double *ray,
                                               const double2 *r) {
    const double ax = r[0].x, ay = r[0].y, az = r[1].x;
    const double e1x = r[1].y, e1y = r[2].x, e1z = r[2].y;
    const double e2x = r[3].x, e2y = r[3].y, e2z = r[4].x;
    const double sx = p[0] - ax, sy = p[1] - ay, sz = p[2] - az;
    // rxe2 = ray x e2
    const double qx = ray[1] * e2z - ray[2] * e2y;
    const double qy = ray[2] * e2x - ray[0] * e2z;
    const double qz = ray[0] * e2y - ray[1] * e2x;
    const double det = e1x * qx + e1y * qy + e1z * qz;
    const double nx = e1y * e2z - e1z * e2y;
    const double ny = e1z * e2x - e1x * e2z;
    const double nz = e1x * e2y - e1y * e2x;
    const double nlen = sqrt(nx * nx + ny * ny + nz * nz);
    const double det_tol = kRayEps * nlen;
    if (fabs(det) <= det_tol) {
        if (nlen == 0.0) return kMiss;
        double es = 1.0;
        const double l1 = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
        const double l2 = sqrt(e2x * e2x + e2y * e2y + e2z * e2z);
        if (es < l1) es = l1;
        if (es < l2) es = l2;
        const double plane = fabs(nx * sx + ny * sy + nz * sz) / nlen;
        return plane <= kRayEps * es ? kAmbiguous : kMiss;
    }
    const double u = (sx * qx + sy * qy + sz * qz) / det;
    if (u < -kRayEps || u - 1.0 > kRayEps) return kMiss;
    // sxe1 = s x e1
    const double tx = sy * e1z - sz * e1y;
    const double ty = sz * e1x - sx * e1z;
    const double tz = sx * e1y - sy * e1x;
    const double v = (ray[0] * tx + ray[1] * ty + ray[2] * tz) / det;
    if (v < -kRayEps || u + v - 1.0 > kRayEps) return kMiss;
    const double t = (e2x * tx + e2y * ty + e2z * tz) / det;
    if (t <= kRayEps) return kMiss;
    const double w = 1.0 - u - v;
    if (u <= kRayEps || v <= kRayEps || w <= kRayEps) return kAmbiguous;
    return kHit;
}

// Parity count of one ray through every node whose padded box it meets
// (src/inside.cpp:78-111); an ambiguous triangle ends the cast.  The count is
// independent of the visiting order.
__device__ __forceinline__ int count_ray_hits(const SceneView &s, const double *p,
                                              const double *ray, bool &ambiguous) {
    ambiguous = false;
    int hits = 0;
    auto leaf = [&](int j) -> bool {
        const int b = leaf_first(j, s.n_prims, s.depth);
        const int e = leaf_first(j + 1, s.n_prims, s.depth);
        for (int k = b; k < e; ++k) {
            const int h = moller_trumbore(p, ray, s.tri64 + 7 * k);
            if (h == kAmbiguous) return true;
            if (h == kHit) ++hits;
        }
        return false;
    };
    if (!ray_box(s.box64 + 6, p, ray)) return 0;
    if (s.depth == 0) {
        ambiguous = leaf(0);
        return hits;
    }
    const unsigned leaf_base = 1u << s.depth;
    const unsigned last_internal = leaf_base >> 1;
    unsigned cur = 1, bits = 0;
    for (;;) {
        const bool hl = ray_box(s.box64 + 6 * (2 * cur), p, ray);
        const bool hr = ray_box(s.box64 + 6 * (2 * cur + 1), p, ray);
        bool descended = false;
        if (cur >= last_internal) {
            if (hl && leaf(static_cast<int>(2 * cur - leaf_base))) {
                ambiguous = true;
                return hits;
            }
            if (hr && leaf(static_cast<int>(2 * cur + 1 - leaf_base))) {
                ambiguous = true;
                return hits;
            }
        } else if (hl) {
            bits = (bits << 1) | (hr ? 1u : 0u);
            cur = 2 * cur;
            descended = true;
        } else if (hr) {
            bits <<= 1;
            cur = 2 * cur + 1;
            descended = true;
        }
        if (descended) continue;
        if (bits == 0) return hits;
        const int tz = __ffs(bits) - 1;
        bits >>= tz;
        cur >>= tz;
        bits ^= 1u;
        cur ^= 1u;  // the right sibling, whose box the ray already meets
    }
}

}  // namespace wosb
