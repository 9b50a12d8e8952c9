// Device build of a scene: the binary FP64 tree, the leaf-slot records, the
// 32-wide FP32 tree with its slab bounds and primitive blocks, written
// straight into the scene arena.  The result is bit-identical to the host
// build (scene_build.cpp), array by array:
//
// * Both trees are median splits at fixed slot positions (the binary tree's
//   implicit layout, the wide tree's chunk multiples) by the order
//   (centroid coordinate on the node's longest axis, primitive id), with the
//   leaves in primitive-id order (src/bvh.cpp:143-230 for the split rule).
//   The set of primitives on each side of a split depends only on that
//   order, not on how a builder arranges them, so the trees are unique.
//   Here every axis keeps a list of the primitives sorted by
//   (centroid, id) (one stable radix sort per axis); a level of splits marks
//   the left part of each node in its axis list and stably partitions all
//   lists by the marks, which keeps every node's lists sorted.
// * Node boxes are minima and maxima of the primitives' boxes (exact in any
//   order); the records, slab fits and rounding repeat the host's
//   expressions operation by operation, and this translation unit is
//   compiled without FMA contraction, so they round alike.
// * Which slot ranges split, and where, depends only on the primitive
//   count: the host lays out every level of splits, the device only
//   decides axes and sides.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "context_internal.h"
#include "kernels.h"

namespace wosb {

namespace {

constexpr long long kKeyMax = 0x7fffffffffffffffLL;
constexpr long long kKeyMin = -0x7fffffffffffffffLL - 1;

// Signed integer keys that order like the doubles (finite values, no -0.0).
__device__ __forceinline__ long long okey(double d) {
    const long long b = __double_as_longlong(d);
    return b >= 0 ? b : b ^ 0x7fffffffffffffffLL;
}
__device__ __forceinline__ double from_okey(long long k) {
    return __longlong_as_double(k >= 0 ? k : k ^ 0x7fffffffffffffffLL);
}

__host__ __device__ __forceinline__ long long first_slot(long long k, long long n, int level) {
    return static_cast<long long>(
        (static_cast<unsigned long long>(k) * static_cast<unsigned long long>(n)) >> level);
}

// Node of `slot` at `level` of the implicit binary tree: the largest k with
// first_slot(k) <= slot.
__device__ __forceinline__ int node_of(long long slot, long long n, int level) {
    const unsigned long long t = static_cast<unsigned long long>(slot + 1) << level;
    return static_cast<int>((t + static_cast<unsigned long long>(n) - 1) /
                            static_cast<unsigned long long>(n)) - 1;
}

struct Items {
    double *lo[3], *hi[3], *c[3];
};

// Primitive boxes and centroids, as build_scene computes them.
__global__ void items_kernel(int dim, const double *__restrict__ verts,
                             const int *__restrict__ prims, int n, Items it) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    auto V = [&](int v, int k) { return verts[static_cast<size_t>(dim) * v + k]; };
    if (dim == 2) {
        const int a = prims[2 * p], b = prims[2 * p + 1];
        for (int k = 0; k < 2; ++k) {
            it.lo[k][p] = fmin(V(a, k), V(b, k)) + 0.0;
            it.hi[k][p] = fmax(V(a, k), V(b, k)) + 0.0;
            it.c[k][p] = (V(a, k) + V(b, k)) / 2.0 + 0.0;
        }
    } else {
        const int a = prims[3 * p], b = prims[3 * p + 1], c = prims[3 * p + 2];
        for (int k = 0; k < 3; ++k) {
            it.lo[k][p] = fmin(fmin(V(a, k), V(b, k)), V(c, k)) + 0.0;
            it.hi[k][p] = fmax(fmax(V(a, k), V(b, k)), V(c, k)) + 0.0;
            it.c[k][p] = (V(a, k) + V(b, k) + V(c, k)) / 3.0 + 0.0;
        }
    }
}

// Radix-sort keys of the centroids along one axis (unsigned, order-preserving).
__global__ void sort_keys_kernel(const double *__restrict__ c, int n,
                                 unsigned long long *keys, int *vals) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const long long b = __double_as_longlong(c[p]);
    keys[p] = b >= 0 ? (static_cast<unsigned long long>(b) | 0x8000000000000000ULL)
                     : ~static_cast<unsigned long long>(b);
    vals[p] = p;
}

// A level of splits.  Binary tree: segment k of `level` is node k, its
// slots [first_slot(k), first_slot(k + 1)), split at first_slot(2k + 1) of
// the next level.  Wide tree: an explicit list of slot ranges and split
// points, sorted by start; slots outside every range stay where they are.
struct Segs {
    int binary;          // 1: the binary tree's level `level`; 0: explicit list
    int level;
    long long n;
    const int3 *list;    // explicit: {start, end, split}
    int count;           // segments of the level
};

__device__ __forceinline__ int seg_of(const Segs &g, long long slot) {
    if (g.binary) return node_of(slot, g.n, g.level);
    int lo = 0, hi = g.count - 1, found = -1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        if (g.list[mid].x <= slot) {
            found = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    return found >= 0 && slot < g.list[found].y ? found : -1;
}
__device__ __forceinline__ void seg_range(const Segs &g, int s, long long &start, long long &end,
                                          long long &split) {
    if (g.binary) {
        start = first_slot(s, g.n, g.level);
        end = first_slot(s + 1, g.n, g.level);
        split = first_slot(2ll * s + 1, g.n, g.level + 1);
    } else {
        const int3 v = g.list[s];
        start = v.x;
        end = v.y;
        split = v.z;
    }
}

__global__ void fill_keys_kernel(long long *box, int count, int dim) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<long long>(count) * 2 * dim) return;
    box[t] = (t % (2 * dim)) < dim ? kKeyMax : kKeyMin;
}

// Box of every segment: min of the primitives' lo, max of their hi, as
// ordered keys.  Each warp reduces runs of lanes in one segment, then one
// lane per run updates the segment atomically.
__global__ void seg_box_kernel(Segs g, int dim, const int *__restrict__ list, Items it,
                               long long *box) {
    const long long slot = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool valid = slot < g.n;
    const int s = valid ? seg_of(g, slot) : -1;
    const int p = valid && s >= 0 ? list[slot] : 0;
    const int next = __shfl_down_sync(0xffffffffu, s, 1);
    const bool tail = lane == 31 || next != s;
    for (int q = 0; q < 2 * dim; ++q) {
        const bool lo = q < dim;
        long long v = lo ? kKeyMax : kKeyMin;
        if (s >= 0) v = lo ? okey(it.lo[q][p]) : okey(it.hi[q - dim][p]);
        for (int off = 1; off < 32; off <<= 1) {
            const long long o = __shfl_up_sync(0xffffffffu, v, off);
            const int os = __shfl_up_sync(0xffffffffu, s, off);
            if (lane >= off && os == s) v = lo ? min(v, o) : max(v, o);
        }
        if (s >= 0 && tail) {
            if (lo) atomicMin(box + static_cast<long long>(s) * 2 * dim + q, v);
            else atomicMax(box + static_cast<long long>(s) * 2 * dim + q, v);
        }
    }
}

// Longest axis of each segment's box, ties to the lower axis (src/bvh.cpp:
// 218-224); for the binary tree also the node's box64 entry.
__global__ void seg_axis_kernel(int count, int dim, const long long *__restrict__ box,
                                int *axis, double *box64, int level) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int k = 0; k < dim; ++k) {
        lo[k] = from_okey(box[static_cast<long long>(s) * 2 * dim + k]);
        hi[k] = from_okey(box[static_cast<long long>(s) * 2 * dim + dim + k]);
    }
    if (box64 != nullptr) {
        double *b = box64 + (static_cast<long long>(1) << level) * 2 * dim +
                    static_cast<long long>(s) * 2 * dim;
        for (int k = 0; k < dim; ++k) {
            b[k] = lo[k];
            b[dim + k] = hi[k];
        }
    }
    const double ex = hi[0] - lo[0], ey = hi[1] - lo[1];
    const double ez = dim == 3 ? hi[2] - lo[2] : -1.0;
    axis[s] = (ex >= ey) ? (ex >= ez ? 0 : 2) : (ey >= ez ? 1 : 2);
}

// Side of every primitive: 1 if it is among the first (split - start)
// entries of its segment's list along the segment's axis (or outside every
// splitting segment).
__global__ void side_kernel(Segs g, const int *__restrict__ l0, const int *__restrict__ l1,
                            const int *__restrict__ l2, const int *__restrict__ axis,
                            unsigned char *left) {
    const long long slot = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (slot >= g.n) return;
    const int s = seg_of(g, slot);
    if (s < 0) {
        left[l0[slot]] = 1;
        return;
    }
    long long start, end, split;
    seg_range(g, s, start, end, split);
    const int a = axis[s];
    const int *l = a == 0 ? l0 : (a == 1 ? l1 : l2);
    left[l[slot]] = slot < split ? 1 : 0;
}

__global__ void gather_side_kernel(long long n, const int *__restrict__ list,
                                   const unsigned char *__restrict__ left, int *flag) {
    const long long slot = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (slot < n) flag[slot] = left[list[slot]];
}

// Stable partition of one list within every splitting segment: the left
// primitives keep their order at the front, the right ones after them.
// `before` is the exclusive prefix sum of the flags over all slots.
__global__ void partition_kernel(Segs g, const int *__restrict__ list,
                                 const int *__restrict__ flag, const int *__restrict__ before,
                                 int *out) {
    const long long slot = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (slot >= g.n) return;
    const int s = seg_of(g, slot);
    if (s < 0) {
        out[slot] = list[slot];
        return;
    }
    long long start, end, split;
    seg_range(g, s, start, end, split);
    const long long lefts = before[slot] - before[start];
    const long long dst = flag[slot] ? start + lefts : split + (slot - start - lefts);
    out[dst] = list[slot];
}

// Groups of at most `width` consecutive slots sorted by primitive id: the
// binary tree's leaves (first_slot boundaries) or the wide tree's 32-slot
// clusters.
__global__ void group_sort_kernel(int binary, int level, long long n, int groups,
                                  const int *__restrict__ list, int *out) {
    const int gidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (gidx >= groups) return;
    const long long s = binary ? first_slot(gidx, n, level) : 32ll * gidx;
    const long long e = binary ? first_slot(gidx + 1, n, level) : min(n, 32ll * gidx + 32);
    int v[32];
    const int m = static_cast<int>(e - s);
    for (int q = 0; q < m; ++q) v[q] = list[s + q];
    for (int q = 1; q < m; ++q) {
        const int x = v[q];
        int u = q - 1;
        while (u >= 0 && v[u] > x) {
            v[u + 1] = v[u];
            --u;
        }
        v[u + 1] = x;
    }
    for (int q = 0; q < m; ++q) out[s + q] = v[q];
}

// Leaf-slot records of the binary tree (build_scene's record loops).
__global__ void records2_kernel(const double *__restrict__ verts, const int *__restrict__ prims,
                                const int *__restrict__ bids, const int *__restrict__ order,
                                int n, double *seg64, int *segid, float *seg32, float *seg32inv,
                                int *slot_verts) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = order[s];
    const int a = prims[2 * p], b = prims[2 * p + 1];
    const double g[4] = {verts[2 * a], verts[2 * a + 1], verts[2 * b], verts[2 * b + 1]};
    for (int k = 0; k < 4; ++k) seg64[4 * s + k] = g[k];
    const float x0 = static_cast<float>(g[0]), y0 = static_cast<float>(g[1]);
    const float vx = static_cast<float>(g[2] - g[0]), vy = static_cast<float>(g[3] - g[1]);
    seg32[4 * s + 0] = x0;
    seg32[4 * s + 1] = y0;
    seg32[4 * s + 2] = vx;
    seg32[4 * s + 3] = vy;
    seg32inv[s] = static_cast<float>(
        1.0 / (static_cast<double>(vx) * vx + static_cast<double>(vy) * vy));
    segid[2 * s] = bids ? bids[p] : 0;
    segid[2 * s + 1] = p;
    slot_verts[2 * s] = a;
    slot_verts[2 * s + 1] = b;
}

__global__ void records3_kernel(const double *__restrict__ verts, const int *__restrict__ prims,
                                const int *__restrict__ order, int n, double *tri64,
                                float *tri32, int *slot_verts) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = order[s];
    const int a = prims[3 * p], b = prims[3 * p + 1], c = prims[3 * p + 2];
    auto V = [&](int v, int k) { return verts[3 * static_cast<size_t>(v) + k]; };
    const double v0[3] = {V(a, 0), V(a, 1), V(a, 2)};
    const double e1[3] = {V(b, 0) - V(a, 0), V(b, 1) - V(a, 1), V(b, 2) - V(a, 2)};
    const double e2[3] = {V(c, 0) - V(a, 0), V(c, 1) - V(a, 1), V(c, 2) - V(a, 2)};
    const double A = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
    const double Bb = e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2];
    const double Cc = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
    const double det = A * Cc - Bb * Bb;
    const double denom = A - 2 * Bb + Cc;
    const double rec64[14] = {v0[0], v0[1], v0[2], e1[0], e1[1], e1[2], e2[0],
                              e2[1], e2[2], A,     Bb,    Cc,    det,   denom};
    for (int k = 0; k < 14; ++k) tri64[14 * static_cast<size_t>(s) + k] = rec64[k];
    float fv[3], fe1[3], fe2[3];
    for (int k = 0; k < 3; ++k) {
        fv[k] = static_cast<float>(v0[k]);
        fe1[k] = static_cast<float>(e1[k]);
        fe2[k] = static_cast<float>(e2[k]);
    }
    double fa = 0, fb = 0, fc = 0;
    for (int k = 0; k < 3; ++k) {
        fa += static_cast<double>(fe1[k]) * fe1[k];
        fb += static_cast<double>(fe1[k]) * fe2[k];
        fc += static_cast<double>(fe2[k]) * fe2[k];
    }
    const double fdet = fa * fc - fb * fb;
    float *o = tri32 + 16 * static_cast<size_t>(s);
    o[0] = fv[0]; o[1] = fv[1]; o[2] = fv[2]; o[3] = static_cast<float>(fa);
    o[4] = fe1[0]; o[5] = fe1[1]; o[6] = fe1[2]; o[7] = static_cast<float>(fb);
    o[8] = fe2[0]; o[9] = fe2[1]; o[10] = fe2[2]; o[11] = static_cast<float>(fc);
    o[12] = static_cast<float>(fdet);
    o[13] = static_cast<float>(1.0 / fdet);
    o[14] = static_cast<float>(1.0 / fa);
    o[15] = static_cast<float>(1.0 / fc);
    slot_verts[3 * s] = a;
    slot_verts[3 * s + 1] = b;
    slot_verts[3 * s + 2] = c;
}

__global__ void inverse_kernel(const int *__restrict__ order, int n, int *bin_of) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) bin_of[order[s]] = s;
}

__global__ void wide2bin_kernel(const int *__restrict__ witem, const int *__restrict__ bin_of,
                                int n, int npad, int *wide2bin) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) wide2bin[s] = bin_of[witem[s]];
    else if (s < npad) wide2bin[s] = -1;
}

// Height-0 boxes of the wide tree: the primitives' boxes in wide-slot order.
__global__ void level0_kernel(int dim, const int *__restrict__ witem, int n, Items it,
                              double *lv) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = witem[s];
    for (int k = 0; k < dim; ++k) {
        lv[static_cast<size_t>(s) * 2 * dim + k] = it.lo[k][p];
        lv[static_cast<size_t>(s) * 2 * dim + dim + k] = it.hi[k][p];
    }
}

// Height-h boxes from height h-1: min / max over the 32 children in order.
__global__ void level_up_kernel(int dim, const double *__restrict__ below, long long cnt_below,
                                long long cnt, double *lv) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const int nc = 2 * dim;
    const long long c0 = 32 * i, c1 = min(cnt_below, 32 * i + 32);
    for (int k = 0; k < nc; ++k) {
        double v = below[c0 * nc + k];
        for (long long c = c0 + 1; c < c1; ++c) {
            const double x = below[c * nc + k];
            v = k < dim ? (x < v ? x : v) : (v < x ? x : v);
        }
        lv[i * nc + k] = v;
    }
}

__device__ __forceinline__ float round_down(double v) {
    float f = static_cast<float>(v);
    if (static_cast<double>(f) > v) f = nextafterf(f, -INFINITY);
    return f;
}
__device__ __forceinline__ float round_up(double v) {
    float f = static_cast<float>(v);
    if (static_cast<double>(f) < v) f = nextafterf(f, INFINITY);
    return f;
}

// Padding of the child-group blocks: empty boxes, unbounded slabs.
__global__ void wbox_fill_kernel(int dim, float *wbox, int total) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int nc = 2 * dim, nbox = nc + dim + 2;
    const int f = (t / 32) % nbox;
    float fill = 0.0f;
    if (f < dim) fill = INFINITY;
    else if (f < nc) fill = -INFINITY;
    else if (f == nbox - 1) fill = INFINITY;
    wbox[t] = fill;
}

// Box and slab of every height-h node (build_wide's node loop, slab_of):
// one warp per node.  Lane c sums the points of the node's child c (its
// `chunk` consecutive points, in wide-slot and vertex order) from zero; lane
// 0 adds the 32 partial sums in child order, as slab_of does, and fits the
// slab; the thickness is a maximum, reduced over the lanes.
__global__ void wide_node_kernel(int dim, long long cnt, long long span, int n,
                                 const double *__restrict__ lv, const int *__restrict__ witem,
                                 const double *__restrict__ verts,
                                 const int *__restrict__ prims, int off, double widen,
                                 float *wbox) {
    constexpr unsigned kAll = 0xffffffffu;
    const long long i = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= cnt) return;  // whole warps leave together
    const int nc = 2 * dim, nbox = nc + dim + 2;
    float *blk = wbox + off + (i / 32) * nbox * 32;
    const int slot_lane = static_cast<int>(i % 32);
    if (lane == 0) {
        for (int k = 0; k < nc; ++k) {
            const double v = lv[i * nc + k];
            blk[k * 32 + slot_lane] = k < dim ? round_down(v - widen) : round_up(v + widen);
        }
    }
    const long long s0 = i * span, s1 = min(static_cast<long long>(n), (i + 1) * span);
    const long long m = (s1 - s0) * dim;
    const long long chunk = (span / 32) * dim;
    const long long q0 = lane * chunk, q1 = min(m, q0 + chunk);
    auto point = [&](long long q, int k) {
        const long long sl = s0 + q / dim;
        const int v = prims[static_cast<size_t>(dim) * witem[sl] + (q % dim)];
        return verts[static_cast<size_t>(dim) * v + k];
    };
    // mean: chunk sums, then their sum in chunk order
    double part[3] = {0, 0, 0};
    for (long long q = q0; q < q1; ++q)
        for (int k = 0; k < dim; ++k) part[k] += point(q, k);
    double mean[3] = {0, 0, 0};
    for (int c = 0; c < 32; ++c) {
        for (int k = 0; k < dim; ++k) {
            const double v = __shfl_sync(kAll, part[k], c);
            if (static_cast<long long>(c) * chunk < m) mean[k] += v;
        }
    }
    for (int k = 0; k < dim; ++k) mean[k] /= static_cast<double>(m);
    // covariance: the same two levels
    double pa[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (long long q = q0; q < q1; ++q) {
        double pt[3];
        for (int k = 0; k < dim; ++k) pt[k] = point(q, k);
        for (int a = 0; a < dim; ++a)
            for (int b = 0; b < dim; ++b) pa[a][b] += (pt[a] - mean[a]) * (pt[b] - mean[b]);
    }
    double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int c = 0; c < 32; ++c) {
        for (int a = 0; a < dim; ++a) {
            for (int b = 0; b < dim; ++b) {
                const double v = __shfl_sync(kAll, pa[a][b], c);
                if (static_cast<long long>(c) * chunk < m) A[a][b] += v;
            }
        }
    }
    // every lane runs the same Jacobi sweeps on the same matrix
    double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 32; ++sweep) {
        double offd = 0.0;
        for (int a = 0; a < dim; ++a)
            for (int b = a + 1; b < dim; ++b) offd += A[a][b] * A[a][b];
        if (offd < 1e-30) break;
        for (int a = 0; a < dim; ++a) {
            for (int b = a + 1; b < dim; ++b) {
                if (fabs(A[a][b]) < 1e-300) continue;
                const double theta = (A[b][b] - A[a][a]) / (2.0 * A[a][b]);
                const double t = fabs(theta) > 1e150
                                     ? 0.5 / theta
                                     : (theta >= 0.0 ? 1.0 : -1.0) /
                                           (fabs(theta) + sqrt(theta * theta + 1.0));
                const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                for (int k = 0; k < dim; ++k) {
                    const double x = A[k][a], y = A[k][b];
                    A[k][a] = cs * x - sn * y;
                    A[k][b] = sn * x + cs * y;
                }
                for (int k = 0; k < dim; ++k) {
                    const double x = A[a][k], y = A[b][k];
                    A[a][k] = cs * x - sn * y;
                    A[b][k] = sn * x + cs * y;
                }
                for (int k = 0; k < dim; ++k) {
                    const double x = V[k][a], y = V[k][b];
                    V[k][a] = cs * x - sn * y;
                    V[k][b] = sn * x + cs * y;
                }
            }
        }
    }
    int best = 0;
    for (int a = 1; a < dim; ++a)
        if (A[a][a] < A[best][best]) best = a;
    double nrm[3] = {0, 0, 0}, len = 0.0;
    for (int k = 0; k < dim; ++k) {
        nrm[k] = V[k][best];
        len += nrm[k] * nrm[k];
    }
    len = sqrt(len);
    for (int k = 0; k < dim; ++k) nrm[k] /= len;
    double c = 0.0;
    for (int k = 0; k < dim; ++k) c += nrm[k] * mean[k];
    float nf[3] = {0, 0, 0};
    for (int k = 0; k < dim; ++k) nf[k] = static_cast<float>(nrm[k]);
    const float cf = static_cast<float>(c);
    double t32 = 0.0;
    for (long long q = q0; q < q1; ++q) {
        double t = -static_cast<double>(cf);
        for (int k = 0; k < dim; ++k) t += static_cast<double>(nf[k]) * point(q, k);
        t32 = t32 < fabs(t) ? fabs(t) : t32;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double other = __shfl_xor_sync(kAll, t32, o);
        t32 = t32 < other ? other : t32;
    }
    if (lane == 0) {
        for (int k = 0; k < dim; ++k) blk[(nc + k) * 32 + slot_lane] = nf[k];
        blk[(nc + dim) * 32 + slot_lane] = cf;
        blk[(nc + dim + 1) * 32 + slot_lane] = round_up(t32 + 4.0 * widen);
    }
}

// Primitive blocks of the wide tree from the binary slots' FP32 records.
__global__ void wprim_kernel(int dim, int n, int npad, const int *__restrict__ wide2bin,
                             const float *__restrict__ rec32, const float *__restrict__ inv32,
                             float *wprim) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= npad) return;
    float rec[16];
    const int na = dim == 2 ? 5 : 16;
    if (s >= n) {
        for (int k = 0; k < 16; ++k) rec[k] = 0.0f;
        rec[0] = rec[1] = 1e30f;
        if (dim == 3) rec[2] = 1e30f;
    } else if (dim == 2) {
        const int b = wide2bin[s];
        for (int k = 0; k < 4; ++k) rec[k] = rec32[4 * static_cast<size_t>(b) + k];
        rec[4] = inv32[b];
    } else {
        const int b = wide2bin[s];
        for (int k = 0; k < 16; ++k) rec[k] = rec32[16 * static_cast<size_t>(b) + k];
    }
    float *blk = wprim + static_cast<size_t>(s / 32) * na * 32;
    for (int k = 0; k < na; ++k) blk[k * 32 + s % 32] = rec[k];
}

unsigned blocks_for(long long n, int threads = 256) {
    return static_cast<unsigned>(std::max<long long>(1, (n + threads - 1) / threads));
}

// The wide tree's levels of splits (WideBuilder in scene_build.cpp): a task
// (s, e, ch) splits [s, e) at chunk multiples of 32^ch; a range of at most
// one chunk becomes a node of height ch, which splits again at 32^(ch-1)
// until it is a cluster of at most 32 primitives.
std::vector<std::vector<int3>> wide_rounds(int n, int H) {
    struct Task {
        long long s, e;
        int ch;
    };
    std::vector<Task> frontier;
    auto node = [&](long long s, long long e, int height, std::vector<Task> &out) {
        // node(s, e, height): a cluster, or a split task at the next height
        while (height > 1) {
            long long chunk = 1;
            for (int h = 1; h < height; ++h) chunk *= 32;
            const long long nch = (e - s + chunk - 1) / chunk;
            if (nch > 1) {
                out.push_back(Task{s, e, height - 1});
                return;
            }
            --height;
        }
    };
    node(0, n, H, frontier);
    std::vector<std::vector<int3>> rounds;
    while (!frontier.empty()) {
        std::vector<int3> round;
        std::vector<Task> next;
        for (const Task &t : frontier) {
            long long chunk = 1;
            for (int h = 0; h < t.ch; ++h) chunk *= 32;
            const long long nch = (t.e - t.s + chunk - 1) / chunk;
            const long long mid = t.s + ((nch + 1) / 2) * chunk;
            round.push_back(make_int3(static_cast<int>(t.s), static_cast<int>(t.e),
                                      static_cast<int>(mid)));
            for (const auto &half : {std::make_pair(t.s, mid), std::make_pair(mid, t.e)}) {
                const long long hn = (half.second - half.first + chunk - 1) / chunk;
                if (hn > 1) next.push_back(Task{half.first, half.second, t.ch});
                else node(half.first, half.second, t.ch, next);
            }
        }
        std::sort(round.begin(), round.end(), [](int3 a, int3 b) { return a.x < b.x; });
        rounds.push_back(std::move(round));
        frontier = std::move(next);
    }
    return rounds;
}

}  // namespace

ArenaLayout arena_layout(const HostScene &m) {
    const size_t n = static_cast<size_t>(m.n_prims);
    const int na = m.dim == 2 ? 5 : 16;
    const size_t bytes[ArenaLayout::kParts] = {
        (static_cast<size_t>(1) << (m.depth + 1)) * 2 * m.dim * sizeof(double),
        m.dim == 2 ? n * 4 * sizeof(double) : 0,
        m.dim == 2 ? n * 2 * sizeof(int) : 0,
        m.dim == 3 ? n * 14 * sizeof(double) : 0,
        static_cast<size_t>(m.w_box_total) * sizeof(float),
        static_cast<size_t>(m.w_npad) * na * sizeof(float),
        static_cast<size_t>(m.w_npad) * sizeof(int),
        8 * sizeof(int),
        n * m.dim * sizeof(int),
    };
    ArenaLayout L{};
    size_t total = 0;
    for (int k = 0; k < ArenaLayout::kParts; ++k) {
        L.bytes[k] = bytes[k];
        L.offset[k] = total;
        total += (std::max<size_t>(bytes[k], 16) + 255) / 256 * 256;
    }
    L.total = total;
    return L;
}

cudaError_t SceneDevice::build_on_device(const HostScene &m, cudaStream_t stream) {
    const int dim = m.dim, n = m.n_prims, D = m.depth, H = m.wH;
    const ArenaLayout L = arena_layout(m);
    cudaError_t e = arena.reserve(L.total);
    if (e != cudaSuccess) return e;
    auto *base = static_cast<char *>(arena.ptr);
    if ((e = cudaMemsetAsync(base, 0, L.total, stream)) != cudaSuccess) return e;
    auto part = [&](int k) { return base + L.offset[k]; };
    auto *box64 = reinterpret_cast<double *>(part(0));
    auto *seg64 = reinterpret_cast<double *>(part(1));
    auto *segid = reinterpret_cast<int *>(part(2));
    auto *tri64 = reinterpret_cast<double *>(part(3));
    auto *wbox = reinterpret_cast<float *>(part(4));
    auto *wprim = reinterpret_cast<float *>(part(5));
    auto *wide2bin = reinterpret_cast<int *>(part(6));
    auto *offs = reinterpret_cast<int *>(part(7));
    auto *sverts = reinterpret_cast<int *>(part(8));

    // the host's plan of the wide tree's splits
    const std::vector<std::vector<int3>> rounds = wide_rounds(n, H);
    size_t max_round = 1, round_total = 0;
    for (const auto &r : rounds) {
        max_round = std::max(max_round, r.size());
        round_total += r.size();
    }
    std::vector<int3> round_host;
    round_host.reserve(round_total);
    for (const auto &r : rounds) round_host.insert(round_host.end(), r.begin(), r.end());
    std::vector<long long> cnt(H + 1);
    cnt[0] = n;
    for (int h = 1; h <= H; ++h) cnt[h] = (cnt[h - 1] + 31) / 32;
    size_t lv_total = 0;
    for (int h = 0; h <= H; ++h) lv_total += static_cast<size_t>(cnt[h]) * 2 * dim;

    // temporaries, one stream-ordered allocation
    size_t sort_bytes = 0, scan_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, static_cast<unsigned long long *>(nullptr),
                                    static_cast<unsigned long long *>(nullptr),
                                    static_cast<int *>(nullptr), static_cast<int *>(nullptr), n,
                                    0, 64, stream);
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, static_cast<int *>(nullptr),
                                  static_cast<int *>(nullptr), n, stream);
    const size_t nn = static_cast<size_t>(n);
    const long long max_nodes = std::max<long long>(static_cast<long long>(max_round),
                                                    1ll << std::min(D, 30));
    struct Slab {
        size_t bytes;
        size_t at;
    };
    std::vector<Slab> slabs;
    size_t total = 0;
    auto take = [&](size_t bytes) {
        slabs.push_back(Slab{bytes, total});
        total += (std::max<size_t>(bytes, 16) + 255) / 256 * 256;
        return slabs.size() - 1;
    };
    const size_t t_verts = take(m.verts.size() * sizeof(double));
    const size_t t_prims = take(m.prims.size() * sizeof(int));
    const size_t t_bids = take(dim == 2 ? nn * sizeof(int) : 0);
    const size_t t_items = take(nn * 9 * sizeof(double));
    const size_t t_keys = take(nn * 2 * sizeof(unsigned long long));
    const size_t t_vals = take(nn * sizeof(int));
    const size_t t_lists = take(nn * 3 * sizeof(int));      // per-axis lists
    const size_t t_lists2 = take(nn * 3 * sizeof(int));     // partition targets
    const size_t t_sorted = take(nn * 3 * sizeof(int));     // the presorted lists
    const size_t t_left = take(nn);
    const size_t t_flag = take(nn * sizeof(int));
    const size_t t_before = take(nn * sizeof(int));
    const size_t t_box = take(static_cast<size_t>(max_nodes) * 2 * dim * sizeof(long long));
    const size_t t_axis = take(static_cast<size_t>(max_nodes) * sizeof(int));
    const size_t t_rounds = take(round_host.size() * sizeof(int3));
    const size_t t_order = take(nn * sizeof(int));
    const size_t t_witem = take(nn * sizeof(int));
    const size_t t_binof = take(nn * sizeof(int));
    const size_t t_rec32 = take(nn * (dim == 2 ? 4 : 16) * sizeof(float));
    const size_t t_inv32 = take(nn * sizeof(float));
    const size_t t_lv = take(lv_total * sizeof(double));
    const size_t t_cub = take(std::max(sort_bytes, scan_bytes));
    void *tmp = nullptr;
    if ((e = cudaMallocAsync(&tmp, total, stream)) != cudaSuccess) return e;
    auto at = [&](size_t k) { return static_cast<char *>(tmp) + slabs[k].at; };
    auto *d_verts = reinterpret_cast<double *>(at(t_verts));
    auto *d_prims = reinterpret_cast<int *>(at(t_prims));
    auto *d_bids = dim == 2 ? reinterpret_cast<int *>(at(t_bids)) : nullptr;
    Items it{};
    auto *itd = reinterpret_cast<double *>(at(t_items));
    for (int k = 0; k < 3; ++k) {
        it.lo[k] = itd + nn * k;
        it.hi[k] = itd + nn * (3 + k);
        it.c[k] = itd + nn * (6 + k);
    }
    auto *keys = reinterpret_cast<unsigned long long *>(at(t_keys));
    auto *vals = reinterpret_cast<int *>(at(t_vals));
    int *lists[3], *lists2[3], *sorted[3];
    for (int k = 0; k < 3; ++k) {
        lists[k] = reinterpret_cast<int *>(at(t_lists)) + nn * k;
        lists2[k] = reinterpret_cast<int *>(at(t_lists2)) + nn * k;
        sorted[k] = reinterpret_cast<int *>(at(t_sorted)) + nn * k;
    }
    auto *left = reinterpret_cast<unsigned char *>(at(t_left));
    auto *flag = reinterpret_cast<int *>(at(t_flag));
    auto *before = reinterpret_cast<int *>(at(t_before));
    auto *segbox = reinterpret_cast<long long *>(at(t_box));
    auto *axis = reinterpret_cast<int *>(at(t_axis));
    auto *d_rounds = reinterpret_cast<int3 *>(at(t_rounds));
    auto *order = reinterpret_cast<int *>(at(t_order));
    auto *witem = reinterpret_cast<int *>(at(t_witem));
    auto *bin_of = reinterpret_cast<int *>(at(t_binof));
    auto *rec32 = reinterpret_cast<float *>(at(t_rec32));
    auto *inv32 = reinterpret_cast<float *>(at(t_inv32));
    auto *lv = reinterpret_cast<double *>(at(t_lv));
    void *cub_tmp = at(t_cub);

    auto run = [&]() -> cudaError_t {
        cudaError_t r;
        if ((r = cudaMemcpyAsync(d_verts, m.verts.data(), m.verts.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, stream)) != cudaSuccess) return r;
        if ((r = cudaMemcpyAsync(d_prims, m.prims.data(), m.prims.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, stream)) != cudaSuccess) return r;
        if (d_bids && (r = cudaMemcpyAsync(d_bids, m.boundary_ids.data(), nn * sizeof(int),
                                           cudaMemcpyHostToDevice, stream)) != cudaSuccess) {
            return r;
        }
        if (!round_host.empty() &&
            (r = cudaMemcpyAsync(d_rounds, round_host.data(), round_host.size() * sizeof(int3),
                                 cudaMemcpyHostToDevice, stream)) != cudaSuccess) {
            return r;
        }
        if ((r = cudaMemcpyAsync(offs, m.w_off, 8 * sizeof(int), cudaMemcpyHostToDevice,
                                 stream)) != cudaSuccess) return r;
        // the permutations start as valid indices (0), whatever a kernel misses
        for (int *perm : {order, witem, bin_of}) {
            if ((r = cudaMemsetAsync(perm, 0, nn * sizeof(int), stream)) != cudaSuccess) return r;
        }
        items_kernel<<<blocks_for(n), 256, 0, stream>>>(dim, d_verts, d_prims, n, it);
        // one list per axis, sorted by (centroid, primitive id): a stable
        // radix sort of the centroid keys over the primitives in id order
        for (int a = 0; a < dim; ++a) {
            sort_keys_kernel<<<blocks_for(n), 256, 0, stream>>>(it.c[a], n, keys, vals);
            size_t tb = std::max(sort_bytes, scan_bytes);
            if ((r = cub::DeviceRadixSort::SortPairs(cub_tmp, tb, keys, keys + nn, vals,
                                                     sorted[a], n, 0, 64, stream)) !=
                cudaSuccess) {
                return r;
            }
            if ((r = cudaMemcpyAsync(lists[a], sorted[a], nn * sizeof(int),
                                     cudaMemcpyDeviceToDevice, stream)) != cudaSuccess) {
                return r;
            }
        }
        // one level of splits over segments g with `count` segments
        auto split_level = [&](const Segs &g, int count, double *b64, int level,
                               bool split) -> cudaError_t {
            cudaError_t q;
            fill_keys_kernel<<<blocks_for(static_cast<long long>(count) * 2 * dim), 256, 0,
                               stream>>>(segbox, count, dim);
            seg_box_kernel<<<blocks_for(n), 256, 0, stream>>>(g, dim, lists[0], it, segbox);
            seg_axis_kernel<<<blocks_for(count), 256, 0, stream>>>(count, dim, segbox, axis, b64,
                                                                   level);
            if (!split) return cudaGetLastError();
            side_kernel<<<blocks_for(n), 256, 0, stream>>>(g, lists[0], lists[1],
                                                           dim == 3 ? lists[2] : lists[0], axis,
                                                           left);
            for (int b = 0; b < dim; ++b) {
                gather_side_kernel<<<blocks_for(n), 256, 0, stream>>>(n, lists[b], left, flag);
                size_t tb = std::max(sort_bytes, scan_bytes);
                if ((q = cub::DeviceScan::ExclusiveSum(cub_tmp, tb, flag, before, n, stream)) !=
                    cudaSuccess) {
                    return q;
                }
                partition_kernel<<<blocks_for(n), 256, 0, stream>>>(g, lists[b], flag, before,
                                                                    lists2[b]);
                std::swap(lists[b], lists2[b]);
            }
            return cudaGetLastError();
        };
        // binary tree: boxes of every level, splits above the leaves
        for (int l = 0; l <= D; ++l) {
            Segs g{1, l, n, nullptr, 1 << l};
            if ((r = split_level(g, 1 << l, box64, l, l < D)) != cudaSuccess) return r;
        }
        const int leaves = 1 << D;
        group_sort_kernel<<<blocks_for(leaves, 128), 128, 0, stream>>>(1, D, n, leaves,
                                                                       lists[0], order);
        if (dim == 2) {
            records2_kernel<<<blocks_for(n), 256, 0, stream>>>(d_verts, d_prims, d_bids, order,
                                                               n, seg64, segid, rec32, inv32,
                                                               sverts);
        } else {
            records3_kernel<<<blocks_for(n), 256, 0, stream>>>(d_verts, d_prims, order, n,
                                                               tri64, rec32, sverts);
        }
        // wide tree: the same splits from the presorted lists
        for (int a = 0; a < dim; ++a) {
            if ((r = cudaMemcpyAsync(lists[a], sorted[a], nn * sizeof(int),
                                     cudaMemcpyDeviceToDevice, stream)) != cudaSuccess) {
                return r;
            }
        }
        size_t done = 0;
        for (const auto &rd : rounds) {
            Segs g{0, 0, n, d_rounds + done, static_cast<int>(rd.size())};
            if ((r = split_level(g, static_cast<int>(rd.size()), nullptr, 0, true)) !=
                cudaSuccess) {
                return r;
            }
            done += rd.size();
        }
        const int clusters = (n + 31) / 32;
        group_sort_kernel<<<blocks_for(clusters, 128), 128, 0, stream>>>(0, 0, n, clusters,
                                                                         lists[0], witem);
        inverse_kernel<<<blocks_for(n), 256, 0, stream>>>(order, n, bin_of);
        wide2bin_kernel<<<blocks_for(m.w_npad), 256, 0, stream>>>(witem, bin_of, n, m.w_npad,
                                                                  wide2bin);
        // node boxes per height, then the child-group blocks
        std::vector<double *> lvh(H + 1);
        size_t o = 0;
        for (int h = 0; h <= H; ++h) {
            lvh[h] = lv + o;
            o += static_cast<size_t>(cnt[h]) * 2 * dim;
        }
        level0_kernel<<<blocks_for(n), 256, 0, stream>>>(dim, witem, n, it, lvh[0]);
        for (int h = 1; h <= H; ++h) {
            level_up_kernel<<<blocks_for(cnt[h]), 256, 0, stream>>>(dim, lvh[h - 1], cnt[h - 1],
                                                                    cnt[h], lvh[h]);
        }
        // (a one-height tree has no child groups: its block stays zero)
        if (H > 1) {
            wbox_fill_kernel<<<blocks_for(m.w_box_total), 256, 0, stream>>>(dim, wbox,
                                                                            m.w_box_total);
        }
        const double widen = std::ldexp(m.scale, -20);
        long long span = 1;
        for (int h = 1; h < H; ++h) {
            span *= 32;
            wide_node_kernel<<<blocks_for(cnt[h] * 32, 128), 128, 0, stream>>>(
                dim, cnt[h], span, n, lvh[h], witem, d_verts, d_prims, m.w_off[h], widen, wbox);
        }
        wprim_kernel<<<blocks_for(m.w_npad), 256, 0, stream>>>(dim, n, m.w_npad, wide2bin, rec32,
                                                               inv32, wprim);
        return cudaGetLastError();
    };
    e = run();
    const cudaError_t f = cudaFreeAsync(tmp, stream);
    if (e == cudaSuccess) e = f;
    if (e != cudaSuccess) return e;
    set_views(m);
    return build_lattice(m, stream);
}

}  // namespace wosb
