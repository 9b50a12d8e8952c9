// Warp-cooperative closest-point queries on a 32-wide BVH (FAST_FP32 path).
//
// Layout (built by scene_build.cpp): primitives sit in "wide slots" ordered by
// recursive median bisection; the node at height h with index i covers slots
// [i * 32^h, (i+1) * 32^h), so the children of node i are nodes 32i .. 32i+31
// one height below and no pointers are stored.  The root has height H
// (32^H >= n).  Data are blocked by 32 (array of structures of arrays): the
// 32 children of a node form one block of NB x 32 floats (field f of child k
// at f*32 + k: box lo, hi, slab normal, slab offset, half-thickness) and the
// 32 primitives of a leaf cluster one block of NF x 32 floats, so lane k of a
// warp reads child k or slot k with one base address, immediate field
// offsets and conflict-free 128-byte rows.  Padding children are empty
// (infinitely far) and padding primitives lie at 1e30, so every lane always
// has something to test.
//
// Traversal: one query at a time per warp, all 32 lanes working on it.  At a
// node every lane computes the box distance of one child; the nearest pending
// child is found with one redux.sync.min over a key (distance bits with the
// lane in the low 5 bits); a leaf cluster's 32 primitives are tested in
// parallel and reduced with redux.sync.min.  It is stackless: the state is
// (height, node); going back up recomputes the parent's child distances and
// keeps the children whose key is above the one just left, which are exactly
// the pending ones because children are taken in increasing key order.
//
// Pruning is conservative to a relative tau above the epsilon shell: while
// best > exact2 a node is skipped when its bound exceeds best * keep, with
// keep = (1 - tau)^2, so nodes that could improve the distance by less than a
// relative tau are skipped and the true distance d satisfies
// (1 - tau) sqrt(best) <= d <= sqrt(best); (1 - tau) sqrt(best) is then a
// radius whose ball lies inside the domain.  Below exact2 (inside the
// epsilon shell) pruning is exact.
#pragma once
#include <cstdint>
#include <type_traits>

namespace wosb {

struct WideView {
    int dim;
    int H;             // root height
    int n;             // primitives
    int npad;          // primitive slots (multiple of 32)
    int box_total;     // floats of the child-group blocks
    const int *off;    // [8]: float offset of the height-h child groups
    const float *box;  // child-group blocks of (3*dim+2) x 32 floats
    const float *prim; // cluster blocks of 5 (2D) or 16 (3D) x 32 floats
    const int *wide2bin;
    // Distance lattice (null when absent): gd[(i*gn[1] + j)*gn[2] + k] is a
    // lower bound of the boundary distance at the node glo + (i, j, k) * gh
    // as computed in FP32, so that d(x) >= gd[node] - |x - node| for every x
    // (the distance function is 1-Lipschitz).
    const float *gd;
    int gn[3];
    float glo[3];
    float gh, ginv;
    // a walk uses the lattice bound D - r (r = |x - node|) only when
    // D >= gratio * r, i.e. when it is at least (gratio - 1) / (gratio + 1)
    // of the upper bound D + r of the true distance
    float gratio;
    // Near-boundary candidate lists (null when absent): gl[node].x is -1 or
    // (offset << 5) | (length - 1), the list's wide slots at gpool + offset,
    // lists packed end to end (at most gk slots each).  The list holds every
    // primitive within d(node) + 2 r_max of the node (r_max the largest
    // distance from a point to its nearest node), so it holds the nearest
    // primitive of every point whose nearest node this is.  2D lists (a few
    // segments, scanned by one lane) keep ascending slot order and .y = 0.
    // 3D lists (scanned by the warp) are ordered by their slots' distance D
    // from the node, and gl[node].y packs, in 6 bits per bucket
    // b < kListBuckets, how many have D <= d(node) + 2 rho_b (+ rounding
    // slack), rho_b = (b + 1) r_max / (kListBuckets + 1): a point within
    // rho_b of the node has its nearest primitive among those (list_prefix).
    // gbinv = (kListBuckets + 1) / r_max.
    const int2 *gl;
    const int *gpool;
    int gk;
    float gbinv;
    // the primitive records again, one per wide slot, contiguous (2D: 5 of 8
    // floats, 3D: 16 floats), for the list scans' per-lane gathers
    const float4 *aos;
};

// Lattice value D at the node nearest to p and the distance r from p to it:
// D - r <= d(p) <= D + r (up to D's downward rounding).
struct LatticeSample {
    float d, r;
    int node;  // lattice index of the node
};

template <int DIM>
__device__ __forceinline__ LatticeSample lattice_sample(const WideView &w, float px, float py,
                                                        float pz) {
    const int i = min(max(__float2int_rn((px - w.glo[0]) * w.ginv), 0), w.gn[0] - 1);
    const int j = min(max(__float2int_rn((py - w.glo[1]) * w.ginv), 0), w.gn[1] - 1);
    const float dx = px - (w.glo[0] + static_cast<float>(i) * w.gh);
    const float dy = py - (w.glo[1] + static_cast<float>(j) * w.gh);
    if (DIM == 2) {
        const int node = i * w.gn[1] + j;
        const float d = __ldg(w.gd + node);
        return LatticeSample{d, sqrtf(dx * dx + dy * dy), node};
    }
    const int k = min(max(__float2int_rn((pz - w.glo[2]) * w.ginv), 0), w.gn[2] - 1);
    const float dz = pz - (w.glo[2] + static_cast<float>(k) * w.gh);
    const int node = (i * w.gn[1] + j) * w.gn[2] + k;
    const float d = __ldg(w.gd + node);
    return LatticeSample{d, sqrtf(dx * dx + dy * dy + dz * dz), node};
}

// Lower bound of the boundary distance at p from the nearest lattice node.
template <int DIM>
__device__ __forceinline__ float lattice_bound(const WideView &w, float px, float py, float pz) {
    const LatticeSample s = lattice_sample<DIM>(w, px, py, pz);
    return s.d - s.r;
}

struct WideResult {
    float best;   // squared distance
    int slot;     // wide slot of the closest primitive
};

__device__ __forceinline__ unsigned order_key(float d, unsigned lane) {
    // non-negative floats order like their bit patterns; the low 5 bits name
    // the lane so keys are unique (ties broken towards the lower lane)
    return (__float_as_uint(d) & ~31u) | lane;
}

// Squared lower bound of the distance from p to the primitives of a node: the
// larger of the box distance and the distance outside the node's slab
// {x : |n.x - c| <= h}.
// Children of node `parent` at height h+1 (so the children have height h).
template <int DIM>
__device__ __forceinline__ float wide_box_dist(const WideView &w, int h, int parent, float px,
                                               float py, float pz) {
    constexpr int NB = 3 * DIM + 2;
    const float *b = w.box + w.off[h] + parent * (NB * 32) + (threadIdx.x & 31u);
    const float lx = b[0], ly = b[32];
    float dx, dy;
    if (DIM == 2) {
        const float hx = b[64], hy = b[96];
        const float nx = b[128], ny = b[160], c = b[192], th = b[224];
        dx = fmaxf(0.0f, fmaxf(lx - px, px - hx));
        dy = fmaxf(0.0f, fmaxf(ly - py, py - hy));
        const float ds = fmaxf(0.0f, fabsf(nx * px + ny * py - c) - th);
        return fmaxf(dx * dx + dy * dy, ds * ds);
    }
    const float lz = b[64], hx = b[96], hy = b[128], hz = b[160];
    const float nx = b[192], ny = b[224], nz = b[256], c = b[288], th = b[320];
    dx = fmaxf(0.0f, fmaxf(lx - px, px - hx));
    dy = fmaxf(0.0f, fmaxf(ly - py, py - hy));
    const float dz = fmaxf(0.0f, fmaxf(lz - pz, pz - hz));
    const float ds = fmaxf(0.0f, fabsf(nx * px + ny * py + nz * pz - c) - th);
    return fmaxf(dx * dx + dy * dy + dz * dz, ds * ds);
}

// Squared distance to the primitive whose record starts at r (fields 32
// floats apart).
template <int DIM>
__device__ __forceinline__ float prim_dist(const float *r, float px, float py, float pz) {
    if (DIM == 2) {
        const float x0 = r[0], y0 = r[32], vx = r[64], vy = r[96], inv = r[128];
        const float wx = px - x0, wy = py - y0;
        const float t = fminf(fmaxf((wx * vx + wy * vy) * inv, 0.0f), 1.0f);
        const float dx = wx - t * vx, dy = wy - t * vy;
        return dx * dx + dy * dy;
    }
    float4 rec[4];
    float *f = reinterpret_cast<float *>(rec);
#pragma unroll
    for (int k = 0; k < 16; ++k) f[k] = r[k * 32];
    return eberly32(px, py, pz, rec);
}

// Primitive of this lane in leaf cluster `cluster`.
template <int DIM>
__device__ __forceinline__ float wide_prim_dist(const WideView &w, int cluster, float px,
                                                float py, float pz) {
    constexpr int NF = DIM == 2 ? 5 : 16;
    return prim_dist<DIM>(w.prim + cluster * (NF * 32) + (threadIdx.x & 31u), px, py, pz);
}

// Closest primitive to (px, py, pz) found by one lane alone, testing every
// primitive in slot order (the first minimum wins, as in wide_nearest).
// For trees of at most kLanePrims primitives: a warp-cooperative query costs
// about as much per query as one lane's whole scan there, and the lanes'
// reads of one record are one broadcast.
template <int DIM>
__device__ __forceinline__ WideResult lane_nearest(const WideView &w, float px, float py,
                                                   float pz) {
    constexpr int NF = DIM == 2 ? 5 : 16;
    float best = INFINITY;
    int slot = -1;
    for (int k = 0; k < w.n; ++k) {
        const float d2 = prim_dist<DIM>(w.prim + (k >> 5) * (NF * 32) + (k & 31), px, py, pz);
        if (d2 < best) {
            best = d2;
            slot = k;
        }
    }
    return WideResult{best, slot};
}

// Squared FP32 distance from p to the primitive in wide slot s, read from
// the contiguous records (w.aos), or from the cluster blocks when a kernel
// staged those in shared memory (aos null).
template <int DIM>
__device__ __forceinline__ float slot_dist(const WideView &w, int s, float px, float py,
                                           float pz) {
    if (w.aos == nullptr) {
        constexpr int NF = DIM == 2 ? 5 : 16;
        return prim_dist<DIM>(w.prim + (s >> 5) * (NF * 32) + (s & 31), px, py, pz);
    }
    if (DIM == 2) {
        const float4 a = __ldg(w.aos + 2 * s);
        const float inv = __ldg(reinterpret_cast<const float *>(w.aos + 2 * s + 1));
        const float wx = px - a.x, wy = py - a.y;
        const float t = fminf(fmaxf((wx * a.z + wy * a.w) * inv, 0.0f), 1.0f);
        const float dx = wx - t * a.z, dy = wy - t * a.w;
        return dx * dx + dy * dy;
    }
    float4 rec[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) rec[f] = __ldg(w.aos + 4 * s + f);
    return eberly32(px, py, pz, rec);
}

// A node's packed list entry gl[node] = (offset << 5) | (length - 1), or -1.
__device__ __forceinline__ const int *list_of(const WideView &w, int packed) {
    return w.gpool + (packed >> 5);
}
__device__ __forceinline__ int list_length(int packed) { return (packed & 31) + 1; }

// Distance buckets of a list entry (WideView::gl).
constexpr int kListBuckets = 5;

// The packed list entry of a query at distance r from its node, its length
// cut to the entries that can hold the query's nearest primitive: with
// r <= rho_b, those with D <= d(node) + 2 rho_b (the list's bucket b), since
// the nearest primitive is within d(p) + r <= d(node) + 2 r of the node.
// The minimum over that prefix is the minimum over the whole list.
__device__ __forceinline__ int list_prefix(const WideView &w, int2 v, float r) {
    const int b = min(static_cast<int>(r * w.gbinv), kListBuckets);
    if (b == kListBuckets) return v.x;
    const int k = max((v.y >> (6 * b)) & 63, 1);
    return (v.x & ~31) | (k - 1);
}

// Closest primitive among a near-boundary candidate list of k wide slots,
// found by this lane alone; the first minimum in list order (ascending
// slots: 2D lists keep slot order) wins.
template <int DIM>
__device__ __forceinline__ WideResult list_nearest(const WideView &w, const int *list, int k,
                                                   float px, float py, float pz) {
    float best = INFINITY;
    int slot = -1;
    for (int q = 0; q < k; ++q) {
        const int s = __ldg(list + q);
        const float d2 = slot_dist<DIM>(w, s, px, py, pz);
        if (d2 < best) {
            best = d2;
            slot = s;
        }
    }
    return WideResult{best, slot};
}

// list_nearest's answer for every lane with `want` (`packed` its node's list
// entry), computed by the whole warp, which must call it converged.  The
// (lane, candidate) pairs of all wanting lanes are laid out 32 at a time
// across the lanes; each lane measures one pair; a segmented minimum over
// (distance bits, slot) keys hands each list's winner to its lane, so ties
// go to the lower slot as in list_nearest.  A lane alone would scan its whole
// list while the others wait.
template <int DIM>
__device__ __forceinline__ WideResult warp_list_nearest(const WideView &w, bool want, int packed,
                                                        float px, float py, float pz) {
    constexpr unsigned kAll = 0xffffffffu;
    constexpr unsigned long long kNone = ~0ull;
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int k = want ? list_length(packed) : 0;
    int inc = k;  // inclusive prefix sum of the lengths
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kAll, inc, o);
        if (lane >= o) inc += t;
    }
    const int total = __shfl_sync(kAll, inc, 31);
    const int off = inc - k;  // this lane's first pair
    const int first = want ? (packed >> 5) : 0;  // the list's offset in the pool
    unsigned long long best = kNone;
    for (int c = 0; c < total; c += 32) {
        const int g = c + lane;  // the pair this lane measures
        // its owner: the last lane whose first pair is at or before g
        // (offsets never decrease along the lanes; j + step stays <= 31)
        int j = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            if (__shfl_sync(kAll, off, j + step) <= g) j += step;
        }
        const int q = g - __shfl_sync(kAll, off, j);
        const int list = __shfl_sync(kAll, first, j);
        const float qx = __shfl_sync(kAll, px, j);
        const float qy = __shfl_sync(kAll, py, j);
        const float qz = DIM == 3 ? __shfl_sync(kAll, pz, j) : 0.0f;
        unsigned long long key = kNone;
        if (g < total) {
            const int s = __ldg(w.gpool + list + q);
            const float d2 = slot_dist<DIM>(w, s, qx, qy, qz);
            if (d2 < INFINITY) {
                key = (static_cast<unsigned long long>(__float_as_uint(d2)) << 32) |
                      static_cast<unsigned>(s);
            }
        }
        // minimum over the rest of this lane's run (one owner's lanes are
        // contiguous; lanes past the total carry no key)
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long other = __shfl_down_sync(kAll, key, o);
            const int jo = __shfl_down_sync(kAll, j, o);
            if (lane + o < 32 && jo == j && other < key) key = other;
        }
        // each owner reads the first lane of its run in this chunk
        const unsigned long long run = __shfl_sync(kAll, key, min(max(off - c, 0), 31));
        if (k > 0 && off < c + 32 && off + k > c && run < best) best = run;
    }
    if (best == kNone) return WideResult{INFINITY, -1};
    return WideResult{__uint_as_float(static_cast<unsigned>(best >> 32)),
                      static_cast<int>(static_cast<unsigned>(best))};
}

// Every primitive within squared FP32 distance r2 of (px, py, pz), found by
// the whole warp (all lanes call it with the same point): the wide slots in
// ascending order go to out[0 .. cap) and their count to every lane.  Once
// more than cap are found the search stops and returns a count above cap.
// Children are visited when their lower bound (box and slab) is within r2.
template <int DIM>
__device__ int wide_range(const WideView &w, float px, float py, float pz, float r2, int *out,
                          int cap) {
    constexpr unsigned kAll = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    int count = 0;
    auto leaf = [&](int cluster) {
        const float d2 = wide_prim_dist<DIM>(w, cluster, px, py, pz);
        const unsigned m = __ballot_sync(kAll, d2 <= r2);
        const int at = count + __popc(m & below);
        if (((m >> lane) & 1u) && at < cap) out[at] = cluster * 32 + static_cast<int>(lane);
        count += __popc(m);
    };
    if (w.H == 1) {
        leaf(0);
        return count;
    }
    // mask[h]: children of height h (of the node parent[h]) still to visit
    unsigned mask[8];
    int parent[8];
    int h = w.H - 1;
    parent[h] = 0;
    mask[h] = __ballot_sync(kAll, wide_box_dist<DIM>(w, h, 0, px, py, pz) <= r2);
    for (;;) {
        if (mask[h] == 0u) {
            if (h == w.H - 1) break;
            ++h;
            continue;
        }
        const int k = __ffs(mask[h]) - 1;
        mask[h] &= mask[h] - 1u;
        const int child = parent[h] * 32 + k;
        if (h == 1) {
            leaf(child);
            if (count > cap) break;
        } else {
            --h;
            parent[h] = child;
            mask[h] = __ballot_sync(kAll, wide_box_dist<DIM>(w, h, child, px, py, pz) <= r2);
        }
    }
    return count;
}

// Traversal classes: a kernel compiled for one class carries only that
// class's code (the other paths cost registers and instruction cache on the
// hot ones).  kHeightAny keeps every path.  kLaneScan: at most kLanePrims
// primitives, which the walk kernels scan lane by lane (lane_nearest);
// wide_nearest treats it like kHeightUpTo2.
enum : int { kHeightAny = -1, kHeightOther = 0, kLaneScan = 1, kHeightUpTo2 = 2, kHeight3 = 3 };

__host__ __device__ __forceinline__ int lane_prims(int dim) { return dim == 2 ? 64 : 32; }

__host__ __device__ __forceinline__ int height_class(int H) {
    return H <= 2 ? kHeightUpTo2 : (H == 3 ? kHeight3 : kHeightOther);
}

__host__ __device__ __forceinline__ int traversal_class(const WideView &w) {
    return w.n <= lane_prims(w.dim) ? kLaneScan : height_class(w.H);
}

// Host dispatch: calls f(std::integral_constant<int, HC>{}) for class hc.
template <class F>
inline auto with_height_class(int hc, F &&f) {
    switch (hc) {
        case kLaneScan: return f(std::integral_constant<int, kLaneScan>{});
        case kHeightUpTo2: return f(std::integral_constant<int, kHeightUpTo2>{});
        case kHeight3: return f(std::integral_constant<int, kHeight3>{});
        default: return f(std::integral_constant<int, kHeightOther>{});
    }
}

// Closest primitive to (px, py, pz); all 32 lanes of the warp must call this
// with the same point and receive the same result.  HC: the height class the
// caller guarantees (height_class(w.H) == HC), or kHeightAny.
template <int DIM, int HC = kHeightAny>
__device__ __forceinline__ WideResult wide_nearest(const WideView &w, float px, float py,
                                                   float pz, float keep, float exact2) {
    constexpr unsigned kAll = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    float best = INFINITY, limit = INFINITY;
    int slot = -1;
    auto leaf = [&](int cluster) {
        const float d2 = wide_prim_dist<DIM>(w, cluster, px, py, pz);
        const unsigned u = __reduce_min_sync(kAll, __float_as_uint(d2));
        const float m = __uint_as_float(u);
        if (m < best) {
            best = m;
            slot = cluster * 32 + (__ffs(__ballot_sync(kAll, __float_as_uint(d2) == u)) - 1);
            limit = best > exact2 ? best * keep : best;
        }
    };
    auto take_nearest = [&](unsigned &m, float d) -> unsigned {
        const unsigned key = ((m >> lane) & 1u) ? order_key(d, lane) : 0xffffffffu;
        const unsigned k = __reduce_min_sync(kAll, key) & 31u;
        m &= ~(1u << k);
        return k;
    };
    if constexpr (HC == kHeightUpTo2 || HC == kLaneScan || HC == kHeightAny) {
    if (w.H == 1) {
        leaf(0);
        return WideResult{best, slot};
    }
    if (w.H == 2) {
        // root children are the leaf clusters: visit them nearest first
        const float d = wide_box_dist<DIM>(w, 1, 0, px, py, pz);
        unsigned m = __ballot_sync(kAll, d < limit);
        while (m) {
            const unsigned k = take_nearest(m, d);
            leaf(static_cast<int>(k));
            m &= __ballot_sync(kAll, d < limit);
        }
        return WideResult{best, slot};
    }
    }
    // Heights 3 and 4: the same nearest-first order with one child bound per
    // level held in a register, so going back up re-reads nothing.
    if constexpr (HC == kHeight3 || HC == kHeightAny) {
    if (w.H == 3) {
        const float d2 = wide_box_dist<DIM>(w, 2, 0, px, py, pz);
        unsigned m2 = __ballot_sync(kAll, d2 < limit);
        while (m2) {
            const int n2 = static_cast<int>(take_nearest(m2, d2));
            const float d1 = wide_box_dist<DIM>(w, 1, n2, px, py, pz);
            unsigned m1 = __ballot_sync(kAll, d1 < limit);
            while (m1) {
                const unsigned k = take_nearest(m1, d1);
                leaf(n2 * 32 + static_cast<int>(k));
                m1 &= __ballot_sync(kAll, d1 < limit);
            }
            m2 &= __ballot_sync(kAll, d2 < limit);
        }
        return WideResult{best, slot};
    }
    }
    if constexpr (HC == kHeightOther || HC == kHeightAny) {
    if (w.H == 4) {
        const float d3 = wide_box_dist<DIM>(w, 3, 0, px, py, pz);
        unsigned m3 = __ballot_sync(kAll, d3 < limit);
        while (m3) {
            const int n3 = static_cast<int>(take_nearest(m3, d3));
            const float d2 = wide_box_dist<DIM>(w, 2, n3, px, py, pz);
            unsigned m2 = __ballot_sync(kAll, d2 < limit);
            while (m2) {
                const int n2 = n3 * 32 + static_cast<int>(take_nearest(m2, d2));
                const float d1 = wide_box_dist<DIM>(w, 1, n2, px, py, pz);
                unsigned m1 = __ballot_sync(kAll, d1 < limit);
                while (m1) {
                    const unsigned k = take_nearest(m1, d1);
                    leaf(n2 * 32 + static_cast<int>(k));
                    m1 &= __ballot_sync(kAll, d1 < limit);
                }
                m2 &= __ballot_sync(kAll, d2 < limit);
            }
            m3 &= __ballot_sync(kAll, d3 < limit);
        }
        return WideResult{best, slot};
    }
    int h = w.H;    // height of the current node
    int node = 0;   // its index at that height
    float d = wide_box_dist<DIM>(w, h - 1, node, px, py, pz);
    unsigned m = __ballot_sync(kAll, d < limit);
    for (;;) {
        if (m == 0u) {
            if (h == w.H) break;
            // back to the parent: its children with a key above ours are pending
            const unsigned left = static_cast<unsigned>(node) & 31u;
            node >>= 5;
            ++h;
            d = wide_box_dist<DIM>(w, h - 1, node, px, py, pz);
            const unsigned key = order_key(d, lane);
            const unsigned key_left = __shfl_sync(kAll, key, left);
            m = __ballot_sync(kAll, key > key_left && d < limit);
            continue;
        }
        const unsigned k = take_nearest(m, d);
        const int child = node * 32 + static_cast<int>(k);
        if (h == 2) {
            leaf(child);
            m &= __ballot_sync(kAll, d < limit);
        } else {
            node = child;
            --h;
            d = wide_box_dist<DIM>(w, h - 1, node, px, py, pz);
            m = __ballot_sync(kAll, d < limit);
        }
    }
    }
    return WideResult{best, slot};
}

}  // namespace wosb
