// Host construction of the device scene: mesh validation, the implicit
// median-split BVH and the FP64 / FP32 primitive records.
#include "scene_build.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <utility>

namespace wosb {

unsigned host_threads() {
    static const unsigned t = [] {
        if (const char *e = std::getenv("WOS_HOST_THREADS")) {
            const int v = std::atoi(e);
            if (v >= 1) return static_cast<unsigned>(v);
        }
        return std::max(1u, std::thread::hardware_concurrency());
    }();
    return t;
}

namespace {

// Subtree recursions split into host threads down to this depth (2^depth
// threads at most); below it, or under kSerialItems items, they run inline.
// Subtrees touch disjoint item ranges and node slots, so the result does not
// depend on the thread count.
int spawn_depth() {
    static const int d = [] {
        const unsigned hw = host_threads();
        int k = 0;
        while ((2u << k) <= hw && k < 6) ++k;
        return k;
    }();
    return d;
}
constexpr int kSerialItems = 8192;

template <class F, class G>
void both(int depth, int items, F &&left, G &&right) {
    if (depth < spawn_depth() && items >= kSerialItems) {
        std::thread t(std::forward<F>(left));
        right();
        t.join();
    } else {
        left();
        right();
    }
}

// Runs f(i) for i in [0, n) on the host threads, in contiguous blocks;
// inline below `min_items` items (small loops of cheap items).
template <class F>
void parallel_for(long long n, F &&f, long long min_items = 64) {
    const long long threads = host_threads();
    if (n < min_items || n < 2 || threads == 1) {
        for (long long i = 0; i < n; ++i) f(i);
        return;
    }
    const long long per = (n + threads - 1) / threads;
    std::vector<std::thread> pool;
    for (long long b = 0; b < n; b += per) {
        const long long e = std::min(n, b + per);
        pool.emplace_back([&f, b, e] {
            for (long long i = b; i < e; ++i) f(i);
        });
    }
    for (auto &t : pool) t.join();
}

struct Item {
    double lo[3], hi[3], c[3];
    int prim;
};

float round_down(double v) {
    float f = static_cast<float>(v);
    if (static_cast<double>(f) > v) f = std::nextafter(f, -INFINITY);
    return f;
}
float round_up(double v) {
    float f = static_cast<float>(v);
    if (static_cast<double>(f) < v) f = std::nextafter(f, INFINITY);
    return f;
}

int first_slot(long long k, long long n, int level) {
    return static_cast<int>((static_cast<unsigned long long>(k) * static_cast<unsigned long long>(n)) >>
                            level);
}

struct Builder {
    HostScene &sc;
    std::vector<Item> items;

    void box_of(int s, int e, double *lo, double *hi) const {
        for (int k = 0; k < 3; ++k) {
            lo[k] = items[s].lo[k];
            hi[k] = items[s].hi[k];
        }
        for (int i = s + 1; i < e; ++i) {
            for (int k = 0; k < sc.dim; ++k) {
                lo[k] = lo[k] < items[i].lo[k] ? lo[k] : items[i].lo[k];
                hi[k] = hi[k] > items[i].hi[k] ? hi[k] : items[i].hi[k];
            }
        }
    }

    // Node `id` (1-based heap index) at `level` covers slots [s, e).
    void build(long long id, int level, int s, int e) {
        double lo[3], hi[3];
        box_of(s, e, lo, hi);
        const int d = sc.dim;
        double *b = sc.box64.data() + static_cast<size_t>(2 * d) * id;
        for (int k = 0; k < d; ++k) {
            b[k] = lo[k];
            b[d + k] = hi[k];
        }
        if (level == sc.depth) {
            // leaf: canonical order by primitive id
            std::sort(items.begin() + s, items.begin() + e,
                      [](const Item &x, const Item &y) { return x.prim < y.prim; });
            return;
        }
        // longest axis of the node box, ties to the lower axis (src/bvh.cpp:218-224)
        const double ex = hi[0] - lo[0], ey = hi[1] - lo[1];
        int axis;
        if (d == 2) {
            axis = ex >= ey ? 0 : 1;
        } else {
            const double ez = hi[2] - lo[2];
            axis = (ex >= ey) ? (ex >= ez ? 0 : 2) : (ey >= ez ? 1 : 2);
        }
        const long long k = id - (1ll << level);
        const int mid = first_slot(2 * k + 1, sc.n_prims, level + 1);
        // median split by (centroid coordinate, primitive id), src/bvh.cpp:143-171
        std::nth_element(items.begin() + s, items.begin() + mid, items.begin() + e,
                         [axis](const Item &x, const Item &y) {
                             if (x.c[axis] < y.c[axis]) return true;
                             if (x.c[axis] > y.c[axis]) return false;
                             return x.prim < y.prim;
                         });
        both(level, e - s, [&] { build(2 * id, level + 1, s, mid); },
             [&] { build(2 * id + 1, level + 1, mid, e); });
    }
};

// 32-wide tree: the node at height h covering [s, e) is split into children
// of 32^(h-1) slots by recursive median bisection along the longest axis, with
// split points on multiples of the child size.
struct WideBuilder {
    int dim;
    std::vector<Item> &items;

    void bbox(int s, int e, double *lo, double *hi) const {
        for (int k = 0; k < 3; ++k) {
            lo[k] = items[s].lo[k];
            hi[k] = items[s].hi[k];
        }
        for (int i = s + 1; i < e; ++i) {
            for (int k = 0; k < dim; ++k) {
                lo[k] = std::min(lo[k], items[i].lo[k]);
                hi[k] = std::max(hi[k], items[i].hi[k]);
            }
        }
    }

    void split(int s, int e, long long chunk, int child_height, int depth = 0) {
        const long long nch = (e - s + chunk - 1) / chunk;
        if (nch <= 1) {
            node(s, e, child_height, depth);
            return;
        }
        const int mid = static_cast<int>(s + ((nch + 1) / 2) * chunk);
        double lo[3], hi[3];
        bbox(s, e, lo, hi);
        const double ex = hi[0] - lo[0], ey = hi[1] - lo[1];
        const double ez = dim == 3 ? hi[2] - lo[2] : -1.0;
        const int axis = (ex >= ey) ? (ex >= ez ? 0 : 2) : (ey >= ez ? 1 : 2);
        std::nth_element(items.begin() + s, items.begin() + mid, items.begin() + e,
                         [axis](const Item &x, const Item &y) {
                             if (x.c[axis] < y.c[axis]) return true;
                             if (x.c[axis] > y.c[axis]) return false;
                             return x.prim < y.prim;
                         });
        both(depth, e - s, [&] { split(s, mid, chunk, child_height, depth + 1); },
             [&] { split(mid, e, chunk, child_height, depth + 1); });
    }

    void node(int s, int e, int height, int depth = 0) {
        if (height <= 1) {
            std::sort(items.begin() + s, items.begin() + e,
                      [](const Item &x, const Item &y) { return x.prim < y.prim; });
            return;
        }
        long long chunk = 1;
        for (int h = 1; h < height; ++h) chunk *= 32;
        split(s, e, chunk, height - 1, depth);
    }
};

}  // namespace

// Principal plane of a point set: unit normal along the smallest-variance
// direction (cyclic Jacobi eigen-decomposition of the covariance, rotations
// from their tangents), offset n.mean and half-thickness max |n.v - offset|.
// Any unit normal gives a valid slab; the thickness is measured for it.
// The sums run in two levels: over consecutive chunks of `chunk` points
// (a node's child subtrees), each from zero, then over the chunk sums in
// order; the device build sums the chunks in parallel in the same order.
static void slab_of(const std::vector<double> &pts, int dim, size_t chunk, double *n, double &c,
                    double &h) {
    const size_t m = pts.size() / dim;
    double mean[3] = {0, 0, 0};
    for (size_t c0 = 0; c0 < m; c0 += chunk) {
        double part[3] = {0, 0, 0};
        for (size_t i = c0; i < std::min(m, c0 + chunk); ++i)
            for (int k = 0; k < dim; ++k) part[k] += pts[i * dim + k];
        for (int k = 0; k < dim; ++k) mean[k] += part[k];
    }
    for (int k = 0; k < dim; ++k) mean[k] /= static_cast<double>(m);
    double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (size_t c0 = 0; c0 < m; c0 += chunk) {
        double part[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (size_t i = c0; i < std::min(m, c0 + chunk); ++i)
            for (int a = 0; a < dim; ++a)
                for (int b = 0; b < dim; ++b)
                    part[a][b] += (pts[i * dim + a] - mean[a]) * (pts[i * dim + b] - mean[b]);
        for (int a = 0; a < dim; ++a)
            for (int b = 0; b < dim; ++b) A[a][b] += part[a][b];
    }
    double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 32; ++sweep) {
        double off = 0.0;
        for (int a = 0; a < dim; ++a)
            for (int b = a + 1; b < dim; ++b) off += A[a][b] * A[a][b];
        if (off < 1e-30) break;
        for (int a = 0; a < dim; ++a) {
            for (int b = a + 1; b < dim; ++b) {
                if (std::fabs(A[a][b]) < 1e-300) continue;
                // the rotation that zeroes A[a][b], from its tangent
                // (t = tan phi, |phi| <= pi/4): +, -, *, / and sqrt only, so
                // every IEEE machine rounds it the same way
                const double theta = (A[b][b] - A[a][a]) / (2.0 * A[a][b]);
                const double t =
                    std::fabs(theta) > 1e150
                        ? 0.5 / theta
                        : (theta >= 0.0 ? 1.0 : -1.0) /
                              (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
                for (int k = 0; k < dim; ++k) {  // A <- A J
                    const double x = A[k][a], y = A[k][b];
                    A[k][a] = cs * x - sn * y;
                    A[k][b] = sn * x + cs * y;
                }
                for (int k = 0; k < dim; ++k) {  // A <- J^T A
                    const double x = A[a][k], y = A[b][k];
                    A[a][k] = cs * x - sn * y;
                    A[b][k] = sn * x + cs * y;
                }
                for (int k = 0; k < dim; ++k) {  // V <- V J
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
    double len = 0.0;
    for (int k = 0; k < dim; ++k) {
        n[k] = V[k][best];
        len += n[k] * n[k];
    }
    len = std::sqrt(len);
    for (int k = 0; k < dim; ++k) n[k] /= len;
    c = 0.0;
    for (int k = 0; k < dim; ++k) c += n[k] * mean[k];
    h = 0.0;
    for (size_t i = 0; i < m; ++i) {
        double t = -c;
        for (int k = 0; k < dim; ++k) t += n[k] * pts[i * dim + k];
        h = std::max(h, std::fabs(t));
    }
}

void wide_layout(HostScene &sc);

static void build_wide(HostScene &sc, std::vector<Item> items, int dim) {
    const int n = sc.n_prims;
    wide_layout(sc);
    const int H = sc.wH;
    WideBuilder W{dim, items};
    W.node(0, n, H);

    // binary slot of every primitive (for the FP64 records)
    std::vector<int> bin_of(n);
    for (int s = 0; s < n; ++s) bin_of[sc.order[s]] = s;
    sc.wide2bin.assign(sc.w_npad, -1);
    for (int s = 0; s < n; ++s) sc.wide2bin[s] = bin_of[items[s].prim];

    // node boxes per height (FP64, then rounded outward and widened)
    const int nc = 2 * dim;
    std::vector<std::vector<double>> lv(H + 1);
    std::vector<long long> cnt(H + 1);
    cnt[0] = n;
    lv[0].resize(static_cast<size_t>(n) * nc);
    for (int s = 0; s < n; ++s) {
        for (int k = 0; k < dim; ++k) {
            lv[0][static_cast<size_t>(s) * nc + k] = items[s].lo[k];
            lv[0][static_cast<size_t>(s) * nc + dim + k] = items[s].hi[k];
        }
    }
    for (int h = 1; h <= H; ++h) {
        cnt[h] = (cnt[h - 1] + 31) / 32;
        lv[h].assign(static_cast<size_t>(cnt[h]) * nc, 0.0);
        parallel_for(cnt[h], [&](long long i) {
            const long long c0 = 32 * i, c1 = std::min(cnt[h - 1], 32 * i + 32);
            for (int k = 0; k < nc; ++k) {
                double v = lv[h - 1][static_cast<size_t>(c0) * nc + k];
                for (long long c = c0 + 1; c < c1; ++c) {
                    const double x = lv[h - 1][static_cast<size_t>(c) * nc + k];
                    v = k < dim ? std::min(v, x) : std::max(v, x);
                }
                lv[h][static_cast<size_t>(i) * nc + k] = v;
            }
        });
    }
    // heights 1..H-1 are children of some node.  Children of one parent form
    // a group block of nbox x 32 floats (field f of child k at f*32 + k):
    // box lo[dim], hi[dim], slab normal[dim], slab offset, half-thickness
    // (offsets w_off and size w_box_total from wide_layout).
    const int nbox = nc + dim + 2;
    const double widen = std::ldexp(sc.scale, -20);
    sc.wbox.assign(static_cast<size_t>(sc.w_box_total), 0.0f);
    // padding children are empty boxes (lo = +inf, hi = -inf) with an
    // unbounded slab: infinitely far
    for (int h = 1; h < H; ++h) {
        for (long long g = 0; g < cnt[h + 1]; ++g) {
            float *blk = sc.wbox.data() + sc.w_off[h] + static_cast<size_t>(g) * nbox * 32;
            for (int f = 0; f < nbox; ++f) {
                float fill = 0.0f;
                if (f < dim) fill = INFINITY;
                else if (f < nc) fill = -INFINITY;
                else if (f == nbox - 1) fill = INFINITY;
                for (int k = 0; k < 32; ++k) blk[f * 32 + k] = fill;
            }
        }
    }
    auto vertex = [&](int prim, int j, double *out) {
        const int v = sc.prims[static_cast<size_t>(dim) * prim + j];
        for (int k = 0; k < dim; ++k) out[k] = sc.verts[static_cast<size_t>(dim) * v + k];
    };
    for (int h = 1; h < H; ++h) {
        long long span_h = 1;
        for (int k = 0; k < h; ++k) span_h *= 32;
        parallel_for(cnt[h], [&](long long i) {
            std::vector<double> pts;
            float *blk = sc.wbox.data() + sc.w_off[h] + static_cast<size_t>(i / 32) * nbox * 32;
            const int lane = static_cast<int>(i % 32);
            for (int k = 0; k < nc; ++k) {
                const double v = lv[h][static_cast<size_t>(i) * nc + k];
                blk[k * 32 + lane] = k < dim ? round_down(v - widen) : round_up(v + widen);
            }
            // slab of every vertex of the node's primitives
            pts.clear();
            const long long s0 = i * span_h, s1 = std::min<long long>(n, (i + 1) * span_h);
            for (long long sl = s0; sl < s1; ++sl) {
                for (int j = 0; j < dim; ++j) {
                    double v[3];
                    vertex(items[sl].prim, j, v);
                    pts.insert(pts.end(), v, v + dim);
                }
            }
            double nrm[3] = {0, 0, 0}, c = 0.0, th = 0.0;
            slab_of(pts, dim, static_cast<size_t>(span_h / 32) * dim, nrm, c, th);
            float nf[3];
            for (int k = 0; k < dim; ++k) nf[k] = static_cast<float>(nrm[k]);
            const float cf = static_cast<float>(c);
            // thickness for the rounded normal and offset, padded for the FP32
            // evaluation at query time
            double t32 = 0.0;
            for (size_t q = 0; q < pts.size() / dim; ++q) {
                double t = -static_cast<double>(cf);
                for (int k = 0; k < dim; ++k) t += static_cast<double>(nf[k]) * pts[q * dim + k];
                t32 = std::max(t32, std::fabs(t));
            }
            for (int k = 0; k < dim; ++k) blk[(nc + k) * 32 + lane] = nf[k];
            blk[(nc + dim) * 32 + lane] = cf;
            blk[(nc + dim + 1) * 32 + lane] = round_up(t32 + 4.0 * widen);
        }, 2);  // the top heights have a few large nodes: thread them too
    }
    // primitives in wide-slot order, one block of na x 32 floats per cluster
    // (field f of slot 32c + k at c*na*32 + f*32 + k); padding primitives are
    // far away
    const int na = dim == 2 ? 5 : 16;
    sc.wprim.assign(static_cast<size_t>(sc.w_npad) * na, 0.0f);
    parallel_for(sc.w_npad, [&](long long sl) {
        const int s = static_cast<int>(sl);
        float rec[16];
        if (s >= n) {
            for (float &x : rec) x = 0.0f;
            rec[0] = rec[1] = 1e30f;
            if (dim == 3) rec[2] = 1e30f;
        } else if (dim == 2) {
            const int b = sc.wide2bin[s];
            for (int k = 0; k < 4; ++k) rec[k] = sc.seg32[4 * static_cast<size_t>(b) + k];
            rec[4] = sc.seg32inv[b];
        } else {
            const int b = sc.wide2bin[s];
            for (int k = 0; k < 16; ++k) rec[k] = sc.tri32[16 * static_cast<size_t>(b) + k];
        }
        float *blk = sc.wprim.data() + static_cast<size_t>(s / 32) * na * 32;
        for (int k = 0; k < na; ++k) blk[k * 32 + s % 32] = rec[k];
    });
}

std::string check_mesh(int dim, const double *verts, int n_verts, const int *prims, int n_prims,
                       int leaf_size) {
    if (dim != 2 && dim != 3) return "mesh dimension must be 2 or 3";
    if (!verts || n_verts <= 0) return "mesh contains no vertices";
    if (!prims || n_prims <= 0) {
        return dim == 2 ? "mesh contains no line primitives" : "mesh contains no triangle primitives";
    }
    if (leaf_size == 0) leaf_size = 4;
    if (leaf_size < 2 || leaf_size > 8) return "leaf_size must be 0 or in [2, 8]";
    for (long long i = 0; i < static_cast<long long>(n_verts) * dim; ++i) {
        if (!std::isfinite(verts[i])) return "vertex coordinates must be finite";
    }
    for (long long i = 0; i < static_cast<long long>(n_prims) * dim; ++i) {
        if (prims[i] < 0 || prims[i] >= n_verts) return "primitive vertex index out of range";
    }
    auto V = [&](int v, int k) { return verts[static_cast<size_t>(dim) * v + k]; };
    for (int p = 0; p < n_prims; ++p) {
        if (dim == 2) {
            const int a = prims[2 * p], b = prims[2 * p + 1];
            const double dx = V(b, 0) - V(a, 0), dy = V(b, 1) - V(a, 1);
            if (!(dx * dx + dy * dy > 0.0)) return "mesh contains a zero-length line segment";
        } else {
            const int a = prims[3 * p], b = prims[3 * p + 1], c = prims[3 * p + 2];
            const double abx = V(b, 0) - V(a, 0), aby = V(b, 1) - V(a, 1), abz = V(b, 2) - V(a, 2);
            const double acx = V(c, 0) - V(a, 0), acy = V(c, 1) - V(a, 1), acz = V(c, 2) - V(a, 2);
            const double cx = aby * acz - abz * acy, cy = abz * acx - abx * acz,
                         cz = abx * acy - aby * acx;
            if (!(cx * cx + cy * cy + cz * cz > 0.0)) return "mesh contains a degenerate triangle";
        }
    }
    int D = 0;
    while (((static_cast<long long>(n_prims) + (1ll << D) - 1) >> D) > leaf_size) ++D;
    if (D > 30) return "mesh too large for the BVH layout";
    return std::string();
}

void wide_layout(HostScene &sc) {
    const int n = sc.n_prims, dim = sc.dim;
    int H = 1;
    long long span = 32;
    while (span < n) {
        span *= 32;
        ++H;
    }
    sc.wH = H;
    sc.w_npad = (n + 31) / 32 * 32;
    std::vector<long long> cnt(H + 1);
    cnt[0] = n;
    for (int h = 1; h <= H; ++h) cnt[h] = (cnt[h - 1] + 31) / 32;
    const int nbox = 2 * dim + dim + 2;
    int total = 0;
    for (int h = 0; h < 8; ++h) sc.w_off[h] = 0;
    for (int h = 1; h < H; ++h) {
        sc.w_off[h] = total;
        total += static_cast<int>(cnt[h + 1]) * nbox * 32;
    }
    sc.w_box_total = std::max(total, nbox * 32);
}

std::string scene_meta(int dim, const double *verts, int n_verts, const int *prims, int n_prims,
                       const int *boundary_ids, int leaf_size, HostScene &sc) {
    std::string err = check_mesh(dim, verts, n_verts, prims, n_prims, leaf_size);
    if (!err.empty()) return err;
    if (leaf_size == 0) leaf_size = 4;
    sc = HostScene{};
    sc.dim = dim;
    sc.n_prims = n_prims;
    sc.n_verts = n_verts;
    sc.leaf_size = leaf_size;
    sc.verts.assign(verts, verts + static_cast<size_t>(n_verts) * dim);
    sc.prims.assign(prims, prims + static_cast<size_t>(n_prims) * dim);
    sc.boundary_ids.assign(n_prims, 0);
    if (dim == 2 && boundary_ids) sc.boundary_ids.assign(boundary_ids, boundary_ids + n_prims);
    auto V = [&](int v, int k) { return verts[static_cast<size_t>(dim) * v + k]; };
    for (int k = 0; k < 3; ++k) {
        sc.bbox[2 * k] = k < dim ? V(0, k) : 0.0;
        sc.bbox[2 * k + 1] = sc.bbox[2 * k];
    }
    for (int v = 1; v < n_verts; ++v) {
        for (int k = 0; k < dim; ++k) {
            const double x = V(v, k);
            if (x < sc.bbox[2 * k]) sc.bbox[2 * k] = x;
            else if (x > sc.bbox[2 * k + 1]) sc.bbox[2 * k + 1] = x;
        }
    }
    sc.scale = std::max({1.0, sc.bbox[1] - sc.bbox[0], sc.bbox[3] - sc.bbox[2],
                         sc.bbox[5] - sc.bbox[4]});
    int D = 0;
    while (((static_cast<long long>(n_prims) + (1ll << D) - 1) >> D) > leaf_size) ++D;
    sc.depth = D;
    wide_layout(sc);
    return std::string();
}

std::string build_scene(int dim, const double *verts, int n_verts, const int *prims, int n_prims,
                        const int *boundary_ids, int leaf_size, HostScene &sc) {
    if (dim != 2 && dim != 3) return "mesh dimension must be 2 or 3";
    if (!verts || n_verts <= 0) return "mesh contains no vertices";
    if (!prims || n_prims <= 0) {
        return dim == 2 ? "mesh contains no line primitives" : "mesh contains no triangle primitives";
    }
    if (leaf_size == 0) leaf_size = 4;
    if (leaf_size < 2 || leaf_size > 8) return "leaf_size must be 0 or in [2, 8]";
    for (long long i = 0; i < static_cast<long long>(n_verts) * dim; ++i) {
        if (!std::isfinite(verts[i])) return "vertex coordinates must be finite";
    }
    for (long long i = 0; i < static_cast<long long>(n_prims) * dim; ++i) {
        if (prims[i] < 0 || prims[i] >= n_verts) return "primitive vertex index out of range";
    }

    sc = HostScene{};
    sc.dim = dim;
    sc.n_prims = n_prims;
    sc.n_verts = n_verts;
    sc.leaf_size = leaf_size;
    sc.verts.assign(verts, verts + static_cast<size_t>(n_verts) * dim);
    sc.prims.assign(prims, prims + static_cast<size_t>(n_prims) * dim);
    sc.boundary_ids.assign(n_prims, 0);
    if (dim == 2 && boundary_ids) sc.boundary_ids.assign(boundary_ids, boundary_ids + n_prims);

    auto V = [&](int v, int k) { return verts[static_cast<size_t>(dim) * v + k]; };

    // mesh bounding box, src/mesh.cpp:297-322
    for (int k = 0; k < 3; ++k) {
        sc.bbox[2 * k] = k < dim ? V(0, k) : 0.0;
        sc.bbox[2 * k + 1] = sc.bbox[2 * k];
    }
    for (int v = 1; v < n_verts; ++v) {
        for (int k = 0; k < dim; ++k) {
            const double x = V(v, k);
            if (x < sc.bbox[2 * k]) sc.bbox[2 * k] = x;
            else if (x > sc.bbox[2 * k + 1]) sc.bbox[2 * k + 1] = x;
        }
    }
    sc.scale = std::max({1.0, sc.bbox[1] - sc.bbox[0], sc.bbox[3] - sc.bbox[2],
                         sc.bbox[5] - sc.bbox[4]});

    // primitive boxes and centroids (src/mesh.cpp:324-366); degeneracy checks
    // (src/mesh.cpp:239-267)
    Builder B{sc, std::vector<Item>(n_prims)};
    for (int p = 0; p < n_prims; ++p) {
        Item &it = B.items[p];
        std::memset(&it, 0, sizeof(it));
        it.prim = p;
        if (dim == 2) {
            const int a = prims[2 * p], b = prims[2 * p + 1];
            const double dx = V(b, 0) - V(a, 0), dy = V(b, 1) - V(a, 1);
            if (!(dx * dx + dy * dy > 0.0)) return "mesh contains a zero-length line segment";
            // "+ 0.0" turns -0.0 into +0.0: the boxes' min / max then do not
            // depend on the order items are visited in (the device build
            // visits them in another order)
            for (int k = 0; k < 2; ++k) {
                it.lo[k] = std::fmin(V(a, k), V(b, k)) + 0.0;
                it.hi[k] = std::fmax(V(a, k), V(b, k)) + 0.0;
                it.c[k] = (V(a, k) + V(b, k)) / 2.0 + 0.0;
            }
        } else {
            const int a = prims[3 * p], b = prims[3 * p + 1], c = prims[3 * p + 2];
            const double abx = V(b, 0) - V(a, 0), aby = V(b, 1) - V(a, 1), abz = V(b, 2) - V(a, 2);
            const double acx = V(c, 0) - V(a, 0), acy = V(c, 1) - V(a, 1), acz = V(c, 2) - V(a, 2);
            const double cx = aby * acz - abz * acy, cy = abz * acx - abx * acz,
                         cz = abx * acy - aby * acx;
            if (!(cx * cx + cy * cy + cz * cz > 0.0)) return "mesh contains a degenerate triangle";
            for (int k = 0; k < 3; ++k) {
                it.lo[k] = std::fmin(std::fmin(V(a, k), V(b, k)), V(c, k)) + 0.0;
                it.hi[k] = std::fmax(std::fmax(V(a, k), V(b, k)), V(c, k)) + 0.0;
                it.c[k] = (V(a, k) + V(b, k) + V(c, k)) / 3.0 + 0.0;
            }
        }
    }

    // depth: the smallest D with ceil(n / 2^D) <= leaf_size
    int D = 0;
    while (((static_cast<long long>(n_prims) + (1ll << D) - 1) >> D) > leaf_size) ++D;
    if (D > 30) return "mesh too large for the BVH layout";
    sc.depth = D;
    const long long n_nodes = 1ll << (D + 1);
    sc.box64.assign(static_cast<size_t>(n_nodes) * 2 * dim, 0.0);
    B.build(1, 0, 0, n_prims);

    sc.order.resize(n_prims);
    for (int s = 0; s < n_prims; ++s) sc.order[s] = B.items[s].prim;

    // leaf-slot primitive records
    if (dim == 2) {
        sc.seg64.resize(static_cast<size_t>(n_prims) * 4);
        sc.segid.resize(static_cast<size_t>(n_prims) * 2);
        sc.seg32.resize(static_cast<size_t>(n_prims) * 4);
        sc.seg32inv.resize(static_cast<size_t>(n_prims));
        parallel_for(n_prims, [&](long long sl) {
            const int s = static_cast<int>(sl);
            const int p = sc.order[s];
            const int a = prims[2 * p], b = prims[2 * p + 1];
            const double g[4] = {V(a, 0), V(a, 1), V(b, 0), V(b, 1)};
            for (int k = 0; k < 4; ++k) sc.seg64[4 * s + k] = g[k];
            // FP32: origin, direction and 1/|direction|^2
            const float x0 = static_cast<float>(g[0]), y0 = static_cast<float>(g[1]);
            const float vx = static_cast<float>(g[2] - g[0]), vy = static_cast<float>(g[3] - g[1]);
            sc.seg32[4 * s + 0] = x0;
            sc.seg32[4 * s + 1] = y0;
            sc.seg32[4 * s + 2] = vx;
            sc.seg32[4 * s + 3] = vy;
            sc.seg32inv[s] = static_cast<float>(
                1.0 / (static_cast<double>(vx) * vx + static_cast<double>(vy) * vy));
            sc.segid[2 * s] = sc.boundary_ids[p];
            sc.segid[2 * s + 1] = p;
        });
    } else {
        sc.tri64.resize(static_cast<size_t>(n_prims) * 14);
        sc.tri32.resize(static_cast<size_t>(n_prims) * 16);
        parallel_for(n_prims, [&](long long sl) {
            const int s = static_cast<int>(sl);
            const int p = sc.order[s];
            const int a = prims[3 * p], b = prims[3 * p + 1], c = prims[3 * p + 2];
            // Eberly cache, src/bvh.cpp:204-217
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
            std::memcpy(sc.tri64.data() + 14 * static_cast<size_t>(s), rec64, sizeof(rec64));
            // FP32 record from the rounded vertex and edges
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
            float *o = sc.tri32.data() + 16 * static_cast<size_t>(s);
            o[0] = fv[0]; o[1] = fv[1]; o[2] = fv[2]; o[3] = static_cast<float>(fa);
            o[4] = fe1[0]; o[5] = fe1[1]; o[6] = fe1[2]; o[7] = static_cast<float>(fb);
            o[8] = fe2[0]; o[9] = fe2[1]; o[10] = fe2[2]; o[11] = static_cast<float>(fc);
            o[12] = static_cast<float>(fdet);
            o[13] = static_cast<float>(1.0 / fdet);
            o[14] = static_cast<float>(1.0 / fa);
            o[15] = static_cast<float>(1.0 / fc);
        });
    }
    sc.slot_verts.resize(static_cast<size_t>(n_prims) * dim);
    for (int s = 0; s < n_prims; ++s) {
        for (int k = 0; k < dim; ++k) sc.slot_verts[dim * s + k] = prims[dim * sc.order[s] + k];
    }
    build_wide(sc, std::move(B.items), dim);  // the binary build is done with them
    return std::string();
}

}  // namespace wosb
