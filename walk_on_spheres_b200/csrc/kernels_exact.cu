// Exact-path kernels: classification, PLAIN_FP64 walks and the FP64
// closest-point / PRNG checks.  This translation unit is compiled with
// --fmad=false so double expressions round exactly like the reference's
// C++17 x86-64 build (no FMA contraction); expression shapes in the device
// headers follow the reference for the same reason.
#include <algorithm>
#include <cmath>

#include "kernels.h"

namespace wosb {

namespace {

constexpr int kExactThreads = 128;

__device__ __forceinline__ double dinf() { return __longlong_as_double(0x7ff0000000000000LL); }

// 3D inside test with the reference's ray budget and majority vote
// (src/inside.cpp:228-260).  Returns the location code; counts retries.
__device__ int classify_3d(const SceneView &s, const double *p, double bdist, double btol,
                           int max_ray_attempts, Xoshiro &rng, int &retries) {
    retries = 0;
    if (bdist <= btol) return 2;
    int valid = 0, votes = 0;
    for (int a = 0; a < max_ray_attempts && valid < 3; ++a) {
        // random_unit_direction, src/inside.cpp:18-25
        const double u = rng.unit();
        const double v = rng.unit();
        const double z = 2 * u - 1;
        const double phi = 2 * kPi * v;
        const double r = sqrt(1 - z * z);
        const double ray[3] = {r * cos(phi), r * sin(phi), z};
        bool amb;
        const int hits = count_ray_hits(s, p, ray, amb);
        if (amb) {
            ++retries;
            continue;
        }
        votes += hits & 1;
        ++valid;
    }
    if (valid < 3) return 3;
    return votes > 1 ? 1 : 0;
}

// Start point, location and (non-inside) fields of point t of `ps`
// (include/wos/runner.hpp:170-206).  A lower bound `lo` of the point's
// distance above `exact_below` (FastStart) becomes the start radius without
// the exact query; its start record then has no nearest point (slot -1),
// which no walk reads: such a point is neither on the boundary nor inside the
// shell.
template <int DIM>
__device__ __forceinline__ void classify_point(const SceneView &s, const PointSet &ps,
                                               long long t, uint64_t seed, int max_ray_attempts,
                                               double btol, const EqDesc &eq, const Fields &out,
                                               uint8_t *location, StartRecord *start,
                                               DeviceCounters *ctr, double lo = -1.0,
                                               double exact_below = 0.0) {
    double p[3];
    uint64_t linear;
    point_at(ps, t, p[0], p[1], p[2], linear);
    StartRecord st;
    if (exact_below >= 0.0 && lo > exact_below) {
        st.radius = lo;
        st.nx = p[0];
        st.ny = p[1];
        st.nz = DIM == 3 ? p[2] : 0.0;
        st.boundary_id = -1;
        st.slot = -1;
    } else {
        const Nearest<double> q = nearest64<DIM>(s, p[0], p[1], p[2], dinf());
        st.radius = sqrt(q.best);
        st.nx = q.x;
        st.ny = q.y;
        st.nz = DIM == 3 ? q.z : 0.0;
        st.boundary_id = (DIM == 2 && q.slot >= 0) ? s.segid[q.slot].x : -1;
        st.slot = q.slot;
    }
    int where;
    if (DIM == 2) {
        where = st.radius <= btol ? 2 : (winding_number(s, p[0], p[1]) != 0 ? 1 : 0);
    } else {
        Xoshiro rng(splitmix64(point_seed(seed, linear) ^ kInsideStream));
        int retries = 0;
        where = classify_3d(s, p, st.radius, btol, max_ray_attempts, rng, retries);
        if (retries) atomicAdd(&ctr->ambiguous_ray_retries, static_cast<unsigned long long>(retries));
        if (where == 3) atomicAdd(&ctr->indeterminate_points, 1ull);
    }
    location[t] = static_cast<uint8_t>(where);
    start[t] = st;
    if (out.location) out.location[t] = static_cast<uint8_t>(where);
    if (where != 1) {
        double m = __longlong_as_double(0x7ff8000000000000LL), zero = m;
        if (where == 2) {
            m = boundary_value<DIM>(eq, V3<double>{st.nx, st.ny, st.nz}, st.boundary_id);
            zero = 0.0;
        }
        if (out.mean) out.mean[t] = m;
        if (out.variance) out.variance[t] = zero;
        if (out.standard_error) out.standard_error[t] = zero;
        if (out.mean_steps) out.mean_steps[t] = zero;
    }
}

template <int DIM>
__global__ void __launch_bounds__(kExactThreads)
    classify_kernel(SceneView s, PointSet ps, uint64_t seed, int max_ray_attempts, double btol,
                    EqDesc eq, Fields out, uint8_t *location, StartRecord *start,
                    DeviceCounters *ctr) {
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < ps.n;
         t += stride) {
        classify_point<DIM>(s, ps, t, seed, max_ray_attempts, btol, eq, out, location, start, ctr);
    }
}

// FastStart lower bounds of the points of a warp: lane j's point (when
// `want`) is queried by the whole warp with the lattice build's conservative
// wide-tree query, on scene w_of(j).  Returns this lane's bound, or -1.
template <int DIM, int HC, class WOf, class MarginOf>
__device__ __forceinline__ float start_bounds(bool want, double x, double y, double z, WOf w_of,
                                              MarginOf margin_of) {
    constexpr unsigned kAll = 0xffffffffu;
    constexpr float kShrink = 1.0f - 0x1p-10f;
    const int lane = static_cast<int>(threadIdx.x & 31u);
    float lo = -1.0f;
    unsigned todo = __ballot_sync(kAll, want);
    while (todo) {
        const int j = __ffs(todo) - 1;
        todo &= todo - 1u;
        const float qx = __shfl_sync(kAll, static_cast<float>(x), j);
        const float qy = __shfl_sync(kAll, static_cast<float>(y), j);
        const float qz = DIM == 3 ? __shfl_sync(kAll, static_cast<float>(z), j) : 0.0f;
        // both lookups may shuffle: every lane takes them here, converged
        const WideView &wj = w_of(j);
        const float mj = margin_of(j);
        const WideResult q = wide_nearest<DIM, HC>(wj, qx, qy, qz, kShrink * kShrink, 0.0f);
        if (lane == j && q.slot >= 0) {
            // the rounding of the point to FP32 and of the distance
            // arithmetic stay within the margin (the lattice's bound)
            const float d = (sqrtf(q.best) * kShrink - mj) * (1.0f - 0x1p-20f);
            lo = d > 0.0f ? d : 0.0f;
        }
    }
    return lo;
}

// classify_kernel with FastStart: one warp per 32 consecutive points.
template <int DIM, int HC>
__global__ void __launch_bounds__(kExactThreads)
    classify_fast_kernel(SceneView s, WideView w, PointSet ps, uint64_t seed, int max_ray_attempts,
                         double btol, double exact_below, float margin, EqDesc eq, Fields out,
                         uint8_t *location, StartRecord *start, DeviceCounters *ctr) {
    const long long lane = threadIdx.x & 31;
    const long long warp = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const long long warps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
    for (long long base = warp * 32; base < ps.n; base += warps * 32) {
        const long long t = base + lane;
        const bool valid = t < ps.n;
        double x = 0.0, y = 0.0, z = 0.0;
        uint64_t linear = 0;
        if (valid) point_at(ps, t, x, y, z, linear);
        const float lo = start_bounds<DIM, HC>(
            valid, x, y, z, [&](int) -> const WideView & { return w; },
            [&](int) { return margin; });
        if (valid) {
            classify_point<DIM>(s, ps, t, seed, max_ray_attempts, btol, eq, out, location, start,
                                ctr, static_cast<double>(lo), exact_below);
        }
    }
}

// Classification of a batch: global point g in [base, base + n) belongs to
// the item with the largest point_begin <= g.  One warp per 32 consecutive
// points, so FAST_FP32 items can take FastStart bounds (items[i].exact_below
// >= 0), each point on its own item's scene.
template <int DIM>
__global__ void __launch_bounds__(kExactThreads)
    classify_batch_kernel(const BatchItem *__restrict__ items, int n_items, long long base,
                          long long n) {
    const long long lane = threadIdx.x & 31;
    const long long warp = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const long long warps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
    for (long long first = warp * 32; first < n; first += warps * 32) {
        const long long t = first + lane;
        const bool valid = t < n;
        const long long g = base + t;
        int lo_i = 0;
        if (valid) {
            int hi = n_items - 1;
            while (lo_i < hi) {
                const int mid = (lo_i + hi + 1) >> 1;
                if (items[mid].point_begin <= g) lo_i = mid;
                else hi = mid - 1;
            }
        }
        const BatchItem &it = items[lo_i];
        double x = 0.0, y = 0.0, z = 0.0;
        uint64_t linear = 0;
        if (valid) point_at(it.a.ps, g - it.point_begin, x, y, z, linear);
        const bool want = valid && it.exact_below >= 0.0;
        const float lo = start_bounds<DIM, kHeightAny>(
            want, x, y, z,
            [&](int j) -> const WideView & { return items[__shfl_sync(0xffffffffu, lo_i, j)].a.w; },
            [&](int j) { return items[__shfl_sync(0xffffffffu, lo_i, j)].start_margin; });
        if (valid) {
            classify_point<DIM>(it.a.s, it.a.ps, g - it.point_begin, it.a.seed,
                                it.max_ray_attempts, it.btol, it.eq, it.out,
                                const_cast<uint8_t *>(it.a.location),
                                const_cast<StartRecord *>(it.a.start), it.a.ctr,
                                static_cast<double>(lo), it.exact_below);
        }
    }
}

template <int DIM, class Eq>
__global__ void __launch_bounds__(kExactThreads)
    walk_plain_kernel(SceneView s, PointSet ps, uint64_t seed, Eq eq, int n_walks, double eps,
                      int max_steps, const uint8_t *__restrict__ location,
                      const StartRecord *__restrict__ start, Fields out, DeviceCounters *ctr) {
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < ps.n;
         t += stride) {
        if (location[t] != 1) continue;
        double x, y, z;
        uint64_t linear;
        point_at(ps, t, x, y, z, linear);
        const uint64_t pseed = point_seed(seed, linear);
        Xoshiro walk(splitmix64(pseed ^ kWalkStream));
        Xoshiro src(DIM == 2 ? splitmix64(pseed ^ kSourceStream) : 0ull);
        const StartRecord st = start[t];
        double mean = 0.0, m2 = 0.0, total_steps = 0.0;
        unsigned long long steps_sum = 0;
        int hits = 0;
        bool overflow = false;
        for (int i = 0; i < n_walks; ++i) {
            // wos_sample, include/wos/wos.hpp:54-138
            V3<double> p{x, y, z};
            V3<double> np{st.nx, st.ny, st.nz};
            int bid = st.boundary_id;
            double R = st.radius;
            double sample = 0.0, weight = 1.0;
            int steps = 0;
            while (R > eps && steps < max_steps) {
                if (DIM == 2) {
                    p = walk_body<2, true, double>(eq, p, R, sample, weight, walk, src, overflow);
                } else {
                    p = walk_body<3, true, double>(eq, p, R, sample, weight, walk, walk, overflow);
                }
                ++steps;
                const Nearest<double> q = nearest64<DIM>(s, p.x, p.y, p.z, dinf());
                R = sqrt(q.best);
                np = V3<double>{q.x, q.y, q.z};
                if (DIM == 2) bid = s.segid[q.slot].x;
            }
            if (R > eps) ++hits;
            sample += weight * eq.boundary(np, bid);
            // Welford update, include/wos/wos.hpp:169-180
            const double count = static_cast<double>(i + 1);
            const double before = sample - mean;
            mean += before / count;
            const double after = sample - mean;
            m2 += before * after;
            total_steps += steps;
            steps_sum += static_cast<unsigned long long>(steps);
        }
        const double variance = n_walks > 1 ? m2 / static_cast<double>(n_walks - 1) : 0.0;
        const double se = n_walks > 0 ? sqrt(variance / static_cast<double>(n_walks)) : 0.0;
        const double mean_steps = n_walks > 0 ? total_steps / static_cast<double>(n_walks) : 0.0;
        if (out.mean) out.mean[t] = mean;
        if (out.variance) out.variance[t] = variance;
        if (out.standard_error) out.standard_error[t] = se;
        if (out.mean_steps) out.mean_steps[t] = mean_steps;
        if (hits) atomicAdd(&ctr->max_steps_hits, static_cast<unsigned long long>(hits));
        atomicAdd(&ctr->total_steps, steps_sum);
        atomicAdd(&ctr->exact_queries, steps_sum);  // one FP64 BVH query per step
        atomicAdd(&ctr->total_walks, static_cast<unsigned long long>(n_walks));
        if (overflow) atomicOr(&ctr->error_flags, kErrRejectionCap);
    }
}

__global__ void prng_kernel(const uint64_t *seeds, long long n, int count, uint64_t *out) {
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < n;
         t += stride) {
        Xoshiro rng(seeds[t]);
        for (int i = 0; i < count; ++i) out[t * count + i] = rng.u64();
    }
}

template <int DIM>
__global__ void closest64_kernel(SceneView s, const double *pts, long long n, double *dist,
                                 double *nearest, int *bid) {
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < n;
         t += stride) {
        const double px = pts[DIM * t], py = pts[DIM * t + 1];
        const double pz = DIM == 3 ? pts[DIM * t + 2] : 0.0;
        const Nearest<double> q = nearest64<DIM>(s, px, py, pz, dinf());
        dist[t] = sqrt(q.best);
        nearest[DIM * t] = q.x;
        nearest[DIM * t + 1] = q.y;
        if (DIM == 3) nearest[DIM * t + 2] = q.z;
        if (bid) bid[t] = (DIM == 2 && q.slot >= 0) ? s.segid[q.slot].x : -1;
    }
}

int blocks_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > (1ll << 30)) b = 1ll << 30;
    return static_cast<int>(b);
}

template <int DIM, class Eq>
void launch_plain_typed(const SceneView &s, const PointSet &ps, uint64_t seed, const Eq &eq,
                        int n_walks, double eps, int max_steps, const uint8_t *location,
                        const StartRecord *start, Fields out, DeviceCounters *ctr,
                        cudaStream_t stream) {
    walk_plain_kernel<DIM, Eq><<<blocks_for(ps.n, kExactThreads), kExactThreads, 0, stream>>>(
        s, ps, seed, eq, n_walks, eps, max_steps, location, start, out, ctr);
}

template <int DIM>
void launch_plain_dim(const SceneView &s, const PointSet &ps, uint64_t seed, EqDesc e,
                      int n_walks, double eps, int max_steps, const uint8_t *location,
                      const StartRecord *start, Fields out, DeviceCounters *ctr,
                      cudaStream_t stream) {
    switch (e.kind) {
        case kLaplace:
            launch_plain_typed<DIM>(s, ps, seed, Laplace<DIM>{}, n_walks, eps, max_steps,
                                    location, start, out, ctr, stream);
            break;
        case kPoisson:
            launch_plain_typed<DIM>(s, ps, seed, Poisson<DIM>{e.mode, e.alpha}, n_walks, eps,
                                    max_steps, location, start, out, ctr, stream);
            break;
        case kScreened:
            launch_plain_typed<DIM>(s, ps, seed, Screened<DIM>{e.mode, e.alpha}, n_walks, eps,
                                    max_steps, location, start, out, ctr, stream);
            break;
        case kTransient:
            if (DIM == 2) {
                launch_plain_typed<2>(s, ps, seed, Transient<2>{kGreen, e.alpha, e.tr}, n_walks,
                                      eps, max_steps, location, start, out, ctr, stream);
            }
            break;
        case kPlate:
            if (DIM == 2) {
                launch_plain_typed<2>(s, ps, seed, Plate<2>{e.mode, *e.pl}, n_walks, eps,
                                      max_steps, location, start, out, ctr, stream);
            }
            break;
        default:
            launch_plain_typed<DIM>(s, ps, seed, Helmholtz<DIM>{}, n_walks, eps, max_steps,
                                    location, start, out, ctr, stream);
            break;
    }
}

}  // namespace

cudaError_t launch_classify(const SceneView &s, const PointSet &ps, uint64_t seed,
                            int max_ray_attempts, double btol, EqDesc eq, Fields out,
                            uint8_t *location, StartRecord *start, DeviceCounters *counters,
                            cudaStream_t stream, const FastStart &fast) {
    if (ps.n <= 0) return cudaSuccess;
    const int blocks = blocks_for(ps.n, kExactThreads);
    if (fast.on && fast.w.n > 0) {
        const WideView &w = fast.w;
        return with_height_class(height_class(w.H), [&](auto h) -> cudaError_t {
            constexpr int HC = decltype(h)::value;
            if (s.dim == 2) {
                classify_fast_kernel<2, HC><<<blocks, kExactThreads, 0, stream>>>(
                    s, w, ps, seed, max_ray_attempts, btol, fast.exact_below, fast.margin, eq,
                    out, location, start, counters);
            } else {
                classify_fast_kernel<3, HC><<<blocks, kExactThreads, 0, stream>>>(
                    s, w, ps, seed, max_ray_attempts, btol, fast.exact_below, fast.margin, eq,
                    out, location, start, counters);
            }
            return cudaGetLastError();
        });
    }
    if (s.dim == 2) {
        classify_kernel<2><<<blocks, kExactThreads, 0, stream>>>(s, ps, seed, max_ray_attempts,
                                                                 btol, eq, out, location, start,
                                                                 counters);
    } else {
        classify_kernel<3><<<blocks, kExactThreads, 0, stream>>>(s, ps, seed, max_ray_attempts,
                                                                 btol, eq, out, location, start,
                                                                 counters);
    }
    return cudaGetLastError();
}

cudaError_t launch_classify_batch(int dim, const BatchItem *items, int n_items,
                                  long long point_base, long long n_points, cudaStream_t stream) {
    if (n_items <= 0 || n_points <= 0) return cudaSuccess;
    long long b = (n_points + kExactThreads - 1) / kExactThreads;
    if (b > 148 * 64) b = 148 * 64;
    if (dim == 2) {
        classify_batch_kernel<2><<<static_cast<int>(b), kExactThreads, 0, stream>>>(
            items, n_items, point_base, n_points);
    } else {
        classify_batch_kernel<3><<<static_cast<int>(b), kExactThreads, 0, stream>>>(
            items, n_items, point_base, n_points);
    }
    return cudaGetLastError();
}

cudaError_t launch_walk_plain(const SceneView &s, const PointSet &ps, uint64_t seed, EqDesc eq,
                              int n_walks, double eps, int max_steps, const uint8_t *location,
                              const StartRecord *start, Fields out, DeviceCounters *counters,
                              cudaStream_t stream) {
    if (ps.n <= 0) return cudaSuccess;
    if (s.dim == 2) {
        launch_plain_dim<2>(s, ps, seed, eq, n_walks, eps, max_steps, location, start, out,
                            counters, stream);
    } else {
        launch_plain_dim<3>(s, ps, seed, eq, n_walks, eps, max_steps, location, start, out,
                            counters, stream);
    }
    return cudaGetLastError();
}

namespace {
__global__ void special64_kernel(const double *x, long long n, double *li0, double *lk0) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    li0[i] = log_i0(x[i]);
    lk0[i] = log_k0(x[i]);
}
}  // namespace

cudaError_t launch_special64(const double *x, long long n, double *log_i0, double *log_k0,
                             cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    special64_kernel<<<blocks_for(n, 128), 128, 0, stream>>>(x, n, log_i0, log_k0);
    return cudaGetLastError();
}

cudaError_t launch_prng(const uint64_t *seeds, long long n, int count, uint64_t *out,
                        cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    prng_kernel<<<blocks_for(n, 128), 128, 0, stream>>>(seeds, n, count, out);
    return cudaGetLastError();
}

cudaError_t launch_closest64(const SceneView &s, const double *pts, long long n, double *dist,
                             double *nearest, int *bid, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    if (s.dim == 2) {
        closest64_kernel<2><<<blocks_for(n, 128), 128, 0, stream>>>(s, pts, n, dist, nearest, bid);
    } else {
        closest64_kernel<3><<<blocks_for(n, 128), 128, 0, stream>>>(s, pts, n, dist, nearest, bid);
    }
    return cudaGetLastError();
}

}  // namespace wosb
