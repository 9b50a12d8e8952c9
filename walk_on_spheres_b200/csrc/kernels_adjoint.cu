// Gaussian heat source: forward walks and their adjoint replay.
//
// Equation.  -Δu = f in the domain with f(x) = Q exp(-|x - x0|^2 / sigma^2)
// and u = g on the boundary, g given per mesh vertex and interpolated at the
// walk's terminal nearest point: linearly along the nearest segment (2D) or
// barycentrically on the nearest triangle (3D).  The reference has no such
// equation and no gradients; the estimator is its Poisson estimator
// (include/wos/wos.hpp:54-138 with the Green kernels of
// include/wos/poisson.hpp:12-51): every step adds green_mass(R) f(y) with y
// Green-distributed in the ball (source mode green), |B(R)| f(y) G(R, |y-x|)
// with y uniform in the ball (uniform), or the balance-heuristic mixture of
// the Green density and a Gaussian proposal (MIS, include/wos/
// source_sampling.hpp:35-78), then moves to a uniform point of the
// sphere; inside the epsilon shell the walk ends with g at the nearest point.
//
// Derivatives.  A walk's geometry -- sphere centres, source samples y_k and
// terminal point -- depends on the mesh and the random numbers only, never on
// (Q, x0, sigma) or g.  With m_k the step's mass and q_k = |y_k - x0|^2/sigma^2:
//     du/dQ     = sum_k m_k exp(-q_k)
//     du/dx0    = sum_k m_k f(y_k) 2 (y_k - x0) / sigma^2
//     du/dsigma = sum_k m_k f(y_k) 2 q_k / sigma
//     du/dg_v   = b_v(terminal point)      (interpolation weight of vertex v)
// are the exact derivatives of that walk's sample, so their walk means are
// unbiased estimates of the derivatives of the probe value, and central
// differences taken with the same seeds (common random numbers) converge to
// them as the step shrinks.  The adjoint pass re-runs every walk from its
// seed (nothing is stored between the passes): one instantiation serves both
// passes, with a uniform runtime flag around the derivative sums, so the
// replayed paths are bit-identical to the forward ones.  Given dL/du_p it
// accumulates the per-probe derivative means and scatter-adds
// dL/du_p * b_v / N into dL/dg_v.
//
// Scheduling and precision are those of the FAST walks (kernels_fast.cu):
// persistent warps over (probe, chunk of walks) tasks, lane regeneration,
// warp-cooperative FP32 queries on the 32-wide tree with an FP64
// re-projection in the epsilon shell (or FP64 queries throughout).  Source
// terms and derivative sums are evaluated and accumulated in FP64 at the
// FP32 sample points.
#include <algorithm>
#include <cmath>
#include <type_traits>

#include "device/fast_walk.cuh"
#include "kernels.h"

namespace wosb {

namespace {

struct HeatArgs {
    SceneView s;
    WideView w;
    PointSet ps;
    uint64_t seed;
    int n_walks;
    double eps;
    int max_steps;
    float keep, shrink, exact2, shell2;  // FP32 query bounds (see kernels_fast.cu)
    float list_t;                        // near-boundary lists below this value (-1: none)
    int chunk;
    int chunks;
    long long n_tasks;
    int stage, stage_box, stage_prim;
    int mode;
    double Q, x0, y0, z0, inv_s2, inv_s;
    double beta;                            // MIS: probability of a Green sample
    double px0, py0, pz0, p_inv_s2, p_norm, p_scale;  // MIS proposal N(px0, psigma^2/2 I)
    const double *g;
    const int *slot_verts;
    int adjoint;
    const double *grad_u;
    double *grad_g;
    const uint8_t *location;
    const StartRecord *start;
    HeatPartial *partials;
    unsigned long long *queue;
    DeviceCounters *ctr;
};

// Interpolation weights of the vertices of binary slot `slot` at its point np.
template <int DIM>
__device__ __forceinline__ void vertex_weights(const SceneView &s, int slot, const V3<double> &np,
                                               double w[3]) {
    if (DIM == 2) {
        const double2 a = s.seg64[2 * slot], c = s.seg64[2 * slot + 1];
        const double vx = c.x - a.x, vy = c.y - a.y;
        double t = ((np.x - a.x) * vx + (np.y - a.y) * vy) / (vx * vx + vy * vy);
        t = fmin(fmax(t, 0.0), 1.0);
        w[0] = 1.0 - t;
        w[1] = t;
        w[2] = 0.0;
        return;
    }
    // record: v0 | e1 | e2 | a = e1.e1, b = e1.e2, c = e2.e2 | det, denom
    const double2 *r = s.tri64 + 7 * slot;
    const double2 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4], r5 = r[5], r6 = r[6];
    const double dx = np.x - r0.x, dy = np.y - r0.y, dz = np.z - r1.x;
    const double d1 = dx * r1.y + dy * r2.x + dz * r2.y;
    const double d2 = dx * r3.x + dy * r3.y + dz * r4.x;
    double su = (r5.y * d1 - r5.x * d2) / r6.x;
    double tu = (r4.y * d2 - r5.x * d1) / r6.x;
    su = fmax(su, 0.0);
    tu = fmax(tu, 0.0);
    const double sum = su + tu;
    if (sum > 1.0) {
        su /= sum;
        tu /= sum;
    }
    w[0] = 1.0 - su - tu;
    w[1] = su;
    w[2] = tu;
}

// Boundary value g(np) on slot `slot`; scatters c * b_v into grad_g when c != 0.
template <int DIM>
__device__ __forceinline__ double boundary_data(const HeatArgs &a, int slot, const V3<double> &np,
                                                double c) {
    double w[3];
    vertex_weights<DIM>(a.s, slot, np, w);
    const int *v = a.slot_verts + DIM * slot;
    double val = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        const int vk = v[k];
        if (a.g) val += w[k] * a.g[vk];
        if (c != 0.0) atomicAdd(a.grad_g + vk, c * w[k]);
    }
    return val;
}

// Source term of one step from the ball B(p, R); adds its parameter
// derivatives to j when `adj`.  Every branch reduces to m * f(y) with a
// weight m that does not depend on (Q, x0, sigma):
//   Green    y ~ Green density of the ball,  m = green_mass(R)
//   uniform  y ~ uniform in the ball,        m = |B(R)| G(R, |y - p|)
//   MIS      y ~ beta Green + (1 - beta) proposal (include/wos/source_sampling.hpp:
//            35-78), m = G / (beta G / green_mass + (1 - beta) p_proposal(y)),
//            0 unless 0 < |y - p| < R; the proposal is a fixed density, so the
//            derivatives are still m * df/dtheta.
template <int DIM, typename T>
__device__ __forceinline__ double heat_source(const HeatArgs &a, V3<T> p, T R, FastRng<T> &rng,
                                              bool adj, double j[5]) {
    double yx, yy, yz;
    double m;
    const double Rd = static_cast<double>(R);
    const double px = static_cast<double>(p.x), py = static_cast<double>(p.y);
    const double pz = DIM == 3 ? static_cast<double>(p.z) : 0.0;
    if (a.mode == kGreen) {
        const T r = DIM == 2 ? pg_sample_radius_2d(R, rng) : pg_sample_radius_3d(R, rng);
        const V3<T> y = direction_at<DIM, false, T>(p, r, rng);
        yx = static_cast<double>(y.x);
        yy = static_cast<double>(y.y);
        yz = DIM == 3 ? static_cast<double>(y.z) : 0.0;
        m = DIM == 2 ? Rd * Rd / 4.0 : Rd * Rd / 6.0;
    } else if (a.mode == kMis) {
        if (static_cast<double>(rng.unit()) < a.beta) {
            const T r = DIM == 2 ? pg_sample_radius_2d(R, rng) : pg_sample_radius_3d(R, rng);
            const V3<T> y = direction_at<DIM, false, T>(p, r, rng);
            yx = static_cast<double>(y.x);
            yy = static_cast<double>(y.y);
            yz = DIM == 3 ? static_cast<double>(y.z) : 0.0;
        } else {
            // Box-Muller normals from FP64 uniforms
            double s0, c0;
            const double rho0 = sqrt(-2.0 * log(rng.s.uniform_d()));
            sincospi(2.0 * rng.s.uniform_d(), &s0, &c0);
            yx = a.px0 + a.p_scale * rho0 * c0;
            yy = a.py0 + a.p_scale * rho0 * s0;
            yz = 0.0;
            if (DIM == 3) {
                const double rho1 = sqrt(-2.0 * log(rng.s.uniform_d()));
                yz = a.pz0 + a.p_scale * rho1 * cospi(2.0 * rng.s.uniform_d());
            }
        }
        const double ex = yx - px, ey = yy - py, ez = yz - pz;
        const double r = sqrt(ex * ex + ey * ey + ez * ez);
        if (!(r > 0.0 && r < Rd)) return 0.0;
        const double G = DIM == 2 ? pg_green_2d(Rd, r) : pg_green_3d(Rd, r);
        const double mass = DIM == 2 ? Rd * Rd / 4.0 : Rd * Rd / 6.0;
        const double qx = yx - a.px0, qy = yy - a.py0, qz = yz - a.pz0;
        const double src_pdf = a.p_norm * exp(-(qx * qx + qy * qy + qz * qz) * a.p_inv_s2);
        const double mix = a.beta * (G / mass) + (1.0 - a.beta) * src_pdf;
        if (!(mix > 0.0)) return 0.0;
        m = G / mix;
    } else {
        const V3<T> y = ball_sample<DIM, false, T>(p, R, rng);
        yx = static_cast<double>(y.x);
        yy = static_cast<double>(y.y);
        yz = DIM == 3 ? static_cast<double>(y.z) : 0.0;
        const double ex = yx - px, ey = yy - py, ez = yz - pz;
        const double r = fmin(sqrt(ex * ex + ey * ey + ez * ez), Rd);
        if (!(r > 0.0)) return 0.0;
        m = ball_volume<DIM, double>(Rd) * (DIM == 2 ? pg_green_2d(Rd, r) : pg_green_3d(Rd, r));
    }
    const double dx = yx - a.x0;
    const double dy = yy - a.y0;
    const double dz = DIM == 3 ? yz - a.z0 : 0.0;
    const double q = (dx * dx + dy * dy + dz * dz) * a.inv_s2;
    const double e = exp(-q);
    const double mf = m * a.Q * e;
    if (adj) {
        j[0] += m * e;
        const double c2 = 2.0 * mf * a.inv_s2;
        j[1] += c2 * dx;
        j[2] += c2 * dy;
        j[3] += c2 * dz;
        j[4] += 2.0 * mf * q * a.inv_s;
    }
    return mf;
}

template <int DIM, typename T, int MIN_BLOCKS, int HC>
__global__ void __launch_bounds__(256, MIN_BLOCKS) heat_walk_kernel(HeatArgs a) {
    constexpr bool kF32 = std::is_same<T, float>::value;
    extern __shared__ float4 smem[];
    __shared__ int s_off[8];
    __shared__ double s_acc[10][256];
    if (threadIdx.x < 8) s_off[threadIdx.x] = a.w.off[threadIdx.x];
    WideView wv = a.w;
    wv.off = s_off;
    if (!kF32 || !a.stage) __syncthreads();
    if (kF32 && a.stage) {
        float *sm = reinterpret_cast<float *>(smem);
        for (int i = threadIdx.x; i < a.stage_box; i += blockDim.x) sm[i] = a.w.box[i];
        for (int i = threadIdx.x; i < a.stage_prim; i += blockDim.x) {
            sm[a.stage_box + i] = a.w.prim[i];
        }
        __syncthreads();
        wv.box = sm;
        if (a.stage_prim) {
            // staged primitives: the list scans read them here, not the copy
            wv.prim = sm + a.stage_box;
            wv.aos = nullptr;
        }
    }
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const double eps = a.eps;
    const bool adj = a.adjoint != 0;

    for (;;) {
        unsigned long long task = 0;
        if (lane == 0) task = atomicAdd(a.queue, 1ull);
        task = __shfl_sync(kFull, task, 0);
        if (task >= static_cast<unsigned long long>(a.n_tasks)) break;
        const long long pidx = static_cast<long long>(task / a.chunks);
        const int c = static_cast<int>(task % a.chunks);
        if (a.location[pidx] != 1) continue;

        double px0, py0, pz0;
        uint64_t linear;
        point_at(a.ps, pidx, px0, py0, pz0, linear);
        const uint64_t pseed = point_seed(a.seed, linear);
        const V3<T> p0{static_cast<T>(px0), static_cast<T>(py0), static_cast<T>(pz0)};
        const StartRecord st0 = a.start[pidx];
        const T R0 = static_cast<T>(st0.radius);
        const bool start_stops = !(st0.radius > eps);
        const double cgrad = adj ? a.grad_u[pidx] / static_cast<double>(a.n_walks) : 0.0;
        const int w0 = c * a.chunk;
        const int w1 = min(a.n_walks, w0 + a.chunk);

        int steps_acc = 0;
        ShiftedSums acc;
        // per-lane sums and sums of squares of the derivatives, in shared
        // memory (touched once per finished walk) to keep registers for the walk
        if (adj) {
#pragma unroll
            for (int k = 0; k < 10; ++k) s_acc[k][threadIdx.x] = 0.0;
        }
        unsigned hits = 0;
        unsigned queries = 0;  // BVH queries of this task (FP32; warp-uniform; < 2^32)
        bool bad = false;  // a closest-point query found no primitive

        int walk = w0 + lane;
        bool active = walk < w1;
        int next = w0 + 32;
        V3<T> p = p0;
        T R = R0;
        double sample = 0.0;
        double j[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        int steps = 0;
        int slot = -1;                    // FP32: wide slot of the last query
        int slot64 = -1;                  // FP64: binary slot of the last query
        V3<double> np64{0.0, 0.0, 0.0};
        const uint2 pkey = PhiloxStream::key_of(pseed);
        FastRng<T> rng(pkey, static_cast<uint32_t>(walk));

        while (__any_sync(kFull, active)) {
            bool need_query = false;
            bool listed = false;  // answered from a near-boundary list
            int packed = -1;      // 3D: the list the warp scans for this lane
            // one step of every walk in flight (none from a start point
            // inside the shell)
            if (active && !start_stops) {
                rng.begin_step(steps);
                sample += heat_source<DIM, T>(a, p, R, rng, adj, j);
                p = sphere_step<DIM, false, T>(p, R, rng);
                ++steps;
                if constexpr (kF32) {
                    need_query = true;
                    // the walk kernels' lattice step: away from the shell a
                    // lattice lower bound is the radius (forward and replay
                    // take the same branches, the lattice is fixed)
                    if (wv.gd != nullptr && steps < a.max_steps) {
                        const LatticeSample ls =
                            lattice_sample<DIM>(wv, p.x, p.y, DIM == 3 ? p.z : 0.0f);
                        const float gb = (ls.d - ls.r) * a.shrink;
                        if (ls.d >= wv.gratio * ls.r && gb > 0.0f && gb * gb > a.shell2) {
                            R = gb;
                            need_query = false;
                        } else if (ls.d <= a.list_t) {
                            // near the boundary: a query over the node's
                            // candidate list, when it has one (2D: this
                            // lane scans it; 3D: the warp, below)
                            const int2 e = __ldg(wv.gl + ls.node);
                            const int v = DIM == 3 && e.x >= 0 ? list_prefix(wv, e, ls.r) : e.x;
                            if (v >= 0) {
                                if constexpr (DIM == 2) {
                                    const WideResult q = list_nearest<DIM>(
                                        wv, list_of(wv, v), list_length(v),
                                        static_cast<float>(p.x), static_cast<float>(p.y), 0.0f);
                                    const float r = sqrtf(q.best);
                                    R = static_cast<T>(q.best > a.shell2 ? r * a.shrink : r);
                                    slot = q.slot;
                                } else {
                                    packed = v;
                                }
                                need_query = false;
                                listed = true;
                            }
                        }
                    }
                } else {
                    const Nearest<double> q = nearest64<DIM>(
                        a.s, static_cast<double>(p.x), static_cast<double>(p.y),
                        static_cast<double>(p.z), dinf());
                    R = static_cast<T>(sqrt(q.best));
                    np64 = V3<double>{q.x, q.y, q.z};
                    slot64 = q.slot;
                }
            }
            if constexpr (kF32 && DIM == 3) {
                const bool want = packed >= 0;
                if (__any_sync(kFull, want)) {
                    const WideResult q = warp_list_nearest<DIM>(
                        wv, want, packed, static_cast<float>(p.x), static_cast<float>(p.y),
                        static_cast<float>(p.z));
                    if (want) {
                        const float r = sqrtf(q.best);
                        R = static_cast<T>(q.best > a.shell2 ? r * a.shrink : r);
                        slot = q.slot;
                    }
                }
            }
            if constexpr (kF32) {
                unsigned pending = __ballot_sync(kFull, need_query);
                queries += __popc(pending) + __popc(__ballot_sync(kFull, listed));
                float qbest = 0.0f;
                int qslot = -1;
                while (pending) {
                    const int jl = __ffs(pending) - 1;
                    pending &= pending - 1u;
                    const float qx = __shfl_sync(kFull, static_cast<float>(p.x), jl);
                    const float qy = __shfl_sync(kFull, static_cast<float>(p.y), jl);
                    const float qz =
                        DIM == 3 ? __shfl_sync(kFull, static_cast<float>(p.z), jl) : 0.0f;
                    const WideResult r = wide_nearest<DIM, HC>(wv, qx, qy, qz, a.keep, a.exact2);
                    if (lane == jl) {
                        qbest = r.best;
                        qslot = r.slot;
                    }
                }
                if (need_query) {
                    const float r = sqrtf(qbest);
                    R = static_cast<T>(qbest > a.shell2 ? r * a.shrink : r);
                    slot = qslot;
                }
            }
            // walks whose new radius is in the shell, or that reached the
            // step cap, end in the iteration of their last step
            bool done = false;
            double value = 0.0;
            if (active) {
                bool stop = false;
                V3<double> np{0.0, 0.0, 0.0};
                int bslot = -1;
                int bid = -1;
                if (start_stops) {
                    stop = true;
                    np = V3<double>{st0.nx, st0.ny, st0.nz};
                    bslot = st0.slot;
                } else if (!kF32) {
                    stop = !(static_cast<double>(R) > eps);
                    np = np64;
                    bslot = slot64;
                } else if (static_cast<float>(R) * static_cast<float>(R) <= a.shell2) {
                    if (slot < 0) {  // a query found no primitive: flag it, stop
                        bad = true;
                        stop = true;
                    } else {
                        bslot = wv.wide2bin[slot];
                        const double d2 = reproject64_sq<DIM>(
                            a.s, bslot, static_cast<double>(p.x), static_cast<double>(p.y),
                            static_cast<double>(p.z), np, bid);
                        if (d2 <= eps * eps) {
                            stop = true;
                        } else {
                            R = static_cast<T>(sqrt(d2));
                        }
                    }
                }
                if (!stop && steps >= a.max_steps) {
                    ++hits;
                    stop = true;
                    if (kF32) {
                        if (slot < 0) {
                            bad = true;
                        } else {
                            bslot = wv.wide2bin[slot];
                            reproject64<DIM>(a.s, bslot, static_cast<double>(p.x),
                                             static_cast<double>(p.y), static_cast<double>(p.z),
                                             np, bid);
                        }
                    } else {
                        np = np64;
                        bslot = slot64;
                    }
                }
                if (stop) {
                    value = sample + (bslot >= 0 ? boundary_data<DIM>(a, bslot, np, cgrad) : 0.0);
                    done = true;
                }
            }
            if (done) {
                acc.add(value);
                steps_acc += steps;
                if (adj) {
#pragma unroll
                    for (int k = 0; k < 5; ++k) {
                        s_acc[k][threadIdx.x] += j[k];
                        s_acc[5 + k][threadIdx.x] += j[k] * j[k];
                    }
                }
            }
            const unsigned done_mask = __ballot_sync(kFull, done);
            if (done_mask) {
                if (done) {
                    walk = next + __popc(done_mask & lt_mask);
                    active = walk < w1;
                    if (active) {
                        p = p0;
                        R = R0;
                        sample = 0.0;
#pragma unroll
                        for (int k = 0; k < 5; ++k) j[k] = 0.0;
                        steps = 0;
                        rng = FastRng<T>(pkey, static_cast<uint32_t>(walk));
                    }
                }
                next += __popc(done_mask);
            }
        }

        if (__ballot_sync(kFull, bad) && lane == 0) atomicOr(&a.ctr->error_flags, kErrBadState);
        double n_tot = static_cast<double>(acc.n);
        double mean_acc, m2_acc;
        acc.finish(mean_acc, m2_acc);
        unsigned long long steps_tot = static_cast<unsigned long long>(steps_acc);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double nb = __shfl_down_sync(kFull, n_tot, o);
            const double mb = __shfl_down_sync(kFull, mean_acc, o);
            const double m2b = __shfl_down_sync(kFull, m2_acc, o);
            const unsigned long long sb = __shfl_down_sync(kFull, steps_tot, o);
            const unsigned hb = __shfl_down_sync(kFull, hits, o);
            chan_merge(n_tot, mean_acc, m2_acc, nb, mb, m2b);
            steps_tot += sb;
            hits += hb;
        }
        double jsum[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, jsq[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (adj) {
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                jsum[k] = s_acc[k][threadIdx.x];
                jsq[k] = s_acc[5 + k][threadIdx.x];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
                for (int k = 0; k < 5; ++k) {
                    jsum[k] += __shfl_down_sync(kFull, jsum[k], o);
                    jsq[k] += __shfl_down_sync(kFull, jsq[k], o);
                }
            }
        }
        if (lane == 0) {
            HeatPartial hp;
            hp.n = n_tot;
            hp.mean = mean_acc;
            hp.m2 = m2_acc;
            hp.steps = static_cast<double>(steps_tot);
            hp.queries = kF32 ? static_cast<double>(queries) : static_cast<double>(steps_tot);
            hp.hits = hits;
            hp.pad = 0;
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                hp.jsum[k] = jsum[k];
                hp.jsq[k] = jsq[k];
            }
            a.partials[task] = hp;
        }
    }
}

// Per-probe merge of the chunk partials; boundary and outside probes.
template <int DIM>
__global__ void heat_merge_kernel(HeatArgs a, HeatOut out) {
    const long long n_points = a.ps.n;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    const bool adj = a.adjoint != 0;
    for (long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
         p < n_points; p += stride) {
        const int where = a.location[p];
        double mean = dnan(), variance = dnan(), se = dnan(), steps_mean = dnan();
        double jm[5], js[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) jm[k] = js[k] = dnan();
        if (where == 1) {
            double n = 0.0, m = 0.0, m2 = 0.0, steps = 0.0, queries = 0.0,
                   sum[5] = {0, 0, 0, 0, 0}, sq[5] = {0, 0, 0, 0, 0};
            unsigned long long hits = 0;
            for (int c = 0; c < a.chunks; ++c) {
                const HeatPartial &hp = a.partials[p * a.chunks + c];
                chan_merge(n, m, m2, hp.n, hp.mean, hp.m2);
                steps += hp.steps;
                queries += hp.queries;
                hits += hp.hits;
                if (adj) {
#pragma unroll
                    for (int k = 0; k < 5; ++k) {
                        sum[k] += hp.jsum[k];
                        sq[k] += hp.jsq[k];
                    }
                }
            }
            const double N = static_cast<double>(a.n_walks);
            mean = m;
            variance = a.n_walks > 1 ? m2 / (N - 1.0) : 0.0;
            se = sqrt(variance / N);
            steps_mean = steps / N;
            if (adj) {
#pragma unroll
                for (int k = 0; k < 5; ++k) {
                    jm[k] = sum[k] / N;
                    const double v = a.n_walks > 1 ? fmax(sq[k] - sum[k] * jm[k], 0.0) / (N - 1.0)
                                                   : 0.0;
                    js[k] = sqrt(v / N);
                }
                const double gu = a.grad_u[p];
                if (gu != 0.0 && out.grad_source) {
#pragma unroll
                    for (int k = 0; k < 5; ++k) atomicAdd(out.grad_source + k, gu * jm[k]);
                }
            }
            if (hits) atomicAdd(&a.ctr->max_steps_hits, hits);
            atomicAdd(&a.ctr->total_steps, static_cast<unsigned long long>(steps));
            atomicAdd(&a.ctr->exact_queries, static_cast<unsigned long long>(queries));
            atomicAdd(&a.ctr->total_walks, static_cast<unsigned long long>(n));
        } else if (where == 2) {
            const StartRecord st = a.start[p];
            const double c = adj ? a.grad_u[p] : 0.0;
            mean = boundary_data<DIM>(a, st.slot, V3<double>{st.nx, st.ny, st.nz}, c);
            variance = se = steps_mean = 0.0;
#pragma unroll
            for (int k = 0; k < 5; ++k) jm[k] = js[k] = 0.0;
        }
        if (out.f.mean) out.f.mean[p] = mean;
        if (out.f.variance) out.f.variance[p] = variance;
        if (out.f.standard_error) out.f.standard_error[p] = se;
        if (out.f.mean_steps) out.f.mean_steps[p] = steps_mean;
        if (adj) {
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                if (out.jac) out.jac[5 * p + k] = jm[k];
                if (out.jac_se) out.jac_se[5 * p + k] = js[k];
            }
        }
    }
}

template <int DIM>
cudaError_t launch_heat_dim(const HeatArgs &a, int precision, const FastPlan &plan,
                            cudaStream_t stream) {
    auto grid_for = [&](auto kernel, int smem, int &blocks) -> cudaError_t {
        if (plan.blocks > 0) {
            blocks = plan.blocks;
            return cudaSuccess;
        }
        int per_sm = 0, dev = 0, sms = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel,
                                                                      plan.threads, smem);
        if (e != cudaSuccess) return e;
        e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        blocks = sms * (per_sm > 0 ? per_sm : 1);
        return cudaSuccess;
    };
    int blocks = 0;
    if (precision == 32) {
        // forward and replay read the same tree, so they use one instantiation
        return with_height_class(height_class(a.w.H), [&](auto h) -> cudaError_t {
            constexpr int HC = decltype(h)::value;
            // 4 blocks / SM (64 registers) for the height <= 3 traversals:
            // the kernel waits on loads, so more resident warps pay
            constexpr int kMinBlocks = (HC == kHeightUpTo2 || HC == kHeight3) ? 4 : 3;
            auto k = heat_walk_kernel<DIM, float, kMinBlocks, HC>;
            // the static accumulators (20 KB) plus the staged scene can pass
            // the 48 KB default: opt in whenever anything is staged
            if (plan.smem_bytes > 0) {
                cudaError_t e = cudaFuncSetAttribute(
                    k, cudaFuncAttributeMaxDynamicSharedMemorySize, plan.smem_bytes);
                if (e != cudaSuccess) return e;
            }
            cudaError_t e = grid_for(k, plan.smem_bytes, blocks);
            if (e != cudaSuccess) return e;
            k<<<blocks, plan.threads, plan.smem_bytes, stream>>>(a);
            return cudaGetLastError();
        });
    } else {
        auto k = heat_walk_kernel<DIM, double, 1, kHeightAny>;
        cudaError_t e = grid_for(k, 0, blocks);
        if (e != cudaSuccess) return e;
        k<<<blocks, plan.threads, 0, stream>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_heat(const SceneView &s, const WideView &w, const PointSet &ps,
                        uint64_t seed, const HeatDesc &h, int n_walks, double epsilon,
                        int max_steps, double shell_delta, int precision, const FastPlan &plan,
                        const uint8_t *location, const StartRecord *start, HeatPartial *partials,
                        unsigned long long *queue, HeatOut out, DeviceCounters *counters,
                        cudaStream_t stream, cudaEvent_t after_walk) {
    if (ps.n <= 0) return cudaSuccess;
    HeatArgs a{};
    a.s = s;
    a.w = w;
    a.ps = ps;
    a.seed = seed;
    a.n_walks = n_walks;
    a.eps = epsilon;
    a.max_steps = max_steps;
    const double tau = 1.0 / 1024.0;
    const double shell = epsilon + shell_delta;
    a.keep = static_cast<float>((1.0 - tau) * (1.0 - tau));
    a.shrink = static_cast<float>(1.0 - tau);
    a.shell2 = static_cast<float>(shell * shell);
    a.exact2 = static_cast<float>(shell * shell / ((1.0 - tau) * (1.0 - tau)));
    a.list_t = w.gl != nullptr ? near_list_threshold(w, epsilon, shell_delta) : -1.0f;
    a.chunk = plan.chunk;
    a.chunks = plan.chunks;
    a.n_tasks = plan.n_tasks;
    a.stage = plan.stage_scene ? 1 : 0;
    a.stage_box = plan.stage_scene ? w.box_total : 0;
    a.stage_prim = plan.stage_prims ? (w.dim == 2 ? 5 : 16) * w.npad : 0;
    a.mode = h.mode;
    a.Q = h.Q;
    a.x0 = h.x0[0];
    a.y0 = h.x0[1];
    a.z0 = s.dim == 3 ? h.x0[2] : 0.0;
    a.inv_s2 = 1.0 / (h.sigma * h.sigma);
    a.inv_s = 1.0 / h.sigma;
    a.beta = h.beta;
    a.px0 = h.px0[0];
    a.py0 = h.px0[1];
    a.pz0 = s.dim == 3 ? h.px0[2] : 0.0;
    a.p_inv_s2 = 1.0 / (h.psigma * h.psigma);
    // N(px0, psigma^2/2 I): density exp(-|y - px0|^2 / psigma^2) / (pi^(d/2) psigma^d)
    a.p_norm = 1.0 / (std::pow(kPi, 0.5 * s.dim) * std::pow(h.psigma, s.dim));
    a.p_scale = h.psigma / std::sqrt(2.0);
    a.g = h.g;
    a.slot_verts = h.slot_verts;
    a.adjoint = h.adjoint;
    a.grad_u = h.grad_u;
    a.grad_g = h.grad_g;
    a.location = location;
    a.start = start;
    a.partials = partials;
    a.queue = queue;
    a.ctr = counters;
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    e = s.dim == 2 ? launch_heat_dim<2>(a, precision, plan, stream)
                   : launch_heat_dim<3>(a, precision, plan, stream);
    if (e != cudaSuccess) return e;
    if (after_walk) {
        e = cudaEventRecord(after_walk, stream);
        if (e != cudaSuccess) return e;
    }
    long long b = (ps.n + 255) / 256;
    if (b < 1) b = 1;
    if (s.dim == 2) {
        heat_merge_kernel<2><<<static_cast<int>(b), 256, 0, stream>>>(a, out);
    } else {
        heat_merge_kernel<3><<<static_cast<int>(b), 256, 0, stream>>>(a, out);
    }
    return cudaGetLastError();
}

}  // namespace wosb
