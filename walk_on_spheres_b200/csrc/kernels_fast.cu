// Fast-path kernels: FAST_FP32 / FAST_FP64 walks and the per-point merge.
//
// Scheduling.  A persistent grid of warps pulls tasks from a device queue
// (one atomicAdd per task).  A task is a chunk of consecutive walks of one
// grid point; its 32 lanes each run one walk at a time and, when a walk
// ends, the lane is regenerated with the next walk index of the chunk
// (warp ballot + popcount rank), so a warp stays full until the chunk's last
// walks.  Every walk of point p with index w draws from its own Philox
// stream keyed by p's reference seed, so results do not depend on which
// lane or warp runs the walk.
//
// Precision (FAST_FP32).  Positions, radii, closest-point queries and the
// sphere step are FP32 against the FP32 scene (staged in shared memory when
// it fits).  When the FP32 radius falls within `shell_delta` of epsilon the
// walk re-projects in FP64: an exact FP64 query at the (exactly widened)
// position decides termination and supplies the nearest point and
// boundary id for the boundary value, evaluated in FP64.  Per-walk values are
// accumulated in FP64 (Welford per lane, Chan's merge across lanes and
// chunks).  FAST_FP64 runs the same scheduling with FP64 everywhere.
#include <algorithm>
#include <cmath>
#include <type_traits>

#include "device/fast_walk.cuh"
#include "kernels.h"

namespace wosb {

namespace {


// One task: walks [c*chunk, min(N, (c+1)*chunk)) of point pidx, written to
// a.partials[task] as Welford statistics.
template <int DIM, class Eq, typename T, int HC>
__device__ __forceinline__ void fast_task(const FastArgs a, const WideView &wv, const Eq &eq,
                                          unsigned long long task, long long pidx, int c) {
    constexpr bool kF32 = std::is_same<T, float>::value;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const double eps = a.eps;
    const double eps2 = eps * eps;

    double x0, y0, z0;
    uint64_t linear;
    point_at(a.ps, pidx, x0, y0, z0, linear);
    const uint64_t pseed = point_seed(a.seed, linear);
    const V3<T> p0{static_cast<T>(x0), static_cast<T>(y0), static_cast<T>(z0)};
    const double r0 = a.start[pidx].radius;
    const T R0 = static_cast<T>(r0);
    const bool start_stops = !(r0 > eps);  // start point already inside the shell
    const int w0 = c * a.chunk;
    const int w1 = min(a.n_walks, w0 + a.chunk);

    // per-lane statistics
    int steps_acc = 0;
    ShiftedSums acc;
    unsigned hits = 0;
    // BVH closest-point queries of this task (warp-uniform; FP32 only: every
    // FP64 step is one).  At most chunk * max_steps < 2^32 (set_chunk).
    unsigned queries = 0;
    bool overflow = false;
    bool bad = false;  // a closest-point query found no primitive

    // per-lane walk state
    int walk = w0 + lane;
    bool active = walk < w1;
    int next = w0 + 32;
    V3<T> p = p0;
    T R = R0;
    T sample = T(0), weight = T(1);
    int steps = 0;
    int slot = -1;                 // FP32: winner of the last query
    V3<double> np64{0.0, 0.0, 0.0};  // FP64: nearest point of the last query
    int bid64 = -1;
    const uint2 pkey = PhiloxStream::key_of(pseed);
    FastRng<T> rng(pkey, static_cast<uint32_t>(walk));

    while (__any_sync(kFull, active)) {
        bool need_query = false;
        bool listed = false;  // answered from a near-boundary list
        int packed = -1;      // 3D: the list the warp scans for this lane
        // One step of every walk in flight (a start point inside the shell
        // takes none: its walks end where they start).
        if (active && !start_stops) {
            rng.begin_step(steps);
            p = walk_body<DIM, false, T>(eq, p, R, sample, weight, rng, rng, overflow);
            ++steps;
            if constexpr (kF32) {
                need_query = true;
                if constexpr (HC != kLaneScan) {
                    // away from the shell a lattice lower bound is a valid
                    // (smaller) radius and spares the exact query; the step
                    // that reaches the cap queries, for its nearest point
                    if (wv.gd != nullptr && steps < a.max_steps) {
                        const LatticeSample ls =
                            lattice_sample<DIM>(wv, p.x, p.y, DIM == 3 ? p.z : 0.0f);
                        const float gb = (ls.d - ls.r) * a.shrink;
                        if (ls.d >= wv.gratio * ls.r && gb > 0.0f && gb * gb > a.shell2) {
                            R = gb;
                            need_query = false;
                        } else if (ls.d <= a.list_t) {
                            // near the boundary: a query over the node's
                            // candidate list, when it has one; in 2D (a
                            // few segments) this lane scans it, in 3D the
                            // warp scans all such lists together below
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
                }
            } else {
                const Nearest<double> q = nearest64<DIM>(
                    a.s, static_cast<double>(p.x), static_cast<double>(p.y),
                    static_cast<double>(p.z), dinf());
                R = static_cast<T>(sqrt(q.best));
                np64 = V3<double>{q.x, q.y, q.z};
                bid64 = bid_of<DIM>(a.s, q.slot);
            }
        }
        if constexpr (kF32 && HC == kLaneScan) {
            // a handful of primitives: every lane scans them for its own query
            queries += __popc(__ballot_sync(kFull, need_query));
            if (need_query) {
                const WideResult q = lane_nearest<DIM>(wv, static_cast<float>(p.x),
                                                       static_cast<float>(p.y),
                                                       static_cast<float>(p.z));
                const float r = sqrtf(q.best);
                R = static_cast<T>(q.best > a.shell2 ? r * a.shrink : r);
                slot = q.slot;
            }
        } else if constexpr (kF32) {
            if constexpr (DIM == 3) {
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
            // the warp resolves every pending closest-point query together
            unsigned pending = __ballot_sync(kFull, need_query);
            queries += __popc(pending) + __popc(__ballot_sync(kFull, listed));
            float qbest = 0.0f;
            int qslot = -1;
            while (pending) {
                const int j = __ffs(pending) - 1;
                pending &= pending - 1u;
                const float qx = __shfl_sync(kFull, static_cast<float>(p.x), j);
                const float qy = __shfl_sync(kFull, static_cast<float>(p.y), j);
                const float qz = DIM == 3 ? __shfl_sync(kFull, static_cast<float>(p.z), j) : 0.0f;
                const WideResult r = wide_nearest<DIM, HC>(wv, qx, qy, qz, a.keep, a.exact2);
                if (lane == j) {
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
        // Walks whose new radius is in the epsilon shell, or that reached
        // the step cap, end in the iteration of their last step, so the lane
        // steps its next walk in the next iteration.
        bool done = false;
        double value = 0.0;
        if (active) {
            bool stop = false;
            V3<double> np{0.0, 0.0, 0.0};
            int bid = -1;
            if (start_stops) {
                stop = true;
                const StartRecord st = a.start[pidx];
                np = V3<double>{st.nx, st.ny, st.nz};
                bid = st.boundary_id;
            } else if (!kF32) {
                stop = !(static_cast<double>(R) > eps);
                np = np64;
                bid = bid64;
            } else if (static_cast<float>(R) * static_cast<float>(R) <= a.shell2) {
                // epsilon shell: FP64 re-projection onto the nearest primitive
                // (a query that found none is a broken walk: flag it, stop)
                if (slot < 0) {
                    bad = true;
                    stop = true;
                } else {
                    const double d2 = reproject64_sq<DIM>(a.s, wv.wide2bin[slot],
                                                          static_cast<double>(p.x),
                                                          static_cast<double>(p.y),
                                                          static_cast<double>(p.z), np, bid);
                    if (d2 <= eps2) {
                        stop = true;
                    } else {
                        R = static_cast<T>(sqrt(d2));
                    }
                }
            }
            if (!stop && steps >= a.max_steps) {
                // step cap: finish at the nearest boundary point
                // (include/wos/wos.hpp:129-137)
                ++hits;
                stop = true;
                if (kF32) {
                    if (slot < 0) {
                        bad = true;
                    } else {
                        reproject64<DIM>(a.s, wv.wide2bin[slot], static_cast<double>(p.x),
                                         static_cast<double>(p.y), static_cast<double>(p.z), np,
                                         bid);
                    }
                } else {
                    np = np64;
                    bid = bid64;
                }
            }
            if (stop) {
                value = static_cast<double>(sample) +
                        static_cast<double>(weight) * eq.boundary(np, bid);
                done = true;
            }
        }
        if (done) {
            acc.add(value);
            steps_acc += steps;
        }
        const unsigned done_mask = __ballot_sync(kFull, done);
        if (done_mask) {
            if (done) {
                walk = next + __popc(done_mask & lt_mask);
                active = walk < w1;
                if (active) {
                    p = p0;
                    R = R0;
                    sample = T(0);
                    weight = T(1);
                    steps = 0;
                    rng = FastRng<T>(pkey, static_cast<uint32_t>(walk));
                }
            }
            next += __popc(done_mask);
        }
    }

    // warp merge of the lanes' statistics
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
    const unsigned any_overflow = __ballot_sync(kFull, overflow);
    const unsigned any_bad = __ballot_sync(kFull, bad);
    if (lane == 0) {
        if (any_bad) atomicOr(&a.ctr->error_flags, kErrBadState);
        TaskPartial tp;
        tp.n = n_tot;
        tp.mean = mean_acc;
        tp.m2 = m2_acc;
        tp.steps = static_cast<double>(steps_tot);
        tp.queries = kF32 ? static_cast<double>(queries) : static_cast<double>(steps_tot);
        tp.hits = hits;
        tp.pad = 0;
        a.partials[task] = tp;
        if (any_overflow) atomicOr(&a.ctr->error_flags, kErrRejectionCap);
    }
}

template <int DIM>
__device__ __forceinline__ Laplace<DIM> eq_from(const EqDesc &, Laplace<DIM> *) {
    return Laplace<DIM>{};
}
template <int DIM>
__device__ __forceinline__ Poisson<DIM> eq_from(const EqDesc &e, Poisson<DIM> *) {
    return Poisson<DIM>{e.mode, e.alpha};
}
template <int DIM>
__device__ __forceinline__ Screened<DIM> eq_from(const EqDesc &e, Screened<DIM> *) {
    return Screened<DIM>{e.mode, e.alpha};
}
template <int DIM>
__device__ __forceinline__ Helmholtz<DIM> eq_from(const EqDesc &, Helmholtz<DIM> *) {
    return Helmholtz<DIM>{};
}

template <int DIM, class Eq, typename T, int MIN_BLOCKS, int HC>
__global__ void __launch_bounds__(256, MIN_BLOCKS) walk_fast_kernel(FastArgs a, Eq eq) {
    constexpr bool kF32 = std::is_same<T, float>::value;
    extern __shared__ float4 smem[];
    __shared__ int s_off[8];
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

    for (;;) {
        unsigned long long task = 0;
        if (lane == 0) task = atomicAdd(a.queue, 1ull);
        task = __shfl_sync(kFull, task, 0);
        if (task >= static_cast<unsigned long long>(a.n_tasks)) break;
        const long long pidx = static_cast<long long>(task / a.chunks);
        const int c = static_cast<int>(task % a.chunks);
        if (a.location[pidx] != 1) continue;
        fast_task<DIM, Eq, T, HC>(a, wv, eq, task, pidx, c);
    }
}

// Walks of one family of batch items: one queue over the items' tasks
// (numbered by task_begin); each task runs the walk_fast_kernel task body
// with its own item's scene, grid, equation and statistics buffers (the
// scene is read through L1/L2, never staged).
template <int DIM, class Eq, typename T, int MIN_BLOCKS, int HC>
__global__ void __launch_bounds__(256, MIN_BLOCKS)
    walk_batch_kernel(const BatchItem *__restrict__ items, int n_items, long long n_tasks,
                      unsigned long long *queue) {
    __shared__ int s_off[8][8];  // per warp: wide-tree offsets of the warp's current item
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    int cur = -1;
    for (;;) {
        unsigned long long task = 0;
        if (lane == 0) task = atomicAdd(queue, 1ull);
        task = __shfl_sync(kFull, task, 0);
        if (task >= static_cast<unsigned long long>(n_tasks)) break;
        const long long t = static_cast<long long>(task);
        int lo = 0, hi = n_items - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (items[mid].task_begin <= t) lo = mid;
            else hi = mid - 1;
        }
        const BatchItem &it = items[lo];
        if (lo != cur) {
            __syncwarp();
            if (lane < 8) s_off[warp][lane] = it.a.w.off[lane];
            __syncwarp();
            cur = lo;
        }
        const long long local = t - it.task_begin;
        const long long pidx = local / it.a.chunks;
        const int c = static_cast<int>(local % it.a.chunks);
        if (it.a.location[pidx] != 1) continue;
        WideView wv = it.a.w;
        wv.off = s_off[warp];
        const Eq eq = eq_from(it.eq, static_cast<Eq *>(nullptr));
        fast_task<DIM, Eq, T, HC>(it.a, wv, eq, static_cast<unsigned long long>(local), pidx, c);
    }
}

// Per-point merge of the chunk statistics (include/wos/wos.hpp:182-190).
__device__ __forceinline__ void merge_point(long long p, int chunks, int n_walks,
                                            const TaskPartial *__restrict__ partials,
                                            const Fields &out, DeviceCounters *ctr) {
    double n = 0.0, mean = 0.0, m2 = 0.0, steps = 0.0, queries = 0.0;
    unsigned long long hits = 0;
    for (int c = 0; c < chunks; ++c) {
        const TaskPartial tp = partials[p * chunks + c];
        chan_merge(n, mean, m2, tp.n, tp.mean, tp.m2);
        steps += tp.steps;
        queries += tp.queries;
        hits += tp.hits;
    }
    const double variance = n_walks > 1 ? m2 / static_cast<double>(n_walks - 1) : 0.0;
    if (out.mean) out.mean[p] = mean;
    if (out.variance) out.variance[p] = variance;
    if (out.standard_error) out.standard_error[p] = sqrt(variance / static_cast<double>(n_walks));
    if (out.mean_steps) out.mean_steps[p] = steps / static_cast<double>(n_walks);
    if (hits) atomicAdd(&ctr->max_steps_hits, hits);
    atomicAdd(&ctr->total_steps, static_cast<unsigned long long>(steps));
    atomicAdd(&ctr->exact_queries, static_cast<unsigned long long>(queries));
    atomicAdd(&ctr->total_walks, static_cast<unsigned long long>(n));
}

__global__ void merge_kernel(long long n_points, int chunks, int n_walks,
                             const uint8_t *__restrict__ location,
                             const TaskPartial *__restrict__ partials, Fields out,
                             DeviceCounters *ctr) {
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
         p < n_points; p += stride) {
        if (location[p] != 1) continue;
        merge_point(p, chunks, n_walks, partials, out, ctr);
    }
}

// ------------------------------------------------------------------ batches

__global__ void merge_batch_kernel(const BatchItem *__restrict__ items, int n_items,
                                   long long n_points) {
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
         t < n_points; t += stride) {
        int lo = 0, hi = n_items - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (items[mid].point_begin <= t) lo = mid;
            else hi = mid - 1;
        }
        const BatchItem &it = items[lo];
        const long long p = t - it.point_begin;
        if (it.a.location[p] != 1) continue;
        merge_point(p, it.a.chunks, it.a.n_walks, it.a.partials, it.out, it.a.ctr);
    }
}

template <int DIM, class Eq>
cudaError_t batch_typed(int precision, int hc, const BatchItem *items, int n_items,
                        long long n_tasks, unsigned long long *queue, int blocks,
                        cudaStream_t stream) {
    if (precision == 32) {
        return with_height_class(hc, [&](auto h) {
            constexpr int HC = decltype(h)::value;
            constexpr int kMinBlocks = (HC == kHeightUpTo2 || HC == kHeight3) ? 4 : 3;
            walk_batch_kernel<DIM, Eq, float, kMinBlocks, HC><<<blocks, 256, 0, stream>>>(
                items, n_items, n_tasks, queue);
            return cudaGetLastError();
        });
    }
    walk_batch_kernel<DIM, Eq, double, 1, kHeightAny><<<blocks, 256, 0, stream>>>(
        items, n_items, n_tasks, queue);
    return cudaGetLastError();
}

template <int DIM, class Eq>
cudaError_t batch_blocks_typed(int precision, int hc, int &blocks) {
    int per_sm = 0, dev = 0, sms = 0;
    cudaError_t e;
    if (precision == 32) {
        e = with_height_class(hc, [&](auto h) {
            constexpr int HC = decltype(h)::value;
            constexpr int kMinBlocks = (HC == kHeightUpTo2 || HC == kHeight3) ? 4 : 3;
            return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, walk_batch_kernel<DIM, Eq, float, kMinBlocks, HC>, 256, 0);
        });
    } else {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, walk_batch_kernel<DIM, Eq, double, 1, kHeightAny>, 256, 0);
    }
    if (e != cudaSuccess) return e;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    blocks = sms * (per_sm > 0 ? per_sm : 1);
    return cudaSuccess;
}

template <int DIM>
cudaError_t batch_dispatch(int kind, int precision, int hc, const BatchItem *items, int n_items,
                           long long n_tasks, unsigned long long *queue, int blocks,
                           cudaStream_t stream, int *blocks_out) {
    switch (kind) {
        case kLaplace:
            return blocks_out
                       ? batch_blocks_typed<DIM, Laplace<DIM>>(precision, hc, *blocks_out)
                       : batch_typed<DIM, Laplace<DIM>>(precision, hc, items, n_items, n_tasks,
                                                        queue, blocks, stream);
        case kPoisson:
            return blocks_out
                       ? batch_blocks_typed<DIM, Poisson<DIM>>(precision, hc, *blocks_out)
                       : batch_typed<DIM, Poisson<DIM>>(precision, hc, items, n_items, n_tasks,
                                                        queue, blocks, stream);
        case kScreened:
            return blocks_out
                       ? batch_blocks_typed<DIM, Screened<DIM>>(precision, hc, *blocks_out)
                       : batch_typed<DIM, Screened<DIM>>(precision, hc, items, n_items, n_tasks,
                                                         queue, blocks, stream);
        default:
            return blocks_out
                       ? batch_blocks_typed<DIM, Helmholtz<DIM>>(precision, hc, *blocks_out)
                       : batch_typed<DIM, Helmholtz<DIM>>(precision, hc, items, n_items, n_tasks,
                                                          queue, blocks, stream);
    }
}

template <int DIM>
__global__ void closest32_kernel(SceneView s, WideView w, const double *pts, long long n,
                                 double *dist, double *nearest, int *bid) {
    // each warp takes 32 queries and resolves them one after another
    const long long base = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) & ~31ll;
    const int lane = threadIdx.x & 31;
    const long long t = base + lane;
    const bool valid = t < n;
    float px = 0.0f, py = 0.0f, pz = 0.0f;
    if (valid) {
        px = static_cast<float>(pts[DIM * t]);
        py = static_cast<float>(pts[DIM * t + 1]);
        pz = DIM == 3 ? static_cast<float>(pts[DIM * t + 2]) : 0.0f;
    }
    float mybest = 0.0f;
    int myslot = -1;
    unsigned pending = __ballot_sync(kFull, valid);
    while (pending) {
        const int j = __ffs(pending) - 1;
        pending &= pending - 1u;
        const float qx = __shfl_sync(kFull, px, j), qy = __shfl_sync(kFull, py, j);
        const float qz = __shfl_sync(kFull, pz, j);
        // exact query (keep = 1)
        const WideResult r = wide_nearest<DIM>(w, qx, qy, qz, 1.0f, 0.0f);
        if (lane == j) {
            mybest = r.best;
            myslot = r.slot;
        }
    }
    if (!valid) return;
    dist[t] = sqrtf(mybest);
    V3<double> np;
    int b = -1;
    reproject64<DIM>(s, w.wide2bin[myslot], px, py, pz, np, b);
    nearest[DIM * t] = np.x;
    nearest[DIM * t + 1] = np.y;
    if (DIM == 3) nearest[DIM * t + 2] = np.z;
    if (bid) bid[t] = b;
}

// The equation object of a descriptor, built on the host for kernel arguments.
template <class Eq>
Eq eq_host(const EqDesc &e);
template <>
Laplace<2> eq_host(const EqDesc &) { return Laplace<2>{}; }
template <>
Laplace<3> eq_host(const EqDesc &) { return Laplace<3>{}; }
template <>
Poisson<2> eq_host(const EqDesc &e) { return Poisson<2>{e.mode, e.alpha}; }
template <>
Poisson<3> eq_host(const EqDesc &e) { return Poisson<3>{e.mode, e.alpha}; }
template <>
Screened<2> eq_host(const EqDesc &e) { return Screened<2>{e.mode, e.alpha}; }
template <>
Screened<3> eq_host(const EqDesc &e) { return Screened<3>{e.mode, e.alpha}; }
template <>
Helmholtz<2> eq_host(const EqDesc &) { return Helmholtz<2>{}; }
template <>
Transient<2> eq_host(const EqDesc &e) { return Transient<2>{kGreen, e.alpha, e.tr}; }
template <>
Plate<2> eq_host(const EqDesc &e) { return Plate<2>{e.mode, *e.pl}; }
template <>
Helmholtz<3> eq_host(const EqDesc &) { return Helmholtz<3>{}; }

template <int DIM, class Eq>
cudaError_t launch_fast_typed(const FastArgs &a, const EqDesc &e, int precision,
                              const FastPlan &plan, cudaStream_t stream) {
    // persistent grid: every block that can be resident at once (plan.blocks
    // overrides when positive)
    auto grid_for = [&](auto kernel, int smem, int &blocks) -> cudaError_t {
        if (plan.blocks > 0) {
            blocks = plan.blocks;
            return cudaSuccess;
        }
        int per_sm = 0, dev = 0, sms = 0;
        cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel,
                                                                        plan.threads, smem);
        if (err != cudaSuccess) return err;
        err = cudaGetDevice(&dev);
        if (err != cudaSuccess) return err;
        err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (err != cudaSuccess) return err;
        blocks = sms * (per_sm > 0 ? per_sm : 1);
        return cudaSuccess;
    };
    int blocks = 0;
    if (precision == 32) {
        return with_height_class(traversal_class(a.w), [&](auto h) -> cudaError_t {
            constexpr int HC = decltype(h)::value;
            // 4 blocks / SM (64 registers) for the height <= 3 traversals,
            // 3 for the generic one
            constexpr int kMinBlocks = (HC == kHeightUpTo2 || HC == kHeight3) ? 4 : 3;
            auto k = walk_fast_kernel<DIM, Eq, float, kMinBlocks, HC>;
            if (plan.smem_bytes > 48 * 1024) {
                cudaError_t err = cudaFuncSetAttribute(
                    k, cudaFuncAttributeMaxDynamicSharedMemorySize, plan.smem_bytes);
                if (err != cudaSuccess) return err;
            }
            cudaError_t err = grid_for(k, plan.smem_bytes, blocks);
            if (err != cudaSuccess) return err;
            k<<<blocks, plan.threads, plan.smem_bytes, stream>>>(a, eq_host<Eq>(e));
            return cudaGetLastError();
        });
    } else {
        auto k = walk_fast_kernel<DIM, Eq, double, 1, kHeightAny>;
        cudaError_t err = grid_for(k, 0, blocks);
        if (err != cudaSuccess) return err;
        k<<<blocks, plan.threads, 0, stream>>>(a, eq_host<Eq>(e));
    }
    return cudaGetLastError();
}

template <int DIM>
cudaError_t launch_fast_dim(const FastArgs &a, EqDesc e, int precision, const FastPlan &plan,
                            cudaStream_t stream) {
    switch (e.kind) {
        case kLaplace:
            return launch_fast_typed<DIM, Laplace<DIM>>(a, e, precision, plan, stream);
        case kPoisson:
            return launch_fast_typed<DIM, Poisson<DIM>>(a, e, precision, plan, stream);
        case kScreened:
            return launch_fast_typed<DIM, Screened<DIM>>(a, e, precision, plan, stream);
        case kTransient:
            return DIM == 2 ? launch_fast_typed<2, Transient<2>>(a, e, precision, plan, stream)
                            : cudaErrorInvalidValue;
        case kPlate:
            return DIM == 2 && e.pl ? launch_fast_typed<2, Plate<2>>(a, e, precision, plan, stream)
                                    : cudaErrorInvalidValue;
        default:
            return launch_fast_typed<DIM, Helmholtz<DIM>>(a, e, precision, plan, stream);
    }
}

}  // namespace

namespace {
__global__ void special32_kernel(const double *x, long long n, double *li0, double *lk0) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float xf = static_cast<float>(x[i]);
    li0[i] = static_cast<double>(log_i0(xf));
    lk0[i] = static_cast<double>(log_k0(xf));
}
}  // namespace

namespace {
// Whether lattice node (i, j, k) and its neighbours all lie outside the mesh
// (the row-parity mask): such a node stores 0 (a valid lower bound, written
// as -0.0 to mark the skip) without a query, since no walk inside the
// domain samples it for a useful bound.
template <int DIM>
__device__ __forceinline__ bool node_skipped(const WideView &w, const uint8_t *outside, int i,
                                             int j, int k) {
    bool all_out = true;
    for (int q = 0; q < (DIM == 2 ? 9 : 27) && all_out; ++q) {
        const int ni = i + q % 3 - 1, nj = j + (q / 3) % 3 - 1;
        const int nk = DIM == 3 ? k + q / 9 - 1 : 0;
        if (ni >= 0 && ni < w.gn[0] && nj >= 0 && nj < w.gn[1] && nk >= 0 && nk < w.gn[2]) {
            all_out = outside[(ni * w.gn[1] + nj) * w.gn[2] + nk] != 0;
        }
    }
    return all_out;
}

// Lattice nodes 32 at a time per warp: each lane decodes one node and
// decides whether it is skipped; the warp then runs the FP32 cooperative
// query for each remaining node in turn, at the node's FP32 position
// glo + (i, j, k) gh, the same position the walks' lattice_sample rebuilds.
// The query prunes conservatively (keep = (1 - tau)^2, as the walks do
// above the shell): it returns a squared distance at most 1 / keep times the
// true one, and a node deep inside a round mesh, nearly equidistant from
// every primitive, does not visit them all.  So the value stored is
// sqrt(best) (1 - tau) minus `margin` (the FP32 rounding of the primitive
// distances, a few ulps of the coordinates), rounded down.  Node indices fit
// in 32 bits (at most 2048^2 in 2D, 256^3 in 3D).
template <int DIM, int HC>
__global__ void __launch_bounds__(256) lattice32_kernel(WideView w, float margin,
                                                        const uint8_t *__restrict__ outside,
                                                        float *out) {
    constexpr float kShrink = 1.0f - 0x1p-10f;
    const int lane = threadIdx.x & 31;
    const int warp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int warps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
    const int n = w.gn[0] * w.gn[1] * w.gn[2];
    for (int base = warp * 32; base < n; base += warps * 32) {
        const int t = base + lane;
        bool query = t < n;
        float x = 0.0f, y = 0.0f, z = 0.0f;
        if (query) {
            const int k = t % w.gn[2];
            const int r = t / w.gn[2];
            const int j = r % w.gn[1];
            const int i = r / w.gn[1];
            if (outside != nullptr && node_skipped<DIM>(w, outside, i, j, k)) {
                out[t] = -0.0f;  // -0.0: a valid bound that marks the node as skipped
                query = false;
            }
            x = w.glo[0] + static_cast<float>(i) * w.gh;
            y = w.glo[1] + static_cast<float>(j) * w.gh;
            z = DIM == 3 ? w.glo[2] + static_cast<float>(k) * w.gh : 0.0f;
        }
        unsigned pending = __ballot_sync(kFull, query);
        while (pending) {
            const int src = __ffs(pending) - 1;
            pending &= pending - 1u;
            const float qx = __shfl_sync(kFull, x, src);
            const float qy = __shfl_sync(kFull, y, src);
            const float qz = __shfl_sync(kFull, z, src);
            const WideResult q = wide_nearest<DIM, HC>(w, qx, qy, qz, kShrink * kShrink, 0.0f);
            if (lane == src) {
                const float d = (sqrtf(q.best) * kShrink - margin) * (1.0f - 0x1p-20f);
                out[t] = d > 0.0f ? d : 0.0f;
            }
        }
    }
}

// 3D lattice by warp tiles of 2 x 4 x 4 nodes (i, j, k), one node per lane.
// The nearest primitive of a node x lies within d(x) + |x - c| <= d(c) +
// 2 |x - c| of the tile centre c, so every primitive within d(c) + 2 r_tile
// (r_tile: the largest |x - c|, plus a rounding slack) is a candidate for
// every node of the tile; the warp collects them once (kTileCap at most) and
// each lane takes the FP32 minimum over the candidates for its node, the
// candidates' contiguous records (w.aos) staged 32 at a time in shared
// memory.  That minimum is the
// unpruned FP32 query's, so each node stores a value at most, and mostly
// exactly, lattice32_kernel's (same (1 - tau) factor and margin).  A tile
// with more candidates (deep inside a large round mesh, where many
// primitives are nearly equidistant) stops collecting them and queries its
// nodes one at a time as lattice32_kernel does.  A candidate costs each
// lane about two warp instructions' worth of its node's time, against about
// 700 for a per-node tree query even on a small mesh.
constexpr int kTileCap = 512;

template <int HC>
__global__ void __launch_bounds__(256) lattice_tile3_kernel(WideView w, float margin,
                                                            float slack,
                                                            const uint8_t *__restrict__ outside,
                                                            float *out) {
    __shared__ int s_cand[8][kTileCap];
    __shared__ float4 s_rec[8][32][4];  // 32 candidate records per warp at a time
    constexpr float kShrink = 1.0f - 0x1p-10f;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int warp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int warps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
    const int tj = (w.gn[1] + 3) / 4, tk = (w.gn[2] + 3) / 4;
    const int tiles = ((w.gn[0] + 1) / 2) * tj * tk;
    for (int tile = warp; tile < tiles; tile += warps) {
        const int i0 = 2 * (tile / (tj * tk)), j0 = 4 * ((tile / tk) % tj), k0 = 4 * (tile % tk);
        const int i = i0 + (lane >> 4), j = j0 + ((lane >> 2) & 3), k = k0 + (lane & 3);
        const bool valid = i < w.gn[0] && j < w.gn[1] && k < w.gn[2];
        const int t = valid ? (i * w.gn[1] + j) * w.gn[2] + k : 0;
        bool query = valid;
        if (valid && outside != nullptr && node_skipped<3>(w, outside, i, j, k)) {
            out[t] = -0.0f;
            query = false;
        }
        const unsigned want = __ballot_sync(kFull, query);
        if (!want) continue;
        const float x = w.glo[0] + static_cast<float>(i) * w.gh;
        const float y = w.glo[1] + static_cast<float>(j) * w.gh;
        const float z = w.glo[2] + static_cast<float>(k) * w.gh;
        // the tile's centre and reach over its nodes inside the lattice
        const int ni = min(2, w.gn[0] - i0), nj = min(4, w.gn[1] - j0), nk = min(4, w.gn[2] - k0);
        const float cx = w.glo[0] + (static_cast<float>(i0) + 0.5f * (ni - 1)) * w.gh;
        const float cy = w.glo[1] + (static_cast<float>(j0) + 0.5f * (nj - 1)) * w.gh;
        const float cz = w.glo[2] + (static_cast<float>(k0) + 0.5f * (nk - 1)) * w.gh;
        const float rt = 0.5f * w.gh *
                         sqrtf(static_cast<float>((ni - 1) * (ni - 1) + (nj - 1) * (nj - 1) +
                                                  (nk - 1) * (nk - 1))) *
                         (1.0f + 0x1p-10f);
        // the conservative query's distance is at least the exact one, so
        // its radius covers the candidates as well
        const WideResult qc = wide_nearest<3, HC>(w, cx, cy, cz, kShrink * kShrink, 0.0f);
        const float radius = (sqrtf(qc.best) + 2.0f * rt) * (1.0f + 0x1p-16f) + slack;
        const int cnt = wide_range<3>(w, cx, cy, cz, radius * radius, s_cand[wib], kTileCap);
        __syncwarp();
        if (cnt <= kTileCap) {
            // 32 records at a time: each lane fetches one (all in flight
            // together), then every lane measures its node against all 32
            float best = INFINITY;
            for (int c0 = 0; c0 < cnt; c0 += 32) {
                const int m = min(32, cnt - c0);
                if (lane < m) {
                    const int sl = s_cand[wib][c0 + lane];
#pragma unroll
                    for (int f = 0; f < 4; ++f) s_rec[wib][lane][f] = __ldg(w.aos + 4 * sl + f);
                }
                __syncwarp();
#pragma unroll 4
                for (int q = 0; q < m; ++q) best = fminf(best, eberly32(x, y, z, s_rec[wib][q]));
                __syncwarp();
            }
            if (query) {
                const float d = (sqrtf(best) * kShrink - margin) * (1.0f - 0x1p-20f);
                out[t] = d > 0.0f ? d : 0.0f;
            }
        } else {
            unsigned pending = want;
            while (pending) {
                const int src = __ffs(pending) - 1;
                pending &= pending - 1u;
                const float qx = __shfl_sync(kFull, x, src);
                const float qy = __shfl_sync(kFull, y, src);
                const float qz = __shfl_sync(kFull, z, src);
                const WideResult q = wide_nearest<3, HC>(w, qx, qy, qz, kShrink * kShrink, 0.0f);
                if (lane == src) {
                    const float d = (sqrtf(q.best) * kShrink - margin) * (1.0f - 0x1p-20f);
                    out[t] = d > 0.0f ? d : 0.0f;
                }
            }
        }
        __syncwarp();
    }
}

// Outside-node classification of the lattice, by the parity of boundary
// crossings along each lattice row (a line along x through the node centres
// (y_j, z_k)).  kRowCrossings crossings are kept per row; a row with more, an
// odd count, or one passing within `tol` of a primitive's edge or vertex is
// left unclassified (none of its nodes is skipped).  Storing 0 at a node is
// always a valid lower bound, so a wrong verdict costs walk speed, never
// correctness.
constexpr int kRowCrossings = 16;
constexpr unsigned kRowUnknown = 0x80000000u;

__device__ __forceinline__ void add_crossing(unsigned *count, float *cross, long long row,
                                             float x) {
    const unsigned c = atomicAdd(count + row, 1u) & ~kRowUnknown;
    if (c < static_cast<unsigned>(kRowCrossings)) cross[row * kRowCrossings + c] = x;
}

// 2D: one thread per segment, rows y_j = glo[1] + j h.  A segment crosses a
// row when min(y) <= y_j < max(y): adjacent segments share their endpoint's
// exact coordinates, so a row through a vertex counts the crossing once (or
// twice at a turning point) and the parity stays right.
__global__ void row_crossings2_kernel(SceneView s, WideView w, unsigned *count, float *cross) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n_prims) return;
    const double2 a = s.seg64[2 * p], b = s.seg64[2 * p + 1];
    const double ylo = fmin(a.y, b.y), yhi = fmax(a.y, b.y);
    if (!(ylo < yhi)) return;  // horizontal: never crosses under the half-open rule
    const double h = w.gh, y0 = w.glo[1];
    const int j0 = max(0, static_cast<int>(floor((ylo - y0) / h)) - 1);
    const int j1 = min(w.gn[1] - 1, static_cast<int>(ceil((yhi - y0) / h)) + 1);
    for (int j = j0; j <= j1; ++j) {
        const double y = static_cast<double>(w.glo[1] + static_cast<float>(j) * w.gh);
        if (!(ylo <= y && y < yhi)) continue;
        const double x = a.x + (y - a.y) * (b.x - a.x) / (b.y - a.y);
        add_crossing(count, cross, j, static_cast<float>(x));
    }
}

// 3D: one thread per triangle, rows through (y_j, z_k); a row crosses the
// triangle where its (y, z) projection contains (y_j, z_k).
__global__ void row_crossings3_kernel(SceneView s, WideView w, double tol, unsigned *count,
                                      float *cross) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n_prims) return;
    const double2 *r = s.tri64 + 7 * p;
    const double2 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4];
    // v0 = (r0.x, r0.y, r1.x), e1 = (r1.y, r2.x, r2.y), e2 = (r3.x, r3.y, r4.x)
    const double v0[3] = {r0.x, r0.y, r1.x};
    const double e1[3] = {r1.y, r2.x, r2.y}, e2[3] = {r3.x, r3.y, r4.x};
    const double P[3][2] = {{v0[1], v0[2]}, {v0[1] + e1[1], v0[2] + e1[2]},
                            {v0[1] + e2[1], v0[2] + e2[2]}};
    const double nx = e1[1] * e2[2] - e1[2] * e2[1];
    const double ny = e1[2] * e2[0] - e1[0] * e2[2];
    const double nz = e1[0] * e2[1] - e1[1] * e2[0];
    const double ylo = fmin(fmin(P[0][0], P[1][0]), P[2][0]);
    const double yhi = fmax(fmax(P[0][0], P[1][0]), P[2][0]);
    const double zlo = fmin(fmin(P[0][1], P[1][1]), P[2][1]);
    const double zhi = fmax(fmax(P[0][1], P[1][1]), P[2][1]);
    const double h = w.gh;
    const int j0 = max(0, static_cast<int>(floor((ylo - tol - w.glo[1]) / h)));
    const int j1 = min(w.gn[1] - 1, static_cast<int>(ceil((yhi + tol - w.glo[1]) / h)));
    const int k0 = max(0, static_cast<int>(floor((zlo - tol - w.glo[2]) / h)));
    const int k1 = min(w.gn[2] - 1, static_cast<int>(ceil((zhi + tol - w.glo[2]) / h)));
    double len[3];
    for (int q = 0; q < 3; ++q) {
        const double dy = P[(q + 1) % 3][0] - P[q][0], dz = P[(q + 1) % 3][1] - P[q][1];
        len[q] = sqrt(dy * dy + dz * dz);
    }
    for (int j = j0; j <= j1; ++j) {
        const double y = static_cast<double>(w.glo[1] + static_cast<float>(j) * w.gh);
        for (int k = k0; k <= k1; ++k) {
            const double z = static_cast<double>(w.glo[2] + static_cast<float>(k) * w.gh);
            const long long row = static_cast<long long>(j) * w.gn[2] + k;
            int pos = 0, neg = 0;
            bool near = false;
            for (int q = 0; q < 3; ++q) {
                const double *A = P[q], *B = P[(q + 1) % 3];
                const double c = (B[0] - A[0]) * (z - A[1]) - (B[1] - A[1]) * (y - A[0]);
                if (fabs(c) <= tol * len[q]) near = true;
                else if (c > 0.0) ++pos;
                else ++neg;
            }
            if (near) {
                // on or next to an edge line of the projection: undecided,
                // unless the point is plainly outside the projected triangle
                if (pos < 1 || neg < 1) atomicOr(count + row, kRowUnknown);
                continue;
            }
            if (pos != 3 && neg != 3) continue;
            const double x = v0[0] - (ny * (y - v0[1]) + nz * (z - v0[2])) / nx;
            add_crossing(count, cross, row, static_cast<float>(x));
        }
    }
}

// One thread per row: sort its crossings and mark the nodes with an even
// number of crossings below them (and none within tol) as outside.
__global__ void row_outside_kernel(WideView w, double tol, const unsigned *count,
                                   const float *cross, uint8_t *outside) {
    const long long rows = static_cast<long long>(w.gn[1]) * w.gn[2];
    const long long row = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (row >= rows) return;
    const unsigned c = count[row];
    const int m = static_cast<int>(c & ~kRowUnknown);
    const bool known = !(c & kRowUnknown) && m <= kRowCrossings && (m % 2) == 0;
    float xs[kRowCrossings];
    for (int q = 0; q < kRowCrossings; ++q) xs[q] = q < m && known ? cross[row * kRowCrossings + q] : 0.0f;
    for (int q = 1; q < m && known; ++q) {  // insertion sort
        const float v = xs[q];
        int u = q - 1;
        while (u >= 0 && xs[u] > v) {
            xs[u + 1] = xs[u];
            --u;
        }
        xs[u + 1] = v;
    }
    int below = 0;
    for (int i = 0; i < w.gn[0]; ++i) {
        const float x = w.glo[0] + static_cast<float>(i) * w.gh;
        bool out = known;
        if (known) {
            while (below < m && xs[below] <= x) ++below;
            out = (below % 2) == 0;
            if (below > 0 && static_cast<double>(x) - xs[below - 1] <= tol) out = false;
            if (below < m && static_cast<double>(xs[below]) - x <= tol) out = false;
        }
        outside[static_cast<long long>(i) * rows + row] = out ? 1 : 0;
    }
}

template <int DIM>
__global__ void lattice_bounds_kernel(WideView w, const double *pts, long long n, double *out) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (w.gd == nullptr) {
        out[i] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const float px = static_cast<float>(pts[DIM * i]);
    const float py = static_cast<float>(pts[DIM * i + 1]);
    const float pz = DIM == 3 ? static_cast<float>(pts[DIM * i + 2]) : 0.0f;
    out[i] = static_cast<double>(lattice_bound<DIM>(w, px, py, pz));
}
}  // namespace

namespace {
// Lattice nodes in the near-boundary band: value in [0, t] (-0.0 marks a
// skipped node).
__global__ void near_band_kernel(const float *__restrict__ gd, long long n, float t,
                                 unsigned *count) {
    unsigned c = 0;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += stride) {
        const float d = gd[i];
        c += (!signbit(d) && d <= t) ? 1u : 0u;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(kFull, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// Bucket b's reach for list_prefix: a list entry at distance D from a node
// at distance d counts in bucket b when D <= d + 2 rho_b + slack,
// rho_b = (b + 1) rmax / (B + 1).
__device__ __forceinline__ float bucket_reach(float dn, int b, float rmax, float slack) {
    const float rho = rmax * static_cast<float>(b + 1) / static_cast<float>(kListBuckets + 1);
    return (dn + 2.0f * rho) * (1.0f + 0x1p-16f) + slack;
}

// One band node's list, built by the whole warp (all lanes call it
// converged with the same node at (x, y, z)): the node's exact FP32
// distance d, then every primitive within d + extra, kept as its list when
// there are at most K.  Lists are packed end to end, so the pool holds about
// the average length per node rather than K: what the walks touch stays
// small enough for L2.  A 3D list's slots are written in increasing
// (distance from the node, slot) order, and the entry's .y holds the bucket
// counts of list_prefix (bucket_reach); `slack` covers the FP32 rounding of
// D, d and the query's distances.  2D lists keep ascending slot order and no
// buckets (one lane scans a few segments; the cut did not pay there).
template <int DIM, int HC>
__device__ void warp_node_list(const WideView &w, int node, float x, float y, float z,
                               float extra, float rmax, float slack, int2 *gl, int *pool,
                               int pool_slots, unsigned *counter, int *s_list) {
    const int lane = threadIdx.x & 31;
    const int K = w.gk;
    const WideResult q = wide_nearest<DIM, HC>(w, x, y, z, 1.0f, 0.0f);
    const float dn = sqrtf(q.best);
    const float radius = dn * (1.0f + 0x1p-16f) + extra;
    const int cnt = wide_range<DIM>(w, x, y, z, radius * radius, s_list, K);
    __syncwarp();
    // the list goes to the next cnt slots of the pool (lists end to end)
    int idx = -1;
    if (cnt >= 1 && cnt <= K) {
        unsigned at = 0;
        if (lane == 0) at = atomicAdd(counter, static_cast<unsigned>(cnt));
        at = __shfl_sync(kFull, at, 0);
        // never short: the pool holds K slots per band node (at most 2^26)
        if (static_cast<long long>(at) + cnt <= pool_slots) idx = static_cast<int>(at);
    }
    if (idx < 0) {
        if (lane == 0) gl[node] = make_int2(-1, 0);
        __syncwarp();
        return;
    }
    if constexpr (DIM == 2) {
        // 2D: ascending slot order, no buckets
        if (lane < cnt) pool[static_cast<long long>(idx) + lane] = s_list[lane];
        if (lane == 0) gl[node] = make_int2((idx << 5) | (cnt - 1), 0);
        __syncwarp();
        return;
    }
    // 3D: each entry's distance from the node, its rank in (distance, slot)
    // order, and the bucket counts
    const bool mine = lane < cnt;
    const int s = mine ? s_list[lane] : 0;
    const float dd = mine ? sqrtf(slot_dist<DIM>(w, s, x, y, z)) : INFINITY;
    const unsigned long long key =
        mine ? (static_cast<unsigned long long>(__float_as_uint(dd)) << 32) |
                   static_cast<unsigned>(s)
             : ~0ull;
    int rank = 0;
    for (int o = 0; o < cnt; ++o) rank += __shfl_sync(kFull, key, o) < key ? 1 : 0;
    if (mine) pool[static_cast<long long>(idx) + rank] = s;
    unsigned buckets = 0;
#pragma unroll
    for (int b = 0; b < kListBuckets; ++b) {
        const float lim = bucket_reach(dn, b, rmax, slack);
        const unsigned c = __popc(__ballot_sync(kFull, mine && dd <= lim));
        buckets |= min(c, 63u) << (6 * b);
    }
    // packed entry: (offset << 5) | (length - 1), offset < 2^26
    if (lane == 0) gl[node] = make_int2((idx << 5) | (cnt - 1), static_cast<int>(buckets));
    __syncwarp();
}

// Band nodes 32 at a time per warp: each lane tests one node for the band
// (0 <= value <= t), then the warp builds the band nodes' lists one after
// another (warp_node_list).
template <int DIM, int HC>
__global__ void __launch_bounds__(256) near_lists_kernel(WideView w, float t, float extra,
                                                         float rmax, float slack, int2 *gl,
                                                         int *pool, int pool_slots,
                                                         unsigned *counter) {
    __shared__ int s_list[8][32];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int warp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int warps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
    const int n = w.gn[0] * w.gn[1] * w.gn[2];  // at most 2^24 nodes
    for (int base = warp * 32; base < n; base += warps * 32) {
        bool in_band = false;
        if (base + lane < n) {
            const float d = w.gd[base + lane];
            in_band = !(signbit(d) || d > t);
            if (!in_band) gl[base + lane] = make_int2(-1, 0);
        }
        unsigned pending = __ballot_sync(kFull, in_band);
        while (pending) {
            const int node = base + __ffs(pending) - 1;
            pending &= pending - 1u;
            const int k = node % w.gn[2];
            const int r = node / w.gn[2];
            const int j = r % w.gn[1];
            const int i = r / w.gn[1];
            const float x = w.glo[0] + static_cast<float>(i) * w.gh;
            const float y = w.glo[1] + static_cast<float>(j) * w.gh;
            const float z = DIM == 3 ? w.glo[2] + static_cast<float>(k) * w.gh : 0.0f;
            warp_node_list<DIM, HC>(w, node, x, y, z, extra, rmax, slack, gl, pool, pool_slots,
                                    counter, s_list[wib]);
        }
    }
}

// 3D lists by warp tiles of 2 x 4 x 4 nodes, one node per lane, as the 3D
// lattice is built: a band node's list holds the primitives within
// d(node) + extra of it, so every primitive within d(c) + 2 r_tile + extra of
// the tile centre c (plus a rounding slack) is a candidate for every node of
// the tile.  Each band lane takes its exact FP32 distance as the minimum over
// the candidates, keeps those within its list radius (the same test as the
// per-node range query, in the same ascending slot order), sorts them by
// (distance, slot) and writes them with their bucket counts; the lanes'
// lists take consecutive pool ranges from one atomic per tile.  A tile with
// more than kTileCap candidates builds its band nodes' lists one by one
// (warp_node_list).  Records come from the contiguous copy (w.aos), staged
// 32 at a time in shared memory.
template <int HC>
__global__ void __launch_bounds__(256) near_lists_tile3_kernel(WideView w, float t, float extra,
                                                               float rmax, float slack,
                                                               int2 *gl, int *pool,
                                                               int pool_slots,
                                                               unsigned *counter) {
    __shared__ int s_cand[8][kTileCap];
    __shared__ float4 s_rec[8][32][4];
    __shared__ int s_list[8][32];
    constexpr float kShrink = 1.0f - 0x1p-10f;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int warp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int warps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
    const int K = w.gk;
    const int tj = (w.gn[1] + 3) / 4, tk = (w.gn[2] + 3) / 4;
    const int tiles = ((w.gn[0] + 1) / 2) * tj * tk;
    for (int tile = warp; tile < tiles; tile += warps) {
        const int i0 = 2 * (tile / (tj * tk)), j0 = 4 * ((tile / tk) % tj), k0 = 4 * (tile % tk);
        const int i = i0 + (lane >> 4), j = j0 + ((lane >> 2) & 3), k = k0 + (lane & 3);
        const bool valid = i < w.gn[0] && j < w.gn[1] && k < w.gn[2];
        const int node = valid ? (i * w.gn[1] + j) * w.gn[2] + k : 0;
        bool in_band = false;
        if (valid) {
            const float d = w.gd[node];
            in_band = !(signbit(d) || d > t);
            if (!in_band) gl[node] = make_int2(-1, 0);
        }
        const unsigned want = __ballot_sync(kFull, in_band);
        if (!want) continue;
        const float x = w.glo[0] + static_cast<float>(i) * w.gh;
        const float y = w.glo[1] + static_cast<float>(j) * w.gh;
        const float z = w.glo[2] + static_cast<float>(k) * w.gh;
        const int ni = min(2, w.gn[0] - i0), nj = min(4, w.gn[1] - j0), nk = min(4, w.gn[2] - k0);
        const float cx = w.glo[0] + (static_cast<float>(i0) + 0.5f * (ni - 1)) * w.gh;
        const float cy = w.glo[1] + (static_cast<float>(j0) + 0.5f * (nj - 1)) * w.gh;
        const float cz = w.glo[2] + (static_cast<float>(k0) + 0.5f * (nk - 1)) * w.gh;
        const float rt = 0.5f * w.gh *
                         sqrtf(static_cast<float>((ni - 1) * (ni - 1) + (nj - 1) * (nj - 1) +
                                                  (nk - 1) * (nk - 1))) *
                         (1.0f + 0x1p-10f);
        // the conservative query's distance is at least the exact one
        const WideResult qc = wide_nearest<3, HC>(w, cx, cy, cz, kShrink * kShrink, 0.0f);
        const float reach = (sqrtf(qc.best) + 2.0f * rt + extra) * (1.0f + 0x1p-16f) + slack;
        const int cnt = wide_range<3>(w, cx, cy, cz, reach * reach, s_cand[wib], kTileCap);
        __syncwarp();
        if (cnt > kTileCap) {
            unsigned pending = want;
            while (pending) {
                const int src = __ffs(pending) - 1;
                pending &= pending - 1u;
                warp_node_list<3, HC>(w, __shfl_sync(kFull, node, src),
                                      __shfl_sync(kFull, x, src), __shfl_sync(kFull, y, src),
                                      __shfl_sync(kFull, z, src), extra, rmax, slack, gl, pool,
                                      pool_slots, counter, s_list[wib]);
            }
            continue;
        }
        // pass 1: each node's exact FP32 distance, the minimum over the
        // candidates (its nearest primitive is one of them)
        float best = INFINITY;
        for (int c0 = 0; c0 < cnt; c0 += 32) {
            const int m = min(32, cnt - c0);
            if (lane < m) {
                const int sl = s_cand[wib][c0 + lane];
#pragma unroll
                for (int f = 0; f < 4; ++f) s_rec[wib][lane][f] = __ldg(w.aos + 4 * sl + f);
            }
            __syncwarp();
#pragma unroll 4
            for (int q = 0; q < m; ++q) best = fminf(best, eberly32(x, y, z, s_rec[wib][q]));
            __syncwarp();
        }
        const float dn = sqrtf(best);
        const float radius = dn * (1.0f + 0x1p-16f) + extra;
        const float r2 = radius * radius;
        // pass 2: the candidates within the node's list radius, ascending slots
        int lst[32];
        float ld[32];
        int len = 0;
        for (int c0 = 0; c0 < cnt; c0 += 32) {
            const int m = min(32, cnt - c0);
            if (lane < m) {
                const int sl = s_cand[wib][c0 + lane];
#pragma unroll
                for (int f = 0; f < 4; ++f) s_rec[wib][lane][f] = __ldg(w.aos + 4 * sl + f);
            }
            __syncwarp();
            for (int q = 0; q < m; ++q) {
                const float d2 = eberly32(x, y, z, s_rec[wib][q]);
                if (in_band && d2 <= r2) {
                    if (len < K) {
                        lst[len] = s_cand[wib][c0 + q];
                        ld[len] = sqrtf(d2);
                    }
                    ++len;
                }
            }
            __syncwarp();
        }
        // the lanes' lists take consecutive pool ranges
        const int take = in_band && len >= 1 && len <= K ? len : 0;
        int incl = take;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(kFull, incl, 31);
        unsigned first = 0;
        if (lane == 0 && total > 0) first = atomicAdd(counter, static_cast<unsigned>(total));
        first = __shfl_sync(kFull, first, 0);
        const long long at = static_cast<long long>(first) + (incl - take);
        // never short: the pool holds K slots per band node (at most 2^26)
        const bool fits = take > 0 && at + take <= pool_slots;
        if (in_band && !fits) gl[node] = make_int2(-1, 0);
        if (fits) {
            // (distance, slot) order, as warp_node_list's ranks give
            for (int a = 1; a < take; ++a) {
                const int sa = lst[a];
                const float da = ld[a];
                int b = a - 1;
                while (b >= 0 && (ld[b] > da || (ld[b] == da && lst[b] > sa))) {
                    lst[b + 1] = lst[b];
                    ld[b + 1] = ld[b];
                    --b;
                }
                lst[b + 1] = sa;
                ld[b + 1] = da;
            }
            for (int a = 0; a < take; ++a) pool[at + a] = lst[a];
            unsigned buckets = 0;
            for (int b = 0; b < kListBuckets; ++b) {
                const float lim = bucket_reach(dn, b, rmax, slack);
                unsigned c = 0;
                for (int a = 0; a < take; ++a) c += ld[a] <= lim ? 1u : 0u;
                buckets |= min(c, 63u) << (6 * b);
            }
            gl[node] = make_int2((static_cast<int>(at) << 5) | (take - 1),
                                 static_cast<int>(buckets));
        }
    }
}
}  // namespace

namespace {
// Contiguous copy of the wide tree's primitive records: slot s at
// aos[s * (2D: 8, 3D: 16) ...], the fields in their block order.
__global__ void prim_aos_kernel(WideView w, float *aos) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= w.npad) return;
    const int nf = w.dim == 2 ? 5 : 16, stride = w.dim == 2 ? 8 : 16;
    const float *b = w.prim + static_cast<size_t>(s / 32) * nf * 32 + (s % 32);
    for (int f = 0; f < stride; ++f) aos[static_cast<size_t>(s) * stride + f] = f < nf ? b[f * 32] : 0.0f;
}
}  // namespace

size_t prim_aos_bytes(const WideView &w) {
    return static_cast<size_t>(w.npad) * (w.dim == 2 ? 8 : 16) * sizeof(float);
}

cudaError_t launch_prim_aos(const WideView &w, float *aos, cudaStream_t stream) {
    if (w.npad <= 0) return cudaSuccess;
    prim_aos_kernel<<<static_cast<unsigned>((w.npad + 255) / 256), 256, 0, stream>>>(w, aos);
    return cudaGetLastError();
}

cudaError_t launch_near_band(const WideView &w, float t, unsigned *count, cudaStream_t stream) {
    const long long n = static_cast<long long>(w.gn[0]) * w.gn[1] * w.gn[2];
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    const long long blocks = std::min<long long>((n + 255) / 256, 148 * 16);
    near_band_kernel<<<static_cast<unsigned>(std::max<long long>(blocks, 1)), 256, 0, stream>>>(
        w.gd, n, t, count);
    return cudaGetLastError();
}

cudaError_t launch_near_lists(const WideView &w, float t, float extra, float rmax, float slack,
                              int2 *gl, int *pool, int pool_slots, unsigned *counter, int sms,
                              cudaStream_t stream) {
    const long long n = static_cast<long long>(w.gn[0]) * w.gn[1] * w.gn[2];
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    const long long blocks = std::min<long long>((n + 255) / 256, static_cast<long long>(sms) * 8);
    const long long tiles = static_cast<long long>((w.gn[0] + 1) / 2) * ((w.gn[1] + 3) / 4) *
                            ((w.gn[2] + 3) / 4);
    const long long tblocks = std::min<long long>((tiles + 7) / 8, static_cast<long long>(sms) * 8);
    return with_height_class(height_class(w.H), [&](auto h) -> cudaError_t {
        constexpr int HC = decltype(h)::value;
        if (w.dim == 2) {
            near_lists_kernel<2, HC><<<static_cast<unsigned>(blocks), 256, 0, stream>>>(
                w, t, extra, rmax, slack, gl, pool, pool_slots, counter);
        } else if (w.aos != nullptr) {
            near_lists_tile3_kernel<HC><<<static_cast<unsigned>(tblocks), 256, 0, stream>>>(
                w, t, extra, rmax, slack, gl, pool, pool_slots, counter);
        } else {
            near_lists_kernel<3, HC><<<static_cast<unsigned>(blocks), 256, 0, stream>>>(
                w, t, extra, rmax, slack, gl, pool, pool_slots, counter);
        }
        return cudaGetLastError();
    });
}

size_t lattice_skip_bytes(const WideView &w) {
    const size_t nodes = static_cast<size_t>(w.gn[0]) * w.gn[1] * w.gn[2];
    const size_t rows = static_cast<size_t>(w.gn[1]) * w.gn[2];
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    return up(nodes) + up(rows * sizeof(unsigned)) + up(rows * kRowCrossings * sizeof(float));
}

cudaError_t launch_lattice32(const SceneView &s, const WideView &w, float margin, float *out,
                             int sms, void *scratch, double tol, cudaStream_t stream) {
    const long long n = static_cast<long long>(w.gn[0]) * w.gn[1] * w.gn[2];
    if (n <= 0) return cudaSuccess;
    uint8_t *outside = nullptr;
    if (scratch != nullptr) {
        auto up = [](size_t b) { return (b + 255) / 256 * 256; };
        const size_t rows = static_cast<size_t>(w.gn[1]) * w.gn[2];
        outside = static_cast<uint8_t *>(scratch);
        auto *count = reinterpret_cast<unsigned *>(outside + up(static_cast<size_t>(n)));
        auto *cross = reinterpret_cast<float *>(reinterpret_cast<char *>(count) +
                                                up(rows * sizeof(unsigned)));
        cudaError_t e = cudaMemsetAsync(count, 0, rows * sizeof(unsigned), stream);
        if (e != cudaSuccess) return e;
        const unsigned pb = static_cast<unsigned>((s.n_prims + 127) / 128);
        if (w.dim == 2) {
            row_crossings2_kernel<<<pb, 128, 0, stream>>>(s, w, count, cross);
        } else {
            row_crossings3_kernel<<<pb, 128, 0, stream>>>(s, w, tol, count, cross);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        row_outside_kernel<<<static_cast<unsigned>((rows + 127) / 128), 128, 0, stream>>>(
            w, tol, count, cross, outside);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    const long long blocks = std::min<long long>((n + 255) / 256, static_cast<long long>(sms) * 8);
    // 3D warp tiles of 32 nodes; their candidate radius carries 12 margins
    // of FP32 rounding (the tile centre, the nodes and the distances)
    const long long tiles = static_cast<long long>((w.gn[0] + 1) / 2) * ((w.gn[1] + 3) / 4) *
                            ((w.gn[2] + 3) / 4);
    const long long tblocks = std::min<long long>((tiles + 7) / 8, static_cast<long long>(sms) * 8);
    // compiled per traversal class, like the walk kernels
    return with_height_class(height_class(w.H), [&](auto h) -> cudaError_t {
        constexpr int HC = decltype(h)::value;
        if (w.dim == 2) {
            lattice32_kernel<2, HC>
                <<<static_cast<unsigned>(blocks), 256, 0, stream>>>(w, margin, outside, out);
        } else if (w.aos != nullptr) {
            lattice_tile3_kernel<HC><<<static_cast<unsigned>(tblocks), 256, 0, stream>>>(
                w, margin, 12.0f * margin, outside, out);
        } else {
            lattice32_kernel<3, HC>
                <<<static_cast<unsigned>(blocks), 256, 0, stream>>>(w, margin, outside, out);
        }
        return cudaGetLastError();
    });
}

cudaError_t launch_lattice_bounds(const WideView &w, const double *pts, long long n, double *out,
                                  cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>((n + 127) / 128);
    if (w.dim == 2) {
        lattice_bounds_kernel<2><<<blocks, 128, 0, stream>>>(w, pts, n, out);
    } else {
        lattice_bounds_kernel<3><<<blocks, 128, 0, stream>>>(w, pts, n, out);
    }
    return cudaGetLastError();
}

cudaError_t launch_special(int precision, const double *x, long long n, double *log_i0,
                           double *log_k0, cudaStream_t stream) {
    if (precision == 64) return launch_special64(x, n, log_i0, log_k0, stream);
    if (n <= 0) return cudaSuccess;
    const long long blocks = (n + 127) / 128;
    special32_kernel<<<static_cast<unsigned>(blocks), 128, 0, stream>>>(x, n, log_i0, log_k0);
    return cudaGetLastError();
}

FastPlan plan_fast(const SceneView &s, const WideView &w, long long n_points, int n_walks,
                   int precision, int device_sms, size_t smem_optin) {
    FastPlan p{};
    p.threads = 256;
    // Walks per task: the longest of 2048 / 1024 / 512 / 256 that still
    // gives about six tasks per resident warp (32 per SM).  A task's last
    // walks leave lanes idle, so longer tasks waste less, but a warp's last
    // task must not run long after the others have finished.  Measured on a
    // B200: 51k points x 4096 walks runs best at 2048, 4096 points x 2048
    // walks at 256 (23.8 -> 22.5 ms), 137k points x 1024 walks at 1024.
    const long long warps = 32LL * (device_sms > 0 ? device_sms : 148);
    int chunk = 256;
    for (int c = 2048; c > 256; c /= 2) {
        if (n_points * ((n_walks + c - 1) / c) >= 6 * warps) {
            chunk = c;
            break;
        }
    }
    p.chunk = n_walks < chunk ? n_walks : chunk;
    if (p.chunk < 1) p.chunk = 1;
    p.chunks = (n_walks + p.chunk - 1) / p.chunk;
    p.n_tasks = n_points * p.chunks;
    // stage the wide boxes, and the primitives too when they fit, in shared memory
    const size_t box_floats = static_cast<size_t>(w.box_total);
    const size_t prim_floats = static_cast<size_t>(w.dim == 2 ? 5 : 16) * w.npad;
    const size_t cap = std::min<size_t>(96 * 1024, smem_optin);
    p.stage_scene = precision == 32 && box_floats * 4 <= cap;
    p.stage_prims = p.stage_scene && (box_floats + prim_floats) * 4 <= cap;
    p.smem_bytes = p.stage_scene
                       ? static_cast<int>((box_floats + (p.stage_prims ? prim_floats : 0)) * 4)
                       : 0;
    p.blocks = 0;  // sized from the occupancy of the chosen kernel at launch
    return p;
}

FastArgs make_fast_args(const SceneView &s, const WideView &w, const PointSet &ps, uint64_t seed,
                        int n_walks, double epsilon, int max_steps, double shell_delta,
                        const FastPlan &plan, const uint8_t *location, const StartRecord *start,
                        TaskPartial *partials, unsigned long long *queue, DeviceCounters *ctr) {
    FastArgs a{};
    a.s = s;
    a.ps = ps;
    a.seed = seed;
    a.n_walks = n_walks;
    a.eps = epsilon;
    a.max_steps = max_steps;
    a.shell_delta = shell_delta;
    a.chunk = plan.chunk;
    a.chunks = plan.chunks;
    a.n_tasks = plan.n_tasks;
    a.w = w;
    a.stage = 0;
    a.stage_box = 0;
    a.stage_prim = 0;
    // FP32 queries are conservative to a relative tau = 2^-10 outside the
    // epsilon shell and exact inside it (see wide_nearest)
    const double tau = 1.0 / 1024.0;
    const double shell = epsilon + shell_delta;
    a.keep = static_cast<float>((1.0 - tau) * (1.0 - tau));
    a.shrink = static_cast<float>(1.0 - tau);
    a.shell2 = static_cast<float>(shell * shell);
    a.exact2 = static_cast<float>(shell * shell / ((1.0 - tau) * (1.0 - tau)));
    a.list_t = w.gl != nullptr ? near_list_threshold(w, epsilon, shell_delta) : -1.0f;
    a.location = location;
    a.start = start;
    a.partials = partials;
    a.queue = queue;
    a.ctr = ctr;
    return a;
}

cudaError_t launch_walk_fast(const SceneView &s, const WideView &w, const PointSet &ps,
                             uint64_t seed, EqDesc eq,
                             int n_walks, double epsilon, int max_steps, double shell_delta,
                             int precision, const FastPlan &plan, const uint8_t *location,
                             const StartRecord *start, TaskPartial *partials,
                             unsigned long long *queue, Fields out, DeviceCounters *counters,
                             cudaStream_t stream, cudaEvent_t after_walk) {
    if (ps.n <= 0) return cudaSuccess;
    FastArgs a = make_fast_args(s, w, ps, seed, n_walks, epsilon, max_steps, shell_delta, plan,
                                location, start, partials, queue, counters);
    a.stage = plan.stage_scene ? 1 : 0;
    a.stage_box = plan.stage_scene ? w.box_total : 0;
    a.stage_prim = plan.stage_prims ? (w.dim == 2 ? 5 : 16) * w.npad : 0;
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    e = s.dim == 2 ? launch_fast_dim<2>(a, eq, precision, plan, stream)
                   : launch_fast_dim<3>(a, eq, precision, plan, stream);
    if (e != cudaSuccess) return e;
    if (after_walk) {
        e = cudaEventRecord(after_walk, stream);
        if (e != cudaSuccess) return e;
    }
    long long b = (ps.n + 255) / 256;
    if (b < 1) b = 1;
    merge_kernel<<<static_cast<int>(b), 256, 0, stream>>>(ps.n, plan.chunks, n_walks, location,
                                                        partials, out, counters);
    return cudaGetLastError();
}

cudaError_t batch_walk_blocks(int dim, int kind, int precision, int hc, int *blocks) {
    return dim == 2 ? batch_dispatch<2>(kind, precision, hc, nullptr, 0, 0, nullptr, 0, nullptr,
                                        blocks)
                    : batch_dispatch<3>(kind, precision, hc, nullptr, 0, 0, nullptr, 0, nullptr,
                                        blocks);
}

cudaError_t launch_walk_batch(int dim, int kind, int precision, int hc, const BatchItem *items,
                              int n_items, long long n_tasks, unsigned long long *queue,
                              int blocks, cudaStream_t stream) {
    if (n_items <= 0 || n_tasks <= 0) return cudaSuccess;
    return dim == 2 ? batch_dispatch<2>(kind, precision, hc, items, n_items, n_tasks, queue,
                                        blocks, stream, nullptr)
                    : batch_dispatch<3>(kind, precision, hc, items, n_items, n_tasks, queue,
                                        blocks, stream, nullptr);
}

cudaError_t launch_merge_batch(const BatchItem *items, int n_items, long long n_points,
                               cudaStream_t stream) {
    if (n_items <= 0 || n_points <= 0) return cudaSuccess;
    long long b = (n_points + 255) / 256;
    if (b > 148 * 64) b = 148 * 64;
    merge_batch_kernel<<<static_cast<int>(b), 256, 0, stream>>>(items, n_items, n_points);
    return cudaGetLastError();
}

cudaError_t launch_closest32(const SceneView &s, const WideView &w, const double *pts,
                             long long n, double *dist, double *nearest, int *bid,
                             cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    long long b = (n + 127) / 128;
    if (s.dim == 2) {
        closest32_kernel<2><<<static_cast<int>(b), 128, 0, stream>>>(s, w, pts, n, dist, nearest,
                                                                     bid);
    } else {
        closest32_kernel<3><<<static_cast<int>(b), 128, 0, stream>>>(s, w, pts, n, dist, nearest,
                                                                     bid);
    }
    return cudaGetLastError();
}

}  // namespace wosb
