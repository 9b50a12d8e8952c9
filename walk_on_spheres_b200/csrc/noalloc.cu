// wos_solve_grid_device_noalloc: a grid sweep that allocates no device memory.
//
// Why it exists.  The regular entry points grow per-context device buffers
// with cudaMalloc on first use (classification records, walk-task partial
// statistics, the work-queue counter).  Some callers cannot allocate at the
// moment they solve: code that runs inside a memory budget enforced by a
// custom allocator or pool (cudaMalloc would bypass it or fail), code that
// must not take the device-wide synchronisation that cudaMalloc / cudaFree
// can cause, and hosts that pre-allocate everything at start-up and forbid
// allocation afterwards.  This entry point serves them: the caller passes the
// outputs, and every temporary lives in one fixed array of static device
// memory in this file.  The call itself still blocks the calling thread until
// the solve has finished on the context's stream (it reads the counters
// back), like wos_solve_grid_device.
//
// The scratch array.  kScratchBytes (8 MiB) of static device memory.  With
// lazy module loading (the CUDA 12 default) it is reserved on a device when
// this file's module is first loaded there, which wos_context_create forces
// by taking the array's address (noalloc_scratch_address below): so the
// reservation happens when a context is created, never inside this call, and
// it stays until the process exits.  A grid needs about 89 bytes per point
// (location, start record, one walk-statistics record) plus 1 KiB, so the
// limit is about 94 000 points; larger grids are rejected with
// WOS_ERR_INVALID before anything runs.  All calls share the array and it
// keeps the last call's contents: each call clears the counters and the work
// queue it relies on before launching, and calls whose work overlaps on the
// GPU (different streams or contexts on one device, or other host threads)
// race on the array, so they must be serialised by the caller.
//
// Device address.  In host code the array's name is only a host-side shadow;
// its device address comes from cudaGetSymbolAddress with the device
// current, taken once per context at creation and kept in the context.  A
// context is tied to its device's primary context, so a cudaDeviceReset by
// the host application invalidates it like every other device pointer the
// context holds.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/wos_b200.h"
#include "context_internal.h"
#include "kernels.h"

namespace {

constexpr size_t kScratchBytes = size_t(8) << 20;
constexpr size_t kAlign = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Bytes of scratch a grid of n points needs with `chunks` walk tasks per point.
size_t scratch_bytes(long long n, int chunks) {
    const size_t m = static_cast<size_t>(std::max<long long>(n, 1));
    return align_up(sizeof(wosb::DeviceCounters)) + align_up(sizeof(unsigned long long)) +
           align_up(m) + align_up(m * sizeof(wosb::StartRecord)) +
           align_up(m * static_cast<size_t>(chunks) * sizeof(wosb::TaskPartial));
}

int fail(wos_context *ctx, int code, const std::string &msg) {
    return wosb::fail(ctx, code, "wos_solve_grid_device_noalloc: " + msg);
}

}  // namespace

cudaError_t wosb::noalloc_scratch_address(void **ptr) {
    *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(ptr, g_noalloc_scratch);
    if (e == cudaSuccess && !*ptr) e = cudaErrorInvalidSymbol;
    return e;
}

extern "C" int wos_solve_grid_device_noalloc(wos_context *ctx, const wos_params *p,
                                             const wos_grid *g, double *mean, double *variance,
                                             double *standard_error, double *mean_steps,
                                             uint8_t *location, wos_counters *counters) {
    if (!ctx) return wosb::fail(nullptr, WOS_ERR_INVALID, "wos_solve_grid_device_noalloc: null context");
    // the same argument rules as wos_solve_grid_device
    std::string err = wosb::check_params(ctx, p);
    if (err.empty()) err = wosb::check_grid(ctx->scene.dim, g);
    if (!err.empty()) return fail(ctx, WOS_ERR_INVALID, err);
    if (!ctx->noalloc_scratch) return fail(ctx, WOS_ERR_INVALID, "the context has no scratch array");
    const wosb::PointSet ps = wosb::grid_points(ctx->scene.dim, *g);

    // walks per task: all of a point's walks in one task, unless a lane's
    // 32-bit step sum could overflow (then as many tasks as that needs)
    wosb::FastPlan plan{};
    const bool fast = p->method != WOS_METHOD_PLAIN_FP64;
    const int precision = p->method == WOS_METHOD_FAST_FP32 ? 32 : 64;
    if (fast) {
        plan = wosb::plan_fast(ctx->view, ctx->wide, ps.n, p->N_walks, precision, ctx->sms,
                               ctx->smem_optin);
        wosb::set_chunk(plan, p->N_walks, p->N_walks, p->max_steps, ps.n);
    }
    const size_t need = scratch_bytes(ps.n, fast ? plan.chunks : 1);
    if (need > kScratchBytes) {
        return fail(ctx, WOS_ERR_INVALID,
                    "a grid of " + std::to_string(ps.n) + " points needs " +
                        std::to_string(need) + " bytes of scratch, more than the static " +
                        std::to_string(kScratchBytes) +
                        "-byte array (about 94000 points); use wos_solve_grid_device");
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return fail(ctx, WOS_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));

    auto *base = static_cast<unsigned char *>(ctx->noalloc_scratch);
    const size_t m = static_cast<size_t>(std::max<long long>(ps.n, 1));
    auto *ctr = reinterpret_cast<wosb::DeviceCounters *>(base);
    size_t at = align_up(sizeof(wosb::DeviceCounters));
    auto *queue = reinterpret_cast<unsigned long long *>(base + at);
    at += align_up(sizeof(unsigned long long));
    auto *loc = base + at;
    at += align_up(m);
    auto *start = reinterpret_cast<wosb::StartRecord *>(base + at);
    at += align_up(m * sizeof(wosb::StartRecord));
    auto *partials = reinterpret_cast<wosb::TaskPartial *>(base + at);

    cudaStream_t s = ctx->stream;
    // the counters keep the previous call's values: clear them
    e = cudaMemsetAsync(ctr, 0, sizeof(wosb::DeviceCounters), s);
    if (e != cudaSuccess) return fail(ctx, WOS_ERR_CUDA, std::string("clear counters: ") + cudaGetErrorString(e));

    wosb::EqDesc eq{p->equation, p->source_mode, p->alpha};
    const double eps = wosb::effective_epsilon(*p);
    const double btol = 1e-10 * ctx->scene.scale;
    wosb::Fields out{mean, variance, standard_error, mean_steps, location};
    cudaEventRecord(ctx->events[0], s);
    // the same start radii as wos_solve_grid_device (FastStart for FAST_FP32)
    wosb::FastStart fs;
    if (p->method == WOS_METHOD_FAST_FP32) {
        fs.on = true;
        fs.w = ctx->wide;
        fs.exact_below = std::max(eps, btol);
        fs.margin = wosb::fp32_distance_margin(ctx->scene.bbox, ctx->scene.dim);
    }
    e = wosb::launch_classify(ctx->view, ps, p->seed, p->max_ray_attempts, btol, eq, out, loc,
                              start, ctr, s, fs);
    if (e != cudaSuccess) return fail(ctx, WOS_ERR_CUDA, std::string("classification kernel: ") + cudaGetErrorString(e));
    cudaEventRecord(ctx->events[1], s);
    if (!fast) {
        e = wosb::launch_walk_plain(ctx->view, ps, p->seed, eq, p->N_walks, eps, p->max_steps, loc,
                                    start, out, ctr, s);
        cudaEventRecord(ctx->events[2], s);
    } else {
        // the queue is cleared by launch_walk_fast before the walk kernel
        e = wosb::launch_walk_fast(ctx->view, ctx->wide, ps, p->seed, eq, p->N_walks, eps,
                                   p->max_steps, std::ldexp(ctx->scene.scale, -16), precision,
                                   plan, loc, start, partials, queue, out, ctr, s,
                                   ctx->events[2]);
    }
    if (e != cudaSuccess) return fail(ctx, WOS_ERR_CUDA, std::string("walk kernel: ") + cudaGetErrorString(e));
    cudaEventRecord(ctx->events[3], s);
    wosb::DeviceCounters hc{};
    e = cudaMemcpyAsync(&hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(ctx, WOS_ERR_CUDA, std::string("solve: ") + cudaGetErrorString(e));
    if (hc.error_flags) return fail(ctx, WOS_ERR_DEVICE, wosb::device_error(hc.error_flags));
    if (counters) {
        std::memset(counters, 0, sizeof(*counters));
        counters->max_steps_hits = static_cast<long long>(hc.max_steps_hits);
        counters->ambiguous_ray_retries = static_cast<long long>(hc.ambiguous_ray_retries);
        counters->indeterminate_points = static_cast<long long>(hc.indeterminate_points);
        counters->total_walks = static_cast<long long>(hc.total_walks);
        counters->total_steps = static_cast<long long>(hc.total_steps);
        counters->exact_queries = static_cast<long long>(hc.exact_queries);
        counters->inside_points = counters->total_walks / p->N_walks;
        counters->effective_epsilon = eps;
        cudaEventElapsedTime(&counters->classify_ms, ctx->events[0], ctx->events[1]);
        cudaEventElapsedTime(&counters->walk_ms, ctx->events[1], ctx->events[2]);
        cudaEventElapsedTime(&counters->total_ms, ctx->events[0], ctx->events[3]);
    }
    return WOS_OK;
}
