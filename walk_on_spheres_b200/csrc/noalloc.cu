// wos_solve_grid_device_noalloc: a grid sweep that allocates no device memory.
//
// Why it exists.  The regular entry points grow per-context device buffers
// with cudaMalloc on first use (classification records, walk-task partial
// statistics, the work-queue counter).  Some callers cannot allocate at the
// moment they solve: code that runs inside a memory budget enforced by a
// custom allocator or pool (cudaMalloc would bypass it or fail), code that
// must not synchronise the device (cudaMalloc / cudaFree can), and hosts that
// pre-allocate everything at start-up and forbid allocation afterwards.  This
// entry point serves them: the caller passes the outputs, and every temporary
// lives in one fixed array of static device memory in this file.
//
// The scratch array.  kScratchBytes (8 MiB) of device memory, reserved on
// every GPU that loads the library, for the life of the process.  A grid needs
// about 81 bytes per point (location, start record, one walk-statistics
// record) plus 1 KiB, so the limit is 103 000 points; larger grids are
// rejected with WOS_ERR_INVALID before anything runs.  All calls share the
// array and it keeps the last call's contents: each call clears the counters
// and the work queue it relies on before launching, and calls whose work
// overlaps on the GPU (different streams or contexts on one device, or other
// host threads) race on the array, so they must be serialised by the caller.
//
// Device address.  In host code the array's name is only a host-side shadow;
// its device address comes from cudaGetSymbolAddress, taken once per device
// (with that device current) by the first call on that device and cached.
// That first call therefore performs a runtime query and should come before
// any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/wos_b200.h"
#include "context_internal.h"
#include "kernels.h"

namespace {

constexpr size_t kScratchBytes = size_t(8) << 20;
constexpr size_t kAlign = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_lock;
void *g_scratch_ptr[kMaxDevices] = {};

size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Bytes of scratch a grid of n points needs (one walk task per point).
size_t scratch_bytes(long long n) {
    const size_t m = static_cast<size_t>(std::max<long long>(n, 1));
    return align_up(sizeof(wosb::DeviceCounters)) + align_up(sizeof(unsigned long long)) +
           align_up(m) + align_up(m * sizeof(wosb::StartRecord)) +
           align_up(m * sizeof(wosb::TaskPartial));
}

int fail(wos_context *ctx, int code, const std::string &msg) {
    ctx->error = msg;
    return code;
}

}  // namespace

extern "C" int wos_solve_grid_device_noalloc(wos_context *ctx, const wos_params *p,
                                             const wos_grid *g, double *mean, double *variance,
                                             double *standard_error, double *mean_steps,
                                             uint8_t *location, wos_counters *counters) {
    if (!ctx) return WOS_ERR_INVALID;
    if (!p || !g) return fail(ctx, WOS_ERR_INVALID, "wos_solve_grid_device_noalloc: null argument");
    if (!ctx->has_mesh) return fail(ctx, WOS_ERR_INVALID, "wos_solve_grid_device_noalloc: no mesh");
    if (p->equation < 0 || p->equation > 3 || (p->source_mode != 0 && p->source_mode != 1) ||
        p->N_walks < 1 || !(p->epsilon > 0.0) || !std::isfinite(p->epsilon) || p->max_steps < 1 ||
        p->max_ray_attempts < 3 || p->method < 0 || p->method > 2 ||
        (p->equation == WOS_EQ_SCREENED_POISSON && !(p->alpha > 0.0))) {
        return fail(ctx, WOS_ERR_INVALID, "wos_solve_grid_device_noalloc: invalid parameters");
    }
    const int dim = ctx->scene.dim;
    if (g->Nx < 1 || g->Ny < 1 || (dim == 3 && g->Nz < 1)) {
        return fail(ctx, WOS_ERR_INVALID, "wos_solve_grid_device_noalloc: grid sizes must be >= 1");
    }
    wosb::PointSet ps{};
    ps.dim = dim;
    ps.Nx = g->Nx;
    ps.Ny = g->Ny;
    ps.Nz = dim == 2 ? 1 : g->Nz;
    ps.lo[0] = g->xmin;
    ps.hi[0] = g->xmax;
    ps.lo[1] = g->ymin;
    ps.hi[1] = g->ymax;
    ps.lo[2] = dim == 3 ? g->zmin : 0.0;
    ps.hi[2] = dim == 3 ? g->zmax : 0.0;
    ps.n = static_cast<long long>(ps.Nx) * ps.Ny * ps.Nz;
    const size_t need = scratch_bytes(ps.n);
    if (need > kScratchBytes) {
        return fail(ctx, WOS_ERR_INVALID,
                    "wos_solve_grid_device_noalloc: a grid of " + std::to_string(ps.n) +
                        " points needs " + std::to_string(need) +
                        " bytes of scratch, more than the static " +
                        std::to_string(kScratchBytes) + "-byte array (at most 103000 points); "
                        "use wos_solve_grid_device");
    }
    if (ctx->device < 0 || ctx->device >= kMaxDevices) {
        return fail(ctx, WOS_ERR_INVALID, "wos_solve_grid_device_noalloc: device index too large");
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return fail(ctx, WOS_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));

    // device address of the scratch array on this device, taken once
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_lock);
        if (!g_scratch_ptr[ctx->device]) {
            void *ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr) {
                return fail(ctx, WOS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") +
                                                   cudaGetErrorString(e));
            }
            g_scratch_ptr[ctx->device] = ptr;
        }
        base = static_cast<unsigned char *>(g_scratch_ptr[ctx->device]);
    }
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
    e = wosb::launch_classify(ctx->view, ps, p->seed, p->max_ray_attempts, btol, eq, out, loc,
                              start, ctr, s);
    if (e != cudaSuccess) return fail(ctx, WOS_ERR_CUDA, std::string("classification kernel: ") + cudaGetErrorString(e));
    cudaEventRecord(ctx->events[1], s);
    if (p->method == WOS_METHOD_PLAIN_FP64) {
        e = wosb::launch_walk_plain(ctx->view, ps, p->seed, eq, p->N_walks, eps, p->max_steps, loc,
                                    start, out, ctr, s);
        cudaEventRecord(ctx->events[2], s);
    } else {
        const int precision = p->method == WOS_METHOD_FAST_FP32 ? 32 : 64;
        wosb::FastPlan plan = wosb::plan_fast(ctx->view, ctx->wide, ps.n, p->N_walks, precision,
                                              ctx->sms, ctx->smem_optin);
        // one walk task per point keeps the partials within the scratch array
        plan.chunk = p->N_walks;
        plan.chunks = 1;
        plan.n_tasks = ps.n;
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
        counters->inside_points = counters->total_walks / p->N_walks;
        counters->effective_epsilon = eps;
        cudaEventElapsedTime(&counters->classify_ms, ctx->events[0], ctx->events[1]);
        cudaEventElapsedTime(&counters->walk_ms, ctx->events[1], ctx->events[2]);
        cudaEventElapsedTime(&counters->total_ms, ctx->events[0], ctx->events[3]);
    }
    return WOS_OK;
}
