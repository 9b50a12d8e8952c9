// C ABI of the transient plate heating solver (include/wos_b200.h): the
// time loop of apps/welding/src/level2_transient_heat.cpp:393-645 with every
// implicit-Euler step solved by the walk kernels (PLAIN_FP64 on the
// reference's streams, or FAST_FP32 / FAST_FP64).
//
// All steps' fields live in one device array, step s in slice s, so step s
// reads slice s-1 through its own TransientDesc and the whole loop is a
// fixed launch sequence that can be captured as one CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wos_b200.h"
#include "context_internal.h"
#include "kernels.h"

using namespace wosb;

namespace {

// GaussianHeatSource2D::gaussian_integral (gaussian_heat_source.hpp:112-123)
double gaussian_integral(double lower, double upper, double centre, double sigma) {
    constexpr double sqrt_two = 1.41421356237309504880168872420969808;
    constexpr double sqrt_pi_over_two = 1.25331413731550025120788264240552263;
    return sigma * sqrt_pi_over_two *
           (std::erf((upper - centre) / (sqrt_two * sigma)) -
            std::erf((lower - centre) / (sqrt_two * sigma)));
}

// heating_fraction (level2_transient_heat.cpp:226-234)
double heating_fraction(double time_begin, double time_end, double heat_on_time) {
    const double overlap_begin = std::max(0.0, time_begin);
    const double overlap_end = std::min(time_end, heat_on_time);
    if (!(overlap_end > overlap_begin)) return 0.0;
    return (overlap_end - overlap_begin) / (time_end - time_begin);
}

int step_count(const wos_transient_params &p) {
    return static_cast<int>(std::llround(p.total_time / p.dt));
}

// The reference's checks (level2_transient_heat.cpp:206-223 and the source's
// constructor, gaussian_heat_source.hpp:28-36), with its messages.
std::string check(const wos_transient_params &p) {
    if (p.scenario != 0 && p.scenario != 2 && p.scenario != 3) return "scenario must be 0, 2 or 3";
    if (p.nx < 3 || p.ny < 3 || p.nx % 2 == 0 || p.ny % 2 == 0) {
        return "--nx and --ny must be odd integers of at least 3";
    }
    if (!(p.dt > 0.0) || !(p.total_time > 0.0) || !(p.epsilon > 0.0) || p.walks < 1 ||
        p.max_steps < 1 || (p.scenario != 0 && !(p.heat_on_time > 0.0))) {
        return "dt, total_time, heat_on_time, epsilon, walks and max_steps must be positive";
    }
    if (p.scenario == 2 && !(p.heat_on_time < p.total_time)) {
        return "--heat-on-time must be smaller than --total-time";
    }
    if (!std::isfinite(p.plate_x0) || !std::isfinite(p.plate_y0)) {
        return "plate corner must be finite";
    }
    if (p.scenario == 3 &&
        (!(p.weld_speed > 0.0) || p.weld_y < p.plate_y0 || p.weld_y > p.plate_y0 + p.length_y)) {
        // moving_gaussian_heat_source.hpp:21-28
        return "invalid moving Gaussian parameters";
    }
    const double steps = p.total_time / p.dt;
    if (std::abs(steps - std::round(steps)) > 1e-10 * std::max(1.0, steps)) {
        return "--total-time must be an integer multiple of --dt";
    }
    if (!(p.epsilon < 0.5 * std::min(p.length_x, p.length_y))) {
        return "--epsilon is too large for the plate";
    }
    if (!(p.length_x > 0.0) || !(p.length_y > 0.0)) return "invalid plate size";
    if (p.scenario != 0 &&
        (!(p.thickness > 0.0) || !(p.electrical_power > 0.0) || !(p.efficiency > 0.0) ||
         p.efficiency > 1.0 || !(p.sigma_x > 0.0) || !(p.sigma_y > 0.0))) {
        return "invalid Gaussian heat-source parameters";
    }
    if (!(p.conductivity > 0.0) || !(p.density > 0.0) || !(p.specific_heat > 0.0)) {
        return "conductivity, density and specific heat must be positive";
    }
    if (p.method < 0 || p.method > 2) return "unknown method";
    return std::string();
}

}  // namespace

extern "C" void wos_transient_defaults(wos_transient_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // Level2Config (level2_transient_heat.cpp:46-78)
    p->nx = 49;
    p->ny = 33;
    p->walks = 500;
    p->max_steps = 1000;
    p->cubic = 1;
    p->dt = 0.1;
    p->total_time = 10.0;
    p->heat_on_time = 3.0;
    p->epsilon = 8e-6;
    p->seed = 20260819ULL;
    p->length_x = 0.12;
    p->length_y = 0.08;
    p->thickness = 0.006;
    p->conductivity = 35.0;
    p->density = 7800.0;
    p->specific_heat = 600.0;
    p->electrical_power = 800.0;
    p->efficiency = 0.75;
    p->sigma_x = 0.006;
    p->sigma_y = 0.006;
    p->method = WOS_METHOD_FAST_FP32;
    p->scenario = 2;
    p->plate_x0 = -0.5 * p->length_x;
    p->plate_y0 = -0.5 * p->length_y;
    // Level3Config (level3_moving_heat.cpp:64-67)
    p->weld_y = 0.0;
    p->source_start_x = -0.05;
    p->weld_speed = 0.02;
}

extern "C" int wos_transient_steps(const wos_transient_params *p) {
    if (!p || !check(*p).empty()) return -1;
    return step_count(*p);
}

extern "C" int wos_transient_solve(wos_context *ctx, const wos_transient_params *pp,
                                   const double *initial, int use_graph, double *fields,
                                   double *standard_error, long long *max_steps_hits,
                                   float *device_ms) {
    if (!ctx) return fail(nullptr, WOS_ERR_INVALID, "null context");
    if (!pp) return fail(ctx, WOS_ERR_INVALID, "wos_transient_solve: null params");
    const wos_transient_params &p = *pp;
    const std::string err = check(p);
    if (!err.empty()) return fail(ctx, WOS_ERR_INVALID, "wos_transient_solve: " + err);
    cudaSetDevice(ctx->device);
    cudaStream_t stream = ctx->stream;

    // the plate (rectangular_plate.hpp:11-34) and its grid
    const double xmin = p.plate_x0, xmax = p.plate_x0 + p.length_x;
    const double ymin = p.plate_y0, ymax = p.plate_y0 + p.length_y;
    const double verts[8] = {xmin, ymin, xmax, ymin, xmax, ymax, xmin, ymax};
    const int prims[8] = {0, 1, 1, 2, 2, 3, 3, 0};
    const int bids[4] = {0, 0, 0, 0};
    HostScene plate;
    const std::string merr = build_scene(2, verts, 4, prims, 4, bids, 0, plate);
    if (!merr.empty()) return fail(ctx, WOS_ERR_MESH, "Mesh: " + merr);
    SceneDevice dev;
    struct Release {
        std::vector<DeviceBuffer *> bufs;
        SceneDevice *scene;
        ~Release() {
            for (DeviceBuffer *b : bufs) b->release();
            scene->release();
        }
    };
    DeviceBuffer d_fields, d_se, d_loc, d_start, d_part, d_queue, d_ctr, d_desc;
    Release guard{{&d_fields, &d_se, &d_loc, &d_start, &d_part, &d_queue, &d_ctr, &d_desc}, &dev};
    WOS_CUDA(ctx, dev.upload(plate, stream), "plate upload");

    PointSet ps{};
    ps.dim = 2;
    ps.Nx = p.nx;
    ps.Ny = p.ny;
    ps.Nz = 1;
    ps.lo[0] = xmin;
    ps.hi[0] = xmax;
    ps.lo[1] = ymin;
    ps.hi[1] = ymax;
    ps.n = static_cast<long long>(p.nx) * p.ny;
    const long long n = ps.n;
    const int steps = step_count(p);
    const size_t field_bytes = sizeof(double) * static_cast<size_t>(n) * (steps + 1);
    WOS_CUDA(ctx, d_fields.reserve(field_bytes), "alloc fields");
    WOS_CUDA(ctx, d_se.reserve(field_bytes), "alloc standard errors");
    WOS_CUDA(ctx, d_loc.reserve(n), "alloc location");
    WOS_CUDA(ctx, d_start.reserve(sizeof(StartRecord) * n), "alloc start");
    WOS_CUDA(ctx, d_ctr.reserve(sizeof(DeviceCounters) * (steps + 1)), "alloc counters");
    WOS_CUDA(ctx, d_desc.reserve(sizeof(TransientDesc) * steps), "alloc step descriptors");
    WOS_CUDA(ctx, cudaMemsetAsync(d_fields.ptr, 0, field_bytes, stream), "clear fields");
    WOS_CUDA(ctx, cudaMemsetAsync(d_se.ptr, 0, field_bytes, stream), "clear fields");
    if (initial) {
        WOS_CUDA(ctx, cudaMemcpyAsync(d_fields.ptr, initial, sizeof(double) * n,
                                      cudaMemcpyHostToDevice, stream),
                 "H2D initial field");
    }
    WOS_CUDA(ctx, cudaMemsetAsync(d_ctr.ptr, 0, sizeof(DeviceCounters) * (steps + 1), stream),
             "clear counters");
    auto *fld = static_cast<double *>(d_fields.ptr);
    auto *se = static_cast<double *>(d_se.ptr);
    auto *loc = static_cast<uint8_t *>(d_loc.ptr);
    auto *st = static_cast<StartRecord *>(d_start.ptr);
    auto *ctr = static_cast<DeviceCounters *>(d_ctr.ptr);
    auto *descs = static_cast<TransientDesc *>(d_desc.ptr);

    // physical constants (level2_transient_heat.cpp:404-409, 430-436)
    const double diffusivity = p.conductivity / (p.density * p.specific_heat);
    const double alpha = 1.0 / std::sqrt(diffusivity * p.dt);
    // the stationary source sits at the plate centre
    const double cx = 0.5 * (xmin + xmax), cy = 0.5 * (ymin + ymax);
    const double ix = p.scenario == 2 ? gaussian_integral(xmin, xmax, cx, p.sigma_x) : 0.0;
    const double iy = p.scenario == 2 ? gaussian_integral(ymin, ymax, cy, p.sigma_y) : 0.0;
    std::vector<TransientDesc> host(steps);
    for (int s = 1; s <= steps; ++s) {
        TransientDesc &t = host[s - 1];
        t = TransientDesc{};
        t.kind = p.scenario;
        t.alpha = alpha;
        t.fraction = p.scenario == 2
                         ? heating_fraction((s - 1) * p.dt, s * p.dt, p.heat_on_time)
                         : 0.0;
        t.conductivity = p.conductivity;
        t.power = p.electrical_power * p.efficiency;
        t.thickness = p.thickness;
        t.ix = ix;
        t.iy = iy;
        t.cx = cx;
        t.cy = cy;
        if (p.scenario == 3) {
            // MovingGaussianStepSource2D (moving_gaussian_heat_source.hpp:16-71)
            const double time_begin = (s - 1) * p.dt, time_end = s * p.dt;
            const double active_begin = std::max(0.0, time_begin);
            const double active_end = std::min(time_end, p.heat_on_time);
            t.moving = 0;
            if (active_end > active_begin) {
                const double active_fraction =
                    (active_end - active_begin) / (time_end - time_begin);
                const double midpoint = 0.5 * (active_begin + active_end);
                const double half_width = 0.5 * (active_end - active_begin);
                constexpr double inverse_sqrt_three = 0.577350269189625764509148780501957456;
                const double times[2] = {midpoint - inverse_sqrt_three * half_width,
                                         midpoint + inverse_sqrt_three * half_width};
                const double absorbed = p.electrical_power * p.efficiency;
                for (int k = 0; k < 2; ++k) {
                    const double mx = p.source_start_x + p.weld_speed * times[k];
                    if (mx < xmin || mx > xmax) {
                        return fail(ctx, WOS_ERR_INVALID,
                                    "wos_transient_solve: moving Gaussian centre leaves the "
                                    "finite plate");
                    }
                    const double gx = gaussian_integral(xmin, xmax, mx, p.sigma_x);
                    const double gy = gaussian_integral(ymin, ymax, p.weld_y, p.sigma_y);
                    t.mx[k] = mx;
                    t.my[k] = p.weld_y;
                    t.mcoef[k] = active_fraction * absorbed / (2.0 * p.thickness * gx * gy);
                }
                t.moving = 2;
            }
        }
        t.sx = p.sigma_x;
        t.sy = p.sigma_y;
        t.prev = fld + static_cast<size_t>(s - 1) * n;
        t.nx = p.nx;
        t.ny = p.ny;
        t.xmin = xmin;
        t.xmax = xmax;
        t.ymin = ymin;
        t.ymax = ymax;
        t.cubic = p.cubic ? 1 : 0;
    }
    WOS_CUDA(ctx, cudaMemcpyAsync(descs, host.data(), sizeof(TransientDesc) * steps,
                                  cudaMemcpyHostToDevice, stream),
             "H2D step descriptors");

    // start points once (the reference computes them once, :411-428); every
    // plate-edge grid point is a boundary point with value 0
    const double btol = 1e-10 * plate.scale;
    const EqDesc cls_eq{kTransient, kGreen, alpha, nullptr};
    WOS_CUDA(ctx, launch_classify(dev.view, ps, p.seed, 12, btol, cls_eq,
                                  Fields{nullptr, nullptr, nullptr, nullptr, nullptr}, loc, st,
                                  ctr + steps, stream),
             "classification kernel");

    const int precision = p.method == WOS_METHOD_FAST_FP64 ? 64 : 32;
    FastPlan plan{};
    if (p.method != WOS_METHOD_PLAIN_FP64) {
        plan = plan_fast(dev.view, dev.wide, n, p.walks, precision, ctx->sms, ctx->smem_optin);
        // a step is small: about two waves of tasks, and at least 256 walks
        // (8 per lane) per task so that a lane whose walk ends takes the
        // next one.  At the level-2 defaults 32 walks per task (one per
        // lane) left a warp waiting for its longest walk: 276 ms for the
        // run, against 184 ms at 256.
        const long long resident = static_cast<long long>(ctx->sms) * 24;
        long long chunk = static_cast<long long>(p.walks) * n / (2 * resident);
        chunk = std::max<long long>(256, std::min<long long>(1024, chunk));
        if (ctx->chunk_override > 0) chunk = ctx->chunk_override;
        set_chunk(plan, chunk, p.walks, p.max_steps, n);
        if (ctx->blocks_override > 0) plan.blocks = ctx->blocks_override;
        WOS_CUDA(ctx, d_part.reserve(sizeof(TaskPartial) * plan.n_tasks), "alloc partials");
        WOS_CUDA(ctx, d_queue.reserve(sizeof(unsigned long long)), "alloc queue");
    }
    const double shell_delta = std::ldexp(plate.scale, -16);

    auto enqueue = [&]() -> cudaError_t {
        for (int s = 1; s <= steps; ++s) {
            const EqDesc e{kTransient, kGreen, alpha, descs + (s - 1)};
            const uint64_t seed = p.seed ^ splitmix64(static_cast<uint64_t>(s));
            const Fields out{fld + static_cast<size_t>(s) * n, nullptr,
                             se + static_cast<size_t>(s) * n, nullptr, nullptr};
            cudaError_t e2;
            if (p.method == WOS_METHOD_PLAIN_FP64) {
                e2 = launch_walk_plain(dev.view, ps, seed, e, p.walks, p.epsilon, p.max_steps,
                                       loc, st, out, ctr + (s - 1), stream);
            } else {
                e2 = launch_walk_fast(dev.view, dev.wide, ps, seed, e, p.walks, p.epsilon,
                                      p.max_steps, shell_delta, precision, plan, loc, st,
                                      static_cast<TaskPartial *>(d_part.ptr),
                                      static_cast<unsigned long long *>(d_queue.ptr), out,
                                      ctr + (s - 1), stream, nullptr);
            }
            if (e2 != cudaSuccess) return e2;
        }
        return cudaSuccess;
    };

    WOS_CUDA(ctx, cudaStreamSynchronize(stream), "transient set-up");
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (use_graph) {
        WOS_CUDA(ctx, cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal),
                 "begin capture");
        const cudaError_t e = enqueue();
        const cudaError_t ee = cudaStreamEndCapture(stream, &graph);
        if (e != cudaSuccess || ee != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            return cuda_fail(ctx, e != cudaSuccess ? e : ee, "transient capture");
        }
        const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
        if (ei != cudaSuccess) {
            cudaGraphDestroy(graph);
            return cuda_fail(ctx, ei, "graph instantiate");
        }
    }
    cudaError_t run = cudaEventRecord(ctx->events[0], stream);
    if (run == cudaSuccess) run = use_graph ? cudaGraphLaunch(exec, stream) : enqueue();
    if (run == cudaSuccess) run = cudaEventRecord(ctx->events[1], stream);
    if (run == cudaSuccess) run = cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (run != cudaSuccess) return cuda_fail(ctx, run, "transient steps");
    if (device_ms) cudaEventElapsedTime(device_ms, ctx->events[0], ctx->events[1]);

    std::vector<DeviceCounters> hc(steps + 1);
    WOS_CUDA(ctx, cudaMemcpy(hc.data(), ctr, sizeof(DeviceCounters) * (steps + 1),
                             cudaMemcpyDeviceToHost),
             "read counters");
    long long hits = 0;
    for (const DeviceCounters &c : hc) {
        if (c.error_flags) {
            return fail(ctx, WOS_ERR_DEVICE, device_error(c.error_flags));
        }
        hits += static_cast<long long>(c.max_steps_hits);
    }
    if (max_steps_hits) *max_steps_hits = hits;
    if (fields) {
        WOS_CUDA(ctx, cudaMemcpy(fields, fld, field_bytes, cudaMemcpyDeviceToHost), "D2H fields");
    }
    if (standard_error) {
        WOS_CUDA(ctx, cudaMemcpy(standard_error, se, field_bytes, cudaMemcpyDeviceToHost),
                 "D2H standard errors");
    }
    return WOS_OK;
}
