// C ABI of the stationary plate heating solver (include/wos_b200.h): the
// three solves of apps/welding/src/level1_stationary_heat.cpp:548-655 (a
// manufactured Poisson problem and a finite-plate Gaussian heat source with
// Green or Green-source MIS sampling) on the walk kernels, PLAIN_FP64 on the
// reference's streams or FAST_FP32 / FAST_FP64.
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

// The reference's per-case stream constants (level1_stationary_heat.cpp:
// 599-600, 623-624, 643-644).
constexpr uint64_t kManufacturedStream = 0x4C4556454C31414FULL;
constexpr uint64_t kGaussianStream = 0x4C4556454C314247ULL;

// GaussianHeatSource2D::gaussian_integral (gaussian_heat_source.hpp:112-123)
double gaussian_integral(double lower, double upper, double centre, double sigma) {
    constexpr double sqrt_two = 1.41421356237309504880168872420969808;
    constexpr double sqrt_pi_over_two = 1.25331413731550025120788264240552263;
    return sigma * sqrt_pi_over_two *
           (std::erf((upper - centre) / (sqrt_two * sigma)) -
            std::erf((lower - centre) / (sqrt_two * sigma)));
}

std::string check(const wos_stationary_params &p) {
    if (p.nx < 3 || p.ny < 3) return "nx and ny must be at least 3";
    if (p.walks < 1 || p.max_steps < 1 || !(p.epsilon > 0.0)) {
        return "walks, max_steps and epsilon must be positive";
    }
    if (!(p.length_x > 0.0) || !(p.length_y > 0.0) || !std::isfinite(p.length_x) ||
        !std::isfinite(p.length_y)) {
        // rectangular_plate.hpp:13-16
        return "rectangular plate requires increasing coordinate bounds";
    }
    if (!(p.epsilon < 0.5 * std::min(p.length_x, p.length_y))) {
        return "epsilon is too large for the plate";
    }
    if (p.source != WOS_PLATE_MANUFACTURED && p.source != WOS_PLATE_GAUSSIAN) {
        return "unknown plate source";
    }
    if (p.source_mode < WOS_SOURCE_UNIFORM || p.source_mode > WOS_SOURCE_MIS) {
        return "unknown source mode";
    }
    if (p.source == WOS_PLATE_MANUFACTURED && p.source_mode == WOS_SOURCE_MIS) {
        // include/wos/wos.hpp:88-91: the manufactured problem has no proposal
        return "GreenSourceMIS requires a source proposal sampler and PDF";
    }
    if (p.source == WOS_PLATE_GAUSSIAN &&
        (!(p.thickness > 0.0) || !(p.electrical_power > 0.0) || !(p.efficiency > 0.0) ||
         p.efficiency > 1.0 || !(p.sigma_x > 0.0) || !(p.sigma_y > 0.0) ||
         p.source_x < 0.0 || p.source_x > p.length_x || p.source_y < 0.0 ||
         p.source_y > p.length_y || !(p.conductivity > 0.0))) {
        // gaussian_heat_source.hpp:28-36
        return "invalid Gaussian heat-source parameters";
    }
    if (p.source_mode == WOS_SOURCE_MIS &&
        (!(p.mis_green_probability > 0.0 && p.mis_green_probability < 1.0) ||
         !std::isfinite(p.mis_green_probability))) {
        // include/wos/source_sampling.hpp:41-47
        return "Green-source MIS probability must be finite and in (0, 1)";
    }
    if (p.source_mode == WOS_SOURCE_MIS && p.max_proposal_attempts < 1) {
        return "max_proposal_attempts must be positive";
    }
    if (p.method < 0 || p.method > 2) return "unknown method";
    return std::string();
}

}  // namespace

extern "C" void wos_stationary_defaults(wos_stationary_params *p, int source) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // Level1Config (level1_stationary_heat.cpp:42-61)
    p->nx = 49;
    p->ny = 33;
    p->walks = 6000;
    p->max_steps = 1000;
    p->epsilon = 8e-6;
    p->seed = 20260818ULL;
    p->length_x = 0.12;
    p->length_y = 0.08;
    p->thickness = 0.006;
    p->conductivity = 35.0;
    p->electrical_power = 800.0;
    p->efficiency = 0.75;
    p->sigma_x = 0.006;
    p->sigma_y = 0.006;
    p->source_x = 0.5 * p->length_x;
    p->source_y = 0.5 * p->length_y;
    p->peak_rise = 100.0;
    p->source = source == WOS_PLATE_MANUFACTURED ? WOS_PLATE_MANUFACTURED : WOS_PLATE_GAUSSIAN;
    p->case_stream = p->source == WOS_PLATE_MANUFACTURED ? kManufacturedStream : kGaussianStream;
    p->source_mode = WOS_SOURCE_GREEN;
    p->mis_green_probability = 0.5;
    p->method = WOS_METHOD_FAST_FP32;
    p->max_proposal_attempts = 1000000;  // gaussian_heat_source.hpp:58
}

extern "C" int wos_stationary_solve(wos_context *ctx, const wos_stationary_params *pp,
                                    double *mean, double *variance, double *standard_error,
                                    double *mean_steps, long long *max_steps_hits,
                                    float *device_ms) {
    if (!ctx) return fail(nullptr, WOS_ERR_INVALID, "null context");
    if (!pp) return fail(ctx, WOS_ERR_INVALID, "wos_stationary_solve: null params");
    const wos_stationary_params &p = *pp;
    const std::string err = check(p);
    if (!err.empty()) return fail(ctx, WOS_ERR_INVALID, "wos_stationary_solve: " + err);
    cudaSetDevice(ctx->device);
    cudaStream_t stream = ctx->stream;

    // make_rectangular_plate (rectangular_plate.hpp:11-34) over [0, Lx] x [0, Ly]
    const double xmin = 0.0, xmax = p.length_x, ymin = 0.0, ymax = p.length_y;
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
    DeviceBuffer d_out, d_loc, d_start, d_part, d_queue, d_ctr;
    Release guard{{&d_out, &d_loc, &d_start, &d_part, &d_queue, &d_ctr}, &dev};
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
    const size_t field_bytes = sizeof(double) * static_cast<size_t>(n);
    WOS_CUDA(ctx, d_out.reserve(4 * field_bytes), "alloc fields");
    WOS_CUDA(ctx, d_loc.reserve(n), "alloc location");
    WOS_CUDA(ctx, d_start.reserve(sizeof(StartRecord) * n), "alloc start");
    WOS_CUDA(ctx, d_ctr.reserve(2 * sizeof(DeviceCounters)), "alloc counters");
    WOS_CUDA(ctx, cudaMemsetAsync(d_out.ptr, 0, 4 * field_bytes, stream), "clear fields");
    WOS_CUDA(ctx, cudaMemsetAsync(d_ctr.ptr, 0, 2 * sizeof(DeviceCounters), stream),
             "clear counters");
    auto *fld = static_cast<double *>(d_out.ptr);
    auto *loc = static_cast<uint8_t *>(d_loc.ptr);
    auto *st = static_cast<StartRecord *>(d_start.ptr);
    auto *ctr = static_cast<DeviceCounters *>(d_ctr.ptr);
    const Fields out{fld, fld + n, fld + 2 * n, fld + 3 * n, nullptr};

    PlateDesc desc{};
    desc.kind = p.source == WOS_PLATE_MANUFACTURED ? 0 : 1;
    desc.max_attempts = p.max_proposal_attempts > 0 ? p.max_proposal_attempts : 1;
    constexpr double pi = 3.141592653589793238462643383279502884;
    desc.peak = p.peak_rise;
    desc.length_x = p.length_x;
    desc.length_y = p.length_y;
    // ManufacturedPoisson2D::source (level1_stationary_heat.cpp:96-101)
    desc.eigen = pi * pi * (1.0 / (p.length_x * p.length_x) + 1.0 / (p.length_y * p.length_y));
    desc.power = p.electrical_power * p.efficiency;
    desc.thickness = p.thickness;
    desc.conductivity = p.conductivity;
    desc.cx = p.source_x;
    desc.cy = p.source_y;
    desc.sx = p.sigma_x;
    desc.sy = p.sigma_y;
    if (desc.kind == 1) {
        desc.ix = gaussian_integral(xmin, xmax, p.source_x, p.sigma_x);
        desc.iy = gaussian_integral(ymin, ymax, p.source_y, p.sigma_y);
    }
    desc.beta = p.mis_green_probability;
    desc.xmin = xmin;
    desc.xmax = xmax;
    desc.ymin = ymin;
    desc.ymax = ymax;

    // start points of every grid point (build_start_points, :207-222); the
    // plate-edge points are boundary points of value 0, which the reference
    // leaves at 0 without walking (:241-243)
    const double btol = 1e-10 * plate.scale;
    const EqDesc eq{kPlate, p.source_mode, 0.0, nullptr, &desc};
    const uint64_t seed = p.seed ^ p.case_stream;
    WOS_CUDA(ctx, launch_classify(dev.view, ps, seed, 12, btol, eq,
                                  Fields{nullptr, nullptr, nullptr, nullptr, nullptr}, loc, st,
                                  ctr + 1, stream),
             "classification kernel");
    WOS_CUDA(ctx, cudaEventRecord(ctx->events[0], stream), "event");
    cudaError_t e = cudaSuccess;
    if (p.method == WOS_METHOD_PLAIN_FP64) {
        e = launch_walk_plain(dev.view, ps, seed, eq, p.walks, p.epsilon, p.max_steps, loc, st,
                              out, ctr, stream);
    } else {
        const int precision = p.method == WOS_METHOD_FAST_FP64 ? 64 : 32;
        FastPlan plan =
            plan_fast(dev.view, dev.wide, n, p.walks, precision, ctx->sms, ctx->smem_optin);
        set_chunk(plan, ctx->chunk_override > 0 ? ctx->chunk_override : plan.chunk, p.walks,
                  p.max_steps, n);
        if (ctx->blocks_override > 0) plan.blocks = ctx->blocks_override;
        WOS_CUDA(ctx, d_part.reserve(sizeof(TaskPartial) * plan.n_tasks), "alloc partials");
        WOS_CUDA(ctx, d_queue.reserve(sizeof(unsigned long long)), "alloc queue");
        const double shell_delta = std::ldexp(plate.scale, -16);
        e = launch_walk_fast(dev.view, dev.wide, ps, seed, eq, p.walks, p.epsilon, p.max_steps,
                             shell_delta, precision, plan, loc, st,
                             static_cast<TaskPartial *>(d_part.ptr),
                             static_cast<unsigned long long *>(d_queue.ptr), out, ctr, stream,
                             nullptr);
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "plate walk kernel");
    WOS_CUDA(ctx, cudaEventRecord(ctx->events[1], stream), "event");
    WOS_CUDA(ctx, cudaStreamSynchronize(stream), "plate walks");
    if (device_ms) cudaEventElapsedTime(device_ms, ctx->events[0], ctx->events[1]);

    DeviceCounters hc[2];
    WOS_CUDA(ctx, cudaMemcpy(hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost), "read counters");
    if (hc[0].error_flags == kErrRejectionCap) {
        // gaussian_heat_source.hpp:70-72
        return fail(ctx, WOS_ERR_DEVICE,
                    "finite-plate Gaussian rejection sampler did not accept a point");
    }
    if (hc[0].error_flags) return fail(ctx, WOS_ERR_DEVICE, device_error(hc[0].error_flags));
    if (max_steps_hits) *max_steps_hits = static_cast<long long>(hc[0].max_steps_hits);
    double *dst[4] = {mean, variance, standard_error, mean_steps};
    for (int k = 0; k < 4; ++k) {
        if (!dst[k]) continue;
        WOS_CUDA(ctx, cudaMemcpy(dst[k], fld + k * n, field_bytes, cudaMemcpyDeviceToHost),
                 "D2H fields");
    }
    return WOS_OK;
}
