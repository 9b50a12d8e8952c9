// C ABI of the Gaussian heat source (include/wos_b200.h): forward solve and
// adjoint replay at probe points.  The kernels are in kernels_adjoint.cu.
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

int wos_context::run_heat(const wos_params &p, const HeatDesc &h, const PointSet &ps,
                          HeatOut out, wos_counters *counters_out) {
    cudaSetDevice(device);
    const long long n = ps.n;
    if (p.method == WOS_METHOD_FAST_FP32) {
        // near-boundary lists for this epsilon (one-time set-up per mesh)
        const float t = near_list_threshold(sdev.wide, p.epsilon, std::ldexp(scene.scale, -16));
        WOS_CUDA(this, sdev.ensure_lists(t, sms, stream), "near-boundary lists");
        wide = sdev.wide;
    }
    WOS_CUDA(this, location.reserve(std::max<long long>(n, 1)), "alloc location");
    WOS_CUDA(this, start.reserve(sizeof(StartRecord) * std::max<long long>(n, 1)), "alloc start");
    WOS_CUDA(this, counters.reserve(sizeof(DeviceCounters)), "alloc counters");
    WOS_CUDA(this, cudaMemsetAsync(counters.ptr, 0, sizeof(DeviceCounters), stream),
             "clear counters");
    auto *loc = static_cast<uint8_t *>(location.ptr);
    auto *st = static_cast<StartRecord *>(start.ptr);
    auto *ctr = static_cast<DeviceCounters *>(counters.ptr);
    // boundary tolerance 1e-10 * max(1, mesh extents), include/wos/runner.hpp:86-88
    const double btol = 1e-10 * scene.scale;
    // classification only: the heat merge writes every field
    const EqDesc eq{kLaplace, 0, 0.0, nullptr};
    const Fields cls{nullptr, nullptr, nullptr, nullptr, out.f.location};

    WOS_CUDA(this, cudaEventRecord(events[0], stream), "event");
    WOS_CUDA(this, launch_classify(view, ps, p.seed, p.max_ray_attempts, btol, eq, cls, loc, st,
                                   ctr, stream),
             "classification kernel");
    WOS_CUDA(this, cudaEventRecord(events[1], stream), "event");
    const int precision = p.method == WOS_METHOD_FAST_FP32 ? 32 : 64;
    FastPlan plan = plan_fast(view, wide, n, p.N_walks, precision, sms, smem_optin);
    set_chunk(plan, chunk_override > 0 ? chunk_override : plan.chunk, p.N_walks, p.max_steps, n);
    if (blocks_override > 0) plan.blocks = blocks_override;
    WOS_CUDA(this, partials.reserve(sizeof(HeatPartial) * std::max<long long>(plan.n_tasks, 1)),
             "alloc partials");
    WOS_CUDA(this, queue.reserve(sizeof(unsigned long long)), "alloc queue");
    const double shell_delta = std::ldexp(scene.scale, -16);
    WOS_CUDA(this, launch_heat(view, wide, ps, p.seed, h, p.N_walks, p.epsilon, p.max_steps,
                               shell_delta, precision, plan, loc, st,
                               static_cast<HeatPartial *>(partials.ptr),
                               static_cast<unsigned long long *>(queue.ptr), out, ctr, stream,
                               events[2]),
             "heat walk kernel");
    WOS_CUDA(this, cudaEventRecord(events[3], stream), "event");
    DeviceCounters hc{};
    WOS_CUDA(this, cudaMemcpyAsync(&hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost, stream),
             "read counters");
    WOS_CUDA(this, cudaStreamSynchronize(stream), "heat solve");
    if (hc.error_flags) return fail(this, WOS_ERR_DEVICE, device_error(hc.error_flags));
    if (counters_out) {
        wos_counters &c = *counters_out;
        std::memset(&c, 0, sizeof(c));
        c.max_steps_hits = static_cast<long long>(hc.max_steps_hits);
        c.ambiguous_ray_retries = static_cast<long long>(hc.ambiguous_ray_retries);
        c.indeterminate_points = static_cast<long long>(hc.indeterminate_points);
        c.total_walks = static_cast<long long>(hc.total_walks);
        c.total_steps = static_cast<long long>(hc.total_steps);
        c.exact_queries = static_cast<long long>(hc.exact_queries);
        c.inside_points = p.N_walks > 0 ? c.total_walks / p.N_walks : 0;
        c.effective_epsilon = p.epsilon;
        cudaEventElapsedTime(&c.classify_ms, events[0], events[1]);
        cudaEventElapsedTime(&c.walk_ms, events[1], events[2]);
        cudaEventElapsedTime(&c.total_ms, events[0], events[3]);
    }
    return WOS_OK;
}

namespace {

std::string check_heat(const wos_context *ctx, const wos_params *p,
                       const wos_gaussian_source *s, const double *probes, long long n) {
    if (!p) return "null params";
    if (!ctx->has_mesh) return "no mesh uploaded";
    if (!s) return "null source";
    if (p->source_mode < 0 || p->source_mode > 2) return "source_mode must be 0, 1 or 2";
    if (p->N_walks < 1) return "N_walks must be >= 1";
    if (!(p->epsilon > 0.0) || !std::isfinite(p->epsilon)) return "epsilon must be positive";
    if (p->max_steps < 1) return "max_steps must be >= 1";
    if (p->max_ray_attempts < 3) return "max_ray_attempts must be >= 3";
    if (p->method != WOS_METHOD_FAST_FP32 && p->method != WOS_METHOD_FAST_FP64) {
        return "method must be FAST_FP32 or FAST_FP64";
    }
    if (!(s->sigma > 0.0) || !std::isfinite(s->sigma)) return "sigma must be positive";
    if (!std::isfinite(s->Q) || !std::isfinite(s->x0[0]) || !std::isfinite(s->x0[1]) ||
        !std::isfinite(s->x0[2])) {
        return "source parameters must be finite";
    }
    if (p->source_mode == WOS_SOURCE_MIS) {
        // include/wos/source_sampling.hpp:44-48
        const double b = s->mis_green_probability;
        if (!(b > 0.0 && b < 1.0) || !std::isfinite(b)) {
            return "Green-source MIS probability must be finite and in (0, 1)";
        }
        if (s->proposal_sigma > 0.0 &&
            (!std::isfinite(s->proposal_sigma) || !std::isfinite(s->proposal_x0[0]) ||
             !std::isfinite(s->proposal_x0[1]) || !std::isfinite(s->proposal_x0[2]))) {
            return "proposal parameters must be finite";
        }
    }
    if (n < 0 || (n > 0 && !probes)) return "null probes";
    // a non-finite probe has no place in the domain; reject it here rather
    // than hand it to the traversals
    for (long long i = 0; i < n * ctx->scene.dim; ++i) {
        if (!std::isfinite(probes[i])) return "probe coordinates must be finite";
    }
    return std::string();
}

// Uploads probes, seeding indices and vertex values; fills ps and h.
int prepare_heat(wos_context *ctx, const wos_params *params, const wos_gaussian_source *src,
                 const double *vertex_values, const double *probes, const uint64_t *point_index,
                 long long n, PointSet &ps, HeatDesc &h) {
    const int dim = ctx->scene.dim;
    ps = PointSet{};
    ps.dim = dim;
    ps.n = n;
    ps.Nx = ps.Ny = ps.Nz = 1;
    for (int k = 0; k < 3; ++k) {
        ps.lo[k] = ctx->scene.bbox[2 * k];
        ps.hi[k] = ctx->scene.bbox[2 * k + 1];
    }
    const long long m = std::max<long long>(n, 1);
    WOS_CUDA(ctx, ctx->points.reserve(sizeof(double) * dim * m), "alloc probes");
    if (n > 0) {
        WOS_CUDA(ctx, cudaMemcpyAsync(ctx->points.ptr, probes, sizeof(double) * dim * n,
                                      cudaMemcpyHostToDevice, ctx->stream),
                 "H2D probes");
    }
    ps.coords = static_cast<const double *>(ctx->points.ptr);
    if (point_index) {
        WOS_CUDA(ctx, ctx->index.reserve(sizeof(uint64_t) * m), "alloc index");
        WOS_CUDA(ctx, cudaMemcpyAsync(ctx->index.ptr, point_index, sizeof(uint64_t) * n,
                                      cudaMemcpyHostToDevice, ctx->stream),
                 "H2D index");
        ps.index = static_cast<const uint64_t *>(ctx->index.ptr);
    }
    h = HeatDesc{};
    h.mode = params->source_mode;
    h.Q = src->Q;
    h.x0[0] = src->x0[0];
    h.x0[1] = src->x0[1];
    h.x0[2] = src->x0[2];
    h.sigma = src->sigma;
    h.beta = src->mis_green_probability;
    const bool own = !(src->proposal_sigma > 0.0);
    for (int k = 0; k < 3; ++k) h.px0[k] = own ? src->x0[k] : src->proposal_x0[k];
    h.psigma = own ? src->sigma : src->proposal_sigma;
    h.slot_verts = ctx->sdev.slot_verts;
    if (vertex_values) {
        const size_t nv = static_cast<size_t>(ctx->scene.n_verts);
        WOS_CUDA(ctx, ctx->h_values.reserve(sizeof(double) * nv), "alloc vertex values");
        WOS_CUDA(ctx, cudaMemcpyAsync(ctx->h_values.ptr, vertex_values, sizeof(double) * nv,
                                      cudaMemcpyHostToDevice, ctx->stream),
                 "H2D vertex values");
        h.g = static_cast<const double *>(ctx->h_values.ptr);
    }
    return WOS_OK;
}

int d2h(wos_context *ctx, void *dst, const void *src, size_t bytes) {
    if (!dst || bytes == 0) return WOS_OK;
    WOS_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    return WOS_OK;
}

}  // namespace

extern "C" int wos_mesh_vertex_count(const wos_context *ctx, int *n_verts) {
    if (!ctx || !ctx->has_mesh || !n_verts) {
        return fail(nullptr, WOS_ERR_INVALID, "wos_mesh_vertex_count: no mesh or null output");
    }
    *n_verts = ctx->scene.n_verts;
    return WOS_OK;
}

extern "C" int wos_heat_forward(wos_context *ctx, const wos_params *params,
                                const wos_gaussian_source *source, const double *vertex_values,
                                const double *probes, const uint64_t *point_index, long long n,
                                double *mean, double *variance, double *standard_error,
                                double *mean_steps, uint8_t *location, wos_counters *counters) {
    if (!ctx) return fail(nullptr, WOS_ERR_INVALID, "null context");
    const std::string err = check_heat(ctx, params, source, probes, n);
    if (!err.empty()) return fail(ctx, WOS_ERR_INVALID, "wos_heat_forward: " + err);
    cudaSetDevice(ctx->device);
    PointSet ps;
    HeatDesc h;
    int rc = prepare_heat(ctx, params, source, vertex_values, probes, point_index, n, ps, h);
    if (rc) return rc;
    Fields dev{};
    rc = ctx->fields_for(n, dev);
    if (rc) return rc;
    HeatOut out{dev, nullptr, nullptr, nullptr};
    rc = ctx->run_heat(*params, h, ps, out, counters);
    if (rc) return rc;
    return ctx->download(n, dev, mean, variance, standard_error, mean_steps, location);
}

extern "C" int wos_heat_adjoint(wos_context *ctx, const wos_params *params,
                                const wos_gaussian_source *source, const double *vertex_values,
                                const double *probes, const uint64_t *point_index, long long n,
                                const double *grad_u, double *grad_source,
                                double *grad_vertex_values, double *jacobian,
                                double *jacobian_se, double *replayed_mean,
                                wos_counters *counters) {
    if (!ctx) return fail(nullptr, WOS_ERR_INVALID, "null context");
    const std::string err = check_heat(ctx, params, source, probes, n);
    if (!err.empty()) return fail(ctx, WOS_ERR_INVALID, "wos_heat_adjoint: " + err);
    cudaSetDevice(ctx->device);
    PointSet ps;
    HeatDesc h;
    int rc = prepare_heat(ctx, params, source, vertex_values, probes, point_index, n, ps, h);
    if (rc) return rc;
    const long long m = std::max<long long>(n, 1);
    const size_t nv = static_cast<size_t>(ctx->scene.n_verts);
    WOS_CUDA(ctx, ctx->h_gradu.reserve(sizeof(double) * m), "alloc probe weights");
    if (grad_u) {
        WOS_CUDA(ctx, cudaMemcpyAsync(ctx->h_gradu.ptr, grad_u, sizeof(double) * n,
                                      cudaMemcpyHostToDevice, ctx->stream),
                 "H2D probe weights");
    } else {
        const std::vector<double> ones(static_cast<size_t>(m), 1.0);
        WOS_CUDA(ctx, cudaMemcpyAsync(ctx->h_gradu.ptr, ones.data(), sizeof(double) * m,
                                      cudaMemcpyHostToDevice, ctx->stream),
                 "H2D probe weights");
        // the host vector must outlive the copy
        WOS_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "H2D probe weights");
    }
    WOS_CUDA(ctx, ctx->h_gradg.reserve(sizeof(double) * std::max<size_t>(nv, 1)), "alloc");
    WOS_CUDA(ctx, ctx->h_grads.reserve(sizeof(double) * 5), "alloc");
    WOS_CUDA(ctx, ctx->h_jac.reserve(sizeof(double) * 5 * m), "alloc");
    WOS_CUDA(ctx, ctx->h_jacse.reserve(sizeof(double) * 5 * m), "alloc");
    WOS_CUDA(ctx, cudaMemsetAsync(ctx->h_gradg.ptr, 0, sizeof(double) * nv, ctx->stream), "clear");
    WOS_CUDA(ctx, cudaMemsetAsync(ctx->h_grads.ptr, 0, sizeof(double) * 5, ctx->stream), "clear");
    h.adjoint = 1;
    h.grad_u = static_cast<const double *>(ctx->h_gradu.ptr);
    h.grad_g = static_cast<double *>(ctx->h_gradg.ptr);
    Fields dev{};
    rc = ctx->fields_for(n, dev);
    if (rc) return rc;
    HeatOut out{dev, static_cast<double *>(ctx->h_jac.ptr),
                static_cast<double *>(ctx->h_jacse.ptr), static_cast<double *>(ctx->h_grads.ptr)};
    rc = ctx->run_heat(*params, h, ps, out, counters);
    if (rc) return rc;
    const size_t b = sizeof(double) * static_cast<size_t>(n);
    if ((rc = d2h(ctx, grad_source, ctx->h_grads.ptr, sizeof(double) * 5))) return rc;
    if ((rc = d2h(ctx, grad_vertex_values, ctx->h_gradg.ptr, sizeof(double) * nv))) return rc;
    if ((rc = d2h(ctx, jacobian, ctx->h_jac.ptr, 5 * b))) return rc;
    if ((rc = d2h(ctx, jacobian_se, ctx->h_jacse.ptr, 5 * b))) return rc;
    if ((rc = d2h(ctx, replayed_mean, dev.mean, b))) return rc;
    WOS_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "D2H");
    return WOS_OK;
}
