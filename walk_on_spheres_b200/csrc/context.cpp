// C ABI of libwos_b200.so (include/wos_b200.h): context, mesh upload,
// solves and kernel-level checks.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/wos_b200.h"
#include "context_internal.h"
#include "kernels.h"
#include "obj_reader.h"

using namespace wosb;

namespace {
thread_local std::string g_error;
}  // namespace

std::string wosb::device_error(unsigned flags) {
    std::string m;
    if (flags & kErrRejectionCap) m = "a rejection sampler reached its proposal cap";
    if (flags & kErrBadState) {
        if (!m.empty()) m += "; ";
        m += "a closest-point query found no boundary primitive";
    }
    return m + " (error flags " + std::to_string(flags) + ")";
}

int wosb::fail(wos_context *ctx, int code, const std::string &msg) {
    if (ctx) ctx->error = msg;
    g_error = msg;
    return code;
}

int wosb::cuda_fail(wos_context *ctx, cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(ctx, WOS_ERR_CUDA, m);
}

// ------------------------------------------------------------- buffers

void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

cudaError_t DeviceBuffer::reserve(size_t n) {
    if (n <= bytes) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return e;
    }
    bytes = n;
    return cudaSuccess;
}

wos_context::~wos_context() {
    for (DeviceBuffer *b : all_buffers()) b->release();
    sdev.release();
    for (auto &ev : events) {
        if (ev) cudaEventDestroy(ev);
    }
    if (stream) cudaStreamDestroy(stream);
}

std::vector<DeviceBuffer *> wos_context::all_buffers() {
    return {&location, &start,
            &f_mean, &f_var, &f_se, &f_steps, &f_loc, &partials, &queue, &counters, &points,
            &index, &scratch_a, &scratch_b, &scratch_c, &scratch_d, &h_values, &h_gradu,
            &h_gradg, &h_grads, &h_jac, &h_jacse};
}

// ------------------------------------------------------------- context

extern "C" int wos_abi_version(void) { return WOS_B200_ABI_VERSION; }

extern "C" const char *wos_last_global_error(void) { return g_error.c_str(); }

extern "C" const char *wos_last_error(const wos_context *ctx) {
    return ctx ? ctx->error.c_str() : g_error.c_str();
}

extern "C" int wos_context_create(int device, wos_context **out) {
    if (!out) return fail(nullptr, WOS_ERR_INVALID, "wos_context_create: null output");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDeviceCount");
    if (device < 0 || device >= count) {
        return fail(nullptr, WOS_ERR_INVALID, "wos_context_create: no CUDA device " +
                                                  std::to_string(device));
    }
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
    auto *ctx = new wos_context();
    ctx->device = device;
    cudaDeviceProp prop{};
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_fail(nullptr, e, "cudaGetDeviceProperties");
    }
    ctx->sms = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    ctx->cc_major = prop.major;
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_fail(nullptr, e, "cudaStreamCreate");
    }
    for (auto &ev : ctx->events) {
        e = cudaEventCreate(&ev);
        if (e != cudaSuccess) {
            delete ctx;
            return cuda_fail(nullptr, e, "cudaEventCreate");
        }
    }
    // the allocation-free entry point's scratch array: looking its address
    // up here loads (and so reserves) it now, while allocating is allowed
    e = noalloc_scratch_address(&ctx->noalloc_scratch);
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_fail(nullptr, e, "cudaGetSymbolAddress (static scratch array)");
    }
    *out = ctx;
    return WOS_OK;
}

extern "C" void wos_context_destroy(wos_context *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (wos_batch *b : ctx->batches) detach_batch(b);
    ctx->batches.clear();
    delete ctx;
}

// ------------------------------------------------------------- mesh

// One device allocation per scene (arrays at 256-byte aligned offsets): a
// set_mesh or batch mesh costs one cudaMalloc instead of one per array.
cudaError_t SceneDevice::upload(const HostScene &h, cudaStream_t stream) {
    const ArenaLayout L = arena_layout(h);
    const std::vector<int> off(h.w_off, h.w_off + 8);
    const void *src[ArenaLayout::kParts] = {h.box64.data(), h.seg64.data(), h.segid.data(),
                                            h.tri64.data(), h.wbox.data(), h.wprim.data(),
                                            h.wide2bin.data(), off.data(), h.slot_verts.data()};
    const size_t have[ArenaLayout::kParts] = {
        h.box64.size() * sizeof(double), h.seg64.size() * sizeof(double),
        h.segid.size() * sizeof(int), h.tri64.size() * sizeof(double),
        h.wbox.size() * sizeof(float), h.wprim.size() * sizeof(float),
        h.wide2bin.size() * sizeof(int), off.size() * sizeof(int),
        h.slot_verts.size() * sizeof(int)};
    for (int k = 0; k < ArenaLayout::kParts; ++k) {
        if (have[k] != L.bytes[k]) return cudaErrorInvalidValue;  // a builder bug
    }
    cudaError_t e = arena.reserve(L.total);
    if (e != cudaSuccess) return e;
    auto *base = static_cast<char *>(arena.ptr);
    if ((e = cudaMemsetAsync(base, 0, L.total, stream)) != cudaSuccess) return e;
    for (int k = 0; k < ArenaLayout::kParts; ++k) {
        if (L.bytes[k] == 0) continue;
        e = cudaMemcpyAsync(base + L.offset[k], src[k], L.bytes[k], cudaMemcpyHostToDevice,
                            stream);
        if (e != cudaSuccess) return e;
    }
    // no wait: a copy from pageable memory returns once its source is staged,
    // and every later use of the scene is ordered after it on `stream`
    set_views(h);
    return build_lattice(h, stream);
}

bool SceneDevice::lists_needed(float t) const {
    if (wide.gd == nullptr || !(t > 0.0f)) return false;
    if (const char *env = std::getenv("WOS_NEAR_LISTS")) {
        if (std::string(env) == "0") return false;
    }
    return !(wide.gl != nullptr && list_built >= t);
}

cudaError_t SceneDevice::lists_count(float t, cudaStream_t stream) {
    const float tb = t * 1.25f;
    const size_t nodes = static_cast<size_t>(wide.gn[0]) * wide.gn[1] * wide.gn[2];
    cudaError_t e = glist.reserve(nodes * sizeof(int2));
    if (e != cudaSuccess) return e;
    if ((e = gcount.reserve(2 * sizeof(unsigned))) != cudaSuccess) return e;
    return launch_near_band(wide, tb, static_cast<unsigned *>(gcount.ptr), stream);
}

cudaError_t SceneDevice::lists_build(float t, unsigned band, int sms, cudaStream_t stream) {
    const float tb = t * 1.25f;
    auto *count = static_cast<unsigned *>(gcount.ptr);
    WideView w = wide;
    w.gk = near_list_capacity(w.dim);
    if (const char *env = std::getenv("WOS_NEAR_CAPACITY")) {
        const int k = std::atoi(env);
        if (k >= 1 && k <= 32) w.gk = k;
    }
    // K slots per band node bound the packed lists; list offsets sit above
    // a 5-bit length in an int, so the pool has at most 2^26 slots (nodes
    // beyond it get no list and query the tree instead)
    const size_t slots = std::min<size_t>(std::max<size_t>(band, 1) * w.gk, size_t(1) << 26);
    cudaError_t e = gpool.reserve(slots * sizeof(int));
    if (e != cudaSuccess) return e;
    // a point is within r_max of its nearest node; 8 lattice margins cover
    // the FP32 rounding of the distances
    const double rmax = 0.5 * w.gh * std::sqrt(static_cast<double>(w.dim)) * (1.0 + 1e-3);
    const float extra = static_cast<float>(2.0 * rmax + 8.0 * lattice_margin);
    // list_prefix's buckets: the same rounding margin as the list radius
    const float slack = static_cast<float>(8.0 * lattice_margin);
    if ((e = launch_near_lists(w, tb, extra, static_cast<float>(rmax), slack,
                               static_cast<int2 *>(glist.ptr), static_cast<int *>(gpool.ptr),
                               static_cast<int>(slots), count + 1, sms, stream)) !=
        cudaSuccess) {
        return e;
    }
    if (wide.aos == nullptr) {
        if ((e = gaos.reserve(prim_aos_bytes(w))) != cudaSuccess) return e;
        if ((e = launch_prim_aos(w, static_cast<float *>(gaos.ptr), stream)) != cudaSuccess) {
            return e;
        }
    }
    wide.gk = w.gk;
    wide.gl = static_cast<const int2 *>(glist.ptr);
    wide.gbinv = static_cast<float>((kListBuckets + 1) / rmax);
    if (const char *env = std::getenv("WOS_LIST_CUT")) {
        // every query past the node itself scans its whole list (the cut
        // never changes a query's answer; this checks that)
        if (std::string(env) == "0") wide.gbinv = 0x1p100f;
    }
    wide.gpool = static_cast<const int *>(gpool.ptr);
    wide.aos = static_cast<const float4 *>(gaos.ptr);
    list_built = tb;
    return cudaSuccess;
}

cudaError_t SceneDevice::ensure_lists(float t, int sms, cudaStream_t stream) {
    if (!lists_needed(t)) return cudaSuccess;
    cudaError_t e = lists_count(t, stream);
    if (e != cudaSuccess) return e;
    unsigned band = 0;
    if ((e = cudaMemcpyAsync(&band, gcount.ptr, sizeof(band), cudaMemcpyDeviceToHost, stream)) !=
        cudaSuccess) {
        return e;
    }
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
    return lists_build(t, band, sms, stream);
}

void SceneDevice::set_views(const HostScene &h) {
    list_built = -1.0f;
    const ArenaLayout L = arena_layout(h);
    auto *base = static_cast<char *>(arena.ptr);
    auto at = [&](int k) { return static_cast<const void *>(base + L.offset[k]); };
    view = SceneView{};
    view.dim = h.dim;
    view.n_prims = h.n_prims;
    view.depth = h.depth;
    view.box64 = static_cast<const double *>(at(0));
    view.seg64 = static_cast<const double2 *>(at(1));
    view.segid = static_cast<const int2 *>(at(2));
    view.tri64 = static_cast<const double2 *>(at(3));
    wide = WideView{};
    wide.dim = h.dim;
    wide.H = h.wH;
    wide.n = h.n_prims;
    wide.npad = h.w_npad;
    wide.box_total = h.w_box_total;
    wide.off = static_cast<const int *>(at(7));
    wide.box = static_cast<const float *>(at(4));
    wide.prim = static_cast<const float *>(at(5));
    wide.wide2bin = static_cast<const int *>(at(6));
    slot_verts = static_cast<const int *>(at(8));
}

// The distance lattice of the FAST_FP32 walks (device/wide.cuh): nodes
// spaced h = (largest bbox extent) / (G - 1) over the bounding box, G = 2048
// in 2D and 256 in 3D (16 MB and 64 MB for a square / cubic box), distances
// at the nodes' FP32 positions from the conservative FP32 cooperative query
// (2D) or from warp tiles' candidate scans over the contiguous records,
// which are made first (3D; launch_lattice32).  Meshes of at most lane_prims
// primitives query exactly at every step and get none; WOS_BOUND_GRID=0
// turns it off.
cudaError_t SceneDevice::build_lattice(const HostScene &h, cudaStream_t stream) {
    wide.gd = nullptr;
    if (h.n_prims <= lane_prims(h.dim)) return cudaSuccess;
    if (const char *env = std::getenv("WOS_BOUND_GRID")) {
        if (std::string(env) == "0") return cudaSuccess;
    }
    const int G = h.dim == 2 ? 2048 : 256;
    double ext = 0.0, mag = 0.0;
    for (int k = 0; k < h.dim; ++k) {
        ext = std::max(ext, h.bbox[2 * k + 1] - h.bbox[2 * k]);
        mag = std::max({mag, std::fabs(h.bbox[2 * k]), std::fabs(h.bbox[2 * k + 1])});
    }
    if (!(ext > 0.0)) return cudaSuccess;
    const double step = ext / (G - 1);
    int n[3] = {1, 1, 1};
    for (int k = 0; k < h.dim; ++k) {
        n[k] = static_cast<int>(std::ceil((h.bbox[2 * k + 1] - h.bbox[2 * k]) / step)) + 1;
        wide.glo[k] = static_cast<float>(h.bbox[2 * k]);
    }
    for (int k = 0; k < 3; ++k) wide.gn[k] = n[k];
    if (h.dim == 2) wide.glo[2] = 0.0f;
    wide.gh = static_cast<float>(step);
    wide.ginv = static_cast<float>(1.0 / step);
    // FP32 primitive distances carry a few ulps of the largest coordinate
    const float margin = fp32_distance_margin(h.bbox, h.dim);
    lattice_margin = margin;
    const size_t count = static_cast<size_t>(n[0]) * n[1] * n[2];
    cudaError_t e = lattice.reserve(sizeof(float) * count);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) {
        return e;
    }
    auto *out = static_cast<float *>(lattice.ptr);
    const char *tiles_env = std::getenv("WOS_LATTICE_TILES");
    if (h.dim == 3 && !(tiles_env && std::string(tiles_env) == "0")) {
        // the 3D tile build scans candidates from the contiguous records
        // (kept for the near-boundary list scans); WOS_LATTICE_TILES=0
        // builds lattice and lists node by node instead
        if ((e = gaos.reserve(prim_aos_bytes(wide))) != cudaSuccess) return e;
        if ((e = launch_prim_aos(wide, static_cast<float *>(gaos.ptr), stream)) != cudaSuccess) {
            return e;
        }
        wide.aos = static_cast<const float4 *>(gaos.ptr);
    }
    // outside-node skip: its row crossings and node mask live in a
    // stream-ordered temporary (WOS_LATTICE_SKIP=0 queries every node)
    void *skip = nullptr;
    const char *skip_env = std::getenv("WOS_LATTICE_SKIP");
    if (!(skip_env && std::string(skip_env) == "0")) {
        if ((e = cudaMallocAsync(&skip, lattice_skip_bytes(wide), stream)) != cudaSuccess) return e;
    }
    const double tol = 1e-5 * std::max(mag, ext);
    e = launch_lattice32(view, wide, margin, out, sms, skip, tol, stream);
    if (skip) {
        const cudaError_t f = cudaFreeAsync(skip, stream);
        if (e == cudaSuccess) e = f;
    }
    if (e != cudaSuccess) return e;
    wide.gd = out;
    wide.gratio = 2.0f;  // bound >= 1/3 of the upper bound
    if (const char *env = std::getenv("WOS_LATTICE_RATIO")) {
        const double r = std::atof(env);
        if (r >= 1.0) wide.gratio = static_cast<float>(r);
    }
    return cudaSuccess;
}

void SceneDevice::release() {
    arena.release();
    lattice.release();
    glist.release();
    gpool.release();
    gcount.release();
    gaos.release();
    list_built = -1.0f;
    slot_verts = nullptr;
}

bool wosb::device_tree_build(bool batch) {
    const char *e = std::getenv("WOS_TREE_BUILD");
    if (e && std::string(e) == "host") return false;
    if (e && std::string(e) == "device") return true;
    return !batch;
}

int wos_context::upload_scene() {
    cudaSetDevice(device);
    if (scene.box64.empty()) {
        WOS_CUDA(this, sdev.build_on_device(scene, stream), "device tree build");
    } else {
        WOS_CUDA(this, sdev.upload(scene, stream), "mesh upload");
    }
    view = sdev.view;
    wide = sdev.wide;
    has_mesh = true;
    return WOS_OK;
}

extern "C" int wos_set_mesh(wos_context *ctx, int dim, const double *verts, int n_verts,
                            const int *prims, int n_prims, const int *boundary_ids,
                            int leaf_size) {
    if (!ctx) return fail(nullptr, WOS_ERR_INVALID, "wos_set_mesh: null context");
    HostScene sc;
    // the device build needs only the checked mesh and its metadata
    const std::string err =
        device_tree_build(false)
            ? scene_meta(dim, verts, n_verts, prims, n_prims, boundary_ids, leaf_size, sc)
            : build_scene(dim, verts, n_verts, prims, n_prims, boundary_ids, leaf_size, sc);
    if (!err.empty()) return fail(ctx, WOS_ERR_MESH, "Mesh: " + err);
    ctx->scene = std::move(sc);
    ctx->has_mesh = false;
    return ctx->upload_scene();
}

extern "C" int wos_scene_arena(wos_context *ctx, void *out, long long capacity,
                               long long *bytes) {
    if (!ctx || !ctx->has_mesh) return fail(ctx, WOS_ERR_INVALID, "wos_scene_arena: no mesh");
    const ArenaLayout L = arena_layout(ctx->scene);
    if (bytes) *bytes = static_cast<long long>(L.total);
    if (!out) return WOS_OK;
    if (capacity < static_cast<long long>(L.total)) {
        return fail(ctx, WOS_ERR_INVALID, "wos_scene_arena: buffer too small");
    }
    cudaSetDevice(ctx->device);
    WOS_CUDA(ctx, cudaMemcpyAsync(out, ctx->sdev.arena.ptr, L.total, cudaMemcpyDeviceToHost,
                                  ctx->stream), "D2H");
    WOS_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "scene arena");
    return WOS_OK;
}

extern "C" int wos_load_obj(wos_context *ctx, const char *path, int leaf_size) {
    if (!ctx) return fail(nullptr, WOS_ERR_INVALID, "wos_load_obj: null context");
    ObjMesh m;
    const std::string err = read_obj(path, m);
    if (!err.empty()) return fail(ctx, WOS_ERR_MESH, err);
    return wos_set_mesh(ctx, m.dim, m.verts.data(), m.n_verts(), m.prims.data(), m.n_prims(),
                        m.dim == 2 ? m.boundary_ids.data() : nullptr, leaf_size);
}

extern "C" int wos_mesh_info(const wos_context *ctx, int *dim, int *n_prims, double bbox[6]) {
    if (!ctx || !ctx->has_mesh) return fail(nullptr, WOS_ERR_INVALID, "wos_mesh_info: no mesh");
    if (dim) *dim = ctx->scene.dim;
    if (n_prims) *n_prims = ctx->scene.n_prims;
    if (bbox) std::memcpy(bbox, ctx->scene.bbox, sizeof(double) * 6);
    return WOS_OK;
}

extern "C" int wos_grid_over_mesh(const wos_context *ctx, int Nx, int Ny, int Nz,
                                  wos_grid *grid) {
    if (!ctx || !ctx->has_mesh || !grid) {
        return fail(nullptr, WOS_ERR_INVALID, "wos_grid_over_mesh: no mesh or null grid");
    }
    grid->Nx = Nx;
    grid->Ny = Ny;
    grid->Nz = ctx->scene.dim == 2 ? 1 : Nz;
    grid->xmin = ctx->scene.bbox[0];
    grid->xmax = ctx->scene.bbox[1];
    grid->ymin = ctx->scene.bbox[2];
    grid->ymax = ctx->scene.bbox[3];
    grid->zmin = ctx->scene.bbox[4];
    grid->zmax = ctx->scene.bbox[5];
    return WOS_OK;
}

// ------------------------------------------------------------- solve

double wosb::effective_epsilon(const wos_params &p) {
    // src/equations/screened_poisson.cpp:22-38
    if (p.equation == WOS_EQ_SCREENED_POISSON) {
        const double limit = 0.05 / p.alpha;
        return std::min(p.epsilon, limit);
    }
    return p.epsilon;
}

std::string wosb::check_params(const wos_context *ctx, const wos_params *p) {
    if (!p) return "null params";
    if (!ctx->has_mesh) return "no mesh uploaded";
    if (p->equation < 0 || p->equation > 3) return "unknown equation kind";
    if (p->source_mode == WOS_SOURCE_MIS &&
        (p->equation == WOS_EQ_POISSON || p->equation == WOS_EQ_SCREENED_POISSON)) {
        // include/wos/wos.hpp:83-92: no registry equation has a source proposal
        return "GreenSourceMIS requires a source proposal sampler and PDF";
    }
    if (p->source_mode < 0 || p->source_mode > 2) return "source_mode must be 0, 1 or 2";
    if (p->N_walks < 1) return "N_walks must be >= 1";
    if (!(p->epsilon > 0.0) || !std::isfinite(p->epsilon)) return "epsilon must be positive";
    if (p->max_steps < 1) return "max_steps must be >= 1";
    if (p->max_ray_attempts < 3) return "max_ray_attempts must be >= 3";
    if (p->equation == WOS_EQ_SCREENED_POISSON && (!(p->alpha > 0.0) || !std::isfinite(p->alpha))) {
        return "alpha must be positive";
    }
    if (p->method < 0 || p->method > 2) return "unknown method";
    return std::string();
}

int wos_context::run(const wos_params &p, const PointSet &ps, Fields out,
                     wos_counters *counters_out) {
    cudaSetDevice(device);
    const long long n = ps.n;
    const int dim = scene.dim;
    WOS_CUDA(this, location.reserve(std::max<long long>(n, 1)), "alloc location");
    WOS_CUDA(this, start.reserve(sizeof(StartRecord) * std::max<long long>(n, 1)), "alloc start");
    WOS_CUDA(this, counters.reserve(sizeof(DeviceCounters)), "alloc counters");
    WOS_CUDA(this, cudaMemsetAsync(counters.ptr, 0, sizeof(DeviceCounters), stream),
             "clear counters");

    EqDesc eq{p.equation, p.source_mode, p.alpha, nullptr};
    const double eps = effective_epsilon(p);
    // boundary tolerance 1e-10 * max(1, mesh extents), include/wos/runner.hpp:86-88
    const double btol = 1e-10 * scene.scale;
    if (p.method == WOS_METHOD_FAST_FP32) {
        // near-boundary lists for this epsilon (one-time set-up per mesh)
        const float t = near_list_threshold(sdev.wide, eps, std::ldexp(scene.scale, -16));
        WOS_CUDA(this, sdev.ensure_lists(t, sms, stream), "near-boundary lists");
        wide = sdev.wide;
    }
    auto *loc = static_cast<uint8_t *>(location.ptr);
    auto *st = static_cast<StartRecord *>(start.ptr);
    auto *ctr = static_cast<DeviceCounters *>(counters.ptr);

    WOS_CUDA(this, cudaEventRecord(events[0], stream), "event");
    FastStart fs;
    if (p.method == WOS_METHOD_FAST_FP32) {
        fs.on = true;
        fs.w = wide;
        fs.exact_below = std::max(eps, btol);
        fs.margin = fp32_distance_margin(scene.bbox, dim);
    }
    WOS_CUDA(this, launch_classify(view, ps, p.seed, p.max_ray_attempts, btol,
                                   eq, out, loc, st, ctr, stream, fs),
             "classification kernel");
    WOS_CUDA(this, cudaEventRecord(events[1], stream), "event");
    if (p.method == WOS_METHOD_PLAIN_FP64) {
        WOS_CUDA(this, launch_walk_plain(view, ps, p.seed, eq, p.N_walks, eps, p.max_steps, loc,
                                         st, out, ctr, stream),
                 "plain walk kernel");
    } else {
        const int precision = p.method == WOS_METHOD_FAST_FP32 ? 32 : 64;
        FastPlan plan = plan_fast(view, wide, n, p.N_walks, precision, sms, smem_optin);
        set_chunk(plan, chunk_override > 0 ? chunk_override : plan.chunk, p.N_walks, p.max_steps,
                  n);
        if (blocks_override > 0) plan.blocks = blocks_override;
        WOS_CUDA(this, partials.reserve(sizeof(TaskPartial) * std::max<long long>(plan.n_tasks, 1)),
                 "alloc partials");
        WOS_CUDA(this, queue.reserve(sizeof(unsigned long long)), "alloc queue");
        // FP32 error margin of the shell test: positions, vertices and the
        // query arithmetic carry ~1e-7 relative error of the mesh scale.
        const double shell_delta = std::ldexp(scene.scale, -16);
        WOS_CUDA(this, launch_walk_fast(view, wide, ps, p.seed, eq, p.N_walks, eps, p.max_steps,
                                        shell_delta, precision, plan, loc, st,
                                        static_cast<TaskPartial *>(partials.ptr),
                                        static_cast<unsigned long long *>(queue.ptr), out, ctr,
                                        stream, events[2]),
                 "fast walk kernel");
    }
    if (p.method == WOS_METHOD_PLAIN_FP64) WOS_CUDA(this, cudaEventRecord(events[2], stream), "event");
    WOS_CUDA(this, cudaEventRecord(events[3], stream), "event");
    DeviceCounters hc{};
    WOS_CUDA(this, cudaMemcpyAsync(&hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost, stream),
             "read counters");
    WOS_CUDA(this, cudaStreamSynchronize(stream), "solve");
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
        c.effective_epsilon = eps;
        cudaEventElapsedTime(&c.classify_ms, events[0], events[1]);
        cudaEventElapsedTime(&c.walk_ms, events[1], events[2]);
        cudaEventElapsedTime(&c.total_ms, events[0], events[3]);
    }
    (void)dim;
    return WOS_OK;
}

PointSet wosb::grid_points(int dim, const wos_grid &g) {
    PointSet ps{};
    ps.dim = dim;
    ps.Nx = g.Nx;
    ps.Ny = g.Ny;
    ps.Nz = dim == 2 ? 1 : g.Nz;
    ps.lo[0] = g.xmin;
    ps.hi[0] = g.xmax;
    ps.lo[1] = g.ymin;
    ps.hi[1] = g.ymax;
    ps.lo[2] = dim == 3 ? g.zmin : 0.0;
    ps.hi[2] = dim == 3 ? g.zmax : 0.0;
    ps.n = static_cast<long long>(ps.Nx) * ps.Ny * ps.Nz;
    return ps;
}

std::string wosb::check_grid(int dim, const wos_grid *g) {
    if (!g) return "null grid";
    if (g->Nx < 1 || g->Ny < 1 || (dim == 3 && g->Nz < 1)) return "grid sizes must be >= 1";
    const double v[6] = {g->xmin, g->xmax, g->ymin, g->ymax, g->zmin, g->zmax};
    for (double x : v) {
        if (!std::isfinite(x)) return "grid bounds must be finite";
    }
    return std::string();
}

extern "C" int wos_solve_grid_device(wos_context *ctx, const wos_params *params,
                                     const wos_grid *grid, double *mean, double *variance,
                                     double *standard_error, double *mean_steps,
                                     uint8_t *location, wos_counters *counters) {
    if (!ctx) return fail(nullptr, WOS_ERR_INVALID, "null context");
    std::string err = check_params(ctx, params);
    if (err.empty()) err = check_grid(ctx->scene.dim, grid);
    if (!err.empty()) return fail(ctx, WOS_ERR_INVALID, "wos_solve_grid: " + err);
    const PointSet ps = grid_points(ctx->scene.dim, *grid);
    Fields out{mean, variance, standard_error, mean_steps, location};
    return ctx->run(*params, ps, out, counters);
}

int wos_context::fields_for(long long n, Fields &out) {
    WOS_CUDA(this, f_mean.reserve(sizeof(double) * std::max<long long>(n, 1)), "alloc mean");
    WOS_CUDA(this, f_var.reserve(sizeof(double) * std::max<long long>(n, 1)), "alloc variance");
    WOS_CUDA(this, f_se.reserve(sizeof(double) * std::max<long long>(n, 1)), "alloc se");
    WOS_CUDA(this, f_steps.reserve(sizeof(double) * std::max<long long>(n, 1)), "alloc steps");
    WOS_CUDA(this, f_loc.reserve(std::max<long long>(n, 1)), "alloc location");
    out = Fields{static_cast<double *>(f_mean.ptr), static_cast<double *>(f_var.ptr),
                 static_cast<double *>(f_se.ptr), static_cast<double *>(f_steps.ptr),
                 static_cast<uint8_t *>(f_loc.ptr)};
    return WOS_OK;
}

int wos_context::download(long long n, const Fields &dev, double *mean, double *variance,
                          double *se, double *steps, uint8_t *loc) {
    const size_t b = sizeof(double) * static_cast<size_t>(n);
    if (mean) WOS_CUDA(this, cudaMemcpyAsync(mean, dev.mean, b, cudaMemcpyDeviceToHost, stream), "D2H");
    if (variance) WOS_CUDA(this, cudaMemcpyAsync(variance, dev.variance, b, cudaMemcpyDeviceToHost, stream), "D2H");
    if (se) WOS_CUDA(this, cudaMemcpyAsync(se, dev.standard_error, b, cudaMemcpyDeviceToHost, stream), "D2H");
    if (steps) WOS_CUDA(this, cudaMemcpyAsync(steps, dev.mean_steps, b, cudaMemcpyDeviceToHost, stream), "D2H");
    if (loc) WOS_CUDA(this, cudaMemcpyAsync(loc, dev.location, static_cast<size_t>(n), cudaMemcpyDeviceToHost, stream), "D2H");
    WOS_CUDA(this, cudaStreamSynchronize(stream), "D2H");
    return WOS_OK;
}

// Host-side diagnostics in grid order (include/wos/runner.hpp:203-236, 265-274).
static void host_sums(long long n, const double *var, const double *se, const double *steps,
                      const uint8_t *loc, wos_counters *c) {
    if (!c || !loc) return;
    double sv = 0.0, ss = 0.0, st = 0.0;
    long long inside = 0;
    for (long long t = 0; t < n; ++t) {
        if (loc[t] != WOS_INSIDE) continue;
        ++inside;
        sv += var ? var[t] : 0.0;
        ss += se ? se[t] : 0.0;
        st += steps ? steps[t] : 0.0;
    }
    c->inside_points = inside;
    c->sum_variance = sv;
    c->sum_standard_error = ss;
    c->sum_mean_steps = st;
}

extern "C" int wos_solve_grid(wos_context *ctx, const wos_params *params, const wos_grid *grid,
                              double *mean, double *variance, double *standard_error,
                              double *mean_steps, uint8_t *location, wos_counters *counters) {
    if (!ctx) return fail(nullptr, WOS_ERR_INVALID, "null context");
    std::string err = check_params(ctx, params);
    if (err.empty()) err = check_grid(ctx->scene.dim, grid);
    if (!err.empty()) return fail(ctx, WOS_ERR_INVALID, "wos_solve_grid: " + err);
    cudaSetDevice(ctx->device);
    const PointSet ps = grid_points(ctx->scene.dim, *grid);
    Fields dev{};
    int rc = ctx->fields_for(ps.n, dev);
    if (rc) return rc;
    rc = ctx->run(*params, ps, dev, counters);
    if (rc) return rc;
    // the diagnostics need the location and statistics even when the caller
    // skips them
    std::vector<double> tv, ts, tst;
    std::vector<uint8_t> tl;
    double *v = variance, *s = standard_error, *m = mean_steps;
    uint8_t *l = location;
    if (counters) {
        if (!v) { tv.resize(ps.n); v = tv.data(); }
        if (!s) { ts.resize(ps.n); s = ts.data(); }
        if (!m) { tst.resize(ps.n); m = tst.data(); }
        if (!l) { tl.resize(ps.n); l = tl.data(); }
    }
    rc = ctx->download(ps.n, dev, mean, v, s, m, l);
    if (rc) return rc;
    host_sums(ps.n, v, s, m, l, counters);
    return WOS_OK;
}

extern "C" int wos_solve_points(wos_context *ctx, const wos_params *params, const double *points,
                                const uint64_t *point_index, long long n, double *mean,
                                double *variance, double *standard_error, double *mean_steps,
                                uint8_t *location, wos_counters *counters) {
    if (!ctx) return fail(nullptr, WOS_ERR_INVALID, "null context");
    std::string err = check_params(ctx, params);
    if (err.empty() && (!points || n < 0)) err = "null points";
    // a non-finite point has no place in the domain; reject it here rather
    // than hand it to the traversals
    for (long long i = 0; err.empty() && i < n * ctx->scene.dim; ++i) {
        if (!std::isfinite(points[i])) err = "point coordinates must be finite";
    }
    if (!err.empty()) return fail(ctx, WOS_ERR_INVALID, "wos_solve_points: " + err);
    cudaSetDevice(ctx->device);
    const int dim = ctx->scene.dim;
    PointSet ps{};
    ps.dim = dim;
    ps.n = n;
    ps.Nx = ps.Ny = ps.Nz = 1;
    // the boundary tolerance scale follows the mesh box (runner.hpp:86-88)
    for (int k = 0; k < 3; ++k) {
        ps.lo[k] = ctx->scene.bbox[2 * k];
        ps.hi[k] = ctx->scene.bbox[2 * k + 1];
    }
    WOS_CUDA(ctx, ctx->points.reserve(sizeof(double) * dim * std::max<long long>(n, 1)), "alloc points");
    WOS_CUDA(ctx, cudaMemcpyAsync(ctx->points.ptr, points, sizeof(double) * dim * n,
                                  cudaMemcpyHostToDevice, ctx->stream), "H2D points");
    ps.coords = static_cast<const double *>(ctx->points.ptr);
    if (point_index) {
        WOS_CUDA(ctx, ctx->index.reserve(sizeof(uint64_t) * std::max<long long>(n, 1)), "alloc index");
        WOS_CUDA(ctx, cudaMemcpyAsync(ctx->index.ptr, point_index, sizeof(uint64_t) * n,
                                      cudaMemcpyHostToDevice, ctx->stream), "H2D index");
        ps.index = static_cast<const uint64_t *>(ctx->index.ptr);
    }
    Fields dev{};
    int rc = ctx->fields_for(n, dev);
    if (rc) return rc;
    rc = ctx->run(*params, ps, dev, counters);
    if (rc) return rc;
    return ctx->download(n, dev, mean, variance, standard_error, mean_steps, location);
}

// ------------------------------------------------------------- checks

extern "C" int wos_prng_u64(wos_context *ctx, const uint64_t *seeds, long long n_seeds, int count,
                            uint64_t *out) {
    if (!ctx || !seeds || !out || n_seeds < 0 || count < 0) {
        return fail(ctx, WOS_ERR_INVALID, "wos_prng_u64: bad arguments");
    }
    cudaSetDevice(ctx->device);
    WOS_CUDA(ctx, ctx->scratch_a.reserve(sizeof(uint64_t) * std::max<long long>(n_seeds, 1)), "alloc");
    WOS_CUDA(ctx, ctx->scratch_b.reserve(sizeof(uint64_t) * std::max<long long>(n_seeds * count, 1)), "alloc");
    WOS_CUDA(ctx, cudaMemcpyAsync(ctx->scratch_a.ptr, seeds, sizeof(uint64_t) * n_seeds,
                                  cudaMemcpyHostToDevice, ctx->stream), "H2D");
    WOS_CUDA(ctx, launch_prng(static_cast<const uint64_t *>(ctx->scratch_a.ptr), n_seeds, count,
                              static_cast<uint64_t *>(ctx->scratch_b.ptr), ctx->stream), "prng kernel");
    WOS_CUDA(ctx, cudaMemcpyAsync(out, ctx->scratch_b.ptr, sizeof(uint64_t) * n_seeds * count,
                                  cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    WOS_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "prng");
    return WOS_OK;
}

extern "C" int wos_special_functions(wos_context *ctx, int precision, const double *x,
                                     long long n, double *log_i0, double *log_k0) {
    if (!ctx || !x || !log_i0 || !log_k0 || n < 0 || (precision != 32 && precision != 64)) {
        return fail(ctx, WOS_ERR_INVALID, "wos_special_functions: bad arguments");
    }
    cudaSetDevice(ctx->device);
    const long long m = std::max<long long>(n, 1);
    WOS_CUDA(ctx, ctx->scratch_a.reserve(sizeof(double) * m), "alloc");
    WOS_CUDA(ctx, ctx->scratch_b.reserve(sizeof(double) * m), "alloc");
    WOS_CUDA(ctx, ctx->scratch_c.reserve(sizeof(double) * m), "alloc");
    WOS_CUDA(ctx, cudaMemcpyAsync(ctx->scratch_a.ptr, x, sizeof(double) * n,
                                  cudaMemcpyHostToDevice, ctx->stream), "H2D");
    auto *di = static_cast<double *>(ctx->scratch_b.ptr);
    auto *dk = static_cast<double *>(ctx->scratch_c.ptr);
    WOS_CUDA(ctx, launch_special(precision, static_cast<const double *>(ctx->scratch_a.ptr), n,
                                 di, dk, ctx->stream),
             "special-function kernel");
    WOS_CUDA(ctx, cudaMemcpyAsync(log_i0, di, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                  ctx->stream), "D2H");
    WOS_CUDA(ctx, cudaMemcpyAsync(log_k0, dk, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                  ctx->stream), "D2H");
    WOS_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "special functions");
    return WOS_OK;
}

extern "C" int wos_distance_bounds(wos_context *ctx, const double *points, long long n,
                                   double *bound) {
    if (!ctx || !ctx->has_mesh || !points || !bound || n < 0) {
        return fail(ctx, WOS_ERR_INVALID, "wos_distance_bounds: bad arguments");
    }
    cudaSetDevice(ctx->device);
    const int dim = ctx->scene.dim;
    const long long m = std::max<long long>(n, 1);
    WOS_CUDA(ctx, ctx->scratch_a.reserve(sizeof(double) * dim * m), "alloc");
    WOS_CUDA(ctx, ctx->scratch_b.reserve(sizeof(double) * m), "alloc");
    WOS_CUDA(ctx, cudaMemcpyAsync(ctx->scratch_a.ptr, points, sizeof(double) * dim * n,
                                  cudaMemcpyHostToDevice, ctx->stream), "H2D");
    WOS_CUDA(ctx, launch_lattice_bounds(ctx->wide, static_cast<const double *>(ctx->scratch_a.ptr),
                                        n, static_cast<double *>(ctx->scratch_b.ptr), ctx->stream),
             "lattice kernel");
    WOS_CUDA(ctx, cudaMemcpyAsync(bound, ctx->scratch_b.ptr, sizeof(double) * n,
                                  cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    WOS_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "distance bounds");
    return WOS_OK;
}

extern "C" int wos_closest_points(wos_context *ctx, int precision, const double *points,
                                  long long n, double *dist, double *nearest, int *boundary_id) {
    if (!ctx || !ctx->has_mesh || !points || !dist || !nearest || n < 0 ||
        (precision != 32 && precision != 64)) {
        return fail(ctx, WOS_ERR_INVALID, "wos_closest_points: bad arguments");
    }
    cudaSetDevice(ctx->device);
    const int dim = ctx->scene.dim;
    const long long m = std::max<long long>(n, 1);
    WOS_CUDA(ctx, ctx->scratch_a.reserve(sizeof(double) * dim * m), "alloc");
    WOS_CUDA(ctx, ctx->scratch_b.reserve(sizeof(double) * m), "alloc");
    WOS_CUDA(ctx, ctx->scratch_c.reserve(sizeof(double) * dim * m), "alloc");
    WOS_CUDA(ctx, ctx->scratch_d.reserve(sizeof(int) * m), "alloc");
    WOS_CUDA(ctx, cudaMemcpyAsync(ctx->scratch_a.ptr, points, sizeof(double) * dim * n,
                                  cudaMemcpyHostToDevice, ctx->stream), "H2D");
    auto *dp = static_cast<const double *>(ctx->scratch_a.ptr);
    auto *dd = static_cast<double *>(ctx->scratch_b.ptr);
    auto *dn = static_cast<double *>(ctx->scratch_c.ptr);
    auto *db = static_cast<int *>(ctx->scratch_d.ptr);
    cudaError_t e = precision == 64 ? launch_closest64(ctx->view, dp, n, dd, dn, db, ctx->stream)
                                    : launch_closest32(ctx->view, ctx->wide, dp, n, dd, dn, db, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "closest-point kernel");
    WOS_CUDA(ctx, cudaMemcpyAsync(dist, dd, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    WOS_CUDA(ctx, cudaMemcpyAsync(nearest, dn, sizeof(double) * dim * n, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    if (boundary_id) {
        WOS_CUDA(ctx, cudaMemcpyAsync(boundary_id, db, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    }
    WOS_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "closest points");
    return WOS_OK;
}

// Tuning knobs for the benchmark's autotuner (not part of the reference
// interface): walks per task, persistent grid size, boundary tolerance.
extern "C" int wos_set_tuning(wos_context *ctx, int chunk, int blocks) {
    if (!ctx) return fail(nullptr, WOS_ERR_INVALID, "null context");
    ctx->chunk_override = chunk;
    ctx->blocks_override = blocks;
    return WOS_OK;
}
