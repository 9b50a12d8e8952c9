// C ABI of solve batches (include/wos_b200.h): many grid sweeps of different
// meshes, grids, equations and walk counts in one launch sequence.
//
// Layout.  Solves are ordered by (dimension, equation kind, precision); the
// order defines the batch's point numbering (2D solves first, so each
// dimension's points are one contiguous range for its classification
// launch) and the walk families (contiguous runs of one kind and precision,
// each with its own task queue numbered from 0).  Every solve owns a slice
// of the concatenated location / start / field / partial buffers and one
// DeviceCounters record; its BatchItem carries the pointers to them.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/wos_b200.h"
#include "context_internal.h"
#include "kernels.h"

using namespace wosb;

namespace {

// A mesh is checked when it is added and built later, with the batch's
// other pending meshes, in parallel (wos_batch::prepare).
struct BatchMesh {
    int dim = 0;
    int leaf_size = 0;
    std::vector<double> verts;   // inputs until built
    std::vector<int> prims, bids;
    bool built = false;
    HostScene scene;
    SceneDevice dev;
};

struct BatchSolve {
    int mesh;
    wos_params p;
    wos_grid g;
    long long n;            // grid points
    long long point_begin;  // in batch order
    long long task_off;     // first partial record
    int item;               // index in the item order
};

struct Family {
    int dim, kind, precision, hc;
    int first, count;  // items
    long long n_tasks;
    int blocks;
};

}  // namespace

struct wos_batch {
    wos_context *ctx = nullptr;
    std::vector<std::unique_ptr<BatchMesh>> meshes;
    std::vector<BatchSolve> solves;
    int chunk_override = 0;
    int blocks_override = 0;

    bool planned = false;
    std::vector<int> order;             // item -> solve
    std::vector<BatchItem> items;
    std::vector<Family> families;
    int n_items2 = 0;
    long long n_points2 = 0, n_points = 0;
    DeviceBuffer d_items, location, start, partials, f_mean, f_var, f_se, f_steps, f_loc,
        counters, queues;
    std::vector<DeviceCounters> host_counters;

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};

    ~wos_batch() { release(); }

    // Frees every device resource (idempotent).
    void release() {
        drop_graph();
        for (DeviceBuffer *b : {&d_items, &location, &start, &partials, &f_mean, &f_var, &f_se,
                                &f_steps, &f_loc, &counters, &queues}) {
            b->release();
        }
        for (auto &m : meshes) m->dev.release();
        for (auto &e : ev) {
            if (e) cudaEventDestroy(e);
            e = nullptr;
        }
        planned = false;
    }

    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }

    void invalidate() {
        planned = false;
        drop_graph();
    }

    int prepare();
    int plan();
    cudaError_t enqueue();
};

// Builds every pending mesh's trees on the host threads (one mesh per
// thread, largest first, each build itself threaded for large meshes) while
// this thread uploads each finished mesh and builds its lattice on the
// context's stream, so the device work overlaps the remaining builds.
int wos_batch::prepare() {
    std::vector<BatchMesh *> todo;
    for (auto &m : meshes) {
        if (!m->built) todo.push_back(m.get());
    }
    if (todo.empty()) return WOS_OK;
    std::stable_sort(todo.begin(), todo.end(), [](const BatchMesh *a, const BatchMesh *b) {
        return a->prims.size() > b->prims.size();
    });
    if (device_tree_build(true)) {
        // every tree on the device, one mesh after another on the stream,
        // each followed by its lattice; the host only checks the meshes
        cudaSetDevice(ctx->device);
        for (BatchMesh *mp : todo) {
            BatchMesh &m = *mp;
            const std::string e =
                scene_meta(m.dim, m.verts.data(), static_cast<int>(m.verts.size()) / m.dim,
                           m.prims.data(), static_cast<int>(m.prims.size()) / m.dim,
                           m.bids.empty() ? nullptr : m.bids.data(), m.leaf_size, m.scene);
            if (!e.empty()) return fail(ctx, WOS_ERR_MESH, "Mesh: " + e);
            WOS_CUDA(ctx, m.dev.build_on_device(m.scene, ctx->stream), "batch tree build");
            m.built = true;
        }
        // the mesh copies serve the build's uploads until it has run
        WOS_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "batch tree build");
        for (BatchMesh *mp : todo) {
            mp->verts.clear();
            mp->verts.shrink_to_fit();
            mp->prims.clear();
            mp->prims.shrink_to_fit();
            mp->bids.clear();
            mp->bids.shrink_to_fit();
        }
        return WOS_OK;
    }
    std::vector<std::string> errs(todo.size());
    std::vector<char> done(todo.size(), 0);
    std::mutex mu;
    std::condition_variable cv;
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (size_t i = next++; i < todo.size(); i = next++) {
            BatchMesh &m = *todo[i];
            std::string e =
                build_scene(m.dim, m.verts.data(), static_cast<int>(m.verts.size()) / m.dim,
                            m.prims.data(), static_cast<int>(m.prims.size()) / m.dim,
                            m.bids.empty() ? nullptr : m.bids.data(), m.leaf_size, m.scene);
            {
                std::lock_guard<std::mutex> lk(mu);
                errs[i] = std::move(e);
                done[i] = 1;
            }
            cv.notify_all();
        }
    };
    std::vector<std::thread> pool;
    const size_t workers = std::min<size_t>(todo.size(), host_threads());
    for (size_t t = 0; t < workers; ++t) pool.emplace_back(work);
    struct Join {
        std::vector<std::thread> &threads;
        ~Join() {
            for (std::thread &t : threads) t.join();
        }
    } join{pool};
    cudaSetDevice(ctx->device);
    // meshes go to the device in the order their builds finish (the largest
    // ready one first), so the device starts on the small meshes while the
    // large ones still build
    std::vector<char> taken(todo.size(), 0);
    for (size_t c = 0; c < todo.size(); ++c) {
        size_t i = 0;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] {
                for (size_t q = 0; q < todo.size(); ++q) {
                    if (done[q] && !taken[q]) {
                        i = q;
                        return true;
                    }
                }
                return false;
            });
        }
        taken[i] = 1;
        if (!errs[i].empty()) {
            // report the first failing mesh in build order, as a serial build would
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] {
                return std::all_of(done.begin(), done.end(), [](char d) { return d != 0; });
            });
            for (size_t q = 0; q < todo.size(); ++q) {
                if (!errs[q].empty()) return fail(ctx, WOS_ERR_MESH, "Mesh: " + errs[q]);
            }
        }
        BatchMesh &m = *todo[i];
        WOS_CUDA(ctx, m.dev.upload(m.scene, ctx->stream), "batch mesh upload");
        m.built = true;
        m.verts.clear();
        m.verts.shrink_to_fit();
        m.prims.clear();
        m.prims.shrink_to_fit();
        m.bids.clear();
        m.bids.shrink_to_fit();
    }
    return WOS_OK;
}

int wos_batch::plan() {
    if (const int rc = prepare()) return rc;
    cudaSetDevice(ctx->device);
    const int n = static_cast<int>(solves.size());
    order.resize(n);
    std::iota(order.begin(), order.end(), 0);
    auto key = [&](int s) {
        const BatchSolve &b = solves[s];
        const int dim = meshes[b.mesh]->scene.dim;
        const int prec = b.p.method == WOS_METHOD_FAST_FP32 ? 0 : 1;
        const int hc = prec == 0 ? traversal_class(meshes[b.mesh]->dev.wide) + 1 : 0;
        return ((dim * 8 + b.p.equation) * 2 + prec) * 8 + hc;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key(a) < key(b); });

    // point and task ranges
    long long points = 0, tasks = 0;
    n_items2 = 0;
    n_points2 = 0;
    std::vector<FastPlan> plans(n);
    for (int i = 0; i < n; ++i) {
        BatchSolve &b = solves[order[i]];
        const BatchMesh &m = *meshes[b.mesh];
        b.item = i;
        b.point_begin = points;
        b.task_off = tasks;
        FastPlan pl{};
        set_chunk(pl, chunk_override > 0 ? chunk_override : 1024, b.p.N_walks, b.p.max_steps,
                  b.n);
        plans[order[i]] = pl;
        points += b.n;
        tasks += pl.n_tasks;
        if (m.scene.dim == 2) {
            ++n_items2;
            n_points2 += b.n;
        }
    }
    n_points = points;
    const long long pm = std::max<long long>(points, 1);
    WOS_CUDA(ctx, location.reserve(pm), "alloc batch location");
    WOS_CUDA(ctx, start.reserve(sizeof(StartRecord) * pm), "alloc batch start");
    WOS_CUDA(ctx, f_mean.reserve(sizeof(double) * pm), "alloc batch mean");
    WOS_CUDA(ctx, f_var.reserve(sizeof(double) * pm), "alloc batch variance");
    WOS_CUDA(ctx, f_se.reserve(sizeof(double) * pm), "alloc batch se");
    WOS_CUDA(ctx, f_steps.reserve(sizeof(double) * pm), "alloc batch steps");
    WOS_CUDA(ctx, f_loc.reserve(pm), "alloc batch locations");
    WOS_CUDA(ctx, partials.reserve(sizeof(TaskPartial) * std::max<long long>(tasks, 1)),
             "alloc batch partials");
    WOS_CUDA(ctx, counters.reserve(sizeof(DeviceCounters) * std::max(n, 1)), "alloc counters");

    auto *loc = static_cast<uint8_t *>(location.ptr);
    auto *st = static_cast<StartRecord *>(start.ptr);
    auto *part = static_cast<TaskPartial *>(partials.ptr);
    auto *ctr = static_cast<DeviceCounters *>(counters.ptr);
    items.assign(n, BatchItem{});
    // near-boundary lists of each mesh, for the largest threshold among its
    // FAST_FP32 solves (the walks read the lists' pointers from the items)
    std::vector<float> list_t(meshes.size(), 0.0f);
    for (const BatchSolve &b : solves) {
        if (b.p.method != WOS_METHOD_FAST_FP32) continue;
        const BatchMesh &m = *meshes[b.mesh];
        list_t[b.mesh] = std::max(list_t[b.mesh],
                                  near_list_threshold(m.dev.wide, effective_epsilon(b.p),
                                                      std::ldexp(m.scene.scale, -16)));
    }
    // every mesh's band count first, one synchronisation, then the lists
    std::vector<size_t> need;
    for (size_t k = 0; k < meshes.size(); ++k) {
        if (!meshes[k]->dev.lists_needed(list_t[k])) continue;
        WOS_CUDA(ctx, meshes[k]->dev.lists_count(list_t[k], ctx->stream), "near-boundary band");
        need.push_back(k);
    }
    if (!need.empty()) {
        WOS_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "near-boundary band");
        // all counts before any build is queued (a plain copy may wait for
        // work on the stream)
        std::vector<unsigned> band(need.size(), 0);
        for (size_t i = 0; i < need.size(); ++i) {
            WOS_CUDA(ctx, cudaMemcpy(&band[i], meshes[need[i]]->dev.gcount.ptr, sizeof(unsigned),
                                     cudaMemcpyDeviceToHost),
                     "near-boundary band");
        }
        for (size_t i = 0; i < need.size(); ++i) {
            const size_t k = need[i];
            WOS_CUDA(ctx, meshes[k]->dev.lists_build(list_t[k], band[i], ctx->sms, ctx->stream),
                     "near-boundary lists");
        }
    }
    families.clear();
    for (int i = 0; i < n; ++i) {
        const BatchSolve &b = solves[order[i]];
        const BatchMesh &m = *meshes[b.mesh];
        const int dim = m.scene.dim;
        const int precision = b.p.method == WOS_METHOD_FAST_FP32 ? 32 : 64;
        PointSet ps{};
        ps.dim = dim;
        ps.Nx = b.g.Nx;
        ps.Ny = b.g.Ny;
        ps.Nz = dim == 2 ? 1 : b.g.Nz;
        ps.lo[0] = b.g.xmin;
        ps.hi[0] = b.g.xmax;
        ps.lo[1] = b.g.ymin;
        ps.hi[1] = b.g.ymax;
        ps.lo[2] = dim == 3 ? b.g.zmin : 0.0;
        ps.hi[2] = dim == 3 ? b.g.zmax : 0.0;
        ps.n = b.n;
        const FastPlan &pl = plans[order[i]];
        BatchItem &it = items[i];
        it.a = make_fast_args(m.dev.view, m.dev.wide, ps, b.p.seed, b.p.N_walks,
                              effective_epsilon(b.p), b.p.max_steps,
                              std::ldexp(m.scene.scale, -16), pl, loc + b.point_begin,
                              st + b.point_begin, part + b.task_off, nullptr, ctr + order[i]);
        it.eq = EqDesc{b.p.equation, b.p.source_mode, b.p.alpha, nullptr};
        it.out = Fields{static_cast<double *>(f_mean.ptr) + b.point_begin,
                        static_cast<double *>(f_var.ptr) + b.point_begin,
                        static_cast<double *>(f_se.ptr) + b.point_begin,
                        static_cast<double *>(f_steps.ptr) + b.point_begin,
                        static_cast<uint8_t *>(f_loc.ptr) + b.point_begin};
        // boundary tolerance 1e-10 * max(1, mesh extents), include/wos/runner.hpp:86-88
        it.btol = 1e-10 * m.scene.scale;
        // FAST_FP32 start radii from FP32 bounds away from the shell, as in
        // a lone solve (FastStart)
        it.exact_below = precision == 32 ? std::max(effective_epsilon(b.p), it.btol) : -1.0;
        it.start_margin = fp32_distance_margin(m.scene.bbox, dim);
        it.max_ray_attempts = b.p.max_ray_attempts;
        it.precision = precision;
        it.point_begin = b.point_begin;
        const int hc = precision == 32 ? traversal_class(m.dev.wide) : kHeightAny;
        if (families.empty() || families.back().dim != dim ||
            families.back().kind != b.p.equation || families.back().precision != precision ||
            families.back().hc != hc) {
            families.push_back(Family{dim, b.p.equation, precision, hc, i, 0, 0, 0});
        }
        Family &f = families.back();
        it.task_begin = f.n_tasks;
        f.n_tasks += pl.n_tasks;
        ++f.count;
    }
    for (Family &f : families) {
        if (blocks_override > 0) {
            f.blocks = blocks_override;
        } else {
            WOS_CUDA(ctx, batch_walk_blocks(f.dim, f.kind, f.precision, f.hc, &f.blocks),
                     "batch occupancy");
        }
    }
    WOS_CUDA(ctx, d_items.reserve(sizeof(BatchItem) * std::max(n, 1)), "alloc batch items");
    WOS_CUDA(ctx, queues.reserve(sizeof(unsigned long long) * std::max<size_t>(families.size(), 1)),
             "alloc batch queues");
    if (n > 0) {
        WOS_CUDA(ctx, cudaMemcpyAsync(d_items.ptr, items.data(), sizeof(BatchItem) * n,
                                      cudaMemcpyHostToDevice, ctx->stream),
                 "H2D batch items");
    }
    WOS_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "batch plan");
    host_counters.assign(n, DeviceCounters{});
    planned = true;
    return WOS_OK;
}

cudaError_t wos_batch::enqueue() {
    cudaStream_t s = ctx->stream;
    const int n = static_cast<int>(items.size());
    const auto *di = static_cast<const BatchItem *>(d_items.ptr);
    auto *q = static_cast<unsigned long long *>(queues.ptr);
    cudaError_t e = cudaMemsetAsync(counters.ptr, 0, sizeof(DeviceCounters) * n, s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(queues.ptr, 0, sizeof(unsigned long long) * families.size(), s);
    if (e != cudaSuccess) return e;
    e = launch_classify_batch(2, di, n_items2, 0, n_points2, s);
    if (e != cudaSuccess) return e;
    e = launch_classify_batch(3, di + n_items2, n - n_items2, n_points2, n_points - n_points2, s);
    if (e != cudaSuccess) return e;
    for (size_t f = 0; f < families.size(); ++f) {
        const Family &fam = families[f];
        e = launch_walk_batch(fam.dim, fam.kind, fam.precision, fam.hc, di + fam.first, fam.count,
                              fam.n_tasks, q + f, fam.blocks, s);
        if (e != cudaSuccess) return e;
    }
    return launch_merge_batch(di, n, n_points, s);
}

void wosb::detach_batch(wos_batch *batch) {
    batch->release();
    batch->ctx = nullptr;
}

// Checks that the batch exists and its context is alive; sets the device.
static int batch_ok(wos_batch *batch, const char *what) {
    if (!batch) return fail(nullptr, WOS_ERR_INVALID, std::string(what) + ": null batch");
    if (!batch->ctx) {
        return fail(nullptr, WOS_ERR_INVALID,
                    std::string(what) + ": the batch's context was destroyed");
    }
    cudaSetDevice(batch->ctx->device);
    return WOS_OK;
}

extern "C" int wos_batch_create(wos_context *ctx, wos_batch **out) {
    if (!ctx || !out) return fail(ctx, WOS_ERR_INVALID, "wos_batch_create: null argument");
    cudaSetDevice(ctx->device);
    auto b = std::make_unique<wos_batch>();
    b->ctx = ctx;
    for (auto &e : b->ev) {
        WOS_CUDA(ctx, cudaEventCreate(&e), "cudaEventCreate");
    }
    ctx->batches.push_back(b.get());
    *out = b.release();
    return WOS_OK;
}

extern "C" void wos_batch_destroy(wos_batch *batch) {
    if (!batch) return;
    if (wos_context *ctx = batch->ctx) {
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        auto &v = ctx->batches;
        v.erase(std::remove(v.begin(), v.end(), batch), v.end());
    }
    delete batch;
}

extern "C" int wos_batch_add_mesh(wos_batch *batch, int dim, const double *verts, int n_verts,
                                  const int *prims, int n_prims, const int *boundary_ids,
                                  int leaf_size, int *mesh_id) {
    if (const int rc = batch_ok(batch, "wos_batch_add_mesh")) return rc;
    wos_context *ctx = batch->ctx;
    const std::string err = check_mesh(dim, verts, n_verts, prims, n_prims, leaf_size);
    if (!err.empty()) return fail(ctx, WOS_ERR_MESH, "Mesh: " + err);
    auto m = std::make_unique<BatchMesh>();
    m->dim = dim;
    m->leaf_size = leaf_size;
    m->verts.assign(verts, verts + static_cast<size_t>(n_verts) * dim);
    m->prims.assign(prims, prims + static_cast<size_t>(n_prims) * dim);
    if (dim == 2 && boundary_ids) m->bids.assign(boundary_ids, boundary_ids + n_prims);
    batch->meshes.push_back(std::move(m));
    if (mesh_id) *mesh_id = static_cast<int>(batch->meshes.size()) - 1;
    batch->invalidate();
    return WOS_OK;
}

extern "C" int wos_batch_add_solve(wos_batch *batch, int mesh_id, const wos_params *p,
                                   const wos_grid *g, int *solve_id) {
    if (const int rc = batch_ok(batch, "wos_batch_add_solve")) return rc;
    wos_context *ctx = batch->ctx;
    std::string err;
    if (mesh_id < 0 || mesh_id >= static_cast<int>(batch->meshes.size())) err = "unknown mesh";
    else if (!p || !g) err = "null params or grid";
    else if (p->equation < 0 || p->equation > 3) err = "unknown equation kind";
    else if (p->source_mode != 0 && p->source_mode != 1) err = "source_mode must be 0 or 1";
    else if (p->N_walks < 1) err = "N_walks must be >= 1";
    else if (!(p->epsilon > 0.0) || !std::isfinite(p->epsilon)) err = "epsilon must be positive";
    else if (p->max_steps < 1) err = "max_steps must be >= 1";
    else if (p->max_ray_attempts < 3) err = "max_ray_attempts must be >= 3";
    else if (p->equation == WOS_EQ_SCREENED_POISSON && (!(p->alpha > 0.0) || !std::isfinite(p->alpha)))
        err = "alpha must be positive";
    else if (p->method != WOS_METHOD_FAST_FP32 && p->method != WOS_METHOD_FAST_FP64)
        err = "batches run FAST_FP32 or FAST_FP64";
    const int dim = err.empty() ? batch->meshes[mesh_id]->dim : 2;
    if (err.empty() && (g->Nx < 1 || g->Ny < 1 || (dim == 3 && g->Nz < 1))) {
        err = "grid sizes must be >= 1";
    }
    if (err.empty()) {
        for (double x : {g->xmin, g->xmax, g->ymin, g->ymax, g->zmin, g->zmax}) {
            if (!std::isfinite(x)) err = "grid bounds must be finite";
        }
    }
    if (!err.empty()) return fail(ctx, WOS_ERR_INVALID, "wos_batch_add_solve: " + err);
    BatchSolve s{};
    s.mesh = mesh_id;
    s.p = *p;
    s.g = *g;
    s.n = static_cast<long long>(g->Nx) * g->Ny * (dim == 3 ? g->Nz : 1);
    batch->solves.push_back(s);
    if (solve_id) *solve_id = static_cast<int>(batch->solves.size()) - 1;
    batch->invalidate();
    return WOS_OK;
}

extern "C" int wos_batch_set_tuning(wos_batch *batch, int chunk, int blocks) {
    if (const int rc = batch_ok(batch, "wos_batch_set_tuning")) return rc;
    batch->chunk_override = chunk;
    batch->blocks_override = blocks;
    batch->invalidate();
    return WOS_OK;
}

extern "C" int wos_batch_prepare(wos_batch *batch) {
    if (const int rc = batch_ok(batch, "wos_batch_prepare")) return rc;
    if (batch->planned) return WOS_OK;
    return batch->plan();
}

extern "C" int wos_batch_run(wos_batch *batch, int use_graph, float *device_ms) {
    if (const int rc = batch_ok(batch, "wos_batch_run")) return rc;
    wos_context *ctx = batch->ctx;
    if (!batch->planned) {
        const int rc = batch->plan();
        if (rc) return rc;
    }
    if (batch->items.empty()) {
        if (device_ms) *device_ms = 0.0f;
        return WOS_OK;
    }
    cudaStream_t s = ctx->stream;
    if (use_graph && !batch->exec) {
        WOS_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
        const cudaError_t e = batch->enqueue();
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(s, &g);
        if (e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return cuda_fail(ctx, e, "batch capture");
        }
        WOS_CUDA(ctx, ee, "end capture");
        batch->graph = g;
        WOS_CUDA(ctx, cudaGraphInstantiate(&batch->exec, g, 0), "graph instantiate");
    }
    WOS_CUDA(ctx, cudaEventRecord(batch->ev[0], s), "event");
    if (use_graph) {
        WOS_CUDA(ctx, cudaGraphLaunch(batch->exec, s), "graph launch");
    } else {
        WOS_CUDA(ctx, batch->enqueue(), "batch launch");
    }
    WOS_CUDA(ctx, cudaEventRecord(batch->ev[1], s), "event");
    const size_t n = batch->items.size();
    if (n) {
        WOS_CUDA(ctx, cudaMemcpyAsync(batch->host_counters.data(), batch->counters.ptr,
                                      sizeof(DeviceCounters) * n, cudaMemcpyDeviceToHost, s),
                 "read batch counters");
    }
    WOS_CUDA(ctx, cudaStreamSynchronize(s), "batch run");
    for (const DeviceCounters &c : batch->host_counters) {
        if (c.error_flags) {
            return fail(ctx, WOS_ERR_DEVICE, device_error(c.error_flags));
        }
    }
    if (device_ms) cudaEventElapsedTime(device_ms, batch->ev[0], batch->ev[1]);
    return WOS_OK;
}

extern "C" int wos_batch_info(const wos_batch *batch, int *n_solves, long long *n_points,
                              long long *total_walks, long long *total_steps) {
    if (!batch) return fail(nullptr, WOS_ERR_INVALID, "wos_batch_info: null batch");
    long long pts = 0, walks = 0, steps = 0;
    for (const BatchSolve &s : batch->solves) pts += s.n;
    for (const DeviceCounters &c : batch->host_counters) {
        walks += static_cast<long long>(c.total_walks);
        steps += static_cast<long long>(c.total_steps);
    }
    if (n_solves) *n_solves = static_cast<int>(batch->solves.size());
    if (n_points) *n_points = pts;
    if (total_walks) *total_walks = walks;
    if (total_steps) *total_steps = steps;
    return WOS_OK;
}

extern "C" int wos_batch_result(wos_batch *batch, int solve_id, double *mean, double *variance,
                                double *standard_error, double *mean_steps, uint8_t *location,
                                wos_counters *counters) {
    if (const int rc = batch_ok(batch, "wos_batch_result")) return rc;
    wos_context *ctx = batch->ctx;
    if (solve_id < 0 || solve_id >= static_cast<int>(batch->solves.size()) || !batch->planned) {
        return fail(ctx, WOS_ERR_INVALID, "wos_batch_result: unknown solve or batch not run");
    }
    cudaSetDevice(ctx->device);
    const BatchSolve &s = batch->solves[solve_id];
    const size_t nb = sizeof(double) * static_cast<size_t>(s.n);
    const long long pb = s.point_begin;
    cudaStream_t st = ctx->stream;
    std::vector<double> tv, ts, tm;
    std::vector<uint8_t> tl;
    double *v = variance, *se = standard_error, *ms = mean_steps;
    uint8_t *l = location;
    if (counters) {
        if (!v) { tv.resize(s.n); v = tv.data(); }
        if (!se) { ts.resize(s.n); se = ts.data(); }
        if (!ms) { tm.resize(s.n); ms = tm.data(); }
        if (!l) { tl.resize(s.n); l = tl.data(); }
    }
    auto copy = [&](void *dst, const void *src, size_t bytes) -> cudaError_t {
        if (!dst || bytes == 0) return cudaSuccess;
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
    };
    WOS_CUDA(ctx, copy(mean, static_cast<double *>(batch->f_mean.ptr) + pb, nb), "D2H");
    WOS_CUDA(ctx, copy(v, static_cast<double *>(batch->f_var.ptr) + pb, nb), "D2H");
    WOS_CUDA(ctx, copy(se, static_cast<double *>(batch->f_se.ptr) + pb, nb), "D2H");
    WOS_CUDA(ctx, copy(ms, static_cast<double *>(batch->f_steps.ptr) + pb, nb), "D2H");
    WOS_CUDA(ctx, copy(l, static_cast<uint8_t *>(batch->f_loc.ptr) + pb, static_cast<size_t>(s.n)),
             "D2H");
    WOS_CUDA(ctx, cudaStreamSynchronize(st), "D2H");
    if (counters) {
        const DeviceCounters &hc = batch->host_counters[solve_id];
        wos_counters &c = *counters;
        std::memset(&c, 0, sizeof(c));
        c.max_steps_hits = static_cast<long long>(hc.max_steps_hits);
        c.ambiguous_ray_retries = static_cast<long long>(hc.ambiguous_ray_retries);
        c.indeterminate_points = static_cast<long long>(hc.indeterminate_points);
        c.total_walks = static_cast<long long>(hc.total_walks);
        c.total_steps = static_cast<long long>(hc.total_steps);
        c.exact_queries = static_cast<long long>(hc.exact_queries);
        c.effective_epsilon = effective_epsilon(s.p);
        long long inside = 0;
        for (long long t = 0; t < s.n; ++t) {
            if (l[t] != WOS_INSIDE) continue;
            ++inside;
            c.sum_variance += v[t];
            c.sum_standard_error += se[t];
            c.sum_mean_steps += ms[t];
        }
        c.inside_points = inside;
    }
    return WOS_OK;
}
