// Internal state behind the opaque wos_context of include/wos_b200.h.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/wos_b200.h"
#include "kernels.h"
#include "scene_build.h"

namespace wosb {

// Grow-only device allocation.
struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t n);
    void release();
};

// Where each array of a scene lives in its arena (one device allocation):
// box64, seg64, segid, tri64, wbox, wprim, wide2bin, the wide tree's height
// offsets and slot_verts, each at a 256-byte aligned offset.  The sizes
// follow from the scene's metadata alone.
struct ArenaLayout {
    static constexpr int kParts = 9;
    size_t offset[kParts];
    size_t bytes[kParts];
    size_t total;
};
ArenaLayout arena_layout(const HostScene &meta);

// Device copy of one HostScene (all tree and primitive arrays) and the
// views the kernels take.
struct SceneDevice {
    DeviceBuffer arena;    // every tree and primitive array, 256-byte aligned
    DeviceBuffer lattice;  // the FAST_FP32 distance lattice
    SceneView view{};
    WideView wide{};
    const int *slot_verts = nullptr;  // binary-tree slot -> the primitive's vertex ids
    // Enqueues the upload of `h` and its lattice build on `stream` (no
    // wait: later work on `stream` is ordered after them) and fills view /
    // wide.
    cudaError_t upload(const HostScene &h, cudaStream_t stream);
    // The same arena built on the device from the mesh alone (`meta` from
    // scene_meta: no host arrays), bit-identical to upload(build_scene(...)),
    // then its lattice; enqueued on `stream` (scene_build_gpu.cu).
    cudaError_t build_on_device(const HostScene &meta, cudaStream_t stream);
    // view / wide / slot_verts over the arena of a scene with this metadata.
    void set_views(const HostScene &meta);

    // Near-boundary candidate lists (wide.gl / gpool): built for every
    // lattice node with value up to 1.25 t, unless lists covering t exist;
    // a scene without a lattice, or WOS_NEAR_LISTS=0, has none.  Waits for
    // the stream once (the band size sizes the list pool).
    cudaError_t ensure_lists(float t, int sms, cudaStream_t stream);
    // ensure_lists in two halves, so a batch can count the bands of all its
    // meshes before one synchronisation: lists_needed(t) says whether lists
    // up to t are missing; lists_count(t) enqueues the band count (into
    // gcount); lists_build(t, band) sizes the pool and builds the lists.
    bool lists_needed(float t) const;
    cudaError_t lists_count(float t, cudaStream_t stream);
    cudaError_t lists_build(float t, unsigned band, int sms, cudaStream_t stream);
    DeviceBuffer glist, gpool, gcount, gaos;
    float list_built = -1.0f;  // the value up to which lists were built
    float lattice_margin = 0.0f;
    // Builds the FAST_FP32 distance lattice into `lattice` and wide.gd.
    cudaError_t build_lattice(const HostScene &h, cudaStream_t stream);
    void release();
};

double effective_epsilon(const wos_params &p);

// Where trees are built; both builders give the same arrays.  A single mesh
// (wos_set_mesh) is built on the device unless WOS_TREE_BUILD=host; a
// batch's meshes on the host threads, in parallel with the device's lattice
// builds, unless WOS_TREE_BUILD=device.
bool device_tree_build(bool batch);

// Argument checks shared by the grid entry points: an empty string when
// `p` (against the context's mesh) or the grid is acceptable, else the
// reason.
std::string check_params(const wos_context *ctx, const wos_params *p);
std::string check_grid(int dim, const wos_grid *g);
// The points of a Cartesian grid of a `dim`-dimensional mesh.
PointSet grid_points(int dim, const wos_grid &g);

// Device address of the allocation-free entry point's static scratch array
// on the current device (noalloc.cu).  Taking it loads the array's module,
// which reserves the array, so the context does it once at creation.
cudaError_t noalloc_scratch_address(void **ptr);

// Frees a batch's device memory and detaches it from its context (called
// for every live batch when the context is destroyed).
void detach_batch(wos_batch *batch);

// Message of a nonzero DeviceCounters::error_flags word.
std::string device_error(unsigned flags);

// Records `msg` as the context's (and the thread's) last error; returns code.
int fail(wos_context *ctx, int code, const std::string &msg);
int cuda_fail(wos_context *ctx, cudaError_t e, const char *what);

}  // namespace wosb

#define WOS_CUDA(ctx, call, what)                                        \
    do {                                                                 \
        cudaError_t e_ = (call);                                         \
        if (e_ != cudaSuccess) return ::wosb::cuda_fail(ctx, e_, what); \
    } while (0)

struct wos_context {
    int device = 0;
    int sms = 148;
    size_t smem_optin = 0;
    int cc_major = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t events[4] = {nullptr, nullptr, nullptr, nullptr};
    std::string error;

    bool has_mesh = false;
    wosb::HostScene scene;
    wosb::SceneView view{};
    wosb::WideView wide{};

    // scene
    wosb::SceneDevice sdev;
    // per solve
    wosb::DeviceBuffer location, start, f_mean, f_var, f_se, f_steps, f_loc, partials, queue,
        counters, points, index;
    // kernel-level checks
    wosb::DeviceBuffer scratch_a, scratch_b, scratch_c, scratch_d;
    // Gaussian heat source: vertex values, probe weights, gradients, Jacobian
    wosb::DeviceBuffer h_values, h_gradu, h_gradg, h_grads, h_jac, h_jacse;

    // live batches created on this context (detached when it is destroyed)
    std::vector<wos_batch *> batches;

    // tuning overrides (<= 0: automatic)
    int chunk_override = 0;
    int blocks_override = 0;

    // this device's address of the allocation-free entry point's static
    // scratch array, taken when the context is created
    void *noalloc_scratch = nullptr;

    ~wos_context();
    std::vector<wosb::DeviceBuffer *> all_buffers();
    int upload_scene();
    int run(const wos_params &p, const wosb::PointSet &ps, wosb::Fields out, wos_counters *c);
    // Heat-source forward (h.adjoint == 0) or adjoint replay over `ps`.
    int run_heat(const wos_params &p, const wosb::HeatDesc &h, const wosb::PointSet &ps,
                 wosb::HeatOut out, wos_counters *c);
    int fields_for(long long n, wosb::Fields &out);
    int download(long long n, const wosb::Fields &dev, double *mean, double *variance, double *se,
                 double *steps, uint8_t *loc);
};
