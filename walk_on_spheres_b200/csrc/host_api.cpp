// Context-free host entry points of include/wos_b200.h: the OBJ reader, the
// host BVH build and the HDF5 result writer (serial, and the parallel path:
// create, then per-rank block writes).
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wos_b200.h"
#include "h5_writer.h"
#include "obj_reader.h"
#include "scene_build.h"

namespace wosb {
// error record of wos_last_global_error (context.cpp)
int fail(wos_context *ctx, int code, const std::string &msg);
}  // namespace wosb

namespace {

double grid_coordinate(double lo, double hi, int i, int n) {
    return n > 1 ? lo + (hi - lo) * static_cast<double>(i) / static_cast<double>(n - 1) : lo;
}

void copy_error(const std::string &msg, char *error, int cap) {
    if (error && cap > 0) {
        std::strncpy(error, msg.c_str(), static_cast<size_t>(cap) - 1);
        error[cap - 1] = '\0';
    }
}

}  // namespace

extern "C" int wos_read_obj(const char *path, int *dim, int *n_verts, int *n_prims,
                            double *verts, int *prims, int *boundary_ids, char *error,
                            int error_capacity) {
    if (!path) {
        copy_error("null path", error, error_capacity);
        return WOS_ERR_INVALID;
    }
    wosb::ObjMesh m;
    const std::string err = wosb::read_obj(path, m);
    if (!err.empty()) {
        copy_error(err, error, error_capacity);
        return WOS_ERR_MESH;
    }
    if (dim) *dim = m.dim;
    if (n_verts) *n_verts = m.n_verts();
    if (n_prims) *n_prims = m.n_prims();
    if (verts) std::memcpy(verts, m.verts.data(), m.verts.size() * sizeof(double));
    if (prims) std::memcpy(prims, m.prims.data(), m.prims.size() * sizeof(int));
    if (boundary_ids && m.dim == 2) {
        std::memcpy(boundary_ids, m.boundary_ids.data(), m.boundary_ids.size() * sizeof(int));
    }
    return WOS_OK;
}

extern "C" int wos_build_bvh(int dim, const double *verts, int n_verts, const int *prims,
                             int n_prims, int leaf_size, int *depth, double *node_boxes,
                             int *order) {
    wosb::HostScene sc;
    const std::string err =
        wosb::build_scene(dim, verts, n_verts, prims, n_prims, nullptr, leaf_size, sc);
    if (!err.empty()) return WOS_ERR_MESH;
    if (depth) *depth = sc.depth;
    if (node_boxes) std::memcpy(node_boxes, sc.box64.data(), sc.box64.size() * sizeof(double));
    if (order) std::memcpy(order, sc.order.data(), sc.order.size() * sizeof(int));
    return WOS_OK;
}

extern "C" int wos_build_wide_bvh(int dim, const double *verts, int n_verts, const int *prims,
                                  int n_prims, int *height, int *entries, int *offsets,
                                  float *nodes, int *order) {
    wosb::HostScene sc;
    const std::string err =
        wosb::build_scene(dim, verts, n_verts, prims, n_prims, nullptr, 0, sc);
    if (!err.empty()) return WOS_ERR_MESH;
    if (height) *height = sc.wH;
    if (entries) *entries = sc.w_box_total;
    if (offsets) std::memcpy(offsets, sc.w_off, sizeof(sc.w_off));
    if (nodes) std::memcpy(nodes, sc.wbox.data(), sc.wbox.size() * sizeof(float));
    if (order) {
        for (int s = 0; s < n_prims; ++s) order[s] = sc.order[sc.wide2bin[s]];
    }
    return WOS_OK;
}

namespace {

// Run settings written under /metadata (include/wos/hdf5_io.hpp:300-322).
struct ResultMeta {
    int N_walks = 0;
    double epsilon = 0.0;
    int max_steps = 0;
    long long max_steps_hits = 0;
    int write_ray_metadata = 0;
    int max_ray_attempts = 0;
    long long ambiguous_ray_retries = 0;
    long long indeterminate_points = 0;
    uint64_t seed = 0;
    int write_source_metadata = 0;
    double alpha = 0.0;
    int source_mode = 0;
};

// The result file's tree: dataset names, order and native types of
// include/wos/hdf5_io.hpp:147-322.  A null field is reserved storage; addr[f]
// receives the file offset of field f's values.  Holds pointers into itself
// and into `m`: build it in place and keep `m` alive while it is written.
struct ResultTree {
    std::vector<double> xs, ys, zs;
    uint64_t addr[5] = {0, 0, 0, 0, 0};
    wosb::H5Group root;

    ResultTree(const wos_grid &g, const void *const fields[5], const ResultMeta &m) {
        xs.resize(g.Nx);
        ys.resize(g.Ny);
        zs.resize(g.Nz);
        for (int i = 0; i < g.Nx; ++i) xs[i] = grid_coordinate(g.xmin, g.xmax, i, g.Nx);
        for (int i = 0; i < g.Ny; ++i) ys[i] = grid_coordinate(g.ymin, g.ymax, i, g.Ny);
        for (int i = 0; i < g.Nz; ++i) zs[i] = grid_coordinate(g.zmin, g.zmax, i, g.Nz);
        const std::vector<uint64_t> d3 = {static_cast<uint64_t>(g.Nx),
                                          static_cast<uint64_t>(g.Ny),
                                          static_cast<uint64_t>(g.Nz)};
        static const char *const kNames[5] = {"mean", "variance", "standard_error",
                                              "mean_steps", "location"};
        for (int f = 0; f < 5; ++f) {
            root.datasets.push_back({kNames[f], f < 4 ? wosb::H5Type::F64 : wosb::H5Type::U8, d3,
                                     fields[f], &addr[f]});
        }
        root.datasets.push_back({"x", wosb::H5Type::F64, {d3[0]}, xs.data()});
        root.datasets.push_back({"y", wosb::H5Type::F64, {d3[1]}, ys.data()});
        root.datasets.push_back({"z", wosb::H5Type::F64, {d3[2]}, zs.data()});
        wosb::H5Group meta;
        meta.name = "metadata";
        meta.datasets = {
            {"N_walks", wosb::H5Type::I32, {}, &m.N_walks},
            {"epsilon", wosb::H5Type::F64, {}, &m.epsilon},
            {"max_steps", wosb::H5Type::I32, {}, &m.max_steps},
            {"max_steps_hits", wosb::H5Type::I64, {}, &m.max_steps_hits},
            {"seed", wosb::H5Type::U64, {}, &m.seed},
        };
        if (m.write_ray_metadata) {
            meta.datasets.push_back({"max_ray_attempts", wosb::H5Type::I32, {}, &m.max_ray_attempts});
            meta.datasets.push_back(
                {"ambiguous_ray_retries", wosb::H5Type::I64, {}, &m.ambiguous_ray_retries});
            meta.datasets.push_back(
                {"indeterminate_points", wosb::H5Type::I64, {}, &m.indeterminate_points});
        }
        if (m.write_source_metadata) {
            meta.datasets.push_back({"alpha", wosb::H5Type::F64, {}, &m.alpha});
            meta.datasets.push_back({"source_mode", wosb::H5Type::I32, {}, &m.source_mode});
        }
        root.groups.push_back(meta);
    }
    ResultTree(const ResultTree &) = delete;
    ResultTree &operator=(const ResultTree &) = delete;
};

bool grid_ok(const wos_grid *g) { return g && g->Nx >= 1 && g->Ny >= 1 && g->Nz >= 1; }

void fill_layout(const ResultTree &t, uint64_t file_size, wos_h5_layout *layout) {
    for (int f = 0; f < 5; ++f) layout->field_offset[f] = static_cast<long long>(t.addr[f]);
    layout->file_size = static_cast<long long>(file_size);
}

int result_layout(const wos_grid &g, int ray, int source, wos_h5_layout *layout) {
    const void *const none[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    ResultMeta m;
    m.write_ray_metadata = ray;
    m.write_source_metadata = source;
    ResultTree t(g, none, m);
    uint64_t size = 0;
    if (!wosb::layout_h5(t.root, &size).empty()) return WOS_ERR_INVALID;
    fill_layout(t, size, layout);
    return WOS_OK;
}

bool same_layout(const wos_h5_layout &a, const wos_h5_layout &b) {
    if (a.file_size != b.file_size) return false;
    for (int f = 0; f < 5; ++f) {
        if (a.field_offset[f] != b.field_offset[f]) return false;
    }
    return true;
}

// A run of grid points: `n` values from source index `src` to file (linear)
// index `dst`.
struct Run {
    long long dst, src, n;
};

// Positioned writes of the runs of every field into a created result file.
int write_runs(const char *path, const wos_h5_layout *layout, const wos_grid &g,
               const std::vector<Run> &runs, const void *const fields[5]) {
    // the layout has to be one of this grid's four (metadata switches on/off)
    bool known = false;
    for (int k = 0; k < 4 && !known; ++k) {
        wos_h5_layout want{};
        if (result_layout(g, k & 1, k >> 1, &want) == WOS_OK) known = same_layout(want, *layout);
    }
    if (!known) return wosb::fail(nullptr, WOS_ERR_INVALID, "HDF5 block write: layout is not this grid's");
    const int fd = ::open(path, O_RDWR);
    if (fd < 0) {
        return wosb::fail(nullptr, WOS_ERR_IO, std::string("HDF5 block write: cannot open ") + path);
    }
    struct stat st {};
    uint8_t sig[8] = {};
    static const uint8_t kSig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    if (::fstat(fd, &st) != 0 || st.st_size < layout->file_size ||
        ::pread(fd, sig, 8, 0) != 8 || std::memcmp(sig, kSig, 8) != 0) {
        ::close(fd);
        return wosb::fail(nullptr, WOS_ERR_IO,
                          std::string("HDF5 block write: ") + path + " is not a created result file");
    }
    bool ok = true;
    for (int f = 0; f < 5 && ok; ++f) {
        const size_t elem = f < 4 ? sizeof(double) : 1;
        const auto *src = static_cast<const uint8_t *>(fields[f]);
        for (const Run &r : runs) {
            size_t left = static_cast<size_t>(r.n) * elem;
            const uint8_t *p = src + static_cast<size_t>(r.src) * elem;
            off_t at = static_cast<off_t>(layout->field_offset[f] +
                                          static_cast<long long>(r.dst) * static_cast<long long>(elem));
            while (left > 0) {
                const ssize_t w = ::pwrite(fd, p, left, at);
                if (w <= 0) {
                    ok = false;
                    break;
                }
                left -= static_cast<size_t>(w);
                p += w;
                at += w;
            }
            if (!ok) break;
        }
    }
    const int c = ::close(fd);
    if (!ok || c != 0) {
        return wosb::fail(nullptr, WOS_ERR_IO, std::string("HDF5 block write: writing ") + path + " failed");
    }
    return WOS_OK;
}

}  // namespace

extern "C" int wos_write_hdf5(const char *path, const wos_grid *grid, const double *mean,
                              const double *variance, const double *standard_error,
                              const double *mean_steps, const uint8_t *location, int N_walks,
                              double epsilon, int max_steps, long long max_steps_hits,
                              int write_ray_metadata, int max_ray_attempts,
                              long long ambiguous_ray_retries, long long indeterminate_points,
                              uint64_t seed, int write_source_metadata, double alpha,
                              int source_mode) {
    if (!path || !mean || !variance || !standard_error || !mean_steps || !location ||
        !grid_ok(grid)) {
        return wosb::fail(nullptr, WOS_ERR_INVALID, "HDF5 write: null argument or empty grid");
    }
    const ResultMeta m{N_walks, epsilon, max_steps, max_steps_hits, write_ray_metadata,
                       max_ray_attempts, ambiguous_ray_retries, indeterminate_points, seed,
                       write_source_metadata, alpha, source_mode};
    const void *const fields[5] = {mean, variance, standard_error, mean_steps, location};
    const ResultTree t(*grid, fields, m);
    const std::string err = wosb::write_h5(path, t.root);
    if (!err.empty()) {
        const std::string msg = std::string("HDF5 error while writing ") + path + ": " + err;
        std::fprintf(stderr, "%s\n", msg.c_str());
        return wosb::fail(nullptr, WOS_ERR_IO, msg);
    }
    return WOS_OK;
}

extern "C" int wos_hdf5_layout(const wos_grid *grid, int write_ray_metadata,
                               int write_source_metadata, wos_h5_layout *layout) {
    if (!grid_ok(grid) || !layout) return WOS_ERR_INVALID;
    return result_layout(*grid, write_ray_metadata ? 1 : 0, write_source_metadata ? 1 : 0,
                         layout);
}

extern "C" int wos_hdf5_create(const char *path, const wos_grid *grid, int N_walks,
                               double epsilon, int max_steps, long long max_steps_hits,
                               int write_ray_metadata, int max_ray_attempts,
                               long long ambiguous_ray_retries, long long indeterminate_points,
                               uint64_t seed, int write_source_metadata, double alpha,
                               int source_mode, wos_h5_layout *layout) {
    if (!path || !grid_ok(grid)) return WOS_ERR_INVALID;
    const ResultMeta m{N_walks, epsilon, max_steps, max_steps_hits, write_ray_metadata ? 1 : 0,
                       max_ray_attempts, ambiguous_ray_retries, indeterminate_points, seed,
                       write_source_metadata ? 1 : 0, alpha, source_mode};
    const void *const none[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    const ResultTree t(*grid, none, m);
    uint64_t size = 0;
    const std::string err = wosb::write_h5(path, t.root, &size);
    if (!err.empty()) {
        return wosb::fail(nullptr, WOS_ERR_IO,
                          std::string("HDF5 error while creating ") + path + ": " + err);
    }
    if (layout) fill_layout(t, size, layout);
    return WOS_OK;
}

extern "C" int wos_hdf5_write_block(const char *path, const wos_h5_layout *layout,
                                    const wos_grid *grid, const int offset[3],
                                    const int count[3], const double *mean,
                                    const double *variance, const double *standard_error,
                                    const double *mean_steps, const uint8_t *location) {
    if (!path || !layout || !grid_ok(grid) || !offset || !count || !mean || !variance ||
        !standard_error || !mean_steps || !location) {
        return wosb::fail(nullptr, WOS_ERR_INVALID, "HDF5 block write: null argument");
    }
    const int N[3] = {grid->Nx, grid->Ny, grid->Nz};
    for (int d = 0; d < 3; ++d) {
        if (offset[d] < 0 || count[d] < 0 || offset[d] > N[d] - count[d]) {
            return wosb::fail(nullptr, WOS_ERR_INVALID, "HDF5 block write: block leaves the grid");
        }
    }
    // one run per (x, y) row of the block, merged where rows are adjacent in
    // the file (full z rows, then full y planes)
    std::vector<Run> runs;
    for (int i = 0; i < count[0]; ++i) {
        for (int j = 0; j < count[1]; ++j) {
            if (count[2] == 0) continue;
            const long long dst =
                (static_cast<long long>(offset[0] + i) * N[1] + (offset[1] + j)) * N[2] + offset[2];
            const long long src = (static_cast<long long>(i) * count[1] + j) * count[2];
            if (!runs.empty() && runs.back().dst + runs.back().n == dst &&
                runs.back().src + runs.back().n == src) {
                runs.back().n += count[2];
            } else {
                runs.push_back({dst, src, count[2]});
            }
        }
    }
    const void *const fields[5] = {mean, variance, standard_error, mean_steps, location};
    return write_runs(path, layout, *grid, runs, fields);
}

extern "C" int wos_hdf5_write_range(const char *path, const wos_h5_layout *layout,
                                    const wos_grid *grid, long long start, long long count,
                                    const double *mean, const double *variance,
                                    const double *standard_error, const double *mean_steps,
                                    const uint8_t *location) {
    if (!path || !layout || !grid_ok(grid) || !mean || !variance || !standard_error ||
        !mean_steps || !location) {
        return wosb::fail(nullptr, WOS_ERR_INVALID, "HDF5 range write: null argument");
    }
    const long long n = static_cast<long long>(grid->Nx) * grid->Ny * grid->Nz;
    if (start < 0 || count < 0 || start > n - count) {
        return wosb::fail(nullptr, WOS_ERR_INVALID, "HDF5 range write: range leaves the grid");
    }
    std::vector<Run> runs;
    if (count > 0) runs.push_back({start, 0, count});
    const void *const fields[5] = {mean, variance, standard_error, mean_steps, location};
    return write_runs(path, layout, *grid, runs, fields);
}
