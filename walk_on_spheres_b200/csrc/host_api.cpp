// Context-free host entry points of include/wos_b200.h: the OBJ reader, the
// host BVH build and the HDF5 result writer.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wos_b200.h"
#include "h5_writer.h"
#include "obj_reader.h"
#include "scene_build.h"

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

extern "C" int wos_write_hdf5(const char *path, const wos_grid *grid, const double *mean,
                              const double *variance, const double *standard_error,
                              const double *mean_steps, const uint8_t *location, int N_walks,
                              double epsilon, int max_steps, long long max_steps_hits,
                              int write_ray_metadata, int max_ray_attempts,
                              long long ambiguous_ray_retries, long long indeterminate_points,
                              uint64_t seed, int write_source_metadata, double alpha,
                              int source_mode) {
    if (!path || !grid || !mean || !variance || !standard_error || !mean_steps || !location) {
        return WOS_ERR_INVALID;
    }
    if (grid->Nx < 1 || grid->Ny < 1 || grid->Nz < 1) return WOS_ERR_INVALID;
    std::vector<double> xs(grid->Nx), ys(grid->Ny), zs(grid->Nz);
    for (int i = 0; i < grid->Nx; ++i) xs[i] = grid_coordinate(grid->xmin, grid->xmax, i, grid->Nx);
    for (int i = 0; i < grid->Ny; ++i) ys[i] = grid_coordinate(grid->ymin, grid->ymax, i, grid->Ny);
    for (int i = 0; i < grid->Nz; ++i) zs[i] = grid_coordinate(grid->zmin, grid->zmax, i, grid->Nz);
    const std::vector<uint64_t> d3 = {static_cast<uint64_t>(grid->Nx),
                                      static_cast<uint64_t>(grid->Ny),
                                      static_cast<uint64_t>(grid->Nz)};
    // dataset order and names of include/wos/hdf5_io.hpp:147-240
    wosb::H5Group root;
    root.datasets = {
        {"mean", wosb::H5Type::F64, d3, mean},
        {"variance", wosb::H5Type::F64, d3, variance},
        {"standard_error", wosb::H5Type::F64, d3, standard_error},
        {"mean_steps", wosb::H5Type::F64, d3, mean_steps},
        {"location", wosb::H5Type::U8, d3, location},
        {"x", wosb::H5Type::F64, {d3[0]}, xs.data()},
        {"y", wosb::H5Type::F64, {d3[1]}, ys.data()},
        {"z", wosb::H5Type::F64, {d3[2]}, zs.data()},
    };
    // /metadata scalars and their native types (hdf5_io.hpp:300-322)
    wosb::H5Group meta;
    meta.name = "metadata";
    meta.datasets = {
        {"N_walks", wosb::H5Type::I32, {}, &N_walks},
        {"epsilon", wosb::H5Type::F64, {}, &epsilon},
        {"max_steps", wosb::H5Type::I32, {}, &max_steps},
        {"max_steps_hits", wosb::H5Type::I64, {}, &max_steps_hits},
        {"seed", wosb::H5Type::U64, {}, &seed},
    };
    if (write_ray_metadata) {
        meta.datasets.push_back({"max_ray_attempts", wosb::H5Type::I32, {}, &max_ray_attempts});
        meta.datasets.push_back({"ambiguous_ray_retries", wosb::H5Type::I64, {}, &ambiguous_ray_retries});
        meta.datasets.push_back({"indeterminate_points", wosb::H5Type::I64, {}, &indeterminate_points});
    }
    if (write_source_metadata) {
        meta.datasets.push_back({"alpha", wosb::H5Type::F64, {}, &alpha});
        meta.datasets.push_back({"source_mode", wosb::H5Type::I32, {}, &source_mode});
    }
    root.groups.push_back(meta);
    const std::string err = wosb::write_h5(path, root);
    if (!err.empty()) {
        std::fprintf(stderr, "HDF5 error while writing %s: %s\n", path, err.c_str());
        return WOS_ERR_IO;
    }
    return WOS_OK;
}
