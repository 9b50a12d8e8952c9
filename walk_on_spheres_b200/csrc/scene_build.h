// Host construction of the device scene (see device/scene.cuh for the layout).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace wosb {

struct HostScene {
    int dim = 0;
    int n_prims = 0;
    int n_verts = 0;
    int depth = 0;
    int leaf_size = 4;
    double bbox[6] = {0, 0, 0, 0, 0, 0};  // xmin, xmax, ymin, ymax, zmin, zmax
    double scale = 1.0;                   // max(1, largest bbox extent)
    std::vector<double> box64;   // (2^(D+1)) * 2*dim
    std::vector<double> seg64;   // 2D: 4 per slot
    std::vector<int> segid;      // 2D: {boundary_id, prim} per slot
    std::vector<double> tri64;   // 3D: 14 per slot
    // FP32 records per binary slot (host only: the wide primitive blocks
    // are filled from them)
    std::vector<float> seg32;    // 2D: {x0, y0, vx, vy} per slot
    std::vector<float> seg32inv; // 2D: 1/|v|^2 per slot
    std::vector<float> tri32;    // 3D: {v0, a} {e1, b} {e2, c} {det, 1/det, 1/a, 1/c}
    std::vector<int> order;      // leaf slot -> primitive id
    // 32-wide FP32 tree (device/wide.cuh): heights 1..wH-1 of child boxes,
    // primitives in wide-slot order, all SoA
    int wH = 1;                  // root height (32^wH >= n_prims)
    int w_npad = 0;              // primitive slots padded to a multiple of 32
    int w_box_total = 0;         // boxes per coordinate array
    int w_off[8] = {0};          // offset of height h's boxes in each coordinate array
    std::vector<float> wbox;     // dim*2 arrays of w_box_total: lo.x lo.y [lo.z] hi.x hi.y [hi.z]
    std::vector<float> wprim;    // 2D: x0 y0 vx vy inv; 3D: v0 e1 e2 a b c det 1/det 1/a 1/c (16)
    std::vector<int> wide2bin;   // wide slot -> binary-tree slot (FP64 records), -1 for padding
    std::vector<int> slot_verts; // binary-tree slot -> the primitive's dim vertex ids
    // the mesh itself (for the adjoint's per-vertex data and the checks)
    std::vector<double> verts;
    std::vector<int> prims;
    std::vector<int> boundary_ids;
};

// Validates the mesh like src/mesh.cpp:239-267 (no zero-length segment, no
// degenerate triangle, indices in range) and builds the scene.  Returns an
// empty string on success, otherwise the error message.
// The checks of build_scene alone (same messages, same order), for callers
// that validate a mesh now and build its trees later.
std::string check_mesh(int dim, const double *verts, int n_verts, const int *prims, int n_prims,
                       int leaf_size);

// Host threads a build may use: WOS_HOST_THREADS when set to a positive
// count, else the hardware's.
unsigned host_threads();

std::string build_scene(int dim, const double *verts, int n_verts, const int *prims, int n_prims,
                        const int *boundary_ids, int leaf_size, HostScene &out);

// The checks of build_scene and everything of the scene but its arrays:
// the mesh itself, bounding box, scale, binary-tree depth and the 32-wide
// tree's layout (wH, w_npad, w_off, w_box_total), for a build on the device.
std::string scene_meta(int dim, const double *verts, int n_verts, const int *prims, int n_prims,
                       const int *boundary_ids, int leaf_size, HostScene &out);

}  // namespace wosb
