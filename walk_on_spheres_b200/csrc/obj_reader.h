// OBJ boundary-mesh reader with the reference's semantics (src/mesh.cpp:51-270).
#pragma once
#include <string>
#include <vector>

namespace wosb {

struct ObjMesh {
    int dim = 0;
    std::vector<double> verts;       // n_verts * dim
    std::vector<int> prims;          // n_prims * dim, 0-based
    std::vector<int> boundary_ids;   // 2D: `l` record of each segment
    std::vector<std::string> warnings;
    int n_verts() const { return dim ? static_cast<int>(verts.size() / dim) : 0; }
    int n_prims() const { return dim ? static_cast<int>(prims.size() / dim) : 0; }
};

// Dimension of the first primitive record: 2 for `l`, 3 for `f`
// (src/mesh.cpp:51-74).  On failure returns 0 and sets `error`.
int peek_obj_dim(const char *path, std::string &error);

// Reads the mesh; returns an empty string or the reference-formatted error
// ("Mesh <path>[:<line>]: <message>", src/mesh.cpp:17-22).  Auto-close
// warnings are printed to stderr as the reference does (src/mesh.cpp:203-211)
// and also kept in `warnings`.
std::string read_obj(const char *path, ObjMesh &out);

}  // namespace wosb
