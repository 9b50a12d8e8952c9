// OBJ boundary-mesh reader with the reference's semantics (src/mesh.cpp:51-270):
// `v x y [z]` vertices (z dropped in 2D); in 2D every `l` record is one
// closed polyline with its own boundary_id (0, 1, ... in file order), closed
// automatically (with a warning) when its last vertex differs from its first;
// in 3D every `f` record must be a triangle.  Vertex references are 1-based,
// may carry "/vt/vn" suffixes, and must be in range.  Comment tokens ('#...')
// end a record.  Zero-length segments and degenerate triangles are rejected.
#include "obj_reader.h"

#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace wosb {

namespace {

struct MeshError {
    std::string text;
};

MeshError mesh_error(const char *path, int line, const std::string &msg) {
    std::string where = std::string("Mesh ") + path;
    if (line > 0) where += ":" + std::to_string(line);
    return MeshError{where + ": " + msg};
}

// 1-based vertex reference before any '/', src/mesh.cpp:24-47
int vertex_ref(const std::string &tok, int n_verts, const char *path, int line) {
    const std::string idx = tok.substr(0, tok.find('/'));
    if (idx.empty()) throw mesh_error(path, line, "missing vertex index in '" + tok + "'");
    char *end = nullptr;
    errno = 0;
    const long v = std::strtol(idx.c_str(), &end, 10);
    if (errno == ERANGE || end == idx.c_str() || *end != '\0' || v <= 0 || v > INT_MAX) {
        throw mesh_error(path, line,
                         "vertex index must be a positive 1-based integer: '" + tok + "'");
    }
    if (v - 1 >= n_verts) throw mesh_error(path, line, "vertex index out of range: '" + tok + "'");
    return static_cast<int>(v - 1);
}

// first token of a record, or "" for blank / comment lines
std::string record_kind(std::istringstream &rec) {
    std::string kind;
    if (!(rec >> kind) || kind[0] == '#') return std::string();
    return kind;
}

}  // namespace

int peek_obj_dim(const char *path, std::string &error) {
    std::ifstream in(path);
    if (!in) {
        error = std::string("Could not read mesh file ") + path;
        return 0;
    }
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream rec(line);
        const std::string kind = record_kind(rec);
        if (kind == "l") return 2;
        if (kind == "f") return 3;
    }
    error = std::string("Could not determine mesh dimension in ") + path +
            " (no 'l' or 'f' entries)";
    return 0;
}

std::string read_obj(const char *path, ObjMesh &out) {
    std::string err;
    const int dim = peek_obj_dim(path, err);
    if (dim == 0) return err;
    out = ObjMesh{};
    out.dim = dim;
    try {
        std::ifstream in(path);
        if (!in) return std::string("Could not read mesh file ") + path;
        // pass 1: counts and record shapes (src/mesh.cpp:83-138)
        int n_verts = 0, n_prims = 0, line_no = 0;
        std::string line;
        while (std::getline(in, line)) {
            ++line_no;
            std::istringstream rec(line);
            const std::string kind = record_kind(rec);
            if (kind.empty()) continue;
            if (kind == "v") {
                ++n_verts;
            } else if (dim == 2 && kind == "l") {
                std::string tok;
                int refs = 0;
                while (rec >> tok && tok[0] != '#') ++refs;
                if (refs < 2) throw mesh_error(path, line_no, "polyline has fewer than 2 vertices");
                n_prims += refs;
            } else if (dim == 3 && kind == "f") {
                std::string tok;
                int refs = 0;
                while (rec >> tok && tok[0] != '#') ++refs;
                if (refs != 3) {
                    throw mesh_error(path, line_no, "face has " + std::to_string(refs) +
                                                        " vertices; only triangles are supported");
                }
                ++n_prims;
            }
        }
        if (n_verts == 0) throw mesh_error(path, 0, "contains no vertices");
        if (n_prims == 0) {
            throw mesh_error(path, 0, dim == 2 ? "contains no line primitives"
                                               : "contains no triangle primitives");
        }
        // pass 2: values (src/mesh.cpp:150-233)
        in.clear();
        in.seekg(0, std::ios::beg);
        out.verts.reserve(static_cast<size_t>(n_verts) * dim);
        out.prims.reserve(static_cast<size_t>(n_prims) * dim);
        int bid = 0;
        line_no = 0;
        while (std::getline(in, line)) {
            ++line_no;
            std::istringstream rec(line);
            const std::string kind = record_kind(rec);
            if (kind.empty()) continue;
            if (kind == "v") {
                double x, y, z = 0.0;
                if (!(rec >> x >> y)) throw mesh_error(path, line_no, "malformed vertex record");
                std::string zt;
                if (rec >> zt && zt[0] != '#') {
                    char *end = nullptr;
                    errno = 0;
                    z = std::strtod(zt.c_str(), &end);
                    if (errno == ERANGE || end == zt.c_str() || *end != '\0') {
                        throw mesh_error(path, line_no, "malformed vertex record");
                    }
                }
                if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z)) {
                    throw mesh_error(path, line_no, "vertex coordinates must be finite");
                }
                out.verts.push_back(x);
                out.verts.push_back(y);
                if (dim == 3) out.verts.push_back(z);
            } else if (dim == 2 && kind == "l") {
                int first = -1, prev = -1;
                std::string tok;
                while (rec >> tok && tok[0] != '#') {
                    const int v = vertex_ref(tok, n_verts, path, line_no);
                    if (first < 0) first = v;
                    if (prev >= 0) {
                        out.prims.push_back(prev);
                        out.prims.push_back(v);
                        out.boundary_ids.push_back(bid);
                    }
                    prev = v;
                }
                if (prev >= 0 && prev != first) {
                    std::fprintf(stderr, "Warning: open polyline in %s auto-closed\n", path);
                    out.warnings.push_back(std::string("open polyline in ") + path + " auto-closed");
                    out.prims.push_back(prev);
                    out.prims.push_back(first);
                    out.boundary_ids.push_back(bid);
                }
                ++bid;
            } else if (dim == 3 && kind == "f") {
                std::string refs[3];
                for (std::string &r : refs) {
                    if (!(rec >> r) || r[0] == '#') {
                        throw mesh_error(path, line_no, "malformed triangle record");
                    }
                }
                for (const std::string &r : refs) out.prims.push_back(vertex_ref(r, n_verts, path, line_no));
            }
        }
        // degeneracy (src/mesh.cpp:239-267)
        auto V = [&](int v, int k) { return out.verts[static_cast<size_t>(dim) * v + k]; };
        for (int p = 0; p < out.n_prims(); ++p) {
            if (dim == 2) {
                const int a = out.prims[2 * p], b = out.prims[2 * p + 1];
                const double dx = V(b, 0) - V(a, 0), dy = V(b, 1) - V(a, 1);
                if (!(dx * dx + dy * dy > 0.0)) {
                    throw mesh_error(path, 0, "contains a zero-length line segment");
                }
            } else {
                const int a = out.prims[3 * p], b = out.prims[3 * p + 1], c = out.prims[3 * p + 2];
                const double abx = V(b, 0) - V(a, 0), aby = V(b, 1) - V(a, 1), abz = V(b, 2) - V(a, 2);
                const double acx = V(c, 0) - V(a, 0), acy = V(c, 1) - V(a, 1), acz = V(c, 2) - V(a, 2);
                const double cx = aby * acz - abz * acy, cy = abz * acx - abx * acz,
                             cz = abx * acy - aby * acx;
                if (!(cx * cx + cy * cy + cz * cz > 0.0)) {
                    throw mesh_error(path, 0, "contains a degenerate triangle");
                }
            }
        }
    } catch (const MeshError &e) {
        out = ObjMesh{};
        return e.text;
    }
    return std::string();
}

}  // namespace wosb
