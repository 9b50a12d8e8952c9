// Minimal HDF5 writer for the reference's result layout (include/wos/hdf5_io.hpp).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace wosb {

enum class H5Type { F64, U8, I32, I64, U64 };

struct H5Dataset {
    std::string name;            // link name inside its group
    H5Type type;
    std::vector<uint64_t> dims;  // empty: scalar
    const void *data;            // little-endian host data, product(dims) elements;
                                 // null: storage reserved, left for later writes
    uint64_t *data_addr = nullptr;  // if set, receives the raw data's file offset
};

struct H5Group {
    std::string name;            // link name ("" for the root group)
    std::vector<H5Dataset> datasets;
    std::vector<H5Group> groups;
};

// Writes `root` as a classic-format HDF5 file (superblock version 0, version-1
// object headers, symbol-table groups, contiguous datasets).  Returns an
// empty string on success, otherwise the error.  The layout (every address)
// depends only on the names, types and shapes, not on the values.
std::string write_h5(const std::string &path, const H5Group &root,
                     uint64_t *file_size = nullptr);

// The same layout without writing anything: fills the datasets' data_addr
// and the file size.
std::string layout_h5(const H5Group &root, uint64_t *file_size);

}  // namespace wosb
