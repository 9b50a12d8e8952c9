// In-memory implementation of the hdf5.h stand-in.  TEST INFRASTRUCTURE ONLY.
//
// Records what include/wos/hdf5_io.hpp:15-338 writes: each dataset keeps its
// full name ("/mean", "/metadata/seed", ...), its dimensions, its element size
// and its bytes.  Hyperslab selections (hdf5_io.hpp:108-135) are honoured so a
// block written at an offset lands at the right place in the full array.
#include "hdf5.h"

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace {

struct Space {
    std::vector<hsize_t> dims;
    std::vector<hsize_t> start;
    std::vector<hsize_t> count;
    bool none = false;
};

struct Dataset {
    std::string name;
    size_t elem = 0;
    std::vector<hsize_t> dims;
    std::vector<unsigned char> bytes;
};

struct Registry {
    std::mutex lock;
    hid_t next = 100;
    std::map<hid_t, std::string> groups;
    std::map<hid_t, Space> spaces;
    std::map<hid_t, std::string> open_sets;
    std::map<std::string, Dataset> datasets;
};

Registry &reg() {
    static Registry r;
    return r;
}

size_t type_size(hid_t type) { return static_cast<size_t>(type & 0xff); }

}  // namespace

extern "C" {

hid_t H5Pcreate(hid_t) { return 1; }
herr_t H5Pclose(hid_t) { return 0; }
herr_t H5Pset_fapl_mpio(hid_t, MPI_Comm, MPI_Info) { return 0; }
herr_t H5Pset_dxpl_mpio(hid_t, int) { return 0; }
hid_t H5Fcreate(const char *, unsigned, hid_t, hid_t) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    r.datasets.clear();
    r.groups[2] = "";
    return 2;
}
herr_t H5Fclose(hid_t) { return 0; }

hid_t H5Gcreate(hid_t loc, const char *name, hid_t, hid_t, hid_t) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    const hid_t id = r.next++;
    std::string base = r.groups.count(loc) ? r.groups[loc] : std::string();
    r.groups[id] = name[0] == '/' ? std::string(name) : base + "/" + name;
    return id;
}
herr_t H5Gclose(hid_t) { return 0; }

hid_t H5Screate_simple(int rank, const hsize_t *dims, const hsize_t *) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    const hid_t id = r.next++;
    Space s;
    s.dims.assign(dims, dims + rank);
    s.start.assign(rank, 0);
    s.count = s.dims;
    r.spaces[id] = s;
    return id;
}
hid_t H5Screate(int) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    const hid_t id = r.next++;
    r.spaces[id] = Space{};
    return id;
}
herr_t H5Sclose(hid_t space) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    r.spaces.erase(space);
    return 0;
}
herr_t H5Sselect_hyperslab(hid_t space, int, const hsize_t *start, const hsize_t *,
                           const hsize_t *count, const hsize_t *) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    Space &s = r.spaces[space];
    for (size_t d = 0; d < s.dims.size(); ++d) {
        s.start[d] = start[d];
        s.count[d] = count[d];
    }
    return 0;
}
herr_t H5Sselect_none(hid_t space) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    r.spaces[space].none = true;
    return 0;
}

hid_t H5Dcreate(hid_t loc, const char *name, hid_t type, hid_t space, hid_t, hid_t, hid_t) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    const hid_t id = r.next++;
    std::string base = r.groups.count(loc) ? r.groups[loc] : std::string();
    std::string full = name[0] == '/' ? std::string(name) : base + "/" + name;
    Dataset d;
    d.name = full;
    d.elem = type_size(type);
    d.dims = r.spaces[space].dims;
    size_t n = 1;
    for (hsize_t v : d.dims) n *= static_cast<size_t>(v);
    d.bytes.assign(n * d.elem, 0);
    r.datasets[full] = d;
    r.open_sets[id] = full;
    return id;
}

herr_t H5Dwrite(hid_t dataset, hid_t, hid_t, hid_t file_space, hid_t, const void *buf) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    Dataset &d = r.datasets[r.open_sets[dataset]];
    const Space &fs = r.spaces[file_space];
    if (fs.none) return 0;
    const unsigned char *src = static_cast<const unsigned char *>(buf);
    if (d.dims.empty()) {
        std::memcpy(d.bytes.data(), src, d.elem);
        return 0;
    }
    // row-major copy of the selected block into the full array
    const size_t rank = d.dims.size();
    std::vector<hsize_t> idx(rank, 0);
    size_t total = 1;
    for (size_t k = 0; k < rank; ++k) total *= static_cast<size_t>(fs.count[k]);
    for (size_t e = 0; e < total; ++e) {
        size_t rem = e;
        for (size_t k = rank; k-- > 0;) {
            idx[k] = rem % fs.count[k];
            rem /= fs.count[k];
        }
        size_t flat = 0;
        for (size_t k = 0; k < rank; ++k) flat = flat * d.dims[k] + (fs.start[k] + idx[k]);
        std::memcpy(d.bytes.data() + flat * d.elem, src + e * d.elem, d.elem);
    }
    return 0;
}
herr_t H5Dclose(hid_t dataset) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    r.open_sets.erase(dataset);
    return 0;
}

// Copy a captured dataset into `out` (at most `capacity` bytes).  Returns its
// size in bytes, or -1 if no dataset of that name was written.
long long refshim_dataset(const char *name, void *out, long long capacity) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    auto it = r.datasets.find(name);
    if (it == r.datasets.end()) return -1;
    const long long n = static_cast<long long>(it->second.bytes.size());
    if (out && capacity > 0) {
        std::memcpy(out, it->second.bytes.data(),
                    static_cast<size_t>(n < capacity ? n : capacity));
    }
    return n;
}

// Names of all captured datasets, '\n'-separated, into `out`.
long long refshim_dataset_names(char *out, long long capacity) {
    Registry &r = reg();
    std::lock_guard<std::mutex> g(r.lock);
    std::string all;
    for (const auto &kv : r.datasets) {
        all += kv.first;
        all += '\n';
    }
    if (out && capacity > 0) {
        const size_t n = all.size() + 1 < static_cast<size_t>(capacity)
                             ? all.size() + 1
                             : static_cast<size_t>(capacity);
        std::memcpy(out, all.c_str(), n);
        out[n - 1] = '\0';
    }
    return static_cast<long long>(all.size());
}

}  // extern "C"
