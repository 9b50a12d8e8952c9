// Minimal HDF5 writer (HDF5 File Format Specification, version-0 superblock).
//
// Structures written, all little-endian with 8-byte offsets and lengths:
//   superblock v0 (96 bytes) with the root group's symbol-table entry;
//   per group: a version-1 object header holding one Symbol Table message,
//     a v1 B-tree node (type 0, one child), one symbol-table node (SNOD) with
//     the entries sorted by name, and a local heap whose data segment holds
//     "" at offset 0, the names (8-byte padded) and one trailing free block
//     (the free list ends with the value 1, as libhdf5 writes it);
//   per dataset: a version-1 object header with Fill Value (v1), Datatype
//     (IEEE double or fixed-point), Dataspace (v1; rank 0 = scalar) and
//     contiguous Data Layout (v3) messages, then the raw data.
// Group node K values are 16 (leaf) and 16 (internal), so one SNOD holds up
// to 32 links, more than the result layout needs.
#include "h5_writer.h"

#include <algorithm>
#include <cstdio>
#include <cstring>

namespace wosb {

namespace {

constexpr int kLeafK = 16;
constexpr int kInternalK = 16;
constexpr uint64_t kUndef = ~0ull;
// datasets of at least this many bytes are written from the caller's array
constexpr size_t kExternalBytes = 1 << 16;

// File image under construction: `b` holds the bytes from file offset `base`
// on; hole(n) closes that segment and leaves n bytes unwritten, storage that
// other writers fill in later (a POSIX file reads zeros there until then).
// external(p, n) is a hole that the file write fills from the caller's array
// p, so large datasets are not copied into the image.
struct Buf {
    struct External {
        uint64_t at;
        const void *p;
        size_t n;
    };
    std::vector<uint8_t> b;
    uint64_t base = 0;
    std::vector<std::pair<uint64_t, std::vector<uint8_t>>> done;  // closed segments
    std::vector<External> ext;
    uint64_t tell() const { return base + b.size(); }
    void hole(uint64_t n) {
        const uint64_t end = tell();
        if (!b.empty()) done.emplace_back(base, std::move(b));
        b.clear();
        base = end + n;
    }
    void external(const void *p, size_t n) {
        ext.push_back({tell(), p, n});
        hole(n);
    }
    // overwrite n bytes at file offset `at` (inside a written segment)
    bool patch(uint64_t at, const uint8_t *p, size_t n) {
        auto fits = [&](uint64_t off, std::vector<uint8_t> &v) {
            if (at < off || at + n > off + v.size()) return false;
            std::memcpy(v.data() + (at - off), p, n);
            return true;
        };
        if (fits(base, b)) return true;
        for (auto &seg : done) {
            if (fits(seg.first, seg.second)) return true;
        }
        return false;
    }
    void u8(uint8_t v) { b.push_back(v); }
    void u16(uint16_t v) { for (int i = 0; i < 2; ++i) b.push_back(static_cast<uint8_t>(v >> (8 * i))); }
    void u32(uint32_t v) { for (int i = 0; i < 4; ++i) b.push_back(static_cast<uint8_t>(v >> (8 * i))); }
    void u64(uint64_t v) { for (int i = 0; i < 8; ++i) b.push_back(static_cast<uint8_t>(v >> (8 * i))); }
    void bytes(const void *p, size_t n) {
        const uint8_t *q = static_cast<const uint8_t *>(p);
        b.insert(b.end(), q, q + n);
    }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void align8() { while (tell() % 8) b.push_back(0); }
};

size_t elem_size(H5Type t) {
    switch (t) {
        case H5Type::F64: return 8;
        case H5Type::U8: return 1;
        case H5Type::I32: return 4;
        default: return 8;
    }
}

// Datatype message body (padded to 8 bytes).
std::vector<uint8_t> datatype_msg(H5Type t) {
    Buf m;
    if (t == H5Type::F64) {
        m.u8(0x11);          // version 1, class 1 (floating point)
        m.u8(0x20);          // little endian, implied mantissa MSB
        m.u8(63);            // sign bit position
        m.u8(0);
        m.u32(8);            // size
        m.u16(0);            // bit offset
        m.u16(64);           // precision
        m.u8(52);            // exponent location
        m.u8(11);            // exponent size
        m.u8(0);             // mantissa location
        m.u8(52);            // mantissa size
        m.u32(1023);         // exponent bias
    } else {
        const bool is_signed = (t == H5Type::I32 || t == H5Type::I64);
        const uint32_t size = static_cast<uint32_t>(elem_size(t));
        m.u8(0x10);          // version 1, class 0 (fixed point)
        m.u8(is_signed ? 0x08 : 0x00);
        m.u8(0);
        m.u8(0);
        m.u32(size);
        m.u16(0);
        m.u16(static_cast<uint16_t>(8 * size));
    }
    m.align8();
    return m.b;
}

void message(Buf &o, uint16_t type, const std::vector<uint8_t> &body, uint8_t flags) {
    o.u16(type);
    o.u16(static_cast<uint16_t>(body.size()));
    o.u8(flags);
    o.zeros(3);
    o.bytes(body.data(), body.size());
}

void object_header(Buf &o, const std::vector<std::pair<uint16_t, std::vector<uint8_t>>> &msgs,
                   const std::vector<uint8_t> &flags) {
    size_t size = 0;
    for (const auto &m : msgs) size += 8 + m.second.size();
    o.u8(1);   // version
    o.u8(0);
    o.u16(static_cast<uint16_t>(msgs.size()));
    o.u32(1);  // reference count
    o.u32(static_cast<uint32_t>(size));
    o.zeros(4);  // alignment of the first message
    for (size_t i = 0; i < msgs.size(); ++i) message(o, msgs[i].first, msgs[i].second, flags[i]);
}

// Writes a dataset (its raw data first, then its object header); returns the
// object header address.  Without data the raw data's storage is a hole.
uint64_t emit_dataset(Buf &o, const H5Dataset &d) {
    uint64_t n = 1;
    for (uint64_t v : d.dims) n *= v;
    const size_t nbytes = static_cast<size_t>(n) * elem_size(d.type);
    o.align8();
    const uint64_t data_addr = o.tell();
    if (d.data_addr) *d.data_addr = data_addr;
    if (nbytes) {
        if (!d.data) {
            o.hole(nbytes);
        } else if (nbytes >= kExternalBytes) {
            o.external(d.data, nbytes);
        } else {
            o.bytes(d.data, nbytes);
        }
    }
    o.align8();
    const uint64_t hdr = o.tell();

    Buf fill;  // fill value message, version 1
    fill.u8(1);
    fill.u8(2);  // late allocation
    fill.u8(2);  // write fill value if set
    fill.u8(1);  // fill value defined (default)
    fill.u32(0);
    Buf space;  // dataspace message, version 1 (rank 0 = scalar)
    space.u8(1);
    space.u8(static_cast<uint8_t>(d.dims.size()));
    space.u8(0);
    space.u8(0);
    space.u32(0);
    for (uint64_t v : d.dims) space.u64(v);
    Buf layout;  // data layout message, version 3, contiguous
    layout.u8(3);
    layout.u8(1);
    layout.u64(data_addr);
    layout.u64(nbytes);
    layout.align8();
    object_header(o, {{0x0005, fill.b}, {0x0003, datatype_msg(d.type)}, {0x0001, space.b},
                      {0x0008, layout.b}},
                  {1, 1, 0, 0});
    return hdr;
}

struct GroupAddrs {
    uint64_t header, btree, heap;
};

GroupAddrs emit_group(Buf &o, const H5Group &g) {
    struct Link {
        std::string name;
        uint64_t header;
        bool group;
        uint64_t btree, heap;
    };
    std::vector<Link> links;
    for (const H5Dataset &d : g.datasets) links.push_back({d.name, emit_dataset(o, d), false, 0, 0});
    for (const H5Group &c : g.groups) {
        const GroupAddrs a = emit_group(o, c);
        links.push_back({c.name, a.header, true, a.btree, a.heap});
    }
    std::sort(links.begin(), links.end(),
              [](const Link &a, const Link &b) { return std::strcmp(a.name.c_str(), b.name.c_str()) < 0; });

    // local heap data: "" at 0, then the names, then a free block
    Buf heap_data;
    heap_data.zeros(8);
    std::vector<uint64_t> name_off;
    for (const Link &l : links) {
        name_off.push_back(heap_data.tell());
        heap_data.bytes(l.name.c_str(), l.name.size() + 1);
        heap_data.align8();
    }
    const uint64_t free_off = heap_data.tell();
    const uint64_t free_size = 32;
    heap_data.u64(1);          // next free block: none
    heap_data.u64(free_size);  // size of this free block
    heap_data.zeros(free_size - 16);

    o.align8();
    const uint64_t heap_data_addr = o.tell();
    o.bytes(heap_data.b.data(), heap_data.b.size());
    const uint64_t heap_addr = o.tell();
    o.bytes("HEAP", 4);
    o.u8(0);
    o.zeros(3);
    o.u64(heap_data.b.size());
    o.u64(free_off);
    o.u64(heap_data_addr);

    // symbol table node
    const uint64_t snod = o.tell();
    o.bytes("SNOD", 4);
    o.u8(1);
    o.u8(0);
    o.u16(static_cast<uint16_t>(links.size()));
    for (int i = 0; i < 2 * kLeafK; ++i) {
        if (i < static_cast<int>(links.size())) {
            const Link &l = links[i];
            o.u64(name_off[i]);
            o.u64(l.header);
            o.u32(l.group ? 1 : 0);
            o.u32(0);
            o.u64(l.group ? l.btree : 0);
            o.u64(l.group ? l.heap : 0);
        } else {
            o.zeros(40);
        }
    }

    // v1 B-tree node (group), one child; allocated for 2K children
    const uint64_t btree = o.tell();
    o.bytes("TREE", 4);
    o.u8(0);   // group node
    o.u8(0);   // leaf level
    o.u16(1);  // entries used
    o.u64(kUndef);
    o.u64(kUndef);
    o.u64(0);  // key 0: ""
    o.u64(snod);
    o.u64(links.empty() ? 0 : name_off.back());  // key 1: last name
    o.zeros(static_cast<size_t>(2 * kInternalK - 1) * 16);

    // group object header: symbol table message
    o.align8();
    const uint64_t hdr = o.tell();
    Buf st;
    st.u64(btree);
    st.u64(heap_addr);
    object_header(o, {{0x0011, st.b}}, {1});
    return GroupAddrs{hdr, btree, heap_addr};
}

}  // namespace

namespace {
std::string build_h5(const H5Group &root, Buf &o) {
    if (root.datasets.size() + root.groups.size() > 2 * kLeafK) return "too many links in one group";
    o.zeros(96);  // superblock, filled below
    const GroupAddrs r = emit_group(o, root);
    Buf sb;
    const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    sb.bytes(sig, 8);
    sb.u8(0);  // superblock version
    sb.u8(0);  // free-space version
    sb.u8(0);  // root group symbol table entry version
    sb.u8(0);
    sb.u8(0);  // shared header message format version
    sb.u8(8);  // size of offsets
    sb.u8(8);  // size of lengths
    sb.u8(0);
    sb.u16(kLeafK);
    sb.u16(kInternalK);
    sb.u32(0);            // consistency flags
    sb.u64(0);            // base address
    sb.u64(kUndef);       // free-space info
    sb.u64(o.tell());     // end of file
    sb.u64(kUndef);       // driver information
    sb.u64(0);            // root: link name offset
    sb.u64(r.header);     // root: object header
    sb.u32(1);            // cache type: symbol table
    sb.u32(0);
    sb.u64(r.btree);
    sb.u64(r.heap);
    if (!o.patch(0, sb.b.data(), 96)) return "superblock outside the written image";
    return std::string();
}
}  // namespace

std::string layout_h5(const H5Group &root, uint64_t *file_size) {
    Buf o;
    const std::string err = build_h5(root, o);
    if (err.empty() && file_size) *file_size = o.tell();
    return err;
}

std::string write_h5(const std::string &path, const H5Group &root, uint64_t *file_size) {
    Buf o;
    std::string err = build_h5(root, o);
    if (!err.empty()) return err;
    const uint64_t eof = o.tell();
    o.hole(0);  // close the last segment
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return "could not create " + path;
    bool ok = true;
    uint64_t at = 0;  // end of the bytes written so far
    auto put = [&](uint64_t off, const void *p, size_t n) {
        ok = ok && fseeko(f, static_cast<off_t>(off), SEEK_SET) == 0 &&
             std::fwrite(p, 1, n, f) == n;
        at = std::max(at, off + n);
    };
    for (const auto &seg : o.done) put(seg.first, seg.second.data(), seg.second.size());
    for (const Buf::External &e : o.ext) put(e.at, e.p, e.n);
    if (ok && at < eof) {
        // the image ends in a hole: extend the file to its full size
        const uint8_t zero = 0;
        ok = fseeko(f, static_cast<off_t>(eof - 1), SEEK_SET) == 0 &&
             std::fwrite(&zero, 1, 1, f) == 1;
    }
    const int c = std::fclose(f);
    if (!ok || c != 0) return "could not write " + path;
    if (file_size) *file_size = eof;
    return std::string();
}

}  // namespace wosb
