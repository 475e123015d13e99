// HDF5-subset reader and writer for the reference's field files (host code, no libhdf5).
//
// Bastr keeps its velocity fields in HDF5 files that libhdf5 writes with its default (earliest)
// file format: datin/flowini2d.h5 / flowini3d.h5 (initial fields, readwrite.F90:114-181) and
// outdat/flowfieldNNNN.h5 (dumps and restarts, readwrite.F90:183-257).  Every field is a dataset
// u1, u2[, u3] of H5T_NATIVE_DOUBLE whose Fortran dimensions are (ia+1, ja+1, ka+1) with the data
// in [0:ia, 0:ja, 0:max(ka,1)) (hdf5io.F90:752-802 write, 204-256 read); the dumps also hold
// nstep (H5T_NATIVE_INTEGER) and time (H5T_NATIVE_DOUBLE) as datasets of one element
// (hdf5io.F90:1009-1184).  This file writes and reads exactly that subset, from the public HDF5
// File Format Specification (version 0 superblock, version 1 object headers, a root group held
// in a symbol table: version 1 B-tree, symbol table nodes and a local heap; datasets with a
// simple dataspace, IEEE little-endian 64-bit float or 32-bit signed integer datatypes, and
// contiguous (or, when reading, compact) storage).  A caller that cannot link libhdf5 (this
// library's own drivers and tests) reads and writes the reference's files through it.
//
// Layout of a file this writer makes (all addresses absolute, base address 0):
//   superblock (96 bytes) | root object header | local heap header + data | B-tree node |
//   symbol table node(s) | per dataset: object header, raw data
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

#include "../../include/bastr_gpu.h"

namespace {

constexpr uint64_t kUndef = ~0ull;          // the undefined address
constexpr int kLeafK = 4;                    // group leaf node K: symbol table nodes hold 2K entries
constexpr int kInternalK = 16;               // group internal node K: B-tree nodes hold 2K children
constexpr int kEntry = 40;                   // symbol table entry bytes (8-byte offsets and lengths)
constexpr uint8_t kSignature[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

enum MsgType : uint16_t {
    MSG_NIL = 0x0000, MSG_DATASPACE = 0x0001, MSG_DATATYPE = 0x0003, MSG_FILL_OLD = 0x0004,
    MSG_FILL = 0x0005, MSG_LAYOUT = 0x0008, MSG_CONTINUATION = 0x0010, MSG_SYMBOL_TABLE = 0x0011,
};

// ------------------------------------------------------------------------------------------
// little-endian byte buffer
// ------------------------------------------------------------------------------------------
struct Buf {
    std::vector<uint8_t> b;
    size_t size() const { return b.size(); }
    void u8(uint64_t v) { b.push_back((uint8_t)v); }
    void u16(uint64_t v) { for (int i = 0; i < 2; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void u32(uint64_t v) { for (int i = 0; i < 4; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void u64(uint64_t v) { for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void bytes(const void* p, size_t n) { const uint8_t* q = (const uint8_t*)p; b.insert(b.end(), q, q + n); }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void pad8() { while (b.size() % 8) b.push_back(0); }
    void put64(size_t at, uint64_t v) { for (int i = 0; i < 8; ++i) b[at + i] = (uint8_t)(v >> (8 * i)); }
};

size_t round8(size_t n) { return (n + 7) & ~(size_t)7; }

// One version 1 object header message: type, data size (a multiple of 8), flags, 3 reserved.
void message(Buf& o, uint16_t type, const Buf& data) {
    o.u16(type);
    o.u16(round8(data.size()));
    o.u8(0);
    o.zeros(3);
    o.bytes(data.b.data(), data.size());
    o.pad8();
}

// Version 1 object header: prefix (16 bytes with the alignment padding) then the messages.
Buf object_header(const std::vector<std::pair<uint16_t, Buf>>& msgs) {
    Buf body;
    for (const auto& m : msgs) message(body, m.first, m.second);
    Buf o;
    o.u8(1);                     // version
    o.u8(0);                     // reserved
    o.u16(msgs.size());          // number of header messages
    o.u32(1);                    // object reference count
    o.u32(body.size());          // object header size (bytes of messages)
    o.zeros(4);                  // padding to an 8-byte boundary
    o.bytes(body.b.data(), body.size());
    return o;
}

Buf dataspace_msg(const std::vector<uint64_t>& dims) {
    Buf d;
    d.u8(1);                     // version 1
    d.u8(dims.size());           // dimensionality
    d.u8(0);                     // flags: no maximum dimensions
    d.u8(0);
    d.u32(0);                    // reserved
    for (uint64_t v : dims) d.u64(v);
    return d;
}

// IEEE 754 binary64, little-endian (H5T_NATIVE_DOUBLE on x86-64 / aarch64).
Buf datatype_f64() {
    Buf d;
    d.u8(0x11);                  // version 1, class 1 (floating point)
    d.u8(0x20);                  // little-endian, no padding, mantissa normalisation: implied MSB
    d.u8(63);                    // sign bit position
    d.u8(0);
    d.u32(8);                    // size
    d.u16(0);                    // bit offset
    d.u16(64);                   // bit precision
    d.u8(52);                    // exponent location
    d.u8(11);                    // exponent size
    d.u8(0);                     // mantissa location
    d.u8(52);                    // mantissa size
    d.u32(1023);                 // exponent bias
    return d;
}

// Two's-complement signed 32-bit, little-endian (H5T_NATIVE_INTEGER).
Buf datatype_i32() {
    Buf d;
    d.u8(0x10);                  // version 1, class 0 (fixed point)
    d.u8(0x08);                  // little-endian, no padding, signed
    d.u8(0);
    d.u8(0);
    d.u32(4);                    // size
    d.u16(0);                    // bit offset
    d.u16(32);                   // bit precision
    return d;
}

Buf fill_msg() {
    Buf d;
    d.u8(2);                     // version 2
    d.u8(2);                     // space allocation time: late
    d.u8(2);                     // fill value write time: if set
    d.u8(0);                     // fill value not defined (the library default)
    return d;
}

Buf layout_contiguous(uint64_t addr, uint64_t size) {
    Buf d;
    d.u8(3);                     // version 3
    d.u8(1);                     // layout class: contiguous
    d.u64(addr);
    d.u64(size);
    return d;
}

}  // namespace

namespace {

struct OutSet {
    std::string name;
    int type;                    // BASTR_H5_F64 or BASTR_H5_I32
    std::vector<uint64_t> dims;  // slowest first (the C order of the array)
    const void* data;
    uint64_t bytes() const {
        uint64_t n = type == BASTR_H5_I32 ? 4 : 8;
        for (uint64_t d : dims) n *= d;
        return n;
    }
};

Buf dataset_header(const OutSet& s, uint64_t data_addr) {
    return object_header({{MSG_DATASPACE, dataspace_msg(s.dims)},
                          {MSG_DATATYPE, s.type == BASTR_H5_I32 ? datatype_i32() : datatype_f64()},
                          {MSG_FILL, fill_msg()},
                          {MSG_LAYOUT, layout_contiguous(data_addr, s.bytes())}});
}

// Builds the whole file in memory.  Datasets are entries of the root group, sorted by name.
int build_file(std::vector<OutSet> sets, Buf& f, std::string& err) {
    std::sort(sets.begin(), sets.end(), [](const OutSet& a, const OutSet& b) { return a.name < b.name; });
    for (size_t i = 0; i < sets.size(); ++i) {
        if (sets[i].name.empty() || sets[i].name.find('/') != std::string::npos) {
            err = "dataset names must be non-empty and contain no '/'";
            return BASTR_E_INVALID;
        }
        if (i && sets[i].name == sets[i - 1].name) {
            err = "duplicate dataset name " + sets[i].name;
            return BASTR_E_INVALID;
        }
    }
    const size_t n = sets.size();
    const size_t nsnod = std::max<size_t>(1, (n + 2 * kLeafK - 1) / (2 * kLeafK));
    if (nsnod > (size_t)(2 * kInternalK)) {
        err = "too many datasets for one group node";
        return BASTR_E_INVALID;
    }
    // local heap data: the empty string at offset 0, then every name
    Buf heap;
    heap.zeros(8);
    std::vector<uint64_t> name_off(n);
    for (size_t i = 0; i < n; ++i) {
        name_off[i] = heap.size();
        heap.bytes(sets[i].name.c_str(), sets[i].name.size() + 1);
        heap.pad8();
    }
    // addresses
    const uint64_t a_root = 96;
    const Buf root_probe = object_header({{MSG_SYMBOL_TABLE, Buf{std::vector<uint8_t>(16, 0)}}});
    const uint64_t a_heap = a_root + root_probe.size();
    const uint64_t a_heapdata = a_heap + 32;
    const uint64_t a_btree = a_heapdata + heap.size();
    const uint64_t btree_size = 24 + (2 * kInternalK * 2 + 1) * 8;
    const uint64_t a_snod = a_btree + btree_size;
    const uint64_t snod_size = 8 + 2 * kLeafK * kEntry;
    uint64_t a = a_snod + nsnod * snod_size;
    std::vector<uint64_t> a_oh(n), a_data(n);
    for (size_t i = 0; i < n; ++i) {
        a_oh[i] = a;
        a += dataset_header(sets[i], 0).size();
        a_data[i] = a;
        a += round8(sets[i].bytes());
    }
    const uint64_t eof = a;

    // superblock, version 0
    f.bytes(kSignature, 8);
    f.u8(0); f.u8(0); f.u8(0); f.u8(0);   // superblock, free-space, root entry versions; reserved
    f.u8(0);                              // shared header message format version
    f.u8(8); f.u8(8);                     // size of offsets, size of lengths
    f.u8(0);
    f.u16(kLeafK);
    f.u16(kInternalK);
    f.u32(0);                             // file consistency flags
    f.u64(0);                             // base address
    f.u64(kUndef);                        // free-space info address
    f.u64(eof);                           // end of file address
    f.u64(kUndef);                        // driver information block address
    // root group symbol table entry: cached B-tree and heap addresses
    f.u64(0);
    f.u64(a_root);
    f.u32(1);
    f.u32(0);
    f.u64(a_btree);
    f.u64(a_heap);
    // root group object header: its symbol table message
    Buf stm;
    stm.u64(a_btree);
    stm.u64(a_heap);
    const Buf root = object_header({{MSG_SYMBOL_TABLE, stm}});
    f.bytes(root.b.data(), root.size());
    // local heap
    f.bytes("HEAP", 4);
    f.u8(0);
    f.zeros(3);
    f.u64(heap.size());
    f.u64(kUndef);                        // no free block
    f.u64(a_heapdata);
    f.bytes(heap.b.data(), heap.size());
    // B-tree node (group, leaf level): children are the symbol table nodes; key i + 1 is the heap
    // offset of the last name in child i, key 0 the empty string
    f.bytes("TREE", 4);
    f.u8(0);
    f.u8(0);
    f.u16(nsnod);
    f.u64(kUndef);
    f.u64(kUndef);
    f.u64(0);
    for (size_t c = 0; c < (size_t)(2 * kInternalK); ++c) {
        if (c < nsnod) {
            const size_t last = std::min(n, (c + 1) * 2 * kLeafK);
            f.u64(a_snod + c * snod_size);
            f.u64(n ? name_off[last - 1] : 0);
        } else {
            f.u64(0);
            f.u64(0);
        }
    }
    // symbol table nodes, 2K entries each
    for (size_t c = 0; c < nsnod; ++c) {
        const size_t lo = c * 2 * kLeafK, hi = std::min(n, lo + 2 * kLeafK);
        f.bytes("SNOD", 4);
        f.u8(1);
        f.u8(0);
        f.u16(hi - lo);
        for (size_t i = lo; i < lo + 2 * kLeafK; ++i) {
            if (i < hi) {
                f.u64(name_off[i]);
                f.u64(a_oh[i]);
                f.u32(0);
                f.u32(0);
                f.zeros(16);
            } else {
                f.zeros(kEntry);
            }
        }
    }
    // datasets
    for (size_t i = 0; i < n; ++i) {
        const Buf oh = dataset_header(sets[i], a_data[i]);
        f.bytes(oh.b.data(), oh.size());
        f.bytes(sets[i].data, sets[i].bytes());
        f.pad8();
    }
    if (f.size() != eof) {
        err = "internal layout error";
        return BASTR_E_INVALID;
    }
    return BASTR_OK;
}

}  // namespace

// ------------------------------------------------------------------------------------------
// reader
// ------------------------------------------------------------------------------------------
namespace {

thread_local std::string g_h5err;

int h5fail(int code, const std::string& msg) {
    g_h5err = msg;
    return code;
}

struct File {
    std::vector<uint8_t> d;
    bool ok(uint64_t at, uint64_t n) const { return at <= d.size() && n <= d.size() - at; }
    uint64_t rd(uint64_t at, int n) const {
        uint64_t v = 0;
        for (int i = 0; i < n; ++i) v |= (uint64_t)d[at + i] << (8 * i);
        return v;
    }
};

struct InSet {
    int type = -1;
    std::vector<uint64_t> dims;
    uint64_t addr = kUndef, size = 0;   // contiguous storage (kUndef: not allocated, fill values)
    std::vector<uint8_t> compact;       // compact storage
    bool is_compact = false;
};

bool read_file(const char* path, File& f) {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return false;
    std::fseek(fp, 0, SEEK_END);
    const long n = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    f.d.resize(n > 0 ? (size_t)n : 0);
    const size_t got = n > 0 ? std::fread(f.d.data(), 1, (size_t)n, fp) : 0;
    std::fclose(fp);
    return got == f.d.size();
}

// Messages of a version 1 object header, following continuation blocks; calls fn(type, at, size).
template <typename Fn> int walk_header(const File& f, uint64_t oh, Fn&& fn) {
    if (!f.ok(oh, 16) || f.d[oh] != 1) return h5fail(BASTR_E_UNSUPPORTED, "object header is not version 1");
    uint64_t left = f.rd(oh + 2, 2);
    std::vector<std::pair<uint64_t, uint64_t>> blocks = {{oh + 16, f.rd(oh + 8, 4)}};
    for (size_t bi = 0; bi < blocks.size() && left > 0; ++bi) {
        uint64_t at = blocks[bi].first;
        const uint64_t end = at + blocks[bi].second;
        if (!f.ok(blocks[bi].first, blocks[bi].second)) return h5fail(BASTR_E_INVALID, "truncated object header");
        while (left > 0 && at + 8 <= end) {
            const uint16_t type = (uint16_t)f.rd(at, 2);
            const uint64_t size = f.rd(at + 2, 2);
            if (at + 8 + size > end) return h5fail(BASTR_E_INVALID, "object header message overruns its block");
            if (type == MSG_CONTINUATION) blocks.push_back({f.rd(at + 8, 8), f.rd(at + 16, 8)});
            else if (type != MSG_NIL) {
                const int r = fn(type, at + 8, size);
                if (r) return r;
            }
            at += 8 + size;
            --left;
        }
    }
    return BASTR_OK;
}

int parse_dataset(const File& f, uint64_t oh, InSet& s) {
    int r = walk_header(f, oh, [&](uint16_t type, uint64_t at, uint64_t size) -> int {
        if (type == MSG_DATASPACE) {
            const int ver = f.d[at], rank = f.d[at + 1], flags = f.d[at + 2];
            const uint64_t dims_at = ver == 1 ? at + 8 : at + 4;
            if (ver != 1 && ver != 2) return h5fail(BASTR_E_UNSUPPORTED, "dataspace message version");
            if (ver == 2 && f.d[at + 3] == 2) return h5fail(BASTR_E_UNSUPPORTED, "null dataspace");
            (void)flags;
            s.dims.clear();
            for (int i = 0; i < rank; ++i) s.dims.push_back(f.rd(dims_at + 8 * i, 8));
        } else if (type == MSG_DATATYPE) {
            const int cls = f.d[at] & 15, bits0 = f.d[at + 1];
            const uint64_t esize = f.rd(at + 4, 4);
            if (bits0 & 1) return h5fail(BASTR_E_UNSUPPORTED, "big-endian data");
            if (cls == 1 && esize == 8) s.type = BASTR_H5_F64;
            else if (cls == 0 && esize == 4 && (bits0 & 8)) s.type = BASTR_H5_I32;
            else return h5fail(BASTR_E_UNSUPPORTED, "datatype other than 64-bit float or signed 32-bit integer");
        } else if (type == MSG_LAYOUT) {
            const int ver = f.d[at];
            if (ver == 3) {
                const int cls = f.d[at + 1];
                if (cls == 1) {
                    s.addr = f.rd(at + 2, 8);
                    s.size = f.rd(at + 10, 8);
                } else if (cls == 0) {
                    const uint64_t n = f.rd(at + 2, 2);
                    if (!f.ok(at + 4, n)) return h5fail(BASTR_E_INVALID, "truncated compact data");
                    s.is_compact = true;
                    s.compact.assign(f.d.begin() + at + 4, f.d.begin() + at + 4 + n);
                } else {
                    return h5fail(BASTR_E_UNSUPPORTED, "chunked or virtual dataset storage");
                }
            } else if (ver == 1 || ver == 2) {
                const int nd = f.d[at + 1], cls = f.d[at + 2];
                if (cls != 1) return h5fail(BASTR_E_UNSUPPORTED, "old-style layout other than contiguous");
                s.addr = f.rd(at + 8, 8);
                uint64_t n = 1;
                for (int i = 0; i < nd; ++i) n *= f.rd(at + 16 + 4 * i, 4);
                s.size = n;   // includes the element size as the last dimension
            } else {
                return h5fail(BASTR_E_UNSUPPORTED, "layout message version");
            }
        }
        (void)size;
        return BASTR_OK;
    });
    if (r) return r;
    if (s.type < 0) return h5fail(BASTR_E_INVALID, "dataset without a datatype message");
    return BASTR_OK;
}

// Object header address of `name` in the root group (a symbol table: B-tree + local heap).
int find_in_root(const File& f, const std::string& name, uint64_t& oh_out, uint64_t& base_out) {
    uint64_t sb = kUndef;
    for (uint64_t at = 0; at + 8 <= f.d.size(); at = at ? at * 2 : 512) {
        if (std::memcmp(f.d.data() + at, kSignature, 8) == 0) { sb = at; break; }
    }
    if (sb == kUndef) return h5fail(BASTR_E_INVALID, "no HDF5 signature");
    const int ver = f.d[sb + 8];
    if (ver > 1) return h5fail(BASTR_E_UNSUPPORTED, "superblock version above 1 (files from libhdf5's latest format)");
    if (f.d[sb + 13] != 8 || f.d[sb + 14] != 8) return h5fail(BASTR_E_UNSUPPORTED, "offsets or lengths not 8 bytes");
    const uint64_t base = f.rd(sb + 24, 8);
    base_out = base;
    const uint64_t root_entry = sb + (ver == 0 ? 56 : 60);
    const uint64_t root_oh = base + f.rd(root_entry + 8, 8);
    uint64_t btree = kUndef, heap = kUndef;
    int r = walk_header(f, root_oh, [&](uint16_t type, uint64_t at, uint64_t) -> int {
        if (type == MSG_SYMBOL_TABLE) {
            btree = base + f.rd(at, 8);
            heap = base + f.rd(at + 8, 8);
        }
        return BASTR_OK;
    });
    if (r) return r;
    if (btree == kUndef) return h5fail(BASTR_E_UNSUPPORTED, "root group is not a symbol table (new-style group)");
    if (!f.ok(heap, 32) || std::memcmp(f.d.data() + heap, "HEAP", 4) != 0) return h5fail(BASTR_E_INVALID, "bad local heap");
    const uint64_t heap_size = f.rd(heap + 8, 8), heap_data = base + f.rd(heap + 24, 8);
    if (!f.ok(heap_data, heap_size)) return h5fail(BASTR_E_INVALID, "truncated local heap");
    // depth-first walk of the B-tree to its symbol table nodes
    std::vector<uint64_t> stack = {btree};
    int guard = 0;
    while (!stack.empty()) {
        if (++guard > 100000) return h5fail(BASTR_E_INVALID, "group B-tree too large or cyclic");
        const uint64_t node = stack.back();
        stack.pop_back();
        if (!f.ok(node, 24) || std::memcmp(f.d.data() + node, "TREE", 4) != 0 || f.d[node + 4] != 0)
            return h5fail(BASTR_E_INVALID, "bad group B-tree node");
        const int level = f.d[node + 5];
        const uint64_t used = f.rd(node + 6, 2);
        for (uint64_t c = 0; c < used; ++c) {
            const uint64_t child = base + f.rd(node + 24 + 8 + 16 * c, 8);
            if (level > 0) {
                stack.push_back(child);
                continue;
            }
            if (!f.ok(child, 8) || std::memcmp(f.d.data() + child, "SNOD", 4) != 0)
                return h5fail(BASTR_E_INVALID, "bad symbol table node");
            const uint64_t nsym = f.rd(child + 6, 2);
            for (uint64_t i = 0; i < nsym; ++i) {
                const uint64_t e = child + 8 + kEntry * i;
                if (!f.ok(e, kEntry)) return h5fail(BASTR_E_INVALID, "truncated symbol table node");
                const uint64_t off = f.rd(e, 8);
                if (off >= heap_size) return h5fail(BASTR_E_INVALID, "name offset outside the local heap");
                const char* nm = (const char*)f.d.data() + heap_data + off;
                const size_t len = strnlen(nm, heap_size - off);
                if (name.size() == len && std::memcmp(nm, name.data(), len) == 0) {
                    oh_out = base + f.rd(e + 8, 8);
                    return BASTR_OK;
                }
            }
        }
    }
    return h5fail(BASTR_E_INVALID, "no dataset named " + name);
}

// Reads dataset `name` of the given type: its dims, and its values into out (when non-null).
int read_set(const File& f, const std::string& name, int type, std::vector<uint64_t>& dims, void* out,
             uint64_t capacity) {
    uint64_t oh = 0, base = 0;
    int r = find_in_root(f, name, oh, base);
    if (r) return r;
    InSet s;
    r = parse_dataset(f, oh, s);
    if (r) return r;
    if (s.type != type) return h5fail(BASTR_E_INVALID, "dataset " + name + " has another datatype");
    dims = s.dims;
    uint64_t bytes = type == BASTR_H5_I32 ? 4 : 8;
    for (uint64_t d : dims) bytes *= d;
    if (!out) return BASTR_OK;
    if (bytes > capacity) return h5fail(BASTR_E_INVALID, "dataset " + name + " is larger than the buffer");
    if (s.is_compact) {
        if (s.compact.size() < bytes) return h5fail(BASTR_E_INVALID, "compact data shorter than the dataspace");
        std::memcpy(out, s.compact.data(), bytes);
    } else if (s.addr == kUndef) {
        std::memset(out, 0, bytes);   // storage never written: the default fill value
    } else {
        const uint64_t at = base + s.addr;
        if (!f.ok(at, bytes)) return h5fail(BASTR_E_INVALID, "dataset " + name + " runs past the end of the file");
        std::memcpy(out, f.d.data() + at, bytes);
    }
    return BASTR_OK;
}

}  // namespace

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------
namespace {

bool field_dims_ok(int ia, int ja, int ka) { return ia >= 1 && ja >= 1 && ka >= 0; }

// The reference's padded field array, C order [ka+1][ja+1][ia+1]: u(1:ia,1:ja,1:nz) in the
// block [0:nz)x[0:ja)x[0:ia), nz = max(ka,1), the rest zero (hdf5io.F90:752-802).
std::vector<double> pad_field(const double* u, int ia, int ja, int ka) {
    const size_t X = (size_t)ia + 1, Y = (size_t)ja + 1, Z = (size_t)ka + 1, nz = ka == 0 ? 1 : ka;
    std::vector<double> p(X * Y * Z, 0.0);
    for (size_t z = 0; z < nz; ++z)
        for (size_t y = 0; y < (size_t)ja; ++y)
            std::memcpy(&p[(z * Y + y) * X], u + (z * ja + y) * (size_t)ia, (size_t)ia * sizeof(double));
    return p;
}

}  // namespace

extern "C" {

BASTR_API int bastr_h5_write(const char* path, const bastr_h5_dataset* sets, int32_t n) {
    if (!path || (n > 0 && !sets) || n < 0) return h5fail(BASTR_E_INVALID, "bastr_h5_write arguments");
    std::vector<OutSet> v;
    for (int i = 0; i < n; ++i) {
        const bastr_h5_dataset& d = sets[i];
        if (!d.name || !d.data || d.rank < 1 || d.rank > 4 || (d.type != BASTR_H5_F64 && d.type != BASTR_H5_I32))
            return h5fail(BASTR_E_INVALID, "dataset description " + std::to_string(i));
        OutSet o{d.name, d.type, {}, d.data};
        for (int k = 0; k < d.rank; ++k) {
            if (d.dims[k] < 1) return h5fail(BASTR_E_INVALID, "dataset dimensions must be positive");
            o.dims.push_back((uint64_t)d.dims[k]);
        }
        v.push_back(o);
    }
    Buf f;
    std::string err;
    const int r = build_file(v, f, err);
    if (r) return h5fail(r, err);
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return h5fail(BASTR_E_INVALID, std::string("cannot create ") + path);
    const size_t put = std::fwrite(f.b.data(), 1, f.size(), fp);
    const int closed = std::fclose(fp);
    if (put != f.size() || closed != 0) return h5fail(BASTR_E_INVALID, std::string("short write to ") + path);
    return BASTR_OK;
}

BASTR_API int bastr_h5_read(const char* path, const char* name, int32_t type, int32_t* rank, int64_t* dims,
                            void* data, int64_t capacity) {
    if (!path || !name) return h5fail(BASTR_E_INVALID, "bastr_h5_read arguments");
    File f;
    if (!read_file(path, f)) return h5fail(BASTR_E_INVALID, std::string("cannot read ") + path);
    std::vector<uint64_t> d;
    const int r = read_set(f, name, type, d, data, capacity < 0 ? 0 : (uint64_t)capacity);
    if (r) return r;
    if (rank) *rank = (int32_t)d.size();
    if (dims)
        for (size_t i = 0; i < d.size() && i < 4; ++i) dims[i] = (int64_t)d[i];
    return BASTR_OK;
}

BASTR_API int bastr_h5_write_field(const char* path, int32_t ia, int32_t ja, int32_t ka, const double* u1,
                                   const double* u2, const double* u3, int64_t nstep, double time) {
    if (!path || !field_dims_ok(ia, ja, ka) || !u1 || !u2 || (ka > 0 && !u3))
        return h5fail(BASTR_E_INVALID, "bastr_h5_write_field arguments");
    const int64_t dims[4] = {ka + 1, ja + 1, ia + 1, 0};
    const double* src[3] = {u1, u2, u3};
    const char* names[3] = {"u1", "u2", "u3"};
    const int nc = ka == 0 ? 2 : 3;
    std::vector<std::vector<double>> padded;
    std::vector<bastr_h5_dataset> sets;
    for (int c = 0; c < nc; ++c) padded.push_back(pad_field(src[c], ia, ja, ka));
    for (int c = 0; c < nc; ++c) sets.push_back({names[c], BASTR_H5_F64, 3, {dims[0], dims[1], dims[2], 0}, padded[c].data()});
    const int32_t ns = (int32_t)nstep;
    if (nstep >= 0) {
        sets.push_back({"nstep", BASTR_H5_I32, 1, {1, 0, 0, 0}, &ns});
        sets.push_back({"time", BASTR_H5_F64, 1, {1, 0, 0, 0}, &time});
    }
    return bastr_h5_write(path, sets.data(), (int32_t)sets.size());
}

BASTR_API int bastr_h5_read_field(const char* path, int32_t ia, int32_t ja, int32_t ka, double* u1, double* u2,
                                  double* u3, int64_t* nstep, double* time) {
    if (!path || !field_dims_ok(ia, ja, ka) || !u1 || !u2 || (ka > 0 && !u3))
        return h5fail(BASTR_E_INVALID, "bastr_h5_read_field arguments");
    File f;
    if (!read_file(path, f)) return h5fail(BASTR_E_INVALID, std::string("cannot read ") + path);
    double* dst[3] = {u1, u2, u3};
    const char* names[3] = {"u1", "u2", "u3"};
    const int nc = ka == 0 ? 2 : 3;
    const size_t X = (size_t)ia + 1, Y = (size_t)ja + 1, Z = (size_t)ka + 1, nz = ka == 0 ? 1 : ka;
    std::vector<double> p(X * Y * Z);
    for (int c = 0; c < nc; ++c) {
        std::vector<uint64_t> d;
        int r = read_set(f, names[c], BASTR_H5_F64, d, nullptr, 0);
        if (r) return r;
        // the reference reads the block (im, jm, km) at offset 0 of the padded (ia+1, ja+1, ka+1)
        if (d.size() != 3 || d[0] < nz || d[1] < (uint64_t)ja || d[2] < (uint64_t)ia)
            return h5fail(BASTR_E_INVALID, std::string("dataset ") + names[c] + " is smaller than the grid");
        const size_t DX = d[2], DY = d[1];
        p.resize(d[0] * d[1] * d[2]);
        r = read_set(f, names[c], BASTR_H5_F64, d, p.data(), p.size() * sizeof(double));
        if (r) return r;
        for (size_t z = 0; z < nz; ++z)
            for (size_t y = 0; y < (size_t)ja; ++y)
                std::memcpy(dst[c] + (z * ja + y) * (size_t)ia, &p[(z * DY + y) * DX], (size_t)ia * sizeof(double));
    }
    if (nstep) {
        std::vector<uint64_t> d;
        int32_t v = 0;
        const int r = read_set(f, "nstep", BASTR_H5_I32, d, &v, sizeof v);
        if (r) return r;
        *nstep = v;
    }
    if (time) {
        std::vector<uint64_t> d;
        const int r = read_set(f, "time", BASTR_H5_F64, d, time, sizeof(double));
        if (r) return r;
    }
    return BASTR_OK;
}

BASTR_API int bastr_h5_last_error(char* buf, int32_t n) {
    const int len = (int)g_h5err.size();
    if (buf && n > 0) {
        const int m = std::min(len, n - 1);
        std::memcpy(buf, g_h5err.data(), m);
        buf[m] = 0;
    }
    return len;
}

}  // extern "C"
