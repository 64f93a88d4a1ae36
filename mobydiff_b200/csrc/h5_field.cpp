// h5_field.cpp -- field checkpoints in HDF5 without libhdf5: the two C entry
// points of src/modules/field_hdf5.c (fdm_h5_write_field :149-184,
// fdm_h5_read_field :186-204) under the same names and signatures, so that
// the reference's io.f90 interfaces (:7-24) bind to this library unchanged.
//
// File content, as field_hdf5.c writes it: root-group attributes nx, ny, nz
// (32-bit signed little-endian integers) and lx, ly, lz, dx, dy, dz, re, dt,
// t_current (IEEE binary64 little-endian), all scalar; datasets un, vn, wn,
// pn of binary64 with dimensions (nx+2, ny+2, nz+2) in C order -- element
// (i, j, k) of the padded Fortran array at ((i (ny+2) + j) (nz+2) + k)
// (field_hdf5.c:4-12, :53-70).
//
// File format (HDF5 file format specification, the structures libhdf5
// writes for this content with its default, earliest-version settings):
//   superblock version 0, 8-byte offsets and lengths, group K 4 / 16;
//   the root group as a version-1 object header holding a symbol-table
//   message and twelve version-1 attribute messages; a local heap with the
//   link names; one version-1 group B-tree leaf with one symbol-table node
//   listing the four datasets in name order;
//   each dataset a version-1 object header with dataspace (v1), datatype
//   (v1, floating point), fill value (v2, never written) and layout (v3,
//   contiguous) messages, its data stored contiguously after the metadata.
// The reader follows the same specification for the subset such files use
// -- superblock 0 or 1, version-1 object headers with continuation blocks,
// symbol-table groups (B-tree nodes of any level), dataspace v1/v2, layout
// v3 contiguous or compact, little-endian binary64 datasets, scalar
// attribute messages v1-v3 -- and rejects anything else with an error
// instead of guessing.
#include "../../include/mobydiff_b200.h"

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

constexpr uint64_t UNDEF = ~0ull;
const uint8_t SIGNATURE[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
constexpr int LEAF_K = 4, NODE_K = 16;   // group leaf / internal node K

size_t pad8(size_t n) { return (n + 7) & ~(size_t)7; }

struct Buf {
    std::vector<uint8_t> b;
    size_t size() const { return b.size(); }
    void u8(unsigned v) { b.push_back((uint8_t)v); }
    void u16(unsigned v) { for (int s = 0; s < 2; ++s) u8((v >> (8 * s)) & 0xff); }
    void u32(uint32_t v) { for (int s = 0; s < 4; ++s) u8((v >> (8 * s)) & 0xff); }
    void u64(uint64_t v) { for (int s = 0; s < 8; ++s) u8((unsigned)((v >> (8 * s)) & 0xff)); }
    void f64(double v) { uint64_t u; std::memcpy(&u, &v, 8); u64(u); }
    void bytes(const void* p, size_t n) { const uint8_t* q = (const uint8_t*)p; b.insert(b.end(), q, q + n); }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void align8() { zeros(pad8(size()) - size()); }
};

// ---- datatype and dataspace encodings ---------------------------------------
void dtype_f64(Buf& o) {   // class 1 (floating point), version 1, IEEE binary64 little-endian
    o.u8(0x11);
    o.u8(0x20);   // byte order LE, no padding, mantissa normalisation 2 (implied msb)
    o.u8(63);     // sign bit position
    o.u8(0);
    o.u32(8);
    o.u16(0);     // bit offset
    o.u16(64);    // precision
    o.u8(52);     // exponent location
    o.u8(11);     // exponent size
    o.u8(0);      // mantissa location
    o.u8(52);     // mantissa size
    o.u32(1023);  // exponent bias
}
void dtype_i32(Buf& o) {   // class 0 (fixed point), version 1, signed 32-bit little-endian
    o.u8(0x10);
    o.u8(0x08);   // byte order LE, no padding, signed
    o.u8(0);
    o.u8(0);
    o.u32(4);
    o.u16(0);
    o.u16(32);
}
void dspace_v1(Buf& o, int rank, const uint64_t* dims) {
    o.u8(1);
    o.u8((unsigned)rank);
    o.u8(0);      // no maximum dimensions
    o.u8(0);
    o.u32(0);
    for (int r = 0; r < rank; ++r) o.u64(dims[r]);
}

// One message of a version-1 object header: type, padded data.
struct Msg {
    unsigned type, flags;
    Buf data;
};
void header_v1(Buf& o, const std::vector<Msg>& msgs) {
    size_t body = 0;
    for (const Msg& m : msgs) body += 8 + pad8(m.data.size());
    o.u8(1);
    o.u8(0);
    o.u16((unsigned)msgs.size());
    o.u32(1);                  // reference count
    o.u32((uint32_t)body);
    o.u32(0);                  // alignment of the first message to 8 bytes
    for (const Msg& m : msgs) {
        o.u16(m.type);
        o.u16((unsigned)pad8(m.data.size()));
        o.u8(m.flags);
        o.zeros(3);
        o.bytes(m.data.b.data(), m.data.size());
        o.align8();
    }
}
size_t header_v1_size(const std::vector<Msg>& msgs) {
    size_t s = 16;
    for (const Msg& m : msgs) s += 8 + pad8(m.data.size());
    return s;
}

Msg attr_msg(const char* name, bool is_int, int iv, double dv) {
    Buf dt, ds;
    if (is_int) dtype_i32(dt);
    else dtype_f64(dt);
    dspace_v1(ds, 0, nullptr);   // scalar
    Msg m{0x000C, 0, {}};
    const size_t nl = std::strlen(name) + 1;
    m.data.u8(1);
    m.data.u8(0);
    m.data.u16((unsigned)nl);
    m.data.u16((unsigned)dt.size());
    m.data.u16((unsigned)ds.size());
    m.data.bytes(name, nl);
    m.data.align8();
    m.data.bytes(dt.b.data(), dt.size());
    m.data.align8();
    m.data.bytes(ds.b.data(), ds.size());
    m.data.align8();
    if (is_int) m.data.u32((uint32_t)iv);
    else m.data.f64(dv);
    return m;
}

std::vector<Msg> dataset_msgs(const uint64_t* dims, uint64_t addr, uint64_t bytes) {
    std::vector<Msg> v;
    Msg sp{0x0001, 0, {}};
    dspace_v1(sp.data, 3, dims);
    v.push_back(sp);
    Msg dt{0x0003, 1, {}};   // constant
    dtype_f64(dt.data);
    v.push_back(dt);
    Msg fv{0x0005, 1, {}};
    fv.data.u8(2);           // version 2
    fv.data.u8(2);           // space allocated late
    fv.data.u8(2);           // fill value written if set
    fv.data.u8(0);           // no fill value defined
    v.push_back(fv);
    Msg ly{0x0008, 0, {}};
    ly.data.u8(3);           // version 3
    ly.data.u8(1);           // contiguous
    ly.data.u64(addr);
    ly.data.u64(bytes);
    v.push_back(ly);
    return v;
}

// Padded Fortran array -> C order (i slowest, k fastest), in tiles of i x k.
void to_c_order(const double* f, double* out, size_t ni, size_t nj, size_t nk) {
    const size_t T = 32;
    for (size_t j = 0; j < nj; ++j)
        for (size_t i0 = 0; i0 < ni; i0 += T)
            for (size_t k0 = 0; k0 < nk; k0 += T) {
                const size_t i1 = std::min(ni, i0 + T), k1 = std::min(nk, k0 + T);
                for (size_t k = k0; k < k1; ++k)
                    for (size_t i = i0; i < i1; ++i) out[(i * nj + j) * nk + k] = f[i + ni * (j + nj * k)];
            }
}
void from_c_order(const double* in, double* f, size_t ni, size_t nj, size_t nk) {
    const size_t T = 32;
    for (size_t j = 0; j < nj; ++j)
        for (size_t k0 = 0; k0 < nk; k0 += T)
            for (size_t i0 = 0; i0 < ni; i0 += T) {
                const size_t i1 = std::min(ni, i0 + T), k1 = std::min(nk, k0 + T);
                for (size_t k = k0; k < k1; ++k)
                    for (size_t i = i0; i < i1; ++i) f[i + ni * (j + nj * k)] = in[(i * nj + j) * nk + k];
            }
}

// ---- reader -----------------------------------------------------------------
struct Reader {
    FILE* fp = nullptr;
    uint64_t eof = 0;
    std::string err;
    ~Reader() { if (fp) std::fclose(fp); }
    bool fail(const char* m) { if (err.empty()) err = m; return false; }
    bool read(uint64_t at, void* dst, size_t n) {
        if (at == UNDEF || at + n > eof || at + n < at) return fail("read past the end of the file");
        if (std::fseek(fp, (long)at, SEEK_SET) != 0 || std::fread(dst, 1, n, fp) != n) return fail("file read failed");
        return true;
    }
    bool bytes(uint64_t at, size_t n, std::vector<uint8_t>& v) { v.resize(n); return n == 0 || read(at, v.data(), n); }
};
uint16_t g16(const uint8_t* p) { return (uint16_t)(p[0] | (p[1] << 8)); }
uint32_t g32(const uint8_t* p) { return (uint32_t)g16(p) | ((uint32_t)g16(p + 2) << 16); }
uint64_t g64(const uint8_t* p) { return (uint64_t)g32(p) | ((uint64_t)g32(p + 4) << 32); }

struct RawMsg {
    unsigned type;
    std::vector<uint8_t> data;
};

// All messages of a version-1 object header, following continuation blocks.
bool read_header(Reader& R, uint64_t addr, std::vector<RawMsg>& out) {
    uint8_t pre[16];
    if (!R.read(addr, pre, 16)) return false;
    if (pre[0] != 1) return R.fail("unsupported object header version (only version 1 is read)");
    const unsigned nmsg = g16(pre + 2);
    std::vector<std::pair<uint64_t, uint64_t>> blocks{{addr + 16, g32(pre + 8)}};
    for (size_t b = 0; b < blocks.size() && out.size() < nmsg; ++b) {
        std::vector<uint8_t> blk;
        if (!R.bytes(blocks[b].first, (size_t)blocks[b].second, blk)) return false;
        size_t p = 0;
        while (p + 8 <= blk.size() && out.size() < nmsg) {
            const unsigned type = g16(&blk[p]), size = g16(&blk[p + 2]);
            if (p + 8 + size > blk.size()) return R.fail("object header message overruns its block");
            RawMsg m{type, std::vector<uint8_t>(blk.begin() + p + 8, blk.begin() + p + 8 + size)};
            if (type == 0x0010) {   // continuation: offset, length
                if (size < 16) return R.fail("short continuation message");
                blocks.push_back({g64(m.data.data()), g64(m.data.data() + 8)});
                if (blocks.size() > 4096) return R.fail("too many continuation blocks");
            }
            out.push_back(std::move(m));
            p += 8 + size;
        }
    }
    return true;
}

// Dataspace message (v1 or v2): rank and dimensions.
bool parse_dspace(Reader& R, const uint8_t* p, size_t n, int* rank, uint64_t* dims) {
    if (n < 8) return R.fail("short dataspace message");
    const int ver = p[0], r = p[1];
    if (r > 8) return R.fail("dataspace rank above 8");
    size_t off;
    if (ver == 1) off = 8;
    else if (ver == 2) {
        if (p[3] == 2) return R.fail("null dataspace");
        off = 4;
    } else return R.fail("unsupported dataspace version");
    if (n < off + 8 * (size_t)r) return R.fail("short dataspace message");
    for (int d = 0; d < r; ++d) dims[d] = g64(p + off + 8 * d);
    *rank = r;
    return true;
}

// Datatype message: 0 = LE binary64, 1 = LE signed 32-bit integer, else -1.
int parse_dtype(const uint8_t* p, size_t n) {
    if (n < 8) return -1;
    const int cls = p[0] & 0x0f;
    const uint32_t size = g32(p + 4);
    const bool le = (p[1] & 1) == 0;
    if (cls == 1 && size == 8 && le && n >= 20 && g16(p + 10) == 64 && p[12] == 52 && p[13] == 11 && p[15] == 52 &&
        g32(p + 16) == 1023)
        return 0;
    if (cls == 0 && size == 4 && le && (p[1] & 0x08)) return 1;
    return -1;
}

struct Dataset {
    int rank = 0;
    uint64_t dims[8] = {0};
    bool compact = false;
    uint64_t addr = UNDEF, bytes = 0;
    std::vector<uint8_t> inline_data;
};

bool parse_dataset(Reader& R, uint64_t oh, Dataset& ds) {
    std::vector<RawMsg> msgs;
    if (!read_header(R, oh, msgs)) return false;
    bool sp = false, ty = false, lay = false;
    for (const RawMsg& m : msgs) {
        const uint8_t* p = m.data.data();
        const size_t n = m.data.size();
        if (m.type == 0x0001) {
            if (!parse_dspace(R, p, n, &ds.rank, ds.dims)) return false;
            sp = true;
        } else if (m.type == 0x0003) {
            if (parse_dtype(p, n) != 0) return R.fail("dataset is not little-endian binary64");
            ty = true;
        } else if (m.type == 0x000B) {
            return R.fail("filtered (compressed) datasets are not read");
        } else if (m.type == 0x0008) {
            if (n < 2 || p[0] != 3) return R.fail("unsupported layout message version (only 3 is read)");
            if (p[1] == 1) {
                if (n < 18) return R.fail("short layout message");
                ds.addr = g64(p + 2);
                ds.bytes = g64(p + 10);
            } else if (p[1] == 0) {
                if (n < 4) return R.fail("short layout message");
                const unsigned sz = g16(p + 2);
                if (n < 4 + (size_t)sz) return R.fail("short compact layout message");
                ds.compact = true;
                ds.inline_data.assign(p + 4, p + 4 + sz);
                ds.bytes = sz;
            } else {
                return R.fail("chunked datasets are not read");
            }
            lay = true;
        }
    }
    if (!sp || !ty || !lay) return R.fail("dataset header lacks dataspace, datatype or layout");
    return true;
}

// Root group: name -> object header address, through the symbol table.
struct Root {
    uint64_t oh = UNDEF, btree = UNDEF, heap = UNDEF;
    std::vector<uint8_t> names;   // local heap data segment
    std::vector<std::pair<std::string, uint64_t>> links;
};

bool heap_name(Reader& R, const Root& rt, uint64_t off, std::string& s) {
    if (off >= rt.names.size()) return R.fail("link name offset outside the local heap");
    const char* b = (const char*)rt.names.data() + off;
    const size_t maxn = rt.names.size() - off;
    const size_t n = strnlen(b, maxn);
    if (n == maxn) return R.fail("unterminated link name");
    s.assign(b, n);
    return true;
}

bool walk_btree(Reader& R, Root& rt, uint64_t addr, int depth) {
    if (depth > 32) return R.fail("group B-tree too deep");
    uint8_t h[24];
    if (!R.read(addr, h, 24)) return false;
    if (std::memcmp(h, "TREE", 4) != 0 || h[4] != 0) return R.fail("bad group B-tree node");
    const int level = h[5];
    const unsigned used = g16(h + 6);
    std::vector<uint8_t> kc;
    if (!R.bytes(addr + 24, (size_t)(16 * used + 8), kc)) return false;
    for (unsigned c = 0; c < used; ++c) {
        const uint64_t child = g64(&kc[8 + 16 * c]);
        if (level > 0) {
            if (!walk_btree(R, rt, child, depth + 1)) return false;
            continue;
        }
        uint8_t sh[8];
        if (!R.read(child, sh, 8)) return false;
        if (std::memcmp(sh, "SNOD", 4) != 0 || sh[4] != 1) return R.fail("bad symbol-table node");
        const unsigned ns = g16(sh + 6);
        std::vector<uint8_t> ent;
        if (!R.bytes(child + 8, (size_t)40 * ns, ent)) return false;
        for (unsigned e = 0; e < ns; ++e) {
            std::string name;
            if (!heap_name(R, rt, g64(&ent[40 * e]), name)) return false;
            rt.links.push_back({name, g64(&ent[40 * e + 8])});
        }
    }
    return true;
}

bool open_root(Reader& R, const char* filename, Root& rt) {
    R.fp = std::fopen(filename, "rb");
    if (!R.fp) return R.fail("cannot open file");
    std::fseek(R.fp, 0, SEEK_END);
    R.eof = (uint64_t)std::ftell(R.fp);
    uint8_t sb[104];
    if (R.eof < 96 || !R.read(0, sb, 96)) return R.fail("not an HDF5 file (too short)");
    if (std::memcmp(sb, SIGNATURE, 8) != 0) return R.fail("not an HDF5 file (no signature at offset 0)");
    const int ver = sb[8];
    if (ver != 0 && ver != 1) return R.fail("unsupported superblock version (0 and 1 are read)");
    if (sb[13] != 8 || sb[14] != 8) return R.fail("only 8-byte offsets and lengths are read");
    size_t p = 24 + (ver == 1 ? 4 : 0);
    if (ver == 1 && !R.read(0, sb, 100)) return false;
    if (g64(sb + p) != 0) return R.fail("non-zero base address");
    if (g64(sb + p + 16) > R.eof) return R.fail("truncated file (end-of-file address beyond the file size)");
    p += 32;   // base, free space, end of file, driver block
    const uint8_t* ent = sb + p;   // root symbol-table entry
    rt.oh = g64(ent + 8);
    std::vector<RawMsg> msgs;
    if (!read_header(R, rt.oh, msgs)) return false;
    for (const RawMsg& m : msgs)
        if (m.type == 0x0011 && m.data.size() >= 16) {
            rt.btree = g64(m.data.data());
            rt.heap = g64(m.data.data() + 8);
        }
    if (rt.btree == UNDEF) return R.fail("root group has no symbol table (newer group formats are not read)");
    uint8_t hh[32];
    if (!R.read(rt.heap, hh, 32)) return false;
    if (std::memcmp(hh, "HEAP", 4) != 0) return R.fail("bad local heap");
    if (!R.bytes(g64(hh + 24), (size_t)g64(hh + 8), rt.names)) return false;
    return walk_btree(R, rt, rt.btree, 0);
}

bool read_dataset3(Reader& R, const Root& rt, const char* name, int nx, int ny, int nz, double* field) {
    uint64_t oh = UNDEF;
    for (const auto& l : rt.links)
        if (l.first == name) oh = l.second;
    if (oh == UNDEF) return R.fail("dataset not found");
    Dataset ds;
    if (!parse_dataset(R, oh, ds)) return false;
    const uint64_t ni = (uint64_t)nx + 2, nj = (uint64_t)ny + 2, nk = (uint64_t)nz + 2;
    if (ds.rank != 3 || ds.dims[0] != ni || ds.dims[1] != nj || ds.dims[2] != nk)   // field_hdf5.c:119-130
        return R.fail("dataset dimensions differ from (nx+2, ny+2, nz+2)");
    const size_t n = (size_t)(ni * nj * nk);
    if (ds.bytes < 8 * (uint64_t)n) return R.fail("dataset storage smaller than its dataspace");
    std::vector<double> buf(n);
    if (ds.compact) std::memcpy(buf.data(), ds.inline_data.data(), 8 * n);
    else if (ds.addr == UNDEF) std::fill(buf.begin(), buf.end(), 0.0);   // never written: fill value 0
    else if (!R.read(ds.addr, buf.data(), 8 * n)) return false;
    from_c_order(buf.data(), field, ni, nj, nk);
    return true;
}

std::string g_h5_err;

}  // namespace

extern "C" {

int fdm_h5_write_field(const char* filename, int nx, int ny, int nz, double lx, double ly, double lz, double dx,
                       double dy, double dz, double re, double dt, double t_current, const double* un,
                       const double* vn, const double* wn, const double* pn) {
    if (!filename || nx < 1 || ny < 1 || nz < 1 || !un || !vn || !wn || !pn) return 1;   // field_hdf5.c:161
    const uint64_t dims[3] = {(uint64_t)nx + 2, (uint64_t)ny + 2, (uint64_t)nz + 2};
    const size_t n = (size_t)(dims[0] * dims[1] * dims[2]);
    const uint64_t data_bytes = 8 * (uint64_t)n;

    // root group: symbol table + attributes (field_hdf5.c:166-177)
    std::vector<Msg> root;
    Msg st{0x0011, 0, {}};
    st.data.u64(0);
    st.data.u64(0);   // B-tree and heap addresses, filled below
    root.push_back(st);
    root.push_back(attr_msg("nx", true, nx, 0.0));
    root.push_back(attr_msg("ny", true, ny, 0.0));
    root.push_back(attr_msg("nz", true, nz, 0.0));
    const char* dn[9] = {"lx", "ly", "lz", "dx", "dy", "dz", "re", "dt", "t_current"};
    const double dvv[9] = {lx, ly, lz, dx, dy, dz, re, dt, t_current};
    for (int a = 0; a < 9; ++a) root.push_back(attr_msg(dn[a], false, 0, dvv[a]));

    // names in the local heap: "" at 0, then the datasets in name order
    const char* names[4] = {"pn", "un", "vn", "wn"};
    const double* src[4] = {pn, un, vn, wn};
    Buf heap_data;
    heap_data.zeros(8);
    uint64_t name_off[4];
    for (int s = 0; s < 4; ++s) {
        name_off[s] = heap_data.size();
        heap_data.bytes(names[s], std::strlen(names[s]) + 1);
        heap_data.align8();
    }

    // addresses
    const uint64_t a_root = 96;
    const uint64_t a_heap = a_root + header_v1_size(root);
    const uint64_t a_heapdata = a_heap + 32;
    const uint64_t a_btree = a_heapdata + heap_data.size();
    const uint64_t btree_bytes = 24 + (2 * NODE_K + 1) * 8 + 2 * NODE_K * 8;
    const uint64_t a_snod = a_btree + btree_bytes;
    const uint64_t snod_bytes = 8 + 2 * LEAF_K * 40;
    uint64_t a_ds[4], a_data[4];
    uint64_t at = a_snod + snod_bytes;
    for (int s = 0; s < 4; ++s) {
        a_ds[s] = at;
        at += header_v1_size(dataset_msgs(dims, 0, data_bytes));
    }
    for (int s = 0; s < 4; ++s) {
        a_data[s] = at;
        at += data_bytes;
    }
    const uint64_t eof = at;

    Buf o;
    // superblock version 0
    o.bytes(SIGNATURE, 8);
    o.u8(0); o.u8(0); o.u8(0); o.u8(0); o.u8(0);   // superblock, free space, root entry, reserved, shared header
    o.u8(8); o.u8(8); o.u8(0);                      // sizes of offsets and lengths, reserved
    o.u16(LEAF_K);
    o.u16(NODE_K);
    o.u32(0);                                       // consistency flags
    o.u64(0);                                       // base address
    o.u64(UNDEF);                                   // free-space info
    o.u64(eof);
    o.u64(UNDEF);                                   // driver information
    o.u64(0);                                       // root entry: link name offset
    o.u64(a_root);
    o.u32(1);                                       // cache type 1: B-tree and heap in the scratch pad
    o.u32(0);
    o.u64(a_btree);
    o.u64(a_heap);
    // root object header
    root[0].data.b.clear();
    root[0].data.u64(a_btree);
    root[0].data.u64(a_heap);
    header_v1(o, root);
    // local heap
    o.bytes("HEAP", 4);
    o.u8(0); o.zeros(3);
    o.u64(heap_data.size());
    o.u64(1);                                       // no free block
    o.u64(a_heapdata);
    o.bytes(heap_data.b.data(), heap_data.size());
    // group B-tree: one leaf child, keys "" and the last name
    o.bytes("TREE", 4);
    o.u8(0); o.u8(0); o.u16(1);
    o.u64(UNDEF); o.u64(UNDEF);
    o.u64(0);
    o.u64(a_snod);
    o.u64(name_off[3]);
    o.zeros((size_t)(a_snod - (a_btree + 24 + 24)));
    // symbol-table node
    o.bytes("SNOD", 4);
    o.u8(1); o.u8(0); o.u16(4);
    for (int s = 0; s < 4; ++s) {
        o.u64(name_off[s]);
        o.u64(a_ds[s]);
        o.u32(0); o.u32(0);
        o.zeros(16);
    }
    o.zeros((size_t)(2 * LEAF_K - 4) * 40);
    // dataset headers
    for (int s = 0; s < 4; ++s) header_v1(o, dataset_msgs(dims, a_data[s], data_bytes));
    if (o.size() != a_data[0]) return 1;   // layout arithmetic

    FILE* fp = std::fopen(filename, "wb");
    if (!fp) return 1;
    bool ok = std::fwrite(o.b.data(), 1, o.size(), fp) == o.size();
    std::vector<double> buf(ok ? n : 0);
    for (int s = 0; s < 4 && ok; ++s) {
        to_c_order(src[s], buf.data(), (size_t)dims[0], (size_t)dims[1], (size_t)dims[2]);
        ok = std::fwrite(buf.data(), 8, n, fp) == n;
    }
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? 0 : 1;
}

int fdm_h5_read_field(const char* filename, int nx, int ny, int nz, double* un, double* vn, double* wn, double* pn) {
    if (!filename || nx < 1 || ny < 1 || nz < 1 || !un || !vn || !wn || !pn) return 1;   // field_hdf5.c:193
    Reader R;
    Root rt;
    bool ok = open_root(R, filename, rt);
    const char* names[4] = {"un", "vn", "wn", "pn"};
    double* dst[4] = {un, vn, wn, pn};
    for (int s = 0; s < 4 && ok; ++s) ok = read_dataset3(R, rt, names[s], nx, ny, nz, dst[s]);
    g_h5_err = ok ? std::string() : (std::string(filename) + ": " + R.err);
    return ok ? 0 : 1;
}

// Scalar root attributes of a field file: dims = nx, ny, nz; vals = lx, ly,
// lz, dx, dy, dz, re, dt, t_current.
int mdx_h5_read_header(const char* filename, int* dims, double* vals) {
    if (!filename || !dims || !vals) return MDX_ERR_ARG;
    Reader R;
    Root rt;
    if (!open_root(R, filename, rt)) {
        g_h5_err = std::string(filename) + ": " + R.err;
        return MDX_ERR_IO;
    }
    std::vector<RawMsg> msgs;
    if (!read_header(R, rt.oh, msgs)) {
        g_h5_err = std::string(filename) + ": " + R.err;
        return MDX_ERR_IO;
    }
    const char* in[3] = {"nx", "ny", "nz"};
    const char* dn[9] = {"lx", "ly", "lz", "dx", "dy", "dz", "re", "dt", "t_current"};
    int found = 0;
    for (const RawMsg& m : msgs) {
        if (m.type != 0x000C || m.data.size() < 8) continue;
        const uint8_t* p = m.data.data();
        const int ver = p[0];
        const unsigned nl = g16(p + 2), tl = g16(p + 4), sl = g16(p + 6);
        size_t off = ver == 3 ? 9 : 8;
        if (ver < 1 || ver > 3) continue;
        const size_t pn_ = ver == 1 ? pad8(nl) : nl, pt = ver == 1 ? pad8(tl) : tl, ps = ver == 1 ? pad8(sl) : sl;
        if (m.data.size() < off + pn_ + pt + ps) continue;
        const std::string name((const char*)p + off, strnlen((const char*)p + off, nl));
        const int ty = parse_dtype(p + off + pn_, tl);
        const uint8_t* val = p + off + pn_ + pt + ps;
        const size_t left = m.data.size() - (off + pn_ + pt + ps);
        for (int a = 0; a < 3; ++a)
            if (name == in[a] && ty == 1 && left >= 4) { dims[a] = (int)g32(val); found |= 1 << a; }
        for (int a = 0; a < 9; ++a)
            if (name == dn[a] && ty == 0 && left >= 8) {
                uint64_t u = g64(val);
                std::memcpy(&vals[a], &u, 8);
                found |= 8 << a;
            }
    }
    if (found != (1 << 12) - 1) {
        g_h5_err = std::string(filename) + ": missing or malformed root attributes";
        return MDX_ERR_IO;
    }
    return MDX_OK;
}

const char* mdx_h5_last_error(void) { return g_h5_err.c_str(); }

}  // extern "C"
