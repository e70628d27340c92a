// hdf5_lite.cpp -- see hdf5_lite.h. Field order and sizes follow the
// published HDF5 file format specification (superblock version 0, B-tree
// version 1, symbol table node, local heap, object header version 1 and
// its messages); the reference's snapshot and raw-point files
// (simulation/snapshotmanager.cpp:60-104, :186-286) use exactly these
// structures.
#include "hdf5_lite.h"

#include <zlib.h>

#include <algorithm>
#include <cstdio>
#include <map>

namespace h5l {

namespace {

constexpr uint64_t kUndef = ~0ull;
constexpr int kLeafK = 4;       // symbol-table node holds up to 2K entries
constexpr int kInternalK = 16;  // group B-tree node holds up to 2K children
constexpr size_t kSuperblockBytes = 96;
constexpr size_t kBtreeNodeBytes = 24 + (2 * kInternalK + 1) * 8 + 2 * kInternalK * 8;
constexpr size_t kSnodBytes = 8 + 2 * kLeafK * 40;
constexpr size_t kHeapHeaderBytes = 32;
constexpr uint64_t kHeapFreeNull = 1;  // "no next free block" in a local heap

// message types
enum : uint16_t {
    kMsgNil = 0x0000, kMsgDataspace = 0x0001, kMsgDatatype = 0x0003, kMsgFillValue = 0x0005,
    kMsgLayout = 0x0008, kMsgFilters = 0x000B, kMsgAttribute = 0x000C, kMsgContinuation = 0x0010,
    kMsgSymbolTable = 0x0011
};

size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }

struct Out {
    std::vector<uint8_t> b;
    void u8(uint64_t v) { b.push_back((uint8_t)v); }
    void u16(uint64_t v) { for (int i = 0; i < 2; i++) b.push_back((uint8_t)(v >> (8 * i))); }
    void u32(uint64_t v) { for (int i = 0; i < 4; i++) b.push_back((uint8_t)(v >> (8 * i))); }
    void u64(uint64_t v) { for (int i = 0; i < 8; i++) b.push_back((uint8_t)(v >> (8 * i))); }
    void bytes(const void *p, size_t n)
    {
        const uint8_t *q = static_cast<const uint8_t *>(p);
        b.insert(b.end(), q, q + n);
    }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void pad_to(size_t n) { if (b.size() < n) zeros(n - b.size()); }
    void align8() { pad_to(pad8(b.size())); }
};

// body of a datatype message, version 1
void put_type(Out &o, const Type &t)
{
    if (t.cls == kFloat) {
        const bool dbl = t.size == 8;
        o.u8(0x10 | kFloat);
        o.u8(0x20);                 // little-endian, no padding, implied mantissa MSB
        o.u8((uint8_t)(8 * t.size - 1));  // sign bit location
        o.u8(0);
        o.u32((uint32_t)t.size);
        o.u16(0);                   // bit offset
        o.u16(8 * t.size);          // precision
        o.u8(dbl ? 52 : 23);        // exponent location
        o.u8(dbl ? 11 : 8);         // exponent size
        o.u8(0);                    // mantissa location
        o.u8(dbl ? 52 : 23);        // mantissa size
        o.u32(dbl ? 1023 : 127);    // exponent bias
    } else {
        o.u8(0x10 | t.cls);
        o.u8(t.cls == kFixed && t.is_signed ? 0x08 : 0x00);
        o.u8(0);
        o.u8(0);
        o.u32((uint32_t)t.size);
        o.u16(0);
        o.u16(8 * t.size);
    }
}
size_t type_bytes(const Type &t) { return t.cls == kFloat ? 20 : 12; }

// body of a dataspace message, version 1, with maximum dimensions = dims
void put_space(Out &o, const std::vector<uint64_t> &dims)
{
    o.u8(1);
    o.u8((uint8_t)dims.size());
    o.u8(1);
    o.u8(0);
    o.u32(0);
    for (uint64_t d : dims) o.u64(d);
    for (uint64_t d : dims) o.u64(d);
}
size_t space_bytes(size_t rank) { return 8 + 16 * rank; }

void put_msg(Out &o, uint16_t type, uint8_t flags, const Out &body)
{
    o.u16(type);
    o.u16(pad8(body.b.size()));
    o.u8(flags);
    o.zeros(3);
    o.bytes(body.b.data(), body.b.size());
    o.align8();
}

uint64_t nbytes(const DatasetSpec &d)
{
    uint64_t n = (uint64_t)d.type.size;
    for (uint64_t x : d.dims) n *= x;
    return n;
}

// object header (version 1) of a contiguous dataset whose data sit at addr
Out dataset_header(const DatasetSpec &d, uint64_t addr)
{
    Out msgs;
    int count = 0;
    {
        Out m;
        put_space(m, d.dims);
        put_msg(msgs, kMsgDataspace, 0, m);
        count++;
    }
    {
        Out m;
        put_type(m, d.type);
        put_msg(msgs, kMsgDatatype, 1, m);
        count++;
    }
    {
        Out m;  // version 2: allocation late, write fill if set, default (zero) fill defined
        m.u8(2);
        m.u8(2);
        m.u8(2);
        m.u8(1);
        m.u32(0);
        put_msg(msgs, kMsgFillValue, 1, m);
        count++;
    }
    {
        Out m;  // version 3, contiguous
        const uint64_t n = nbytes(d);
        m.u8(3);
        m.u8(1);
        m.u64(n ? addr : kUndef);
        m.u64(n);
        put_msg(msgs, kMsgLayout, 0, m);
        count++;
    }
    for (const Attr &a : d.attrs) {
        Out m;  // version 1: name, datatype and dataspace each padded to 8 bytes
        m.u8(1);
        m.u8(0);
        m.u16(a.name.size() + 1);
        m.u16(type_bytes(a.type));
        m.u16(space_bytes(1));
        m.bytes(a.name.c_str(), a.name.size() + 1);
        m.align8();
        put_type(m, a.type);
        m.align8();
        put_space(m, {1});
        m.align8();
        m.bytes(a.value.data(), a.value.size());
        put_msg(msgs, kMsgAttribute, 0, m);
        count++;
    }
    Out h;
    h.u8(1);
    h.u8(0);
    h.u16(count);
    h.u32(1);
    h.u32(msgs.b.size());
    h.u32(0);
    h.bytes(msgs.b.data(), msgs.b.size());
    return h;
}

}  // namespace

std::string write_file(const std::string &path, const std::vector<DatasetSpec> &datasets)
{
    if (datasets.empty() || datasets.size() > 2 * kLeafK) return "between 1 and 8 datasets per file";
    for (const DatasetSpec &d : datasets) {
        if (d.type.size <= 0 || (nbytes(d) && !d.data)) return "dataset " + d.name + ": no data";
        for (const Attr &a : d.attrs)
            if ((int)a.value.size() != a.type.size) return "attribute " + a.name + ": value size";
    }
    // link names in the local heap, in name order (the symbol-table node's order)
    std::vector<size_t> order(datasets.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return datasets[a].name < datasets[b].name; });
    Out heap;
    heap.zeros(8);  // offset 0: the empty name
    std::vector<uint64_t> name_off(datasets.size());
    for (size_t k : order) {
        name_off[k] = heap.b.size();
        heap.bytes(datasets[k].name.c_str(), datasets[k].name.size() + 1);
        heap.align8();
    }
    const uint64_t free_off = heap.b.size();
    heap.u64(kHeapFreeNull);
    heap.u64(16);

    const uint64_t root_ohdr = kSuperblockBytes;
    const uint64_t btree = root_ohdr + 16 + 24;
    const uint64_t heap_hdr = btree + kBtreeNodeBytes;
    const uint64_t heap_data = heap_hdr + kHeapHeaderBytes;
    const uint64_t snod = heap_data + heap.b.size();
    uint64_t pos = snod + kSnodBytes;
    // dataset object headers need the data addresses, which follow all
    // headers: size the headers first (their size does not depend on addr)
    std::vector<uint64_t> ohdr(datasets.size()), data_at(datasets.size());
    for (size_t i = 0; i < datasets.size(); i++) {
        ohdr[i] = pos;
        pos = pad8(pos + dataset_header(datasets[i], 0).b.size());
    }
    for (size_t i = 0; i < datasets.size(); i++) {
        data_at[i] = pos;
        pos = pad8(pos + nbytes(datasets[i]));
    }
    const uint64_t eof = pos;

    Out o;
    // superblock version 0
    const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    o.bytes(sig, 8);
    o.u8(0); o.u8(0); o.u8(0); o.u8(0);  // superblock, free space, root entry, reserved
    o.u8(0); o.u8(8); o.u8(8); o.u8(0);  // shared header version, offset size, length size, reserved
    o.u16(kLeafK);
    o.u16(kInternalK);
    o.u32(0);              // consistency flags
    o.u64(0);              // base address
    o.u64(kUndef);         // free-space info
    o.u64(eof);
    o.u64(kUndef);         // driver info
    o.u64(0);              // root entry: link name offset
    o.u64(root_ohdr);
    o.u32(1);              // cache type 1: scratch pad holds B-tree and heap addresses
    o.u32(0);
    o.u64(btree);
    o.u64(heap_hdr);
    // root object header: one symbol-table message
    {
        Out m;
        m.u64(btree);
        m.u64(heap_hdr);
        Out msgs;
        put_msg(msgs, kMsgSymbolTable, 0, m);
        o.u8(1); o.u8(0); o.u16(1); o.u32(1); o.u32(msgs.b.size()); o.u32(0);
        o.bytes(msgs.b.data(), msgs.b.size());
    }
    // group B-tree: one leaf node pointing at one symbol-table node
    {
        const size_t start = o.b.size();
        o.bytes("TREE", 4);
        o.u8(0);  // group node
        o.u8(0);  // leaf
        o.u16(1);
        o.u64(kUndef);
        o.u64(kUndef);
        o.u64(0);                          // key 0: the empty name
        o.u64(snod);
        o.u64(name_off[order.back()]);     // key 1: the largest name
        o.pad_to(start + kBtreeNodeBytes);
    }
    // local heap
    o.bytes("HEAP", 4);
    o.u8(0);
    o.zeros(3);
    o.u64(heap.b.size());
    o.u64(free_off);
    o.u64(heap_data);
    o.bytes(heap.b.data(), heap.b.size());
    // symbol-table node
    {
        const size_t start = o.b.size();
        o.bytes("SNOD", 4);
        o.u8(1);
        o.u8(0);
        o.u16(datasets.size());
        for (size_t k : order) {
            o.u64(name_off[k]);
            o.u64(ohdr[k]);
            o.u32(0);
            o.u32(0);
            o.zeros(16);
        }
        o.pad_to(start + kSnodBytes);
    }
    for (size_t i = 0; i < datasets.size(); i++) {
        o.pad_to(ohdr[i]);
        Out h = dataset_header(datasets[i], data_at[i]);
        o.bytes(h.b.data(), h.b.size());
    }
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return "cannot create " + path;
    bool ok = std::fwrite(o.b.data(), 1, o.b.size(), f) == o.b.size();
    uint64_t at = o.b.size();
    static const uint8_t zero[8] = {0};
    for (size_t i = 0; i < datasets.size() && ok; i++) {
        if (at < data_at[i]) ok = std::fwrite(zero, 1, data_at[i] - at, f) == data_at[i] - at;
        at = data_at[i];
        const uint64_t n = nbytes(datasets[i]);
        if (n) ok = ok && std::fwrite(datasets[i].data, 1, n, f) == n;
        at += n;
    }
    if (ok && at < eof) ok = std::fwrite(zero, 1, eof - at, f) == eof - at;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? "" : "write failed: " + path;
}

// ---------------------------------------------------------------- reader

namespace {

struct Msg {
    uint16_t type;
    const uint8_t *d;
    size_t n;
};

struct Layout {
    int cls = -1;  // 0 compact, 1 contiguous, 2 chunked
    uint64_t addr = kUndef, size = 0;
    const uint8_t *compact = nullptr;
    std::vector<uint64_t> chunk;  // chunk dims (without the element-size entry)
};

struct Filter { int id; uint32_t flags; std::vector<uint32_t> vals; };

uint64_t rd(const uint8_t *p, int n)
{
    uint64_t v = 0;
    for (int i = 0; i < n; i++) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

}  // namespace

#define H5L_NEED(cond, what) \
    do {                      \
        if (!(cond)) return what; \
    } while (0)

namespace {

struct View {
    const std::vector<uint8_t> &b;
    bool in(uint64_t at, uint64_t n) const { return at <= b.size() && n <= b.size() - at; }
    const uint8_t *p(uint64_t at) const { return b.data() + at; }
};

std::string object_messages(const View &v, uint64_t at, std::vector<Msg> &out)
{
    H5L_NEED(v.in(at, 16), "object header out of file");
    const uint8_t *h = v.p(at);
    H5L_NEED(h[0] == 1, "object header version " + std::to_string(h[0]) + " not supported");
    const int nmsgs = (int)rd(h + 2, 2);
    std::vector<std::pair<uint64_t, uint64_t>> blocks{{at + 16, rd(h + 8, 4)}};
    for (size_t bi = 0; bi < blocks.size() && (int)out.size() < nmsgs; bi++) {
        uint64_t p = blocks[bi].first, end = p + blocks[bi].second;
        H5L_NEED(v.in(p, blocks[bi].second), "object header block out of file");
        while (p + 8 <= end && (int)out.size() < nmsgs) {
            const uint16_t type = (uint16_t)rd(v.p(p), 2);
            const size_t n = (size_t)rd(v.p(p + 2), 2);
            H5L_NEED(p + 8 + n <= end, "object header message overruns its block");
            out.push_back({type, v.p(p + 8), n});
            if (type == kMsgContinuation) {
                H5L_NEED(n >= 16, "bad continuation message");
                blocks.push_back({rd(v.p(p + 8), 8), rd(v.p(p + 16), 8)});
            }
            p += 8 + n;
        }
    }
    return "";
}

std::string parse_type(const uint8_t *d, size_t n, Type &t)
{
    H5L_NEED(n >= 8, "short datatype message");
    t.cls = d[0] & 0x0f;
    t.size = (int)rd(d + 4, 4);
    H5L_NEED(t.cls == kFixed || t.cls == kFloat || t.cls == kBitfield,
             "datatype class " + std::to_string(t.cls) + " not supported");
    H5L_NEED((d[1] & 0x01) == 0, "big-endian data not supported");
    if (t.cls == kFloat) H5L_NEED((d[1] & 0x40) == 0, "VAX float order not supported");
    t.is_signed = t.cls == kFixed ? (d[1] & 0x08) != 0 : t.cls == kFloat;
    return "";
}

std::string parse_space(const uint8_t *d, size_t n, std::vector<uint64_t> &dims)
{
    H5L_NEED(n >= 4, "short dataspace message");
    const int ver = d[0], rank = d[1];
    const size_t at = ver == 1 ? 8 : 4;
    H5L_NEED(ver == 1 || ver == 2, "dataspace version not supported");
    if (ver == 2 && d[3] == 0) {  // scalar
        dims.clear();
        return "";
    }
    H5L_NEED(n >= at + 8 * (size_t)rank, "short dataspace message");
    dims.resize(rank);
    for (int i = 0; i < rank; i++) dims[i] = rd(d + at + 8 * i, 8);
    return "";
}

std::string parse_layout(const uint8_t *d, size_t n, Layout &L)
{
    H5L_NEED(n >= 2, "short layout message");
    const int ver = d[0];
    if (ver == 3) {
        L.cls = d[1];
        if (L.cls == 0) {
            L.size = rd(d + 2, 2);
            L.compact = d + 4;
        } else if (L.cls == 1) {
            L.addr = rd(d + 2, 8);
            L.size = rd(d + 10, 8);
        } else if (L.cls == 2) {
            const int r1 = d[2];
            L.addr = rd(d + 3, 8);
            L.chunk.resize(r1 - 1);
            for (int i = 0; i < r1 - 1; i++) L.chunk[i] = rd(d + 11 + 4 * i, 4);
        } else {
            return "layout class not supported";
        }
        return "";
    }
    H5L_NEED(ver == 1 || ver == 2, "layout version not supported");
    const int r = d[1];
    L.cls = d[2];
    size_t p = 8;
    if (L.cls != 0) {
        L.addr = rd(d + p, 8);
        p += 8;
    }
    std::vector<uint64_t> dims(r);
    for (int i = 0; i < r; i++) dims[i] = rd(d + p + 4 * i, 4);
    p += 4 * r;
    if (L.cls == 2) L.chunk.assign(dims.begin(), dims.end() - 1);
    if (L.cls == 0) {
        L.size = rd(d + p, 4);
        L.compact = d + p + 4;
    }
    if (L.cls == 1) {
        L.size = 1;
        for (uint64_t x : dims) L.size *= x;
    }
    return "";
}

std::string parse_filters(const uint8_t *d, size_t n, std::vector<Filter> &fs)
{
    H5L_NEED(n >= 2, "short filter message");
    const int ver = d[0], count = d[1];
    size_t p = ver == 1 ? 8 : 2;
    for (int k = 0; k < count; k++) {
        Filter f;
        H5L_NEED(p + 4 <= n, "short filter message");
        f.id = (int)rd(d + p, 2);
        p += 2;
        size_t namelen = 0;
        if (ver == 1 || f.id >= 256) {
            namelen = rd(d + p, 2);
            p += 2;
        }
        f.flags = (uint32_t)rd(d + p, 2);
        const int nv = (int)rd(d + p + 2, 2);
        p += 4;
        p += ver == 1 ? pad8(namelen) : namelen;
        for (int i = 0; i < nv; i++) f.vals.push_back((uint32_t)rd(d + p + 4 * i, 4));
        p += 4 * nv;
        if (ver == 1 && (nv & 1)) p += 4;
        fs.push_back(f);
    }
    return "";
}

struct Dataset {
    Type type;
    std::vector<uint64_t> dims;
    Layout layout;
    std::vector<Filter> filters;
    std::vector<Msg> msgs;
};

std::string load_dataset(const View &v, uint64_t at, Dataset &ds)
{
    std::string e = object_messages(v, at, ds.msgs);
    if (!e.empty()) return e;
    bool have_t = false, have_s = false, have_l = false;
    for (const Msg &m : ds.msgs) {
        if (m.type == kMsgDatatype) { if (!(e = parse_type(m.d, m.n, ds.type)).empty()) return e; have_t = true; }
        if (m.type == kMsgDataspace) { if (!(e = parse_space(m.d, m.n, ds.dims)).empty()) return e; have_s = true; }
        if (m.type == kMsgLayout) { if (!(e = parse_layout(m.d, m.n, ds.layout)).empty()) return e; have_l = true; }
        if (m.type == kMsgFilters) { if (!(e = parse_filters(m.d, m.n, ds.filters)).empty()) return e; }
    }
    H5L_NEED(have_t && have_s && have_l, "object is not a dataset");
    return "";
}

std::string undo_filters(const std::vector<Filter> &fs, uint32_t mask, int elem, std::vector<uint8_t> &data,
                         size_t expect)
{
    for (int k = (int)fs.size() - 1; k >= 0; k--) {
        if (mask & (1u << k)) continue;
        const Filter &f = fs[k];
        if (f.id == 1) {  // deflate
            std::vector<uint8_t> out(expect);
            uLongf len = (uLongf)expect;
            const int rc = uncompress(out.data(), &len, data.data(), (uLong)data.size());
            H5L_NEED(rc == Z_OK, "deflate: corrupt chunk");
            out.resize(len);
            data.swap(out);
        } else if (f.id == 2) {  // shuffle: byte planes back to elements
            const int s = f.vals.empty() ? elem : (int)f.vals[0];
            const size_t ne = data.size() / s;
            std::vector<uint8_t> out(data.size());
            for (int b = 0; b < s; b++)
                for (size_t i = 0; i < ne; i++) out[i * s + b] = data[b * ne + i];
            std::copy(data.begin() + ne * s, data.end(), out.begin() + ne * s);
            data.swap(out);
        } else {
            return "filter " + std::to_string(f.id) + " not supported";
        }
    }
    return "";
}

// copies one decoded chunk at element offset off into the dataset image
void place_chunk(const std::vector<uint64_t> &dims, const std::vector<uint64_t> &chunk,
                 const std::vector<uint64_t> &off, int elem, const uint8_t *src, size_t src_bytes, uint8_t *dst)
{
    const int r = (int)dims.size();
    uint64_t total = 1;
    for (uint64_t c : chunk) total *= c;
    std::vector<uint64_t> idx(r, 0);
    for (uint64_t li = 0; li < total && (li + 1) * elem <= src_bytes; li++) {
        uint64_t rem = li, g = 0;
        bool inside = true;
        for (int k = r - 1; k >= 0; k--) {
            idx[k] = rem % chunk[k];
            rem /= chunk[k];
        }
        for (int k = 0; k < r; k++) {
            const uint64_t x = off[k] + idx[k];
            if (x >= dims[k]) { inside = false; break; }
            g = g * dims[k] + x;
        }
        if (inside) std::memcpy(dst + g * elem, src + li * elem, elem);
    }
}

std::string walk_chunks(const View &v, const Dataset &ds, uint64_t node, uint8_t *dst, int depth)
{
    H5L_NEED(depth < 64, "chunk index too deep");
    H5L_NEED(v.in(node, 24), "chunk index out of file");
    const uint8_t *h = v.p(node);
    H5L_NEED(std::memcmp(h, "TREE", 4) == 0 && h[4] == 1, "bad chunk index node");
    const int level = h[5], used = (int)rd(h + 6, 2);
    const int r = (int)ds.dims.size();
    const size_t key = 8 + 8 * (size_t)(r + 1);
    uint64_t p = node + 24;
    const int elem = ds.type.size;
    size_t expect = (size_t)elem;
    for (uint64_t c : ds.layout.chunk) expect *= c;
    for (int i = 0; i < used; i++) {
        H5L_NEED(v.in(p, key + 8), "chunk index entry out of file");
        const uint32_t size = (uint32_t)rd(v.p(p), 4), mask = (uint32_t)rd(v.p(p + 4), 4);
        std::vector<uint64_t> off(r);
        for (int k = 0; k < r; k++) off[k] = rd(v.p(p + 8 + 8 * k), 8);
        const uint64_t child = rd(v.p(p + key), 8);
        if (level > 0) {
            std::string e = walk_chunks(v, ds, child, dst, depth + 1);
            if (!e.empty()) return e;
        } else {
            H5L_NEED(v.in(child, size), "chunk out of file");
            std::vector<uint8_t> data(v.p(child), v.p(child) + size);
            std::string e = undo_filters(ds.filters, mask, elem, data, expect);
            if (!e.empty()) return e;
            place_chunk(ds.dims, ds.layout.chunk, off, elem, data.data(), data.size(), dst);
        }
        p += key + 8;
    }
    return "";
}

}  // namespace

std::string File::open(const std::string &path)
{
    entries_.clear();
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return "cannot open " + path;
    std::fseek(f, 0, SEEK_END);
    const long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf_.resize(len > 0 ? (size_t)len : 0);
    const bool ok = len > 0 && std::fread(buf_.data(), 1, buf_.size(), f) == buf_.size();
    std::fclose(f);
    if (!ok) return "cannot read " + path;
    const View v{buf_};
    static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    uint64_t sb = kUndef;
    for (uint64_t at = 0; v.in(at, 8); at = at ? 2 * at : 512)
        if (std::memcmp(v.p(at), sig, 8) == 0) { sb = at; break; }
    H5L_NEED(sb != kUndef, "not an HDF5 file: " + path);
    H5L_NEED(v.in(sb, 96), "truncated superblock");
    const uint8_t *s = v.p(sb);
    H5L_NEED(s[8] <= 1, "superblock version " + std::to_string(s[8]) + " not supported");
    H5L_NEED(s[13] == 8 && s[14] == 8, "only 8-byte offsets and lengths are supported");
    const size_t ste = s[8] == 0 ? 56 : 60;
    H5L_NEED(rd(s + 24, 8) == 0, "non-zero base address not supported");
    const uint64_t root = rd(s + ste + 8, 8);
    uint64_t btree = rd(s + ste + 24, 8), heap = rd(s + ste + 32, 8);
    std::vector<Msg> msgs;
    std::string e = object_messages(v, root, msgs);
    if (!e.empty()) return e;
    for (const Msg &m : msgs)
        if (m.type == kMsgSymbolTable && m.n >= 16) {
            btree = rd(m.d, 8);
            heap = rd(m.d + 8, 8);
        }
    H5L_NEED(v.in(heap, kHeapHeaderBytes) && std::memcmp(v.p(heap), "HEAP", 4) == 0, "bad local heap");
    const uint64_t heap_size = rd(v.p(heap + 8), 8), heap_data = rd(v.p(heap + 24), 8);
    H5L_NEED(v.in(heap_data, heap_size), "local heap out of file");
    // group B-tree, depth first
    std::vector<std::pair<uint64_t, int>> stack{{btree, 0}};
    while (!stack.empty()) {
        auto [node, depth] = stack.back();
        stack.pop_back();
        H5L_NEED(depth < 64 && v.in(node, 24), "bad group B-tree");
        const uint8_t *h = v.p(node);
        H5L_NEED(std::memcmp(h, "TREE", 4) == 0 && h[4] == 0, "bad group B-tree node");
        const int level = h[5], used = (int)rd(h + 6, 2);
        for (int i = 0; i < used; i++) {
            const uint64_t child = rd(v.p(node + 24 + 8 + 16 * (uint64_t)i), 8);
            if (level > 0) {
                stack.push_back({child, depth + 1});
                continue;
            }
            H5L_NEED(v.in(child, 8) && std::memcmp(v.p(child), "SNOD", 4) == 0, "bad symbol-table node");
            const int count = (int)rd(v.p(child + 6), 2);
            for (int k = 0; k < count; k++) {
                const uint64_t e0 = child + 8 + 40 * (uint64_t)k;
                H5L_NEED(v.in(e0, 40), "symbol-table entry out of file");
                const uint64_t off = rd(v.p(e0), 8);
                H5L_NEED(off < heap_size, "link name out of heap");
                const char *nm = reinterpret_cast<const char *>(v.p(heap_data + off));
                const size_t max = heap_size - off;
                entries_.push_back({std::string(nm, strnlen(nm, max)), rd(v.p(e0 + 8), 8)});
            }
        }
    }
    return "";
}

uint64_t File::find(const std::string &name) const
{
    for (const Entry &e : entries_)
        if (e.name == name) return e.ohdr;
    return kUndef;
}

bool File::has(const std::string &name) const { return find(name) != kUndef; }

std::vector<std::string> File::names() const
{
    std::vector<std::string> r;
    for (const Entry &e : entries_) r.push_back(e.name);
    return r;
}

std::string File::info(const std::string &name, Info &out) const
{
    const uint64_t at = find(name);
    if (at == kUndef) return "no dataset " + name;
    Dataset ds;
    std::string e = load_dataset(View{buf_}, at, ds);
    if (!e.empty()) return name + ": " + e;
    out.type = ds.type;
    out.dims = ds.dims;
    return "";
}

std::string File::read(const std::string &name, void *out, size_t out_bytes) const
{
    const uint64_t at = find(name);
    if (at == kUndef) return "no dataset " + name;
    const View v{buf_};
    Dataset ds;
    std::string e = load_dataset(v, at, ds);
    if (!e.empty()) return name + ": " + e;
    uint64_t n = (uint64_t)ds.type.size;
    for (uint64_t d : ds.dims) n *= d;
    if (n > out_bytes) return name + ": output buffer too small";
    uint8_t *dst = static_cast<uint8_t *>(out);
    std::memset(dst, 0, n);
    if (ds.layout.cls == 0) {
        std::memcpy(dst, ds.layout.compact, std::min<uint64_t>(n, ds.layout.size));
    } else if (ds.layout.cls == 1) {
        if (ds.layout.addr == kUndef || n == 0) return "";
        if (!v.in(ds.layout.addr, n)) return name + ": data out of file";
        std::memcpy(dst, v.p(ds.layout.addr), n);
    } else {
        if (ds.layout.chunk.size() != ds.dims.size()) return name + ": chunk rank mismatch";
        if (ds.layout.addr == kUndef) return "";
        e = walk_chunks(v, ds, ds.layout.addr, dst, 0);
        if (!e.empty()) return name + ": " + e;
    }
    return "";
}

std::string File::read_attr(const std::string &name, const std::string &attr, Type &type,
                            std::vector<uint8_t> &value) const
{
    const uint64_t at = find(name);
    if (at == kUndef) return "no dataset " + name;
    std::vector<Msg> msgs;
    std::string e = object_messages(View{buf_}, at, msgs);
    if (!e.empty()) return e;
    for (const Msg &m : msgs) {
        if (m.type != kMsgAttribute || m.n < 8) continue;
        const uint8_t *d = m.d;
        const int ver = d[0];
        const size_t nl = rd(d + 2, 2), tl = rd(d + 4, 2), sl = rd(d + 6, 2);
        size_t p = ver == 3 ? 9 : 8;
        auto adv = [&](size_t x) { return ver == 1 ? pad8(x) : x; };
        if (p + adv(nl) + adv(tl) + adv(sl) > m.n) return "attribute message overruns";
        const std::string an(reinterpret_cast<const char *>(d + p), strnlen(reinterpret_cast<const char *>(d + p), nl));
        p += adv(nl);
        if (an != attr) continue;
        if (!(e = parse_type(d + p, tl, type)).empty()) return e;
        p += adv(tl);
        std::vector<uint64_t> dims;
        if (!(e = parse_space(d + p, sl, dims)).empty()) return e;
        p += adv(sl);
        uint64_t cnt = 1;
        for (uint64_t x : dims) cnt *= x;
        const uint64_t bytes = cnt * (uint64_t)type.size;
        if (p + bytes > m.n) return "attribute value overruns";
        value.assign(d + p, d + p + bytes);
        return "";
    }
    return "no attribute " + attr + " on " + name;
}

}  // namespace h5l
