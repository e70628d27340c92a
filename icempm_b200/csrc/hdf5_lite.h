// hdf5_lite.h -- the subset of the HDF5 file format iceMPM's files use,
// written and read without libhdf5.
//
// iceMPM writes its snapshots and reads its raw point clouds through the
// HDF5 C++ API (simulation/snapshotmanager.cpp:14-304). Files here follow
// the layout that library produces for such files (the reference's
// geometries_2d/*.h5 are examples):
//   superblock version 0, 8-byte offsets and lengths, group K = 4 / 16;
//   the root group as a symbol table: a version-1 B-tree node (type 0), one
//   symbol-table node ("SNOD") and a local heap holding the link names;
//   version-1 object headers with dataspace (v1), datatype (v1), fill value
//   (v2), data layout (v3) and attribute (v1) messages.
// The writer emits contiguous datasets of little-endian integers, floats
// and bitfields with one-element attributes. The reader also takes chunked
// datasets (version-1 B-tree chunk index) with the deflate and shuffle
// filters, and object-header continuation blocks. Everything is
// little-endian; big-endian types are rejected.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace h5l {

// datatype classes of the HDF5 datatype message
enum : int { kFixed = 0, kFloat = 1, kBitfield = 4 };

struct Type {
    int cls = kFixed;
    int size = 0;         // bytes
    bool is_signed = true;  // fixed-point only
};
inline Type f64() { return {kFloat, 8, true}; }
inline Type f32() { return {kFloat, 4, true}; }
inline Type i16() { return {kFixed, 2, true}; }
inline Type i32() { return {kFixed, 4, true}; }
inline Type i64() { return {kFixed, 8, true}; }
inline Type b8() { return {kBitfield, 1, false}; }

struct Attr {
    std::string name;
    Type type;
    std::vector<uint8_t> value;  // one element, little-endian
};
template <class T> Attr attr(const std::string &name, Type t, T v)
{
    Attr a{name, t, std::vector<uint8_t>(sizeof(T))};
    static_assert(sizeof(T) <= 8, "scalar attribute");
    std::memcpy(a.value.data(), &v, sizeof(T));
    return a;
}

struct DatasetSpec {
    std::string name;
    Type type;
    std::vector<uint64_t> dims;
    const void *data = nullptr;  // product(dims) * type.size bytes
    std::vector<Attr> attrs;
};

// Writes the datasets into a new file at path (truncating it). Returns an
// empty string on success, else the reason.
std::string write_file(const std::string &path, const std::vector<DatasetSpec> &datasets);

class File {
public:
    // Opens and indexes the root group; "" on success, else the reason.
    std::string open(const std::string &path);
    bool has(const std::string &name) const;
    std::vector<std::string> names() const;
    struct Info {
        Type type;
        std::vector<uint64_t> dims;
    };
    std::string info(const std::string &name, Info &out) const;
    // Reads the whole dataset as stored (its own type) into out, which
    // holds out_bytes bytes.
    std::string read(const std::string &name, void *out, size_t out_bytes) const;
    // Reads attribute `attr` of dataset `name` (type and raw little-endian
    // bytes of all its elements).
    std::string read_attr(const std::string &name, const std::string &attr, Type &type,
                          std::vector<uint8_t> &value) const;

private:
    std::vector<uint8_t> buf_;
    struct Entry { std::string name; uint64_t ohdr; };
    std::vector<Entry> entries_;
    uint64_t find(const std::string &name) const;
};

}  // namespace h5l
