// h5file.h -- a self-contained writer and reader of HDF5 files for the
// checkpoint, snapshot and trajectory layouts of src/checkpoint.jl and
// src/io.jl (no HDF5 library is linked).
//
// Files follow the published HDF5 file format specification: a version-2
// superblock, version-2 object headers ("OHDR", Jenkins lookup3 checksums),
// groups in compact link storage (Link Info, Group Info and Link messages),
// attributes in the object header (Attribute message version 3) and datasets
// with contiguous layout (Dataspace v2, Datatype v1, Fill Value v3, Data
// Layout v3).  Datasets are float64 or int64, little-endian; attributes are
// float64, int64 or null-terminated ASCII strings.  Array dimensions are
// stored in HDF5 order (slowest first), i.e. reversed from the column-major
// (Julia) shape, and the bytes are the column-major buffer unchanged -- the
// way HDF5.jl stores a Julia array.  The reader accepts the files this writer
// produces (superblock v2, version-2 object headers, compact groups,
// contiguous datasets) and rejects anything else with a message.
#pragma once

#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

namespace bsn {
namespace h5 {

// Bob Jenkins' lookup3 hashlittle (public domain, 2006), the checksum of
// HDF5's version-2 metadata.
uint32_t lookup3(const uint8_t* key, size_t length, uint32_t initval = 0);

enum Kind { F64 = 0, I64 = 1, STR = 2 };

struct Attr {
    std::string name;
    Kind kind = F64;
    double d = 0.0;
    int64_t i = 0;
    std::string s;
};

struct Dataset {
    std::string name;
    Kind kind = F64;                 // F64 or I64
    std::vector<uint64_t> dims;      // HDF5 order (slowest first); empty = scalar
    const void* data = nullptr;      // writer: the element bytes (column-major source order)
    std::vector<Attr> attrs;
    uint64_t bytes() const;
};

struct Group {
    std::string name;
    std::vector<Attr> attrs;
    std::vector<Group> groups;
    std::vector<Dataset> dsets;
};

Attr attr_f64(const std::string& n, double v);
Attr attr_i64(const std::string& n, int64_t v);
Attr attr_str(const std::string& n, const std::string& v);

// Write root (its name is ignored) to path, replacing the file.
bool write_file(const std::string& path, const Group& root, std::string* err);

// The reader: the tree of a file with, per dataset, its file offset and size;
// read_data copies a dataset's bytes into dst.
struct RDataset {
    Kind kind = F64;
    std::vector<uint64_t> dims;
    uint64_t addr = 0, size = 0;
    std::map<std::string, Attr> attrs;
    uint64_t count() const;
};
struct RGroup {
    std::map<std::string, Attr> attrs;
    std::map<std::string, RGroup> groups;
    std::map<std::string, RDataset> dsets;
};

class Reader {
public:
    ~Reader();
    bool open(const std::string& path, std::string* err);
    const RGroup& root() const { return root_; }
    // the group or dataset at a '/'-separated path (nullptr if absent)
    const RGroup* group(const std::string& path) const;
    const RDataset* dataset(const std::string& path) const;
    bool read_data(const RDataset& d, void* dst, uint64_t cap_bytes, std::string* err) const;

private:
    bool parse_object(uint64_t addr, RGroup* g, RDataset* d, bool* is_dataset, int depth, std::string* err);
    bool read_at(uint64_t off, void* dst, uint64_t n) const;
    FILE* f_ = nullptr;
    uint64_t eof_ = 0;
    RGroup root_;
};

// Attribute lookup helpers for readers of the layouts (false if absent or of
// another kind; integers convert to double for f64 requests).
bool get_f64(const std::map<std::string, Attr>& a, const char* name, double* v);
bool get_i64(const std::map<std::string, Attr>& a, const char* name, int64_t* v);
bool get_str(const std::map<std::string, Attr>& a, const char* name, std::string* v);

}  // namespace h5
}  // namespace bsn
