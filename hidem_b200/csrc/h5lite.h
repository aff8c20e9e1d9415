// Minimal HDF5 writer / reader for the checkpoint layout and the reference's input files
// (written from the public HDF5 file-format specification).
// Writer: superblock version 2, version-2 object headers, groups with compact link storage
// (Link Info + Group Info + Link messages), 1-D contiguous datasets, version-3 attribute
// messages, little-endian integer and IEEE float types, Jenkins lookup3 checksums.
// Reader: that layout, and what libhdf5 writes by default — superblock version 0 / 1,
// version-1 object headers with continuation blocks, symbol-table groups (version-1 group
// B-tree, symbol nodes, local heap), contiguous, compact and chunked datasets (version-1
// chunk B-tree) with the deflate (zlib) and shuffle filters, attribute messages 1-3.
// Anything else (dense link storage, version-4 layouts, other filters, big-endian or
// compound types, shared messages) is reported as unsupported rather than guessed.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace h5lite {

enum class Type : uint8_t { I8, U8, I32, U32, I64, U64, F32, F64 };

size_t type_size(Type t);

struct Attr {
    std::string name;
    Type type = Type::I32;
    bool scalar = true;          // scalar dataspace, else 1-D of data.size()/type_size
    std::vector<uint8_t> data;   // little-endian element bytes
};

struct Filter {
    uint16_t id = 0;              // 1 deflate, 2 shuffle
    bool optional = false;
    std::vector<uint32_t> values; // client data (deflate level; shuffle element size)
};

struct Dataset {
    std::string name;
    Type type = Type::F64;
    uint64_t count = 0;
    const void *data = nullptr;  // writer: element bytes (count * type_size)
    uint64_t fileOffset = 0;     // reader: where the elements are (contiguous storage)
    std::vector<Attr> attrs;
    // reader: storage of the dataset
    int layout = 1;                          // 0 compact, 1 contiguous, 2 chunked
    std::vector<uint64_t> dims;              // dataspace extent, row-major
    uint64_t storedBytes = ~0ull;            // contiguous: bytes stored
    std::vector<uint8_t> compact;            // compact: the element bytes
    std::vector<uint64_t> chunk;             // chunked: chunk extent per dimension
    uint64_t chunkIndex = ~0ull;             // chunked: version-1 B-tree of the chunks
    std::vector<Filter> filters;             // chunked: the filter pipeline in order
};

struct Group {
    std::string name;
    std::vector<Attr> attrs;
    std::vector<Group> groups;
    std::vector<Dataset> datasets;

    const Group *group(const std::string &n) const;
    const Dataset *dataset(const std::string &n) const;
    const Attr *attr(const std::string &n) const;
};

template <class T>
Attr scalar_attr(const std::string &name, Type t, T v) {
    Attr a;
    a.name = name;
    a.type = t;
    a.scalar = true;
    a.data.resize(sizeof(T));
    std::memcpy(a.data.data(), &v, sizeof(T));
    return a;
}

template <class T>
Attr array_attr(const std::string &name, Type t, const std::vector<T> &v) {
    Attr a;
    a.name = name;
    a.type = t;
    a.scalar = false;
    a.data.resize(sizeof(T) * v.size());
    if (!v.empty()) std::memcpy(a.data.data(), v.data(), a.data.size());
    return a;
}

// HDF5's metadata checksum: Bob Jenkins' lookup3 hashlittle over bytes, initial value 0.
uint32_t lookup3(const uint8_t *key, size_t length, uint32_t initval = 0);

bool write_file(const std::string &path, const Group &root, std::string &err);
bool read_file(const std::string &path, Group &root, std::string &err);
// copies a dataset's elements (count * type_size bytes) out of the file
bool read_dataset(const std::string &path, const Dataset &d, void *out, std::string &err);

}  // namespace h5lite
