// h5file.hpp -- a writer for the subset of the HDF5 file format that the
// reference's output files use (include/ssf_manager.hpp:375-557,
// include/energy_manager.hpp, src/MC.cpp:371-454): groups, contiguous
// datasets of little-endian integers and doubles, variable-length UTF-8
// string datasets, and attributes, with space for a dataset reserved up front
// and filled slice by slice (the reference's H5D_ALLOC_TIME_EARLY streaming
// of /ssf). libhdf5 is not available to this build; this is written from the
// published format specification (superblock version 2, version 2 object
// headers with compact link storage, global heap collections for the strings,
// Jenkins lookup3 checksums).
//
// Layout: the superblock sits at offset 0; dataset data and object headers are
// appended. commit() appends the object headers that changed since the last
// commit (a group changes when a member is added or its header moves) and
// rewrites the superblock to point at the current root, so after every commit
// the file is a complete HDF5 file; superseded headers stay behind as unused
// bytes. Slices written into reserved space need no commit.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace CMC {

// Jenkins' lookup3 hashlittle (byte-wise), the checksum of HDF5 metadata.
uint32_t h5_lookup3(const unsigned char* p, size_t n, uint32_t init);

class H5File {
public:
    explicit H5File(const std::string& path);
    ~H5File();
    H5File(const H5File&) = delete;
    H5File& operator=(const H5File&) = delete;

    // dtype: NumPy-style "<f8", "<i8", "<i4", "<u8", "<u4"; shape {} = scalar.
    void dataset(const std::string& path, const std::string& dtype, const std::vector<uint64_t>& shape,
                 const void* data);
    // Reserves zero-filled contiguous space for a dataset; returns a handle
    // for write_at (byte offsets into the dataset's row-major data).
    size_t reserve(const std::string& path, const std::string& dtype, const std::vector<uint64_t>& shape);
    void write_at(size_t handle, uint64_t byte_offset, const void* data, size_t nbytes);
    // Variable-length UTF-8 strings (one global heap collection).
    void strings(const std::string& path, const std::vector<std::string>& s);
    // Attribute of a group or dataset (created as a group if absent).
    void attribute(const std::string& path, const std::string& name, const std::string& dtype,
                   const std::vector<uint64_t>& shape, const void* data);
    void commit();
    void close();
    const std::string& path() const { return path_; }

private:
    struct Node;
    std::string path_;
    void* fp_ = nullptr;
    uint64_t eof_ = 0;
    std::unique_ptr<Node> root_;
    std::vector<Node*> reserved_;
    bool closed_ = false;

    Node* group_at(const std::string& path, bool create);
    Node* new_dataset(const std::string& path);
    uint64_t append(const std::vector<unsigned char>& b);
    uint64_t append_zeros(uint64_t n);
    uint64_t commit_node(Node& n, bool* moved);
    void write_superblock(uint64_t root_addr);
};

}  // namespace CMC
