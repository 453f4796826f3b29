// h5out.hpp -- the output container of the drivers.
//
// The reference writes /geometry, /energy and /ssf groups to HDF5
// (src/anneal.cpp:171-232). libhdf5 is not available to this build, so the
// same tree -- group paths, dataset names, shapes, dtypes and attributes --
// is written as an uncompressed NumPy .npz archive: dataset "/ssf/static_corr"
// is the member "ssf/static_corr.npy", attribute k_dims of /ssf is the member
// "ssf/@k_dims.npy". pyro_cmc_b200.h5compat.File reads it back with the
// h5py-style access the reference's scripts use (f["/ssf/static_corr"][:],
// f["/ssf"].attrs["k_dims"]).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace CMC {

class OutFile {
public:
    explicit OutFile(const std::string& path);
    ~OutFile();  // finishes the archive if close() was not called
    OutFile(const OutFile&) = delete;
    OutFile& operator=(const OutFile&) = delete;

    // dtype: NumPy descr, e.g. "<f8", "<i8", "<i4", "<u8", "|S2"
    void dataset(const std::string& path, const std::string& dtype, const std::vector<uint64_t>& shape,
                 const void* data, size_t itemsize);
    void attribute(const std::string& group, const std::string& name, const std::string& dtype,
                   const std::vector<uint64_t>& shape, const void* data, size_t itemsize);

    void dataset_f64(const std::string& path, const std::vector<uint64_t>& shape, const double* d) {
        dataset(path, "<f8", shape, d, 8);
    }
    void dataset_i64(const std::string& path, const std::vector<uint64_t>& shape, const int64_t* d) {
        dataset(path, "<i8", shape, d, 8);
    }
    void dataset_i32(const std::string& path, const std::vector<uint64_t>& shape, const int32_t* d) {
        dataset(path, "<i4", shape, d, 4);
    }
    void dataset_u64(const std::string& path, const std::vector<uint64_t>& shape, const uint64_t* d) {
        dataset(path, "<u8", shape, d, 8);
    }
    // fixed-length byte strings (the reference's variable-length UTF-8
    // corr_lookup labels; readers decode bytes, scripts/plot_ssf.py:25-26)
    void dataset_strings(const std::string& path, const std::vector<std::string>& s);

    void close();
    const std::string& path() const { return path_; }

private:
    struct Entry {
        std::string name;
        uint32_t crc;
        uint64_t size;
        uint64_t offset;
    };
    std::string path_;
    void* fp_ = nullptr;
    std::vector<Entry> entries_;
    uint64_t pos_ = 0;
    bool closed_ = false;
    void member(const std::string& name, const std::string& dtype, const std::vector<uint64_t>& shape,
                const void* data, size_t nbytes);
};

}  // namespace CMC
