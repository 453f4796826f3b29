// h5out.hpp -- the output container of the drivers.
//
// The reference writes /geometry, /energy and /ssf groups to HDF5
// (src/anneal.cpp:171-232). A path ending in ".npz" gets the same tree --
// group paths, dataset names, shapes, dtypes and attributes -- as an
// uncompressed NumPy .npz archive (dataset "/ssf/static_corr" is the member
// "ssf/static_corr.npy", attribute k_dims of /ssf is the member
// "ssf/@k_dims.npy"); any other path gets an HDF5 file written by H5File
// (h5file.hpp). pyro_cmc_b200.h5compat.File reads both back with the h5py-style
// access the reference's scripts use (f["/ssf/static_corr"][:],
// f["/ssf"].attrs["k_dims"]), and h5py reads the HDF5 files.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "h5file.hpp"

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
    // the reference's variable-length UTF-8 corr_lookup labels (HDF5), or
    // fixed-length byte strings (.npz); readers decode bytes,
    // scripts/plot_ssf.py:25-26
    void dataset_strings(const std::string& path, const std::vector<std::string>& s);

    // A dataset whose space is reserved now and filled by write_slice (byte
    // offsets into its row-major data), as the reference streams /ssf with
    // H5D_ALLOC_TIME_EARLY (include/ssf_manager.hpp:375-557). In HDF5 the
    // slices land in the file as they are written, and after commit() the file
    // holds the dataset, so an interrupted run leaves the slices written so far
    // readable; an .npz archive is written at close().
    size_t reserve(const std::string& path, const std::string& dtype, const std::vector<uint64_t>& shape,
                   size_t itemsize);
    void write_slice(size_t handle, uint64_t byte_offset, const void* data, size_t nbytes);
    // Makes everything written so far part of the file (HDF5; no-op for .npz).
    void commit();
    bool hdf5() const { return bool(h5_); }

    void close();
    const std::string& path() const { return path_; }

private:
    struct Entry {
        std::string name;
        uint32_t crc;
        uint64_t size;
        uint64_t offset;
    };
    struct Pending {
        std::string path, dtype;
        std::vector<uint64_t> shape;
        std::vector<unsigned char> data;
    };
    std::string path_;
    std::unique_ptr<H5File> h5_;
    void* fp_ = nullptr;
    std::vector<Entry> entries_;
    std::vector<Pending> pending_;
    uint64_t pos_ = 0;
    bool closed_ = false;
    void member(const std::string& name, const std::string& dtype, const std::vector<uint64_t>& shape,
                const void* data, size_t nbytes);
};

}  // namespace CMC
