// h5_stub.h -- TEST INFRASTRUCTURE ONLY: declarations standing in for the
// HDF5 C API (absent from this image) so that the reference's src/MC.cpp
// compiles unchanged into oracle/_ref/. Every function does nothing and
// reports failure; the compiled reference is only used for its Monte Carlo
// functions, never for file output.
#pragma once
#include <cstdint>

typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;

#define H5P_DEFAULT ((hid_t)0)
#define H5S_ALL ((hid_t)0)
#define H5F_ACC_TRUNC 2u
#define H5T_IEEE_F64LE ((hid_t)1)
#define H5T_NATIVE_DOUBLE ((hid_t)2)
#define H5T_STD_I32LE ((hid_t)3)
#define H5T_NATIVE_INT32 ((hid_t)4)
#define H5T_NATIVE_INT64 ((hid_t)5)
#define H5T_NATIVE_HSIZE ((hid_t)6)

inline hid_t H5Fcreate(const char*, unsigned, hid_t, hid_t) { return -1; }
inline herr_t H5Fclose(hid_t) { return -1; }
inline hid_t H5Screate_simple(int, const hsize_t*, const hsize_t*) { return -1; }
inline herr_t H5Sclose(hid_t) { return -1; }
inline hid_t H5Dcreate(hid_t, const char*, hid_t, hid_t, hid_t, hid_t, hid_t) { return -1; }
inline hid_t H5Dcreate2(hid_t, const char*, hid_t, hid_t, hid_t, hid_t, hid_t) { return -1; }
inline herr_t H5Dwrite(hid_t, hid_t, hid_t, hid_t, hid_t, const void*) { return -1; }
inline herr_t H5Dclose(hid_t) { return -1; }
inline hid_t H5Gcreate2(hid_t, const char*, hid_t, hid_t, hid_t) { return -1; }
inline herr_t H5Gclose(hid_t) { return -1; }
