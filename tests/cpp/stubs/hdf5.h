// Stand-in for the HDF5 C API (declarations only): just what include/green/gpu/gpu_factory.h
// calls, so that the drop-in header can be compiled without libhdf5.  Compile check only.
#pragma once
#include <cstdint>
typedef int64_t hid_t;
typedef int herr_t;
#define H5F_ACC_RDONLY 0u
#define H5P_DEFAULT ((hid_t)0)
hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl);
herr_t H5Fclose(hid_t file);
