// Stand-in for the HDF5 lite API (declarations only); see hdf5.h.
#pragma once
#include "hdf5.h"
herr_t H5LTread_dataset_long(hid_t loc, const char* name, long* buf);
herr_t H5LTread_dataset_double(hid_t loc, const char* name, double* buf);
