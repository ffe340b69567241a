/* No-op HDF5 interface used only to compile the reference's own sources into the oracle
 * harness (the container has no HDF5; the harness writes no HDF5 output).
 * Test infrastructure only. */
#pragma once
#include <stddef.h>
typedef int hid_t; typedef int herr_t; typedef unsigned long long hsize_t;
#define H5P_DEFAULT 0
#define H5S_ALL 0
#define H5F_ACC_RDONLY 0
#define H5F_ACC_TRUNC 1
#define H5P_DATASET_CREATE 2
#define H5P_FILE_ACCESS 3
#define H5T_NATIVE_CHAR 1
#define H5T_NATIVE_DOUBLE 2
#define H5T_NATIVE_FLOAT 3
#define H5T_NATIVE_INT 4
#define H5T_NATIVE_UINT 5
#ifdef __cplusplus
extern "C" {
#endif
hid_t H5Fcreate(const char*, unsigned, hid_t, hid_t); hid_t H5Fopen(const char*, unsigned, hid_t); herr_t H5Fclose(hid_t);
hid_t H5Gcreate(hid_t, const char*, ...); hid_t H5Gopen(hid_t, const char*, ...); herr_t H5Gclose(hid_t);
hid_t H5Dcreate(hid_t, const char*, hid_t, hid_t, ...); hid_t H5Dcreate2(hid_t, const char*, hid_t, hid_t, hid_t, hid_t, hid_t);
hid_t H5Dopen(hid_t, const char*, ...); herr_t H5Dclose(hid_t); hid_t H5Dget_space(hid_t); hid_t H5Dget_create_plist(hid_t);
herr_t H5Dread(hid_t, hid_t, hid_t, hid_t, hid_t, void*); herr_t H5Dwrite(hid_t, hid_t, hid_t, hid_t, hid_t, const void*);
hid_t H5Pcreate(hid_t); herr_t H5Pclose(hid_t); herr_t H5Pset_cache(hid_t, int, size_t, size_t, double);
herr_t H5Pset_chunk(hid_t, int, const hsize_t*); herr_t H5Pset_deflate(hid_t, unsigned);
hid_t H5Screate_simple(int, const hsize_t*, const hsize_t*); herr_t H5Sclose(hid_t); int H5Sget_simple_extent_dims(hid_t, hsize_t*, hsize_t*);
hid_t H5Tcopy(hid_t);
#ifdef __cplusplus
}
#endif
