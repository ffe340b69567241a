// No-op HDF5 for the oracle harness (test infrastructure): the harness writes no HDF5.
#include <hdf5.h>

extern "C" {
hid_t H5Fcreate(const char *, unsigned, hid_t, hid_t) { return -1; }
hid_t H5Fopen(const char *, unsigned, hid_t) { return -1; }
herr_t H5Fclose(hid_t) { return 0; }
hid_t H5Gcreate(hid_t, const char *, ...) { return -1; }
hid_t H5Gopen(hid_t, const char *, ...) { return -1; }
herr_t H5Gclose(hid_t) { return 0; }
hid_t H5Dcreate(hid_t, const char *, hid_t, hid_t, ...) { return -1; }
hid_t H5Dcreate2(hid_t, const char *, hid_t, hid_t, hid_t, hid_t, hid_t) { return -1; }
hid_t H5Dopen(hid_t, const char *, ...) { return -1; }
herr_t H5Dclose(hid_t) { return 0; }
hid_t H5Dget_space(hid_t) { return -1; }
hid_t H5Dget_create_plist(hid_t) { return -1; }
herr_t H5Dread(hid_t, hid_t, hid_t, hid_t, hid_t, void *) { return -1; }
herr_t H5Dwrite(hid_t, hid_t, hid_t, hid_t, hid_t, const void *) { return -1; }
hid_t H5Pcreate(hid_t) { return -1; }
herr_t H5Pclose(hid_t) { return 0; }
herr_t H5Pset_cache(hid_t, int, size_t, size_t, double) { return 0; }
herr_t H5Pset_chunk(hid_t, int, const hsize_t *) { return 0; }
herr_t H5Pset_deflate(hid_t, unsigned) { return 0; }
hid_t H5Screate_simple(int, const hsize_t *, const hsize_t *) { return -1; }
herr_t H5Sclose(hid_t) { return 0; }
int H5Sget_simple_extent_dims(hid_t, hsize_t *, hsize_t *) { return 0; }
hid_t H5Tcopy(hid_t) { return -1; }
}
