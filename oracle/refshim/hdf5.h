// Test infrastructure only: inert stand-in for the HDF5 C API subset used by
// MPulse's hdfstream.{cpp,t} (HDF5 is not installed).  The oracle harness reads
// fields straight from Storage, so every call here succeeds and does nothing.
#ifndef MPB_REFSHIM_HDF5_H
#define MPB_REFSHIM_HDF5_H
// The real hdf5.h pulls in <assert.h>; hdfstream.t relies on that.
#include <cassert>
typedef long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
enum {
  H5S_ALL = 0, H5P_DEFAULT = 0, H5T_NATIVE_INT = 1, H5T_NATIVE_FLOAT = 2,
  H5T_NATIVE_DOUBLE = 3, H5F_ACC_RDONLY = 0, H5F_ACC_TRUNC = 1,
  H5S_SELECT_SET = 0, H5P_FILE_ACCESS = 0
};
inline hid_t H5Dopen(hid_t, const char *) { return 1; }
inline hid_t H5Dget_space(hid_t) { return 1; }
inline herr_t H5Sselect_hyperslab(hid_t, int, const hsize_t *, const hsize_t *,
                                  const hsize_t *, const hsize_t *) { return 0; }
inline herr_t H5Dread(hid_t, hid_t, hid_t, hid_t, hid_t, void *) { return 0; }
inline herr_t H5Dwrite(hid_t, hid_t, hid_t, hid_t, hid_t, const void *) { return 0; }
inline herr_t H5Dclose(hid_t) { return 0; }
inline hid_t H5Screate_simple(int, const hsize_t *, const hsize_t *) { return 1; }
inline hid_t H5Dcreate(hid_t, const char *, hid_t, hid_t, hid_t) { return 1; }
inline herr_t H5Sclose(hid_t) { return 0; }
inline herr_t H5Fclose(hid_t) { return 0; }
inline hid_t H5Fopen(const char *, unsigned, hid_t) { return 1; }
inline hid_t H5Fcreate(const char *, unsigned, hid_t, hid_t) { return 1; }
inline hid_t H5Pcreate(int) { return 1; }
inline herr_t H5Pclose(hid_t) { return 0; }
#endif
