// Test infrastructure only: stand-in for the HDF5 C API subset used by
// MPulse's hdfstream.{cpp,t} (HDF5 is not installed).  The oracle harness
// reads fields straight from Storage, so every call succeeds.  With the
// environment variable MPULSE_REF_HDF5_LOG set, the writing calls are recorded
// instead of doing nothing: for each H5Fcreate(name) a text file
// "<name>.calls" lists the created datasets ("dataset <name> <type> <rank>
// <dims...> <offset> <bytes>") and "<name>.raw" holds the bytes each
// H5Dwrite was given, one dataset after the other.  That is what MPulse's
// FieldDiag / FieldSliceDiag hand to HDF5: the dataset names, the dataspace
// and the data (the grid in this shim's C-order layout).
#ifndef MPB_REFSHIM_HDF5_H
#define MPB_REFSHIM_HDF5_H
// The real hdf5.h pulls in <assert.h>; hdfstream.t relies on that.
#include <cassert>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>
typedef long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
enum {
  H5S_ALL = 0, H5P_DEFAULT = 0, H5T_NATIVE_INT = 1, H5T_NATIVE_FLOAT = 2,
  H5T_NATIVE_DOUBLE = 3, H5F_ACC_RDONLY = 0, H5F_ACC_TRUNC = 1,
  H5S_SELECT_SET = 0, H5P_FILE_ACCESS = 0
};

namespace mpb_h5log {
struct File {
  std::FILE *calls = nullptr, *raw = nullptr;
  long offset = 0;
};
struct Set {
  std::string name;
  hid_t file, type;
  std::vector<hsize_t> dims;
};
struct State {
  hid_t next = 100;
  std::map<hid_t, File> files;
  std::map<hid_t, std::vector<hsize_t> > spaces;
  std::map<hid_t, Set> sets;
};
inline State &state() {
  static State s;
  return s;
}
inline bool on() {
  const char *e = std::getenv("MPULSE_REF_HDF5_LOG");
  return e && *e;
}
inline long type_size(hid_t t) { return t == H5T_NATIVE_DOUBLE ? 8 : 4; }
}  // namespace mpb_h5log

inline hid_t H5Dopen(hid_t, const char *) { return 1; }
inline hid_t H5Dget_space(hid_t) { return 1; }
inline herr_t H5Sselect_hyperslab(hid_t, int, const hsize_t *, const hsize_t *,
                                  const hsize_t *, const hsize_t *) { return 0; }
inline herr_t H5Dread(hid_t, hid_t, hid_t, hid_t, hid_t, void *) { return 0; }
inline herr_t H5Dwrite(hid_t dset, hid_t type, hid_t, hid_t, hid_t, const void *data) {
  mpb_h5log::State &s = mpb_h5log::state();
  if (!s.sets.count(dset)) return 0;
  const mpb_h5log::Set &d = s.sets[dset];
  if (!s.files.count(d.file)) return 0;
  mpb_h5log::File &f = s.files[d.file];
  long n = 1;
  for (size_t q = 0; q < d.dims.size(); ++q) n *= long(d.dims[q]);
  const long bytes = n * mpb_h5log::type_size(type);
  std::fprintf(f.calls, "dataset %s %ld %d", d.name.c_str(), long(d.type), int(d.dims.size()));
  for (size_t q = 0; q < d.dims.size(); ++q) std::fprintf(f.calls, " %llu", d.dims[q]);
  std::fprintf(f.calls, " %ld %ld\n", f.offset, bytes);
  std::fwrite(data, 1, size_t(bytes), f.raw);
  f.offset += bytes;
  // the harness ends with _Exit: keep the record complete after every write
  std::fflush(f.calls);
  std::fflush(f.raw);
  return 0;
}
inline herr_t H5Dclose(hid_t) { return 0; }
inline hid_t H5Screate_simple(int rank, const hsize_t *dims, const hsize_t *) {
  mpb_h5log::State &s = mpb_h5log::state();
  const hid_t id = s.next++;
  s.spaces[id] = std::vector<hsize_t>(dims, dims + rank);
  return id;
}
inline hid_t H5Dcreate(hid_t file, const char *name, hid_t type, hid_t sid, hid_t) {
  mpb_h5log::State &s = mpb_h5log::state();
  const hid_t id = s.next++;
  mpb_h5log::Set d;
  d.name = name;
  d.file = file;
  d.type = type;
  d.dims = s.spaces[sid];
  s.sets[id] = d;
  return id;
}
inline herr_t H5Sclose(hid_t) { return 0; }
inline herr_t H5Fclose(hid_t file) {
  mpb_h5log::State &s = mpb_h5log::state();
  if (s.files.count(file)) {
    std::fclose(s.files[file].calls);
    std::fclose(s.files[file].raw);
    s.files.erase(file);
  }
  return 0;
}
inline hid_t H5Fopen(const char *, unsigned, hid_t) { return 1; }
inline hid_t H5Fcreate(const char *name, unsigned, hid_t, hid_t) {
  mpb_h5log::State &s = mpb_h5log::state();
  const hid_t id = s.next++;
  if (mpb_h5log::on()) {
    mpb_h5log::File f;
    f.calls = std::fopen((std::string(name) + ".calls").c_str(), "w");
    f.raw = std::fopen((std::string(name) + ".raw").c_str(), "wb");
    if (f.calls && f.raw) s.files[id] = f;
  }
  return id;
}
inline hid_t H5Pcreate(int) { return 1; }
inline herr_t H5Pclose(hid_t) { return 0; }
#endif
