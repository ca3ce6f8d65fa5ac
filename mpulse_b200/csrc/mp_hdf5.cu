// mp_hdf5.cu - HDF5 field dumps of the device state, the output of MPulse's
// FieldDiag (fielddiag.cpp:17-24, diagnostic.t:1-30) and FieldSliceDiag
// (fielddiag.cpp:46-115) through HDFostream (hdfstream.cpp:189-212,
// hdfstream.t:87-187).
//
// HDF5 is not a dependency of this library: the file is written by the small
// encoder below, which emits the subset of the HDF5 file format (version 0
// superblock, the root group as a symbol table with a version 1 B-tree and a
// local heap, version 1 object headers, contiguous datasets of little-endian
// IEEE doubles) that a single-process HDFostream produces.  What MPulse's
// stream does, and this file does the same way:
//   - datasets are named by HDFstream::getNextBlockName (hdfstream.cpp:70-81)
//     after HDFostream::open set the count to 0: "data0", "data1", "data2",
//     ... in the order they are written;
//   - a grid of MPulse's full index range (ghost cells included) with index
//     (i, j, k) has the dataspace {nz+2, ny+2, nx+2}, the dims reversed
//     (hdfstream.t:110), i.e. the element of (i, j, k) is dataset[k][j][i];
//     a slice is a rank-2 grid the same way (dataset[i2][i1]);
//   - the file name is the pattern after DiagnosticInterface::parsedFileName
//     (diagnostic.cpp:52-70): the first "#p" becomes the process id, the
//     first "#t" the time step.
// The data of a dataset is written when the field is added (downloaded from
// the device, converted to double); the metadata when the file is closed.
#include "mpulse_b200.h"

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace mpb {
void set_global_error(const char *msg);  // mp_api.cu: message for mp_last_error(NULL, ..)
int ctx_grid(const mp_ctx *c, int *nx, int *ny, int *nz);  // mp_api.cu
}  // namespace mpb

namespace {

const uint64_t kUndef = ~uint64_t(0);
const int kLeafK = 4;       // group leaf node K: 2K = 8 entries per symbol table node
const int kInternalK = 16;  // group internal node K: 2K = 32 children per B-tree node
const int kMaxDatasets = 2 * kLeafK * 2 * kInternalK;  // one B-tree node of full symbol table nodes

struct Dataset {
  std::string name;
  int rank = 3;
  uint64_t dims[3];
  uint64_t data_addr, data_size;
  uint64_t header_addr = 0, name_off = 0;
};

}  // namespace

struct mp_hdf5 {
  FILE *fp = nullptr;
  std::string path;
  uint64_t end = 0;  // next free address
  std::vector<Dataset> sets;
};

namespace {

// Little-endian byte buffer.
struct Buf {
  std::vector<unsigned char> b;
  void u8(unsigned v) { b.push_back((unsigned char)v); }
  void u16(unsigned v) { for (int q = 0; q < 2; ++q) u8((v >> (8 * q)) & 0xff); }
  void u32(uint32_t v) { for (int q = 0; q < 4; ++q) u8((v >> (8 * q)) & 0xff); }
  void u64(uint64_t v) { for (int q = 0; q < 8; ++q) u8((unsigned)((v >> (8 * q)) & 0xff)); }
  void bytes(const char *s, size_t n) { b.insert(b.end(), s, s + n); }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void pad8() { while (b.size() % 8) u8(0); }
  size_t size() const { return b.size(); }
};

bool write_at(FILE *fp, uint64_t addr, const Buf &buf) {
  if (fseek(fp, long(addr), SEEK_SET) != 0) return false;
  return fwrite(buf.b.data(), 1, buf.b.size(), fp) == buf.b.size();
}

// One header message of a version 1 object header: type, size of the data
// (padded to 8 bytes), flags, 3 reserved bytes, the data.
void message(Buf &h, unsigned type, const Buf &data, unsigned flags = 0) {
  Buf d = data;
  d.pad8();
  h.u16(type);
  h.u16(unsigned(d.size()));
  h.u8(flags);
  h.zeros(3);
  h.b.insert(h.b.end(), d.b.begin(), d.b.end());
}

// Version 1 object header: version, reserved, number of messages, reference
// count, size of the message data, 4 bytes of padding, then the messages.
Buf object_header(int nmsg, const Buf &msgs) {
  Buf h;
  h.u8(1);
  h.u8(0);
  h.u16(unsigned(nmsg));
  h.u32(1);
  h.u32(uint32_t(msgs.size()));
  h.zeros(4);
  h.b.insert(h.b.end(), msgs.b.begin(), msgs.b.end());
  return h;
}

// The object header of a dataset: dataspace (version 1), datatype (IEEE
// double, little endian), fill value (version 2, none defined), layout
// (version 3, contiguous).
Buf dataset_header(const Dataset &s) {
  Buf msgs;
  Buf sp;  // dataspace
  sp.u8(1);
  sp.u8(uint8_t(s.rank));
  sp.u8(0);  // no maximum dimensions
  sp.u8(0);
  sp.u32(0);
  for (int q = 0; q < s.rank; ++q) sp.u64(s.dims[q]);
  message(msgs, 0x0001, sp);
  Buf ty;  // datatype: class 1 (floating point), version 1
  ty.u8(0x11);
  ty.u8(0x20);  // byte order little endian, mantissa normalisation: msb implied
  ty.u8(63);    // sign bit position
  ty.u8(0);
  ty.u32(8);    // size
  ty.u16(0);    // bit offset
  ty.u16(64);   // bit precision
  ty.u8(52);    // exponent location
  ty.u8(11);    // exponent size
  ty.u8(0);     // mantissa location
  ty.u8(52);    // mantissa size
  ty.u32(1023); // exponent bias
  message(msgs, 0x0003, ty, 1);
  Buf fv;  // fill value, version 2: allocation time late, write time if set, none defined
  fv.u8(2);
  fv.u8(2);
  fv.u8(2);
  fv.u8(0);
  message(msgs, 0x0005, fv, 1);
  Buf ly;  // layout, version 3: contiguous
  ly.u8(3);
  ly.u8(1);
  ly.u64(s.data_addr);
  ly.u64(s.data_size);
  message(msgs, 0x0008, ly);
  return object_header(4, msgs);
}

int fail(const char *msg) {
  mpb::set_global_error(msg);
  return MP_ERR_INVALID;
}

}  // namespace

extern "C" {

int mp_diag_file_name(const char *pattern, int proc_id, long long time, char *out, size_t n) {
  if (!pattern || !out || n == 0) return MP_ERR_INVALID;
  std::string s = pattern;
  size_t pos = s.find("#p");
  if (pos != std::string::npos) s.replace(pos, 2, std::to_string(proc_id));
  pos = s.find("#t");
  if (pos != std::string::npos) s.replace(pos, 2, std::to_string(time));
  if (s.size() + 1 > n) return fail("mp_diag_file_name: output buffer too small");
  memcpy(out, s.c_str(), s.size() + 1);
  return MP_OK;
}

int mp_hdf5_create(const char *pattern, int proc_id, long long time, mp_hdf5 **out) {
  if (!pattern || !out) return fail("mp_hdf5_create: pattern and out must not be NULL");
  *out = nullptr;
  std::vector<char> name(strlen(pattern) + 64);
  int rc = mp_diag_file_name(pattern, proc_id, time, name.data(), name.size());
  if (rc != MP_OK) return rc;
  FILE *fp = fopen(name.data(), "wb");
  if (!fp) return fail("mp_hdf5_create: cannot create the file");
  mp_hdf5 *f = new mp_hdf5;
  f->fp = fp;
  f->path = name.data();
  f->end = 96;  // superblock with the root group's symbol table entry
  *out = f;
  return MP_OK;
}

}  // extern "C"

namespace {

// The next dataset of the file: a rank-1..3 grid of doubles, C order.
int write_dataset(mp_hdf5 *f, const double *data, int rank, const size_t *dims) {
  if (int(f->sets.size()) >= kMaxDatasets) return fail("mp_hdf5: at most 256 datasets per file");
  Dataset s;
  const size_t n = f->sets.size();
  s.name = "data" + std::to_string(n);
  s.rank = rank;
  size_t count = 1;
  for (int q = 0; q < rank; ++q) {
    s.dims[q] = uint64_t(dims[q]);
    count *= dims[q];
  }
  s.data_addr = f->end;
  s.data_size = uint64_t(count) * 8;
  Buf d;
  d.b.resize(s.data_size);
  for (size_t q = 0; q < count; ++q) {
    uint64_t bits;
    memcpy(&bits, &data[q], 8);
    for (int b = 0; b < 8; ++b) d.b[q * 8 + b] = (unsigned char)((bits >> (8 * b)) & 0xff);
  }
  if (!write_at(f->fp, s.data_addr, d)) return fail("mp_hdf5: write failed");
  f->end += s.data_size;
  f->sets.push_back(s);
  return MP_OK;
}

// The field `field` of ctx over MPulse's full index range: (nx+2) (ny+2)
// (nz+2) values, x fastest; x / y ghost cells are the periodic images.
int full_grid(mp_ctx *ctx, const char *field, std::vector<double> &g, int dims[3]) {
  size_t count = 0;
  int rc = mp_field_size(ctx, field, &count);
  if (rc != MP_OK) return rc;
  // the grid's interior x / y and stored planes, in the plane layout
  std::vector<double> plane(count);
  rc = mp_download(ctx, field, plane.data(), count);
  if (rc != MP_OK) return rc;
  // the plane layout holds (nz + 2) planes of ny * nx
  int nx = 0, ny = 0, nz = 0;
  rc = mpb::ctx_grid(ctx, &nx, &ny, &nz);
  if (rc != MP_OK) return rc;
  if (size_t(nz + 2) * ny * nx != count) return fail("mp_hdf5: not a full-grid field");
  const int NX = nx + 2, NY = ny + 2, NZ = nz + 2;
  g.assign(size_t(NX) * NY * NZ, 0.0);
  for (int k = 0; k < NZ; ++k)
    for (int j = 0; j < NY; ++j)
      for (int i = 0; i < NX; ++i) {
        const int ii = i == 0 ? nx : (i == nx + 1 ? 1 : i);
        const int jj = j == 0 ? ny : (j == ny + 1 ? 1 : j);
        g[(size_t(k) * NY + j) * NX + i] = plane[(size_t(k) * ny + (jj - 1)) * nx + (ii - 1)];
      }
  dims[0] = NX;
  dims[1] = NY;
  dims[2] = NZ;
  return MP_OK;
}

}  // namespace

extern "C" {

int mp_hdf5_write_grid(mp_hdf5 *f, const double *data, const size_t dims[3]) {
  if (!f || !data || !dims) return fail("mp_hdf5_write_grid: NULL argument");
  return write_dataset(f, data, 3, dims);
}

int mp_hdf5_write_field(mp_hdf5 *f, mp_ctx *ctx, const char *field) {
  if (!f || !ctx || !field) return fail("mp_hdf5_write_field: NULL argument");
  if (int(f->sets.size()) >= kMaxDatasets) return fail("mp_hdf5_write_field: at most 256 datasets per file");
  std::vector<double> g;
  int n[3];
  const int rc = full_grid(ctx, field, g, n);
  if (rc != MP_OK) return rc;
  const size_t dims[3] = {size_t(n[2]), size_t(n[1]), size_t(n[0])};
  return write_dataset(f, g.data(), 3, dims);
}

int mp_hdf5_write_slice(mp_hdf5 *f, mp_ctx *ctx, const char *field, int normal, int pos) {
  if (!f || !ctx || !field) return fail("mp_hdf5_write_slice: NULL argument");
  if (normal < 0 || normal > 2) return fail("mp_hdf5_write_slice: normal must be 0 (x), 1 (y) or 2 (z)");
  std::vector<double> g;
  int n[3];
  int rc = full_grid(ctx, field, g, n);
  if (rc != MP_OK) return rc;
  // FieldSliceDiag::fetchField: the slice is written only where pos lies
  // strictly inside the index range (the stream is inactive otherwise)
  if (!(pos > 0 && pos < n[normal] - 1)) return MP_OK;
  if (int(f->sets.size()) >= kMaxDatasets) return fail("mp_hdf5_write_slice: at most 256 datasets per file");
  const int d1 = normal == 0 ? 1 : 0, d2 = normal == 2 ? 1 : 2;
  std::vector<double> sl(size_t(n[d1]) * n[d2]);
  int i[3];
  i[normal] = pos;
  for (i[d2] = 0; i[d2] < n[d2]; ++i[d2])
    for (i[d1] = 0; i[d1] < n[d1]; ++i[d1])
      sl[size_t(i[d2]) * n[d1] + i[d1]] = g[(size_t(i[2]) * n[1] + i[1]) * n[0] + i[0]];
  const size_t dims[2] = {size_t(n[d2]), size_t(n[d1])};
  return write_dataset(f, sl.data(), 2, dims);
}

int mp_hdf5_close(mp_hdf5 *f) {
  if (!f) return MP_OK;
  int rc = MP_OK;
  std::vector<Dataset> &sets = f->sets;
  // dataset object headers
  for (Dataset &s : sets) {
    s.header_addr = f->end;
    const Buf h = dataset_header(s);
    if (!write_at(f->fp, s.header_addr, h)) rc = MP_ERR_INVALID;
    f->end += h.size();
  }
  // local heap of the root group: the empty string, then the names, each
  // NUL-terminated and padded to 8 bytes
  Buf heapdata;
  heapdata.zeros(8);
  for (Dataset &s : sets) {
    s.name_off = heapdata.size();
    heapdata.bytes(s.name.c_str(), s.name.size() + 1);
    heapdata.pad8();
  }
  // symbol table nodes hold the entries sorted by name
  std::vector<const Dataset *> sorted;
  for (const Dataset &s : sets) sorted.push_back(&s);
  std::sort(sorted.begin(), sorted.end(), [](const Dataset *a, const Dataset *b) { return a->name < b->name; });
  const int per = 2 * kLeafK;
  // (a file with no dataset: a B-tree without entries, as HDF5 creates an
  // empty group)
  const int nnodes = int((sorted.size() + per - 1) / per);
  std::vector<uint64_t> snod_addr(nnodes), last_name(nnodes, 0);
  for (int q = 0; q < nnodes; ++q) {
    Buf sn;
    sn.bytes("SNOD", 4);
    sn.u8(1);
    sn.u8(0);
    const int first = q * per, cnt = std::min(per, int(sorted.size()) - first);
    sn.u16(unsigned(std::max(cnt, 0)));
    for (int e = 0; e < per; ++e) {
      if (e < cnt) {
        const Dataset *s = sorted[first + e];
        sn.u64(s->name_off);
        sn.u64(s->header_addr);
        sn.u32(0);  // cache type: nothing cached
        sn.u32(0);
        sn.zeros(16);
        last_name[q] = s->name_off;
      } else {
        sn.zeros(40);
      }
    }
    snod_addr[q] = f->end;
    if (!write_at(f->fp, f->end, sn)) rc = MP_ERR_INVALID;
    f->end += sn.size();
  }
  // one leaf B-tree node (group, level 0) over the symbol table nodes: key i
  // is the heap offset of the last name of child i - 1, key 0 the empty string
  Buf bt;
  bt.bytes("TREE", 4);
  bt.u8(0);
  bt.u8(0);
  bt.u16(unsigned(nnodes));
  bt.u64(kUndef);
  bt.u64(kUndef);
  bt.u64(0);
  for (int q = 0; q < nnodes; ++q) {
    bt.u64(snod_addr[q]);
    bt.u64(last_name[q]);
  }
  bt.zeros(size_t(2 * kInternalK - nnodes) * 16);  // the node's full size
  const uint64_t btree_addr = f->end;
  if (!write_at(f->fp, btree_addr, bt)) rc = MP_ERR_INVALID;
  f->end += bt.size();
  // local heap header, then its data segment (no free block: offset 1)
  const uint64_t heap_addr = f->end;
  Buf hh;
  hh.bytes("HEAP", 4);
  hh.u8(0);
  hh.zeros(3);
  hh.u64(heapdata.size());
  hh.u64(1);
  hh.u64(heap_addr + 32);
  if (!write_at(f->fp, heap_addr, hh) || !write_at(f->fp, heap_addr + 32, heapdata)) rc = MP_ERR_INVALID;
  f->end = heap_addr + 32 + heapdata.size();
  // the root group's object header: a symbol table message, and a null
  // message as padding
  Buf msgs;
  Buf st;
  st.u64(btree_addr);
  st.u64(heap_addr);
  message(msgs, 0x0011, st);
  Buf nul;
  nul.zeros(8);
  message(msgs, 0x0000, nul);
  const Buf root = object_header(2, msgs);
  const uint64_t root_addr = f->end;
  if (!write_at(f->fp, root_addr, root)) rc = MP_ERR_INVALID;
  f->end += root.size();
  // superblock version 0 with the root group's symbol table entry
  Buf sb;
  const char sig[8] = {'\x89', 'H', 'D', 'F', '\r', '\n', '\x1a', '\n'};
  sb.bytes(sig, 8);
  sb.u8(0);  // superblock version
  sb.u8(0);  // free-space storage version
  sb.u8(0);  // root group symbol table entry version
  sb.u8(0);
  sb.u8(0);  // shared header message format version
  sb.u8(8);  // size of offsets
  sb.u8(8);  // size of lengths
  sb.u8(0);
  sb.u16(kLeafK);
  sb.u16(kInternalK);
  sb.u32(0);  // file consistency flags
  sb.u64(0);  // base address
  sb.u64(kUndef);  // free-space info
  sb.u64(f->end);  // end of file
  sb.u64(kUndef);  // driver information block
  sb.u64(0);  // root: link name offset
  sb.u64(root_addr);
  sb.u32(1);  // cache type 1: symbol table, scratch = B-tree, heap
  sb.u32(0);
  sb.u64(btree_addr);
  sb.u64(heap_addr);
  if (!write_at(f->fp, 0, sb)) rc = MP_ERR_INVALID;
  if (fclose(f->fp) != 0) rc = MP_ERR_INVALID;
  delete f;
  if (rc != MP_OK) return fail("mp_hdf5_close: write failed");
  return MP_OK;
}

}  // extern "C"
