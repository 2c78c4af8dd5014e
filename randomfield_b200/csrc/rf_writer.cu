// rf_writer.cu -- result files of a generated field (host code only).
//
// The reference writes each field as an HDF5 file holding the dataset
// "samples" and an XDMF file describing the mesh (write_MONO_proc_result,
// writeResultFile_RF.f90:737-829; write_XMF_Elements, :835-938), and puts the
// run's parameters on the HDF5 file as attributes (write_HDF5_attributes,
// :1758-1849).  No HDF5 library is available to this build, so the HDF5 file
// is produced directly from the published file-format specification, in its
// oldest layout, which every HDF5 reader accepts:
//   superblock version 0 (8-byte offsets and lengths, group K 4 / 16);
//   root group: version-1 object header with a symbol-table message (v1
//     B-tree, local heap, one symbol-table node) and one attribute message per
//     run parameter;
//   each dataset: version-1 object header with dataspace (version 1),
//     datatype (IEEE little-endian double), fill value (version 2) and
//     contiguous layout (version 3) messages, data stored contiguously.
// The local heap marks "no free block" with offset 1, as the HDF5 library
// does (valid offsets are multiples of 8).
#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rf_internal.h"

using namespace rfh;

namespace {

constexpr uint64_t kUndef = ~0ull;  // undefined address
constexpr uint64_t kHeapFreeNull = 1;
constexpr int kLeafK = 4, kInternalK = 16;

struct Buf {
  std::vector<unsigned char> b;
  size_t size() const { return b.size(); }
  void u8(unsigned v) { b.push_back((unsigned char)v); }
  void u16(unsigned v) { for (int i = 0; i < 2; ++i) u8((v >> (8 * i)) & 0xff); }
  void u32(uint32_t v) { for (int i = 0; i < 4; ++i) u8((v >> (8 * i)) & 0xff); }
  void u64(uint64_t v) { for (int i = 0; i < 8; ++i) u8((unsigned)((v >> (8 * i)) & 0xff)); }
  void bytes(const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    b.insert(b.end(), c, c + n);
  }
  void pad8() { while (b.size() % 8) u8(0); }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void put64(size_t at, uint64_t v) { for (int i = 0; i < 8; ++i) b[at + i] = (unsigned char)((v >> (8 * i)) & 0xff); }
};

size_t pad8(size_t n) { return (n + 7) / 8 * 8; }

// Datatype message bodies (class and version 1 in the first byte).
Buf dtype_f64() {
  Buf d;
  d.u8(0x11);            // version 1, class 1 (floating point)
  d.u8(0x20);            // little-endian, no padding, mantissa normalisation: implied msb
  d.u8(63);              // sign bit position
  d.u8(0);
  d.u32(8);              // size
  d.u16(0);              // bit offset
  d.u16(64);             // bit precision
  d.u8(52);              // exponent location
  d.u8(11);              // exponent size
  d.u8(0);               // mantissa location
  d.u8(52);              // mantissa size
  d.u32(1023);           // exponent bias
  return d;
}
Buf dtype_i32() {
  Buf d;
  d.u8(0x10);            // version 1, class 0 (fixed point)
  d.u8(0x08);            // little-endian, signed
  d.u8(0);
  d.u8(0);
  d.u32(4);
  d.u16(0);              // bit offset
  d.u16(32);             // bit precision
  return d;
}
// Dataspace message version 1: rank 0 is a scalar.
Buf dspace(const std::vector<uint64_t>& dims) {
  Buf d;
  d.u8(1);
  d.u8((unsigned)dims.size());
  d.u8(0);  // no maximum dimensions
  d.u8(0);
  d.u32(0);
  for (uint64_t v : dims) d.u64(v);
  return d;
}

struct Message {
  unsigned type;
  unsigned flags;
  Buf body;
};

// Version-1 object header at the end of `f`: 16-byte prefix, then the
// messages (8-byte header each, bodies padded to 8 bytes).
void object_header(Buf& f, const std::vector<Message>& msgs) {
  size_t total = 0;
  for (const Message& m : msgs) total += 8 + pad8(m.body.size());
  f.u8(1);
  f.u8(0);
  f.u16((unsigned)msgs.size());
  f.u32(1);  // reference count
  f.u32((uint32_t)total);
  f.u32(0);  // alignment of the first message
  for (const Message& m : msgs) {
    f.u16(m.type);
    f.u16((unsigned)pad8(m.body.size()));
    f.u8(m.flags);
    f.u8(0);
    f.u8(0);
    f.u8(0);
    f.bytes(m.body.b.data(), m.body.size());
    f.pad8();
  }
}

Message attribute(const std::string& name, const Buf& dt, const std::vector<uint64_t>& dims, const void* data,
                  size_t bytes) {
  const Buf ds = dspace(dims);
  Message m{0x000C, 0, Buf()};
  Buf& a = m.body;
  a.u8(1);
  a.u8(0);
  a.u16((unsigned)(name.size() + 1));
  a.u16((unsigned)dt.size());
  a.u16((unsigned)ds.size());
  a.bytes(name.c_str(), name.size() + 1);
  a.pad8();
  a.bytes(dt.b.data(), dt.size());
  a.pad8();
  a.bytes(ds.b.data(), ds.size());
  a.pad8();
  a.bytes(data, bytes);
  return m;
}

struct Dataset {
  std::string name;
  std::vector<uint64_t> dims;  // C order (last fastest)
  const double* data;
};

// The whole file in memory: superblock, root group (object header, local
// heap, B-tree node, symbol-table node), dataset headers, raw data.
int build_h5(const std::vector<Dataset>& sets, const std::vector<Message>& rootAttrs, Buf& f) {
  if (sets.empty() || (int)sets.size() > 2 * kLeafK) return fail(RF_EINVAL_ARG, "1 to %d datasets per file", 2 * kLeafK);
  // local heap data segment: "" at 0, then the names (sorted, 8-byte aligned)
  std::vector<size_t> order(sets.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return sets[a].name < sets[b].name; });
  Buf heap;
  heap.zeros(8);
  std::vector<size_t> nameOff(sets.size());
  for (size_t i : order) {
    nameOff[i] = heap.size();
    heap.bytes(sets[i].name.c_str(), sets[i].name.size() + 1);
    heap.pad8();
  }

  // superblock (96 bytes); addresses patched below
  f.bytes("\x89HDF\r\n\x1a\n", 8);
  f.u8(0);  // superblock version
  f.u8(0);  // free-space version
  f.u8(0);  // root group symbol table entry version
  f.u8(0);
  f.u8(0);  // shared header message version
  f.u8(8);  // size of offsets
  f.u8(8);  // size of lengths
  f.u8(0);
  f.u16(kLeafK);
  f.u16(kInternalK);
  f.u32(0);  // consistency flags
  f.u64(0);  // base address
  f.u64(kUndef);  // free-space info
  const size_t eofAt = f.size();
  f.u64(0);  // end of file (patched)
  f.u64(kUndef);  // driver information block
  // root group symbol table entry
  f.u64(0);  // link name offset
  const size_t rootOhAt = f.size();
  f.u64(0);  // object header address (patched)
  f.u32(1);  // cache type 1: B-tree and heap addresses in the scratch pad
  f.u32(0);
  const size_t scratchAt = f.size();
  f.u64(0);  // B-tree address (patched)
  f.u64(0);  // heap address (patched)

  // root object header: symbol table message + attributes
  const uint64_t rootOh = f.size();
  const size_t heapHdrSize = 32, btreeSize = 24 + (2 * kInternalK + 1) * 8 + 2 * kInternalK * 8;
  const size_t snodSize = 8 + 2 * kLeafK * 40;
  std::vector<Message> rootMsgs;
  Message stab{0x0011, 0, Buf()};
  stab.body.u64(0);
  stab.body.u64(0);  // patched once the addresses are known
  rootMsgs.push_back(stab);
  for (const Message& m : rootAttrs) rootMsgs.push_back(m);
  object_header(f, rootMsgs);
  const size_t stabBodyAt = rootOh + 16 + 8;  // first message's body
  // local heap
  const uint64_t heapAddr = f.size();
  f.bytes("HEAP", 4);
  f.u8(0);
  f.zeros(3);
  f.u64(heap.size());
  f.u64(kHeapFreeNull);
  f.u64(heapAddr + heapHdrSize);
  f.bytes(heap.b.data(), heap.size());
  // B-tree node (group node, level 0, one child)
  const uint64_t btreeAddr = f.size();
  const uint64_t snodAddr = btreeAddr + btreeSize;
  f.bytes("TREE", 4);
  f.u8(0);  // group node
  f.u8(0);  // leaf level
  f.u16(1);
  f.u64(kUndef);
  f.u64(kUndef);
  f.u64(0);                      // key 0: "" (below every name)
  f.u64(snodAddr);               // child 0
  f.u64(nameOff[order.back()]);  // key 1: the largest name in child 0
  f.zeros(btreeSize - 24 - 3 * 8);
  // symbol table node; entries sorted by name, object headers patched below
  f.bytes("SNOD", 4);
  f.u8(1);
  f.u8(0);
  f.u16((unsigned)sets.size());
  std::vector<size_t> entryOhAt(sets.size());
  for (size_t i : order) {
    f.u64(nameOff[i]);
    entryOhAt[i] = f.size();
    f.u64(0);
    f.u32(0);  // cache type 0
    f.u32(0);
    f.zeros(16);
  }
  f.zeros(snodSize - 8 - sets.size() * 40);
  // dataset headers, then the data
  std::vector<uint64_t> ohAddr(sets.size());
  std::vector<size_t> layoutAddrAt(sets.size());
  for (size_t i = 0; i < sets.size(); ++i) {
    uint64_t count = 1;
    for (uint64_t d : sets[i].dims) count *= d;
    std::vector<Message> m;
    m.push_back({0x0001, 0, dspace(sets[i].dims)});
    m.push_back({0x0003, 1, dtype_f64()});
    Message fill{0x0005, 1, Buf()};
    fill.body.u8(2);  // version 2
    fill.body.u8(1);  // space allocated early
    fill.body.u8(2);  // fill value written if set
    fill.body.u8(0);  // no fill value defined
    m.push_back(fill);
    Message lay{0x0008, 0, Buf()};
    lay.body.u8(3);  // version 3
    lay.body.u8(1);  // contiguous
    lay.body.u64(0);  // address (patched)
    lay.body.u64(count * 8);
    m.push_back(lay);
    ohAddr[i] = f.size();
    object_header(f, m);
    // the layout message is the last one: its body starts 8 bytes into it
    size_t at = ohAddr[i] + 16;
    for (size_t k = 0; k + 1 < m.size(); ++k) at += 8 + pad8(m[k].body.size());
    layoutAddrAt[i] = at + 8 + 2;
  }
  for (size_t i = 0; i < sets.size(); ++i) {
    f.pad8();
    uint64_t count = 1;
    for (uint64_t d : sets[i].dims) count *= d;
    f.put64(layoutAddrAt[i], f.size());
    f.bytes(sets[i].data, count * 8);  // IEEE little-endian doubles, as the host holds them
    f.put64(entryOhAt[i], ohAddr[i]);
  }
  f.put64(eofAt, f.size());
  f.put64(rootOhAt, rootOh);
  f.put64(scratchAt, btreeAddr);
  f.put64(scratchAt + 8, heapAddr);
  f.put64(stabBodyAt, btreeAddr);
  f.put64(stabBodyAt + 8, heapAddr);
  return RF_OK;
}

// Creates `dir` if it does not exist (its parent must).
int ensure_dir(const std::string& dir) {
  if (mkdir(dir.c_str(), 0755) == 0 || errno == EEXIST) return RF_OK;
  return fail(RF_EINVAL_ARG, "cannot create folder %s (%s)", dir.c_str(), strerror(errno));
}

int write_file(const std::string& path, const void* p, size_t n) {
  FILE* fp = fopen(path.c_str(), "wb");
  if (!fp) return fail(RF_EINVAL_ARG, "cannot open %s for writing (%s)", path.c_str(), strerror(errno));
  const size_t w = fwrite(p, 1, n, fp);
  const int c = fclose(fp);
  if (w != n || c != 0) return fail(RF_EINVAL_ARG, "short write to %s", path.c_str());
  return RF_OK;
}

std::string num(double v) {
  char s[64];
  snprintf(s, sizeof(s), "%.17g", v);
  return s;
}

// XDMF 2.0 description of one structured field (write_XMF_Elements,
// writeResultFile_RF.f90:835-938): the dataset, a CoRectMesh topology of
// the grid (dimensions slowest axis first), its origin and step, and the
// node-centred scalar "RF1".
std::string xmf_text(const std::string& h5Rel, int nDim, const int64_t* nStep, const double* xMin,
                     const double* xStep) {
  std::string dims, origin, step;
  for (int d = nDim - 1; d >= 0; --d) {
    dims += std::to_string((long long)nStep[d]) + (d ? " " : "");
    origin += num(xMin[d]) + (d ? " " : "");
    step += num(xStep[d]) + (d ? " " : "");
  }
  const std::string topo = nDim == 2 ? "2DCoRectMesh" : "3DCoRectMesh";
  const std::string geo = nDim == 2 ? "ORIGIN_DXDY" : "ORIGIN_DXDYDZ";
  std::string x;
  x += "<?xml version=\"1.0\" ?>\n<Xdmf Version=\"2.0\">\n <Domain>\n";
  x += "   <DataItem Name=\"RF_1\" Format=\"HDF\" DataType=\"Float\" Precision=\"8\" Dimensions=\"" + dims + "\">\n";
  x += "        " + h5Rel + ":/samples\n   </DataItem>\n";
  x += "  <Grid GridType=\"Collection\" CollectionType=\"Spatial\">\n   <Grid Name=\"Group1\">\n";
  x += "     <Topology TopologyType=\"" + topo + "\" Dimensions=\"" + dims + "\"/>\n";
  x += "     <Geometry GeometryType=\"" + geo + "\">\n";
  x += "   <DataItem Name=\"origin\" Format=\"XML\" DataType=\"Float\" Precision=\"8\" Dimensions=\"" +
       std::to_string(nDim) + "\">\n    " + origin + "\n   </DataItem>\n";
  x += "   <DataItem Name=\"step\" Format=\"XML\" DataType=\"Float\" Precision=\"8\" Dimensions=\"" +
       std::to_string(nDim) + "\">\n    " + step + "\n   </DataItem>\n";
  x += "     </Geometry>\n";
  x += "     <Attribute Name=\"RF1\" Center=\"Node\" AttributeType=\"Scalar\">\n";
  x += "       <DataItem Reference=\"XML\">\n         /Xdmf/Domain/DataItem[@Name=\"RF_1\"]\n       </DataItem>\n";
  x += "     </Attribute>\n   </Grid>\n  </Grid>\n </Domain>\n</Xdmf>\n";
  return x;
}

}  // namespace

extern "C" {

int rf_write_result_grid(const char* folder, const char* fileName, int nDim, const double* xMin, const double* xMax,
                         const double* xStep, const double* field, const rf_result_attributes* attr) {
  g_err.clear();
  if (!folder || !fileName || !xMin || !xMax || !xStep || !field) return fail(RF_EINVAL_ARG, "null pointer argument");
  if (nDim < 1 || nDim > 3) return fail(RF_EINVAL_NDIM, "nDim must be 1, 2 or 3 (got %d)", nDim);
  int64_t nStep[3] = {1, 1, 1};
  for (int d = 0; d < nDim; ++d) {
    if (!(xStep[d] > 0.0) || !(xMax[d] >= xMin[d])) return fail(RF_EINVAL_ARG, "axis %d: need xStep > 0, xMax >= xMin", d + 1);
    const double r = (xMax[d] - xMin[d]) / xStep[d];
    if (r > 1e9) return fail(RF_EINVAL_ARG, "axis %d: too many points", d + 1);
    nStep[d] = (int64_t)std::llround(r) + 1;  // nint((xMax - xMin)/xStep) + 1 (:790)
  }
  // dataset dimensions in C order: the slowest axis first (h5screate_simple_f
  // from Fortran reverses the order of its dims array)
  std::vector<uint64_t> dims;
  for (int d = nDim - 1; d >= 0; --d) dims.push_back((uint64_t)nStep[d]);
  std::vector<Message> attrs;
  if (attr) {
    const Buf i32 = dtype_i32(), f64 = dtype_f64();
    auto scalar = [&](const char* nm, int32_t v) { attrs.push_back(attribute(nm, i32, {}, &v, 4)); };
    auto ivec = [&](const char* nm, const int32_t* v) { attrs.push_back(attribute(nm, i32, {(uint64_t)nDim}, v, 4 * (size_t)nDim)); };
    auto dvec = [&](const char* nm, const double* v) { attrs.push_back(attribute(nm, f64, {(uint64_t)nDim}, v, 8 * (size_t)nDim)); };
    scalar("nb_procs", attr->nb_procs);
    scalar("nDim", attr->nDim);
    scalar("Nmc", attr->Nmc);
    scalar("method", attr->method);
    scalar("seedStart", attr->seedStart);
    scalar("corrMod", attr->corrMod);
    scalar("margiFirst", attr->margiFirst);
    scalar("localizationLevel", attr->localizationLevel);
    ivec("kNStep", attr->kNStep);
    ivec("nFields", attr->nFields);
    dvec("xMinGlob", attr->xMinGlob);
    dvec("xMaxGlob", attr->xMaxGlob);
    dvec("xStep", attr->xStep);
    dvec("corrL", attr->corrL);
    dvec("overlap", attr->overlap);
    dvec("procExtent", attr->procExtent);
    dvec("kMax_out", attr->kMax_out);
  }
  Buf f;
  if (int rc = build_h5({{"samples", dims, field}}, attrs, f)) return rc;
  const std::string base(folder);
  if (int rc = ensure_dir(base + "/h5")) return rc;
  if (int rc = write_file(base + "/h5/" + fileName + ".h5", f.b.data(), f.size())) return rc;
  if (nDim >= 2) {  // the reference prepares no XDMF model for 1-D (:876-880)
    const std::string x = xmf_text(std::string("../h5/") + fileName + ".h5", nDim, nStep, xMin, xStep);
    if (int rc = ensure_dir(base + "/xmf")) return rc;
    if (int rc = write_file(base + "/xmf/" + fileName + ".xmf", x.data(), x.size())) return rc;
  }
  return RF_OK;
}

}  // extern "C"
