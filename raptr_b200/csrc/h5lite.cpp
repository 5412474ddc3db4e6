// Minimal HDF5 files for the reference's two data layouts, without libhdf5.
//
// Writes (and reads) what the reference's tools exchange
// (README.md "Data Formats"): a measurement file with the 5-D float32
// dataset "messung" and a density file with the 3-D float32 dataset
// "density" carrying scalar attributes xmin/xmax/ymin/ymax/zmin/zmax
// (float32) and xnbin/ynbin/znbin (int32).  The structures follow the
// HDF5 file format specification in its earliest form, the one libhdf5
// writes by default: superblock version 0 (8-byte offsets and lengths),
// version-1 object headers, a root group held by a symbol table (version-1
// B-tree, symbol table node, local heap), datasets with a version-1
// dataspace, a floating-point or fixed-point datatype, a fill-value message
// and a contiguous version-3 layout, and version-1 attribute messages.
//
// The reader walks these structures and also the later forms libhdf5 and
// h5py write with their latest-format settings and for chunked datasets
// (see "reading" below).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/raptr_b200_h5.h"

namespace {

constexpr uint64_t kUndef = ~uint64_t(0);
constexpr int kGroupLeafK = 4;       // symbol table node holds 2K entries
constexpr int kGroupInternalK = 16;  // B-tree node holds 2K children

thread_local std::string g_h5_error;

int h5_fail(int code, const std::string& msg) {
  g_h5_error = msg;
  return code;
}

// ---- writing ------------------------------------------------------------------

struct Buf {
  std::vector<uint8_t> b;
  size_t size() const { return b.size(); }
  void u8(uint8_t v) { b.push_back(v); }
  void u16(uint16_t v) { put(&v, 2); }
  void u32(uint32_t v) { put(&v, 4); }
  void u64(uint64_t v) { put(&v, 8); }
  void put(const void* p, size_t n) {  // little-endian host
    const uint8_t* c = static_cast<const uint8_t*>(p);
    b.insert(b.end(), c, c + n);
  }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void pad8() {
    while (b.size() % 8) b.push_back(0);
  }
  void set_u64(size_t at, uint64_t v) { std::memcpy(&b[at], &v, 8); }
  void set_u32(size_t at, uint32_t v) { std::memcpy(&b[at], &v, 4); }
  void set_u16(size_t at, uint16_t v) { std::memcpy(&b[at], &v, 2); }
};

size_t up8(size_t n) { return (n + 7) & ~size_t(7); }

// Datatype message bodies.
std::vector<uint8_t> dtype_f32() {
  Buf m;
  m.u8(0x11);             // version 1, class 1 (floating point)
  m.u8(0x20);             // little endian, no padding, mantissa normalisation 2 (implied msb)
  m.u8(31);               // sign bit location
  m.u8(0);
  m.u32(4);               // size
  m.u16(0);               // bit offset
  m.u16(32);              // precision
  m.u8(23);               // exponent location
  m.u8(8);                // exponent size
  m.u8(0);                // mantissa location
  m.u8(23);               // mantissa size
  m.u32(127);             // exponent bias
  return m.b;
}

std::vector<uint8_t> dtype_i32() {
  Buf m;
  m.u8(0x10);  // version 1, class 0 (fixed point)
  m.u8(0x08);  // little endian, signed
  m.u8(0);
  m.u8(0);
  m.u32(4);
  m.u16(0);    // bit offset
  m.u16(32);   // precision
  return m.b;
}

std::vector<uint8_t> dataspace(const std::vector<uint64_t>& dims) {
  Buf m;
  m.u8(1);  // version 1
  m.u8(uint8_t(dims.size()));
  m.u8(0);  // no maximum dimensions
  m.u8(0);
  m.u32(0);
  for (uint64_t d : dims) m.u64(d);
  return m.b;
}

struct Attr {
  std::string name;
  bool is_int;
  float f;
  int32_t i;
};

void message(Buf& oh, uint16_t type, const std::vector<uint8_t>& body, int* count) {
  oh.u16(type);
  oh.u16(uint16_t(up8(body.size())));
  oh.u8(0);  // flags
  oh.zeros(3);
  oh.put(body.data(), body.size());
  oh.pad8();
  (*count)++;
}

std::vector<uint8_t> attribute(const Attr& a) {
  Buf m;
  const std::vector<uint8_t> dt = a.is_int ? dtype_i32() : dtype_f32();
  const std::vector<uint8_t> ds = dataspace({});  // scalar
  m.u8(1);  // version 1
  m.u8(0);
  m.u16(uint16_t(a.name.size() + 1));
  m.u16(uint16_t(dt.size()));
  m.u16(uint16_t(ds.size()));
  m.put(a.name.c_str(), a.name.size() + 1);
  m.pad8();
  m.put(dt.data(), dt.size());
  m.pad8();
  m.put(ds.data(), ds.size());
  m.pad8();
  if (a.is_int)
    m.put(&a.i, 4);
  else
    m.put(&a.f, 4);
  return m.b;
}

// Object header (version 1) from its message region.
void object_header(Buf& f, const Buf& msgs, int nmsgs) {
  f.u8(1);
  f.u8(0);
  f.u16(uint16_t(nmsgs));
  f.u32(1);                       // reference count
  f.u32(uint32_t(msgs.size()));   // header data size
  f.u32(0);                       // alignment to 8
  f.put(msgs.b.data(), msgs.size());
}

// One float32 dataset `name` of shape dims in the root group of a new file.
int write_file(const char* path, const char* name, const float* data, const std::vector<uint64_t>& dims,
               const std::vector<Attr>& attrs) {
  if (!path || !name || !*name || !data) return h5_fail(RAPTR_H5_INVALID, "bad argument");
  uint64_t count = 1;
  for (uint64_t d : dims) count *= d;
  Buf f;
  // superblock v0, filled in at the end
  const char sig[8] = {char(0x89), 'H', 'D', 'F', '\r', '\n', char(0x1a), '\n'};
  f.put(sig, 8);
  f.u8(0);  // superblock version
  f.u8(0);  // free-space storage version
  f.u8(0);  // root group symbol table entry version
  f.u8(0);
  f.u8(0);  // shared header message format version
  f.u8(8);  // size of offsets
  f.u8(8);  // size of lengths
  f.u8(0);
  f.u16(kGroupLeafK);
  f.u16(kGroupInternalK);
  f.u32(0);  // file consistency flags
  f.u64(0);  // base address
  f.u64(kUndef);  // free-space info
  const size_t at_eof = f.size();
  f.u64(0);  // end of file address
  f.u64(kUndef);  // driver information block
  // root group symbol table entry
  f.u64(0);  // link name offset (the empty name)
  const size_t at_root_oh = f.size();
  f.u64(0);  // object header address
  f.u32(1);  // cache type: scratch pad holds the B-tree and heap addresses
  f.u32(0);
  const size_t at_scratch = f.size();
  f.u64(0);  // B-tree
  f.u64(0);  // heap
  f.pad8();

  // root group object header: one symbol table message
  const uint64_t root_oh = f.size();
  Buf rm;
  int nrm = 0;
  std::vector<uint8_t> stab(16, 0);
  message(rm, 0x0011, stab, &nrm);
  const size_t stab_body = 16 + 8;  // offset of the message body in the header
  object_header(f, rm, nrm);
  f.pad8();

  // local heap: "" at 0, the dataset name at 8
  const std::string nm(name);
  const size_t name_off = 8;
  const size_t heap_data_size = up8(name_off + nm.size() + 1);
  const uint64_t heap = f.size();
  f.put("HEAP", 4);
  f.u8(0);
  f.zeros(3);
  f.u64(heap_data_size);
  f.u64(kUndef);  // no free block
  const size_t at_heap_data = f.size();
  f.u64(0);
  f.pad8();
  const uint64_t heap_data = f.size();
  f.zeros(heap_data_size);
  std::memcpy(&f.b[heap_data + name_off], nm.c_str(), nm.size() + 1);

  // B-tree (group, leaf) with one child: the symbol table node
  const uint64_t btree = f.size();
  f.put("TREE", 4);
  f.u8(0);  // group node
  f.u8(0);  // leaf
  f.u16(1);  // entries used
  f.u64(kUndef);
  f.u64(kUndef);
  f.u64(0);  // key 0: ""
  const size_t at_child = f.size();
  f.u64(0);  // child 0
  f.u64(name_off);  // key 1: the largest name in child 0
  f.zeros(size_t(2 * kGroupInternalK - 1) * 16);  // unused keys and children

  // symbol table node with the dataset's entry
  const uint64_t snod = f.size();
  f.put("SNOD", 4);
  f.u8(1);
  f.u8(0);
  f.u16(1);
  f.u64(name_off);
  const size_t at_ds_oh = f.size();
  f.u64(0);  // dataset object header
  f.u32(0);  // no cache
  f.u32(0);
  f.zeros(16);
  f.zeros(size_t(2 * kGroupLeafK - 1) * 40);

  // dataset object header
  const uint64_t ds_oh = f.size();
  Buf dm;
  int ndm = 0;
  message(dm, 0x0001, dataspace(dims), &ndm);
  message(dm, 0x0003, dtype_f32(), &ndm);
  {
    Buf fv;  // fill value message v2: early allocation, write if set, none defined
    fv.u8(2);
    fv.u8(1);
    fv.u8(2);
    fv.u8(0);
    message(dm, 0x0005, fv.b, &ndm);
  }
  const size_t layout_at = dm.size() + 8;  // body offset within the message region
  {
    Buf lo;
    lo.u8(3);  // version 3
    lo.u8(1);  // contiguous
    lo.u64(0);  // address, set below
    lo.u64(count * 4);
    message(dm, 0x0008, lo.b, &ndm);
  }
  for (const Attr& a : attrs) message(dm, 0x000C, attribute(a), &ndm);
  object_header(f, dm, ndm);
  f.pad8();

  // raw data
  const uint64_t raw = f.size();
  f.put(data, size_t(count) * 4);

  // addresses
  f.set_u64(at_eof, f.size());
  f.set_u64(at_root_oh, root_oh);
  f.set_u64(at_scratch, btree);
  f.set_u64(at_scratch + 8, heap);
  f.set_u64(root_oh + stab_body, btree);
  f.set_u64(root_oh + stab_body + 8, heap);
  f.set_u64(at_heap_data, heap_data);
  f.set_u64(at_child, snod);
  f.set_u64(at_ds_oh, ds_oh);
  f.set_u64(ds_oh + 16 + layout_at + 2, raw);

  FILE* fp = std::fopen(path, "wb");
  if (!fp) return h5_fail(RAPTR_H5_IO, std::string("cannot open ") + path + " for writing");
  const size_t w = std::fwrite(f.b.data(), 1, f.size(), fp);
  const int c = std::fclose(fp);
  if (w != f.size() || c != 0) return h5_fail(RAPTR_H5_IO, std::string("short write to ") + path);
  return RAPTR_H5_OK;
}

// ---- reading ------------------------------------------------------------------
//
// The reader follows the HDF5 file format specification (version 3.0) for
// the forms libhdf5 and h5py write for these files, in their default and
// in their latest-format settings:
//   * superblock versions 0 and 1 (root group as a symbol table) and 2 and 3
//     (root group object header address), 8-byte offsets and lengths;
//   * object headers of version 1 and 2 ("OHDR", continuation blocks
//     "OCHK"); checksums are not verified;
//   * groups held by a symbol table (version-1 B-tree, "SNOD" nodes, local
//     heap) or by link messages in the header (compact storage);
//   * dataspace messages of version 1 and 2, datatype messages of versions
//     1-4 (little-endian float32, float64, int32), attribute messages of
//     version 1, 2 and 3 stored in the header;
//   * data layout messages of version 3 and 4: contiguous data; chunked
//     data indexed by a version-1 B-tree (layout version 3) or, in layout
//     version 4, by the single-chunk, implicit or (unpaged) fixed-array
//     index -- without filters (a filter pipeline means compressed data).
// Other forms (dense link or attribute storage in fractal heaps, extensible
// arrays and version-2 B-trees as chunk indexes, paged fixed arrays,
// filters) are reported as unsupported.

struct File {
  std::vector<uint8_t> b;
  bool ok(uint64_t at, uint64_t n) const { return at <= b.size() && n <= b.size() - at; }
  template <class T>
  T get(uint64_t at) const {
    T v{};
    std::memcpy(&v, &b[at], sizeof(T));
    return v;
  }
  // little-endian unsigned integer of n bytes (1..8)
  uint64_t getn(uint64_t at, int n) const {
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; i--) v = (v << 8) | b[at + uint64_t(i)];
    return v;
  }
};

struct Dataset {
  std::vector<uint64_t> dims;
  int cls = -1;  // 0 fixed point, 1 floating point
  uint32_t size = 0;
  bool big_endian = false;
  bool is_signed = true;
  uint64_t addr = kUndef, nbytes = 0;
  int layout = -1;          // 1 contiguous, 2 chunked
  int layout_version = 0;
  std::vector<uint64_t> chunk;  // chunk dimensions in elements (rank entries)
  int index_type = 0;       // layout 4: 1 single chunk, 2 implicit, 3 fixed array; layout 3: B-tree (0)
  bool filtered = false;    // a filter pipeline message is present
  std::map<std::string, double> attrs;
};

// What an object header holds for a group: a symbol table, links, or dense
// link storage (not read).
struct GroupInfo {
  uint64_t btree = kUndef, heap = kUndef;
  std::map<std::string, uint64_t> links;
  bool dense_links = false;
};

bool parse_dtype(const File& f, uint64_t at, uint64_t len, int* cls, uint32_t* size, bool* be, bool* sg) {
  if (len < 8 || !f.ok(at, len)) return false;
  const uint8_t cv = f.b[at];
  *cls = cv & 0x0f;
  *be = (f.b[at + 1] & 1) != 0;
  *sg = (f.b[at + 1] & 0x08) != 0;
  *size = f.get<uint32_t>(at + 4);
  return true;
}

bool parse_dataspace(const File& f, uint64_t at, uint64_t len, std::vector<uint64_t>* dims) {
  if (len < 4 || !f.ok(at, len)) return false;
  const int ver = f.b[at], rank = f.b[at + 1];
  uint64_t p = at + (ver == 1 ? 8 : 4);
  dims->clear();
  for (int i = 0; i < rank; i++) {
    if (!f.ok(p, 8)) return false;
    dims->push_back(f.get<uint64_t>(p));
    p += 8;
  }
  return true;
}

double scalar_value(const File& f, uint64_t at, int cls, uint32_t size, bool be) {
  if (be) return 0.0;
  if (cls == 1 && size == 4) return f.get<float>(at);
  if (cls == 1 && size == 8) return f.get<double>(at);
  if (cls == 0 && size == 4) return f.get<int32_t>(at);
  if (cls == 0 && size == 8) return double(f.get<int64_t>(at));
  return 0.0;
}

// Attribute message (versions 1-3) holding a scalar or one-element value.
void parse_attribute(const File& f, uint64_t body, uint64_t len, Dataset* ds) {
  if (len < 8 || !f.ok(body, len)) return;
  const int ver = f.b[body];
  if (ver < 1 || ver > 3) return;
  const uint16_t nlen = f.get<uint16_t>(body + 2), tlen = f.get<uint16_t>(body + 4), slen = f.get<uint16_t>(body + 6);
  uint64_t q = body + 8 + (ver == 3 ? 1 : 0);  // version 3: character set of the name
  auto step = [&](uint64_t n) { return ver == 1 ? up8(n) : n; };  // version 1 pads to 8 bytes
  if (!f.ok(q, nlen)) return;
  std::string an(reinterpret_cast<const char*>(&f.b[q]), strnlen(reinterpret_cast<const char*>(&f.b[q]), nlen));
  q += step(nlen);
  int cls = -1;
  uint32_t sz = 0;
  bool be = false, sg = true;
  if (!parse_dtype(f, q, tlen, &cls, &sz, &be, &sg)) return;
  q += step(tlen) + step(slen);
  if (f.ok(q, sz)) ds->attrs[an] = scalar_value(f, q, cls, sz, be);
}

// Data layout message, versions 3 and 4.
void parse_layout(const File& f, uint64_t body, uint64_t len, Dataset* ds) {
  if (len < 2 || !f.ok(body, len)) return;
  const int ver = f.b[body];
  ds->layout_version = ver;
  if (ver != 3 && ver != 4) return;
  ds->layout = f.b[body + 1];
  if (ds->layout == 1 && len >= 18) {  // contiguous: address, size
    ds->addr = f.get<uint64_t>(body + 2);
    ds->nbytes = f.get<uint64_t>(body + 10);
    return;
  }
  if (ds->layout != 2) return;
  ds->chunk.clear();
  if (ver == 3) {
    // dimensionality (rank + 1), B-tree address, 4-byte sizes (the last
    // one is the element size)
    if (len < 11) return;
    const int nd = f.b[body + 2];
    ds->addr = f.get<uint64_t>(body + 3);
    if (!f.ok(body + 11, uint64_t(nd) * 4)) return;
    for (int i = 0; i + 1 < nd; i++) ds->chunk.push_back(f.get<uint32_t>(body + 11 + 4 * uint64_t(i)));
    ds->index_type = 0;
    return;
  }
  // version 4: flags, dimensionality, size of the encoded dimensions,
  // dimensions, index type, index-specific fields, address
  if (len < 5) return;
  const int flags = f.b[body + 2], nd = f.b[body + 3], enc = f.b[body + 4];
  uint64_t q = body + 5;
  if (enc < 1 || enc > 8 || !f.ok(q, uint64_t(nd) * enc + 1)) return;
  for (int i = 0; i < nd; i++) ds->chunk.push_back(f.getn(q + uint64_t(i) * enc, enc));
  if (!ds->chunk.empty()) ds->chunk.pop_back();  // the element size
  q += uint64_t(nd) * enc;
  ds->index_type = f.b[q++];
  if (ds->index_type == 1) {  // single chunk: [filtered size, filter mask]
    if (flags & 2) q += 8 + 4;
  } else if (ds->index_type == 3) {  // fixed array: page bits
    q += 1;
  } else if (ds->index_type == 4) {  // extensible array parameters
    q += 5;
  } else if (ds->index_type == 5) {  // version-2 B-tree parameters
    q += 6;
  }
  if (f.ok(q, 8)) ds->addr = f.get<uint64_t>(q);
}

// The messages of an object header of version 1 or 2 (with its
// continuation blocks): dataset fields into *ds, group fields into *grp.
bool parse_object(const File& f, uint64_t oh, Dataset* ds, GroupInfo* grp) {
  struct Block {
    uint64_t at, len;
  };
  std::vector<Block> blocks;
  int version = 0, nmsg = 1 << 30;
  bool creation_order = false;
  if (f.ok(oh, 16) && f.b[oh] == 1) {
    version = 1;
    nmsg = f.get<uint16_t>(oh + 2);
    blocks.push_back({oh + 16, f.get<uint32_t>(oh + 8)});
  } else if (f.ok(oh, 6) && std::memcmp(&f.b[oh], "OHDR", 4) == 0 && f.b[oh + 4] == 2) {
    version = 2;
    const int flags = f.b[oh + 5];
    uint64_t q = oh + 6;
    if (flags & 0x20) q += 16;  // access, modification, change, birth times
    if (flags & 0x10) q += 4;   // attribute storage phase change values
    const int sz = 1 << (flags & 3);
    if (!f.ok(q, uint64_t(sz))) return false;
    const uint64_t chunk0 = f.getn(q, sz);
    q += uint64_t(sz);
    blocks.push_back({q, chunk0});
    creation_order = (flags & 0x04) != 0;
  } else {
    return false;
  }
  int seen = 0;
  for (size_t bi = 0; bi < blocks.size() && seen < nmsg && bi < 64; bi++) {
    uint64_t p = blocks[bi].at;
    const uint64_t end = blocks[bi].at + blocks[bi].len;
    if (!f.ok(p, blocks[bi].len)) return false;
    const uint64_t hsize = version == 1 ? 8 : (creation_order ? 6 : 4);
    while (p + hsize <= end && seen < nmsg) {
      uint16_t type;
      uint64_t len;
      if (version == 1) {
        type = f.get<uint16_t>(p);
        len = f.get<uint16_t>(p + 2);
      } else {
        type = f.b[p];
        len = f.get<uint16_t>(p + 1);
      }
      const uint64_t body = p + hsize;
      if (!f.ok(body, len) || body + len > end) return false;
      seen++;
      switch (type) {
        case 0x0001:
          if (ds) parse_dataspace(f, body, len, &ds->dims);
          break;
        case 0x0002:  // link info: a fractal heap address means dense links
          if (grp && len >= 10) {
            const int lflags = f.b[body + 1];
            const uint64_t heap_at = body + 2 + ((lflags & 1) ? 8 : 0);
            if (f.ok(heap_at, 8) && f.get<uint64_t>(heap_at) != kUndef) grp->dense_links = true;
          }
          break;
        case 0x0003:
          if (ds) parse_dtype(f, body, len, &ds->cls, &ds->size, &ds->big_endian, &ds->is_signed);
          break;
        case 0x0006:  // link (version 1)
          if (grp && len >= 4 && f.b[body] == 1) {
            const int lf = f.b[body + 1];
            uint64_t q = body + 2;
            int ltype = 0;
            if (lf & 0x08) ltype = f.b[q++];
            if (lf & 0x04) q += 8;
            if (lf & 0x10) q += 1;
            const int nb = 1 << (lf & 3);
            if (!f.ok(q, uint64_t(nb))) break;
            const uint64_t nl = f.getn(q, nb);
            q += uint64_t(nb);
            if (ltype != 0 || !f.ok(q, nl + 8)) break;  // hard links only
            grp->links[std::string(reinterpret_cast<const char*>(&f.b[q]), size_t(nl))] = f.get<uint64_t>(q + nl);
          }
          break;
        case 0x0008:
          if (ds) parse_layout(f, body, len, ds);
          break;
        case 0x000B:  // filter pipeline: compressed or otherwise filtered data
          if (ds) ds->filtered = true;
          break;
        case 0x000C:
          if (ds) parse_attribute(f, body, len, ds);
          break;
        case 0x0010:  // continuation
          if (len >= 16) {
            const uint64_t at = f.get<uint64_t>(body), l = f.get<uint64_t>(body + 8);
            if (version == 1) {
              blocks.push_back({at, l});
            } else if (f.ok(at, 4) && std::memcmp(&f.b[at], "OCHK", 4) == 0 && l >= 8) {
              blocks.push_back({at + 4, l - 8});  // signature and checksum
            }
          }
          break;
        case 0x0011:
          if (grp && len >= 16) {
            grp->btree = f.get<uint64_t>(body);
            grp->heap = f.get<uint64_t>(body + 8);
          }
          break;
        default:
          break;
      }
      p = body + len;
    }
  }
  return true;
}

// Object header address of `name` in the group with this B-tree and heap.
uint64_t find_in_group(const File& f, uint64_t btree, uint64_t heap, const std::string& name, int depth = 0) {
  if (depth > 32 || !f.ok(heap, 32) || std::memcmp(&f.b[heap], "HEAP", 4) != 0) return kUndef;
  const uint64_t heap_data = f.get<uint64_t>(heap + 24), heap_size = f.get<uint64_t>(heap + 8);
  if (!f.ok(btree, 24) || std::memcmp(&f.b[btree], "TREE", 4) != 0) return kUndef;
  const int level = f.b[btree + 5], used = f.get<uint16_t>(btree + 6);
  for (int i = 0; i < used; i++) {
    const uint64_t child_at = btree + 24 + 8 + uint64_t(i) * 16;
    if (!f.ok(child_at, 8)) return kUndef;
    const uint64_t child = f.get<uint64_t>(child_at);
    if (level > 0) {
      const uint64_t r = find_in_group(f, child, heap, name, depth + 1);
      if (r != kUndef) return r;
      continue;
    }
    if (!f.ok(child, 8) || std::memcmp(&f.b[child], "SNOD", 4) != 0) continue;
    const int nsym = f.get<uint16_t>(child + 6);
    for (int s = 0; s < nsym; s++) {
      const uint64_t e = child + 8 + uint64_t(s) * 40;
      if (!f.ok(e, 40)) break;
      const uint64_t off = f.get<uint64_t>(e);
      if (off >= heap_size || !f.ok(heap_data + off, 1)) continue;
      const char* nm = reinterpret_cast<const char*>(&f.b[heap_data + off]);
      if (name == std::string(nm, strnlen(nm, size_t(heap_size - off)))) return f.get<uint64_t>(e + 8);
    }
  }
  return kUndef;
}

uint64_t element_count(const Dataset& ds) {
  uint64_t count = 1;
  for (uint64_t d : ds.dims) count *= d;
  return count;
}

int open_dataset(const char* path, const char* name, File* f, Dataset* ds) {
  if (!path || !name) return h5_fail(RAPTR_H5_INVALID, "bad argument");
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return h5_fail(RAPTR_H5_IO, std::string("cannot open ") + path);
  std::fseek(fp, 0, SEEK_END);
  const long n = std::ftell(fp);
  std::fseek(fp, 0, SEEK_SET);
  f->b.resize(size_t(n > 0 ? n : 0));
  const size_t r = f->b.empty() ? 0 : std::fread(f->b.data(), 1, f->b.size(), fp);
  std::fclose(fp);
  if (r != f->b.size()) return h5_fail(RAPTR_H5_IO, std::string("cannot read ") + path);
  const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  if (f->b.size() < 48 || std::memcmp(f->b.data(), sig, 8) != 0)
    return h5_fail(RAPTR_H5_FORMAT, std::string(path) + " is not an HDF5 file");
  const int sbv = f->b[8];
  GroupInfo root;
  if (sbv <= 1) {
    if (f->b.size() < 96 || f->b[13] != 8 || f->b[14] != 8)
      return h5_fail(RAPTR_H5_UNSUPPORTED, "only 8-byte offsets and lengths are read");
    // root symbol table entry follows the fixed fields (v1 has 4 more bytes)
    const uint64_t at = 24 + (sbv == 1 ? 4 : 0) + 32;
    const uint64_t root_oh = f->get<uint64_t>(at + 8);
    if (f->get<uint32_t>(at + 16) == 1) {
      root.btree = f->get<uint64_t>(at + 24);
      root.heap = f->get<uint64_t>(at + 32);
    }
    if (root.btree == kUndef && !parse_object(*f, root_oh, nullptr, &root))
      return h5_fail(RAPTR_H5_FORMAT, "cannot read the root group");
  } else if (sbv == 2 || sbv == 3) {
    if (f->b[9] != 8 || f->b[10] != 8) return h5_fail(RAPTR_H5_UNSUPPORTED, "only 8-byte offsets and lengths are read");
    const uint64_t root_oh = f->get<uint64_t>(36);
    if (!parse_object(*f, root_oh, nullptr, &root)) return h5_fail(RAPTR_H5_FORMAT, "cannot read the root group");
  } else {
    return h5_fail(RAPTR_H5_UNSUPPORTED, "superblock version " + std::to_string(sbv) + " is not read");
  }
  uint64_t oh = kUndef;
  if (root.btree != kUndef) {
    oh = find_in_group(*f, root.btree, root.heap, name);
  } else {
    auto it = root.links.find(name);
    if (it != root.links.end()) oh = it->second;
    else if (root.dense_links)
      return h5_fail(RAPTR_H5_UNSUPPORTED, "the root group keeps its links in dense storage (a fractal heap)");
  }
  if (oh == kUndef) return h5_fail(RAPTR_H5_NOT_FOUND, std::string("no dataset \"") + name + "\" in " + path);
  if (!parse_object(*f, oh, ds, nullptr)) return h5_fail(RAPTR_H5_FORMAT, "cannot read the dataset header");
  if (ds->big_endian || !((ds->cls == 1 && (ds->size == 4 || ds->size == 8)) || (ds->cls == 0 && ds->size == 4)))
    return h5_fail(RAPTR_H5_UNSUPPORTED, "only little-endian float32/float64/int32 datasets are read");
  if (ds->filtered) return h5_fail(RAPTR_H5_UNSUPPORTED, "filtered (compressed) datasets are not read");
  const uint64_t count = element_count(*ds);
  if (ds->layout == 1) {
    if (ds->addr == kUndef) return h5_fail(RAPTR_H5_FORMAT, "contiguous dataset without data");
    if (ds->nbytes < count * ds->size || !f->ok(ds->addr, count * ds->size))
      return h5_fail(RAPTR_H5_FORMAT, "dataset extends past the end of the file");
    return RAPTR_H5_OK;
  }
  if (ds->layout == 2) {
    if (ds->chunk.size() != ds->dims.size() || ds->addr == kUndef)
      return h5_fail(RAPTR_H5_FORMAT, "chunked dataset without its chunk dimensions or index");
    for (uint64_t c : ds->chunk)
      if (c == 0) return h5_fail(RAPTR_H5_FORMAT, "zero chunk dimension");
    if (ds->layout_version == 4 && !(ds->index_type >= 1 && ds->index_type <= 3))
      return h5_fail(RAPTR_H5_UNSUPPORTED, "chunk index type " + std::to_string(ds->index_type) +
                                               " (extensible array or version-2 B-tree) is not read");
    return RAPTR_H5_OK;
  }
  return h5_fail(RAPTR_H5_UNSUPPORTED, "only contiguous and chunked datasets are read");
}

float element_at(const File& f, const Dataset& ds, uint64_t at) {
  return ds.cls == 1 ? (ds.size == 4 ? f.get<float>(at) : float(f.get<double>(at))) : float(f.get<int32_t>(at));
}

// Copies one chunk (dense, chunk dims, at file offset `at`) whose first
// element sits at dataset coordinates `org` into out (row-major dataset),
// clipping at the dataset's edges.
bool copy_chunk(const File& f, const Dataset& ds, uint64_t at, const std::vector<uint64_t>& org, float* out) {
  const size_t r = ds.dims.size();
  uint64_t celems = 1;
  for (uint64_t c : ds.chunk) celems *= c;
  if (!f.ok(at, celems * ds.size)) return false;
  for (size_t d = 0; d < r; d++)
    if (org[d] >= ds.dims[d]) return false;
  std::vector<uint64_t> idx(r, 0);
  for (uint64_t e = 0; e < celems; e++) {
    // element e of the chunk, row-major: idx
    uint64_t rem = e, flat = 0;
    bool inside = true;
    for (size_t d = r; d-- > 0;) {
      idx[d] = rem % ds.chunk[d];
      rem /= ds.chunk[d];
    }
    for (size_t d = 0; d < r; d++) {
      const uint64_t c = org[d] + idx[d];
      if (c >= ds.dims[d]) {
        inside = false;
        break;
      }
      flat = flat * ds.dims[d] + c;
    }
    if (inside) out[flat] = element_at(f, ds, at + e * ds.size);
  }
  return true;
}

// Chunks of a version-1 B-tree (node type 1) below `node`.
bool read_btree_chunks(const File& f, const Dataset& ds, uint64_t node, float* out, int depth, uint64_t* nchunks) {
  if (depth > 64 || !f.ok(node, 24) || std::memcmp(&f.b[node], "TREE", 4) != 0 || f.b[node + 4] != 1) return false;
  const int level = f.b[node + 5], used = f.get<uint16_t>(node + 6);
  const size_t r = ds.dims.size();
  const uint64_t key = 8 + 8 * (r + 1);  // chunk size, filter mask, r + 1 offsets
  uint64_t p = node + 24;
  for (int i = 0; i < used; i++) {
    if (!f.ok(p, key + 8)) return false;
    const uint32_t mask = f.get<uint32_t>(p + 4);
    std::vector<uint64_t> org(r);
    for (size_t d = 0; d < r; d++) org[d] = f.get<uint64_t>(p + 8 + 8 * d);
    const uint64_t child = f.get<uint64_t>(p + key);
    if (level > 0) {
      if (!read_btree_chunks(f, ds, child, out, depth + 1, nchunks)) return false;
    } else {
      if (mask != 0) return false;
      if (!copy_chunk(f, ds, child, org, out)) return false;
      ++*nchunks;
    }
    p += key + 8;
  }
  return true;
}

// Reads every element of the dataset into out (row-major, count elements).
int read_elements(const File& f, const Dataset& ds, float* out) {
  const uint64_t count = element_count(ds);
  if (ds.layout == 1) {
    for (uint64_t i = 0; i < count; i++) out[i] = element_at(f, ds, ds.addr + i * ds.size);
    return RAPTR_H5_OK;
  }
  // chunked: elements no chunk covers keep the fill value 0
  std::fill(out, out + count, 0.f);
  const size_t r = ds.dims.size();
  std::vector<uint64_t> grid(r);  // chunks per dimension
  uint64_t nchunk_all = 1;
  for (size_t d = 0; d < r; d++) {
    grid[d] = (ds.dims[d] + ds.chunk[d] - 1) / ds.chunk[d];
    nchunk_all *= grid[d];
  }
  uint64_t celems = 1;
  for (uint64_t c : ds.chunk) celems *= c;
  auto origin = [&](uint64_t k) {  // chunk k in row-major chunk order
    std::vector<uint64_t> org(r);
    for (size_t d = r; d-- > 0;) {
      org[d] = (k % grid[d]) * ds.chunk[d];
      k /= grid[d];
    }
    return org;
  };
  if (ds.layout_version == 3) {
    uint64_t n = 0;
    if (!read_btree_chunks(f, ds, ds.addr, out, 0, &n))
      return h5_fail(RAPTR_H5_FORMAT, "damaged or filtered chunk B-tree");
    return RAPTR_H5_OK;
  }
  if (ds.index_type == 1) {  // one chunk holds the whole dataset
    if (!copy_chunk(f, ds, ds.addr, std::vector<uint64_t>(r, 0), out))
      return h5_fail(RAPTR_H5_FORMAT, "single chunk extends past the end of the file");
    return RAPTR_H5_OK;
  }
  if (ds.index_type == 2) {  // implicit: every chunk, in chunk order, back to back
    for (uint64_t k = 0; k < nchunk_all; k++)
      if (!copy_chunk(f, ds, ds.addr + k * celems * ds.size, origin(k), out))
        return h5_fail(RAPTR_H5_FORMAT, "implicit chunks extend past the end of the file");
    return RAPTR_H5_OK;
  }
  // fixed array: header "FAHD" -> data block "FADB" of chunk addresses
  const uint64_t h = ds.addr;
  if (!f.ok(h, 28) || std::memcmp(&f.b[h], "FAHD", 4) != 0)
    return h5_fail(RAPTR_H5_FORMAT, "fixed-array chunk index without its header");
  const int client = f.b[h + 5], esize = f.b[h + 6], page_bits = f.b[h + 7];
  const uint64_t nelem = f.get<uint64_t>(h + 8), block = f.get<uint64_t>(h + 16);
  if (client != 0 || esize != 8) return h5_fail(RAPTR_H5_UNSUPPORTED, "filtered fixed-array chunk index");
  if (page_bits < 64 && nelem > (uint64_t(1) << page_bits))
    return h5_fail(RAPTR_H5_UNSUPPORTED, "paged fixed-array chunk index");
  if (nelem != nchunk_all || !f.ok(block, 14 + nelem * 8) || std::memcmp(&f.b[block], "FADB", 4) != 0)
    return h5_fail(RAPTR_H5_FORMAT, "fixed-array chunk index does not match the dataset");
  for (uint64_t k = 0; k < nelem; k++) {
    const uint64_t at = f.get<uint64_t>(block + 14 + k * 8);
    if (at == kUndef) continue;  // never written: fill value
    if (!copy_chunk(f, ds, at, origin(k), out))
      return h5_fail(RAPTR_H5_FORMAT, "chunk extends past the end of the file");
  }
  return RAPTR_H5_OK;
}

}  // namespace

extern "C" {

const char* raptr_h5_last_error(void) { return g_h5_error.c_str(); }

int raptr_h5_write_measurement(const char* path, const float* data, const int64_t dims[5]) {
  std::vector<uint64_t> d;
  for (int i = 0; i < 5; i++) {
    if (dims[i] <= 0) return h5_fail(RAPTR_H5_INVALID, "dimensions must be positive");
    d.push_back(uint64_t(dims[i]));
  }
  return write_file(path, "messung", data, d, {});
}

int raptr_h5_write_density(const char* path, const float* data, const int32_t n[3], const float lo[3],
                           const float hi[3]) {
  if (!n || !lo || !hi || n[0] <= 0 || n[1] <= 0 || n[2] <= 0) return h5_fail(RAPTR_H5_INVALID, "bad grid");
  std::vector<Attr> a;
  const char ax[3] = {'x', 'y', 'z'};
  for (int i = 0; i < 3; i++) {
    a.push_back({std::string(1, ax[i]) + "min", false, lo[i], 0});
    a.push_back({std::string(1, ax[i]) + "max", false, hi[i], 0});
    a.push_back({std::string(1, ax[i]) + "nbin", true, 0.f, n[i]});
  }
  return write_file(path, "density", data, {uint64_t(n[0]), uint64_t(n[1]), uint64_t(n[2])}, a);
}

int raptr_h5_dataset_info(const char* path, const char* name, int32_t* rank, int64_t dims[8]) {
  File f;
  Dataset ds;
  const int st = open_dataset(path, name, &f, &ds);
  if (st != RAPTR_H5_OK) return st;
  if (ds.dims.size() > 8) return h5_fail(RAPTR_H5_UNSUPPORTED, "rank above 8");
  if (rank) *rank = int32_t(ds.dims.size());
  if (dims)
    for (size_t i = 0; i < ds.dims.size(); i++) dims[i] = int64_t(ds.dims[i]);
  return RAPTR_H5_OK;
}

int raptr_h5_read_f32(const char* path, const char* name, float* out, int64_t capacity, int64_t* count) {
  File f;
  Dataset ds;
  const int st = open_dataset(path, name, &f, &ds);
  if (st != RAPTR_H5_OK) return st;
  uint64_t n = 1;
  for (uint64_t d : ds.dims) n *= d;
  if (count) *count = int64_t(n);
  if (!out) return RAPTR_H5_OK;
  if (int64_t(n) > capacity) return h5_fail(RAPTR_H5_INVALID, "buffer too small");
  return read_elements(f, ds, out);
}

int raptr_h5_read_density_grid(const char* path, int32_t n[3], float lo[3], float hi[3]) {
  File f;
  Dataset ds;
  const int st = open_dataset(path, "density", &f, &ds);
  if (st != RAPTR_H5_OK) return st;
  const char ax[3] = {'x', 'y', 'z'};
  for (int i = 0; i < 3; i++) {
    const std::string a(1, ax[i]);
    if (!ds.attrs.count(a + "min") || !ds.attrs.count(a + "max") || !ds.attrs.count(a + "nbin"))
      return h5_fail(RAPTR_H5_FORMAT, "density without its grid attributes");
    lo[i] = float(ds.attrs[a + "min"]);
    hi[i] = float(ds.attrs[a + "max"]);
    n[i] = int32_t(ds.attrs[a + "nbin"]);
  }
  return RAPTR_H5_OK;
}

}  // extern "C"
