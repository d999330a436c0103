// h5lite.cpp -- see h5lite.hpp.  Structure names follow the HDF5 File Format
// Specification version 3.0 (superblock, object header, symbol table, local
// heap, v1 B-tree, symbol table node, dataspace / datatype / layout messages).
#include "h5lite.hpp"

#include <algorithm>
#include <cstring>
#include <fstream>
#include <functional>

namespace h5 {
namespace {

constexpr uint64_t kUndef = ~0ull;
const unsigned char kSig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

// ---------------------------------------------------------------- reading
struct File {
  std::vector<unsigned char> b;
  int so = 8, sl = 8;  // size of offsets, size of lengths
  uint64_t base = 0;

  uint64_t u(uint64_t at, int n) const {
    if (at + n > b.size()) throw Error("HDF5: read past the end of the file");
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; --i) v = (v << 8) | b[at + i];
    return v;
  }
  // A stored address, made absolute: addresses are relative to the base
  // address (the superblock's position when a user block precedes it).
  uint64_t addr(uint64_t at) const {
    const uint64_t v = u(at, so);
    if (v == kUndef || (so < 8 && v == ((1ull << (8 * so)) - 1))) return kUndef;
    return v + base;
  }
  bool sig(uint64_t at, const char* s) const {
    return at + 4 <= b.size() && std::memcmp(&b[at], s, 4) == 0;
  }
};

struct Msg {
  int type;
  uint64_t at;   // start of the message data
  uint64_t size;
};

void collect_v1(const File& f, uint64_t at, uint64_t len, std::vector<Msg>& out,
                std::vector<std::pair<uint64_t, uint64_t>>& cont) {
  uint64_t p = at;
  const uint64_t end = at + len;
  while (p + 8 <= end) {
    const int type = (int)f.u(p, 2);
    const uint64_t size = f.u(p + 2, 2);
    const uint64_t data = p + 8;
    if (type == 0x10) cont.emplace_back(f.addr(data), f.u(data + f.so, f.sl));
    else out.push_back({type, data, size});
    p = data + size;
  }
}

void collect_v2(const File& f, uint64_t at, uint64_t len, int hflags, std::vector<Msg>& out,
                std::vector<std::pair<uint64_t, uint64_t>>& cont) {
  uint64_t p = at;
  const uint64_t end = at + len;
  const int hdr = 4 + ((hflags & 4) ? 2 : 0);
  while (p + hdr <= end) {
    const int type = (int)f.u(p, 1);
    const uint64_t size = f.u(p + 1, 2);
    const uint64_t data = p + hdr;
    if (type == 0x10) cont.emplace_back(f.addr(data), f.u(data + f.so, f.sl));
    else if (type != 0) out.push_back({type, data, size});
    p = data + size;
  }
}

std::vector<Msg> object_messages(const File& f, uint64_t oh) {
  std::vector<Msg> msgs;
  std::vector<std::pair<uint64_t, uint64_t>> cont;
  int hflags = 0;
  bool v2 = false;
  if (f.sig(oh, "OHDR")) {
    v2 = true;
    if (f.u(oh + 4, 1) != 2) throw Error("HDF5: unsupported object header version");
    hflags = (int)f.u(oh + 5, 1);
    uint64_t p = oh + 6;
    if (hflags & 0x20) p += 16;
    if (hflags & 0x10) p += 4;
    const int csz = 1 << (hflags & 3);
    const uint64_t len = f.u(p, csz);
    p += csz;
    collect_v2(f, p, len, hflags, msgs, cont);
  } else {
    if (f.u(oh, 1) != 1) throw Error("HDF5: unsupported object header version");
    const uint64_t len = f.u(oh + 8, 4);
    collect_v1(f, oh + 16, len, msgs, cont);
  }
  for (size_t i = 0; i < cont.size(); ++i) {
    const uint64_t at = cont[i].first, len = cont[i].second;
    if (v2) {
      if (!f.sig(at, "OCHK")) throw Error("HDF5: bad continuation block");
      collect_v2(f, at + 4, len - 8, hflags, msgs, cont);
    } else {
      collect_v1(f, at, len, msgs, cont);
    }
  }
  return msgs;
}

std::string heap_name(const File& f, uint64_t heap_data, uint64_t off) {
  std::string s;
  for (uint64_t p = heap_data + off; p < f.b.size() && f.b[p]; ++p) s.push_back((char)f.b[p]);
  return s;
}

// Looks `name` up in a group with a symbol table (v1 B-tree + local heap).
uint64_t symtab_lookup(const File& f, uint64_t btree, uint64_t heap, const std::string& name) {
  if (!f.sig(heap, "HEAP")) throw Error("HDF5: bad local heap");
  const uint64_t heap_data = f.addr(heap + 8 + 2 * f.sl);
  std::function<uint64_t(uint64_t)> walk = [&](uint64_t node) -> uint64_t {
    if (!f.sig(node, "TREE")) throw Error("HDF5: bad B-tree node");
    const int level = (int)f.u(node + 5, 1);
    const int used = (int)f.u(node + 6, 2);
    uint64_t p = node + 8 + 2 * f.so;  // first key
    for (int e = 0; e < used; ++e) {
      const uint64_t child = f.addr(p + f.sl);
      p += f.sl + f.so;
      if (level > 0) {
        const uint64_t r = walk(child);
        if (r != kUndef) return r;
        continue;
      }
      if (!f.sig(child, "SNOD")) throw Error("HDF5: bad symbol table node");
      const int nsym = (int)f.u(child + 6, 2);
      uint64_t q = child + 8;
      for (int k = 0; k < nsym; ++k) {
        const uint64_t noff = f.u(q, f.so);
        const uint64_t ohad = f.addr(q + f.so);
        if (heap_name(f, heap_data, noff) == name) return ohad;
        q += 2 * f.so + 8 + 16;
      }
    }
    return kUndef;
  };
  return walk(btree);
}

uint64_t find_in_group(const File& f, uint64_t group_oh, const std::string& name) {
  for (const Msg& m : object_messages(f, group_oh)) {
    if (m.type == 0x11) {
      const uint64_t r = symtab_lookup(f, f.addr(m.at), f.addr(m.at + f.so), name);
      if (r != kUndef) return r;
    } else if (m.type == 0x06) {
      const int flags = (int)f.u(m.at + 1, 1);
      uint64_t p = m.at + 2;
      int ltype = 0;
      if (flags & 8) ltype = (int)f.u(p++, 1);
      if (flags & 4) p += 8;
      if (flags & 16) p += 1;
      const int lsz = 1 << (flags & 3);
      const uint64_t nlen = f.u(p, lsz);
      p += lsz;
      const std::string nm(reinterpret_cast<const char*>(&f.b[p]), nlen);
      p += nlen;
      if (ltype == 0 && nm == name) return f.addr(p);
    } else if (m.type == 0x02) {
      // link info: dense storage if the fractal heap address is defined
      const int flags = (int)f.u(m.at + 1, 1);
      const uint64_t heap = f.addr(m.at + 2 + ((flags & 1) ? 8 : 0));
      if (heap != kUndef) throw Error("HDF5: dense link storage is not supported");
    }
  }
  throw Error("HDF5: no dataset '" + name + "' in the root group");
}

File load(const std::string& path) {
  File f;
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error("HDF5: cannot open " + path);
  f.b.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
  return f;
}

uint64_t root_object(File& f) {
  uint64_t sb = kUndef;
  for (uint64_t at = 0; at + 8 <= f.b.size(); at = at ? at * 2 : 512) {
    if (std::memcmp(&f.b[at], kSig, 8) == 0) {
      sb = at;
      break;
    }
  }
  if (sb == kUndef) throw Error("HDF5: no superblock (not an HDF5 file)");
  const int ver = (int)f.u(sb + 8, 1);
  if (ver == 0 || ver == 1) {
    f.so = (int)f.u(sb + 13, 1);
    f.sl = (int)f.u(sb + 14, 1);
    uint64_t p = sb + 24 + (ver == 1 ? 4 : 0);
    f.base = f.u(p, f.so);
    p += 4 * f.so;                   // base, free space, EOF, driver info
    return f.addr(p + f.so);         // root symbol table entry: object header
  }
  if (ver == 2 || ver == 3) {
    f.so = (int)f.u(sb + 9, 1);
    f.sl = (int)f.u(sb + 10, 1);
    f.base = f.u(sb + 12, f.so);
    return f.addr(sb + 12 + 3 * f.so);
  }
  throw Error("HDF5: unsupported superblock version");
}

Dataset read_impl(const std::string& path, const std::string& name, uint64_t rows,
                  uint64_t cols, bool block) {
  File f = load(path);
  const uint64_t root = root_object(f);
  const uint64_t oh = find_in_group(f, root, name);
  Dataset d;
  bool have_space = false, have_type = false, big_endian = false;
  uint64_t data_at = kUndef, data_size = 0;
  for (const Msg& m : object_messages(f, oh)) {
    if (m.type == 0x01) {
      const int ver = (int)f.u(m.at, 1);
      const int rank = (int)f.u(m.at + 1, 1);
      const uint64_t p = m.at + (ver == 1 ? 8 : 4);
      d.dims.clear();
      for (int i = 0; i < rank; ++i) d.dims.push_back(f.u(p + (uint64_t)i * f.sl, f.sl));
      have_space = true;
    } else if (m.type == 0x03) {
      const int cls = (int)(f.u(m.at, 1) & 0x0f);
      const uint64_t size = f.u(m.at + 4, 4);
      if (cls != 1 || size != 8) throw Error("HDF5: dataset '" + name + "' is not float64");
      big_endian = (f.u(m.at + 1, 1) & 1) != 0;
      have_type = true;
    } else if (m.type == 0x08 && (f.u(m.at, 1) == 1 || f.u(m.at, 1) == 2)) {
      // layout versions 1 and 2: version, dimensionality, class, 5 reserved
      // bytes, [address], dimensionality 4-byte sizes (the last = element size)
      const int nd = (int)f.u(m.at + 1, 1);
      const int cls = (int)f.u(m.at + 2, 1);
      uint64_t p = m.at + 8;
      if (cls == 1 || cls == 2) {
        data_at = f.addr(p);
        p += f.so;
      }
      uint64_t bytes = 1;
      for (int i = 0; i < nd; ++i) bytes *= f.u(p + 4 * (uint64_t)i, 4);
      p += 4 * (uint64_t)nd;
      if (cls == 0) {
        data_size = f.u(p, 4);
        data_at = p + 4;
      } else if (cls == 1) {
        data_size = bytes;
      } else {
        throw Error("HDF5: chunked storage is not supported");
      }
    } else if (m.type == 0x08) {
      const int ver = (int)f.u(m.at, 1);
      if (ver != 3) throw Error("HDF5: unsupported data layout message version");
      const int cls = (int)f.u(m.at + 1, 1);
      if (cls == 0) {
        data_size = f.u(m.at + 2, 2);
        data_at = m.at + 4;
      } else if (cls == 1) {
        data_at = f.addr(m.at + 2);
        data_size = f.u(m.at + 2 + f.so, f.sl);
      } else {
        throw Error("HDF5: chunked or virtual storage is not supported");
      }
    }
  }
  if (!have_space || !have_type) throw Error("HDF5: incomplete dataset header");
  uint64_t n = 1;
  for (uint64_t x : d.dims) n *= x;
  if (data_at == kUndef) {  // never written: the fill value (zeros)
    d.data.assign(n, 0.0);
  } else {
    if (data_size < n * 8 || data_at + n * 8 > f.b.size())
      throw Error("HDF5: dataset storage shorter than its extent");
  }
  auto get = [&](uint64_t k) {
    if (data_at == kUndef) return 0.0;
    unsigned char t[8];
    std::memcpy(t, &f.b[data_at + 8 * k], 8);
    if (big_endian) std::reverse(t, t + 8);
    double v;
    std::memcpy(&v, t, 8);
    return v;
  };
  if (!block) {
    d.data.resize(n);
    for (uint64_t k = 0; k < n; ++k) d.data[k] = get(k);
    return d;
  }
  if (d.dims.size() == 1) {
    if (rows > d.dims[0]) throw Error("HDF5: '" + name + "' has fewer entries than requested");
    d.data.resize(rows);
    for (uint64_t k = 0; k < rows; ++k) d.data[k] = get(k);
  } else if (d.dims.size() == 2) {
    if (rows > d.dims[0] || cols > d.dims[1])
      throw Error("HDF5: '" + name + "' is smaller than the requested block");
    d.data.resize(rows * cols);
    for (uint64_t r = 0; r < rows; ++r)
      for (uint64_t c = 0; c < cols; ++c) d.data[r * cols + c] = get(r * d.dims[1] + c);
  } else {
    throw Error("HDF5: only 1-D and 2-D datasets are supported");
  }
  return d;
}

// ---------------------------------------------------------------- writing
struct Out {
  std::vector<unsigned char> b;
  void put(uint64_t v, int n) {
    for (int i = 0; i < n; ++i) b.push_back((unsigned char)(v >> (8 * i)));
  }
  void set(uint64_t at, uint64_t v, int n) {
    for (int i = 0; i < n; ++i) b[at + i] = (unsigned char)(v >> (8 * i));
  }
  void bytes(const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    b.insert(b.end(), c, c + n);
  }
  void align8() {
    while (b.size() % 8) b.push_back(0);
  }
};

}  // namespace

Dataset read(const std::string& path, const std::string& name) {
  return read_impl(path, name, 0, 0, false);
}

std::vector<double> read_block(const std::string& path, const std::string& name, uint64_t rows,
                               uint64_t cols) {
  return read_impl(path, name, rows, cols, true).data;
}

void write(const std::string& path, const std::vector<NamedArray>& sets_in) {
  std::vector<NamedArray> sets = sets_in;
  std::sort(sets.begin(), sets.end(),
            [](const NamedArray& a, const NamedArray& b) { return a.name < b.name; });
  Out o;
  // superblock v0 (96 bytes); addresses patched below
  o.bytes(kSig, 8);
  o.put(0, 1); o.put(0, 1); o.put(0, 1); o.put(0, 1);  // versions, reserved
  o.put(0, 1); o.put(8, 1); o.put(8, 1); o.put(0, 1);  // shared hdr ver, sizes, reserved
  o.put(4, 2); o.put(16, 2);                            // group leaf / internal K
  o.put(0, 4);                                          // consistency flags
  o.put(0, 8);                                          // base address
  o.put(kUndef, 8);                                     // free-space info
  const uint64_t eof_at = o.b.size();
  o.put(0, 8);                                          // end of file (patched)
  o.put(kUndef, 8);                                     // driver info
  // root symbol table entry
  o.put(0, 8);                                          // link name offset
  const uint64_t root_oh_at = o.b.size();
  o.put(0, 8);                                          // object header (patched)
  o.put(1, 4); o.put(0, 4);                             // cache type 1, reserved
  const uint64_t scratch_at = o.b.size();
  o.put(0, 8); o.put(0, 8);                             // B-tree, heap (patched)

  // root group object header (v1) with one symbol-table message
  const uint64_t root_oh = o.b.size();
  o.put(1, 1); o.put(0, 1); o.put(1, 2); o.put(1, 4); o.put(24, 4); o.put(0, 4);
  o.put(0x11, 2); o.put(16, 2); o.put(0, 1); o.put(0, 3);
  const uint64_t stab_at = o.b.size();
  o.put(0, 8); o.put(0, 8);

  // local heap with the names (offset 0: the empty name)
  std::vector<uint64_t> name_off;
  std::vector<unsigned char> heap(8, 0);
  for (const auto& s : sets) {
    name_off.push_back(heap.size());
    heap.insert(heap.end(), s.name.begin(), s.name.end());
    heap.push_back(0);
    while (heap.size() % 8) heap.push_back(0);
  }
  const uint64_t heap_at = o.b.size();
  o.bytes("HEAP", 4); o.put(0, 1); o.put(0, 3);
  o.put(heap.size(), 8); o.put(kUndef, 8);
  const uint64_t heap_data_ptr = o.b.size();
  o.put(0, 8);
  const uint64_t heap_data = o.b.size();
  o.bytes(heap.data(), heap.size());
  o.set(heap_data_ptr, heap_data, 8);

  // v1 B-tree leaf with one child: the symbol table node
  const uint64_t btree_at = o.b.size();
  o.bytes("TREE", 4); o.put(0, 1); o.put(0, 1); o.put(1, 2);
  o.put(kUndef, 8); o.put(kUndef, 8);
  o.put(0, 8);
  const uint64_t child_at = o.b.size();
  o.put(0, 8);
  o.put(sets.empty() ? 0 : name_off.back(), 8);

  // symbol table node
  const uint64_t snod_at = o.b.size();
  o.set(child_at, snod_at, 8);
  o.bytes("SNOD", 4); o.put(1, 1); o.put(0, 1); o.put(sets.size(), 2);
  std::vector<uint64_t> entry_oh;
  for (size_t i = 0; i < sets.size(); ++i) {
    o.put(name_off[i], 8);
    entry_oh.push_back(o.b.size());
    o.put(0, 8);
    o.put(0, 4); o.put(0, 4);
    o.put(0, 8); o.put(0, 8);
  }
  o.align8();

  // datasets: v1 object header (dataspace, datatype, fill value, layout)
  std::vector<uint64_t> layout_addr_at;
  for (size_t i = 0; i < sets.size(); ++i) {
    const auto& s = sets[i];
    const uint64_t oh = o.b.size();
    o.set(entry_oh[i], oh, 8);
    const int rank = (int)s.dims.size();
    const uint64_t sp = 8 + 8 * rank;                  // dataspace v1
    const uint64_t msgs = (8 + sp) + (8 + 24) + (8 + 8) + (8 + 24);
    o.put(1, 1); o.put(0, 1); o.put(4, 2); o.put(1, 4); o.put(msgs, 4); o.put(0, 4);
    // dataspace
    o.put(0x01, 2); o.put(sp, 2); o.put(0, 1); o.put(0, 3);
    o.put(1, 1); o.put(rank, 1); o.put(0, 1); o.put(0, 1); o.put(0, 4);
    for (uint64_t x : s.dims) o.put(x, 8);
    // datatype: IEEE float64 little-endian
    o.put(0x03, 2); o.put(24, 2); o.put(1, 1); o.put(0, 3);
    o.put(0x11, 1); o.put(0x20, 1); o.put(0x3f, 1); o.put(0x00, 1);
    o.put(8, 4);
    o.put(0, 2); o.put(64, 2); o.put(52, 1); o.put(11, 1); o.put(0, 1); o.put(52, 1);
    o.put(1023, 4);
    o.put(0, 4);
    // fill value (version 2, late allocation, never written, undefined)
    o.put(0x05, 2); o.put(8, 2); o.put(1, 1); o.put(0, 3);
    o.put(2, 1); o.put(2, 1); o.put(2, 1); o.put(0, 1); o.put(0, 4);
    // layout (version 3, contiguous)
    o.put(0x08, 2); o.put(24, 2); o.put(0, 1); o.put(0, 3);
    o.put(3, 1); o.put(1, 1);
    layout_addr_at.push_back(o.b.size());
    uint64_t n = 1;
    for (uint64_t x : s.dims) n *= x;
    o.put(0, 8); o.put(8 * n, 8);
    o.put(0, 6);
  }
  for (size_t i = 0; i < sets.size(); ++i) {
    o.align8();
    uint64_t n = 1;
    for (uint64_t x : sets[i].dims) n *= x;
    o.set(layout_addr_at[i], o.b.size(), 8);
    o.bytes(sets[i].data, 8 * n);
  }
  o.set(eof_at, o.b.size(), 8);
  o.set(root_oh_at, root_oh, 8);
  o.set(scratch_at, btree_at, 8);
  o.set(scratch_at + 8, heap_at, 8);
  o.set(stab_at, btree_at, 8);
  o.set(stab_at + 8, heap_at, 8);
  std::ofstream out(path, std::ios::binary);
  if (!out) throw Error("HDF5: cannot create " + path);
  out.write(reinterpret_cast<const char*>(o.b.data()), (std::streamsize)o.b.size());
  if (!out) throw Error("HDF5: write failed for " + path);
}

}  // namespace h5
