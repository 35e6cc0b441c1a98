// HDF5 container writer and reader: see h5file.hpp.  Structures and field orders
// follow the public HDF5 file format specification (superblock version 0; version-1
// object headers; local heaps; version-1 B-tree group nodes; symbol-table nodes;
// dataspace, datatype, layout, attribute, continuation and symbol-table messages).
#include "h5file.hpp"

#include <algorithm>
#include <cstring>

namespace h5 {
namespace {

constexpr uint64_t UNDEF = ~0ull;
constexpr int LEAF_K = 32;              // a symbol-table node holds up to 2K entries
constexpr int INTERNAL_K = 16;          // a group B-tree node has room for 2K children
constexpr uint64_t HEAP_FREE_NULL = 1;  // "no free block" in a local heap's free-list head
constexpr size_t ENTRY = 40;            // symbol-table entry with 8-byte offsets
constexpr size_t SNOD_SIZE = 8 + 2 * LEAF_K * ENTRY;
constexpr size_t BTREE_SIZE = 24 + 2 * INTERNAL_K * 8 + (2 * INTERNAL_K + 1) * 8;
constexpr uint8_t SIGNATURE[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

enum : int { MSG_DATASPACE = 1, MSG_DATATYPE = 3, MSG_LAYOUT = 8, MSG_FILTERS = 11, MSG_ATTRIBUTE = 12,
             MSG_CONTINUATION = 16, MSG_SYMTAB = 17 };

uint64_t pad8(uint64_t n) { return (n + 7) & ~7ull; }

struct Buf {
  std::vector<uint8_t> b;
  void u8(unsigned v) { b.push_back((uint8_t)v); }
  void u16(unsigned v) { u8(v & 255), u8((v >> 8) & 255); }
  void u32(uint32_t v) {
    for (int i = 0; i < 4; i++) u8((v >> (8 * i)) & 255);
  }
  void u64(uint64_t v) {
    for (int i = 0; i < 8; i++) u8((unsigned)((v >> (8 * i)) & 255));
  }
  void raw(const void* p, size_t n) {
    const uint8_t* q = (const uint8_t*)p;
    b.insert(b.end(), q, q + n);
  }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void pad_to(size_t n) { zeros(n - b.size()); }
  void align8() { zeros(pad8(b.size()) - b.size()); }
  size_t size() const { return b.size(); }
};

uint64_t get(const uint8_t* p, int n) {
  uint64_t v = 0;
  for (int i = n - 1; i >= 0; i--) v = (v << 8) | p[i];
  return v;
}

// datatype message bodies ------------------------------------------------------------

void put_float(Buf& o, int fsize) {
  o.u8(0x11);  // version 1, class 1 (floating point)
  o.u8(0x20);  // little-endian, no padding bits, mantissa normalised with an implied 1
  o.u8(fsize == 8 ? 63 : 31);  // sign bit
  o.u8(0);
  o.u32(fsize);
  o.u16(0);          // bit offset
  o.u16(fsize * 8);  // precision
  o.u8(fsize == 8 ? 52 : 23);  // exponent location
  o.u8(fsize == 8 ? 11 : 8);   // exponent size
  o.u8(0);                     // mantissa location
  o.u8(fsize == 8 ? 52 : 23);  // mantissa size
  o.u32(fsize == 8 ? 1023 : 127);
}

void put_type(Buf& o, const Type& t) {
  if (t.kind == Type::FLOAT) return put_float(o, (int)t.size);
  if (t.kind == Type::INT32) {
    o.u8(0x10);  // version 1, class 0 (fixed point)
    o.u8(0x08);  // little-endian, signed
    o.u8(0);
    o.u8(0);
    o.u32(4);
    o.u16(0);
    o.u16(32);
    return;
  }
  o.u8(0x16);  // version 1, class 6 (compound)
  o.u16((unsigned)t.members.size());
  o.u8(0);
  o.u32(t.size);
  for (const Member& m : t.members) {
    o.raw(m.name.c_str(), m.name.size() + 1);
    o.zeros(pad8(m.name.size() + 1) - (m.name.size() + 1));
    o.u32(m.offset);
    o.u8(0);  // no member array dimensions
    o.zeros(3 + 4 + 4 + 16);
    put_float(o, m.fsize);
  }
}

void put_space(Buf& o, const std::vector<uint64_t>& dims) {
  o.u8(1);  // version 1
  o.u8((unsigned)dims.size());
  o.u8(0);  // no maximum dimensions
  o.u8(0);
  o.u32(0);
  for (uint64_t d : dims) o.u64(d);
}

uint64_t elements(const std::vector<uint64_t>& dims) {
  uint64_t n = 1;
  for (uint64_t d : dims) n *= d;
  return n;
}

struct Msg {
  int type;
  Buf body;
};

// version-1 object header: 16-byte prefix, then messages padded to 8 bytes
bool put_header(Buf& o, const std::vector<Msg>& msgs, std::string& err) {
  size_t total = 0;
  for (const Msg& m : msgs) {
    if (pad8(m.body.size()) > 0xfff8) return err = "an HDF5 header message larger than 64 KiB", false;
    total += 8 + pad8(m.body.size());
  }
  o.u8(1);
  o.u8(0);
  o.u16((unsigned)msgs.size());
  o.u32(1);  // reference count
  o.u32((uint32_t)total);
  o.u32(0);  // alignment of the first message
  for (const Msg& m : msgs) {
    o.u16(m.type);
    o.u16((unsigned)pad8(m.body.size()));
    o.u8(0);
    o.zeros(3);
    o.raw(m.body.b.data(), m.body.size());
    o.align8();
  }
  return true;
}

Buf attribute_body(const Attribute& a) {
  Buf t, s, o;
  put_type(t, a.type);
  put_space(s, a.dims);
  o.u8(1);  // version 1
  o.u8(0);
  o.u16((unsigned)a.name.size() + 1);
  o.u16((unsigned)t.size());
  o.u16((unsigned)s.size());
  o.raw(a.name.c_str(), a.name.size() + 1);
  o.align8();
  o.raw(t.b.data(), t.size());
  o.align8();
  o.raw(s.b.data(), s.size());
  o.align8();
  o.raw(a.data.data(), a.data.size());
  return o;
}

// a symbol-table group: name heap, one-leaf B-tree, one symbol-table node
struct Children {
  std::vector<std::string> names;  // sorted
  std::vector<uint64_t> offsets;   // in the heap
  Buf heap_data;
};

Children children_of(std::vector<std::string> names) {
  Children c;
  std::sort(names.begin(), names.end());
  c.names = names;
  c.heap_data.zeros(8);  // offset 0: the empty name
  for (const std::string& n : names) {
    c.offsets.push_back(c.heap_data.size());
    c.heap_data.raw(n.c_str(), n.size() + 1);
    c.heap_data.align8();
  }
  return c;
}

void put_heap(Buf& o, const Children& c, uint64_t at) {
  o.raw("HEAP", 4);
  o.u8(0);
  o.zeros(3);
  o.u64(c.heap_data.size());
  o.u64(HEAP_FREE_NULL);
  o.u64(at + 32);  // data segment right after the header
  o.raw(c.heap_data.b.data(), c.heap_data.size());
}

void put_btree(Buf& o, const Children& c, uint64_t snod) {
  const size_t start = o.size();
  o.raw("TREE", 4);
  o.u8(0);  // group node
  o.u8(0);  // leaf
  o.u16(c.names.empty() ? 0 : 1);
  o.u64(UNDEF);
  o.u64(UNDEF);
  o.u64(0);  // left key: the empty name
  if (!c.names.empty()) {
    o.u64(snod);
    o.u64(c.offsets.back());  // right key: the last name in the node
  }
  o.zeros(start + BTREE_SIZE - o.size());
}

struct Entry {
  uint64_t header;
  bool group;
  uint64_t btree, heap;
};

void put_snod(Buf& o, const Children& c, const std::vector<Entry>& e) {
  const size_t start = o.size();
  o.raw("SNOD", 4);
  o.u8(1);
  o.u8(0);
  o.u16((unsigned)c.names.size());
  for (size_t i = 0; i < c.names.size(); i++) {
    o.u64(c.offsets[i]);
    o.u64(e[i].header);
    o.u32(e[i].group ? 1 : 0);  // cache type 1: B-tree and heap addresses in the scratch pad
    o.u32(0);
    o.u64(e[i].group ? e[i].btree : 0);
    o.u64(e[i].group ? e[i].heap : 0);
  }
  o.zeros(start + SNOD_SIZE - o.size());
}

}  // namespace

Type Type::compound(const std::vector<std::string>& names, int fsize) {
  Type t;
  t.kind = COMPOUND;
  t.size = 0;
  for (const std::string& n : names) {
    t.members.push_back(Member{n, t.size, fsize});
    t.size += fsize;
  }
  return t;
}

bool write_file(const std::string& path, const std::vector<Group>& groups, std::string& err) {
  for (const Group& g : groups) {
    if (g.datasets.size() > 2 * LEAF_K)
      return err = "more than " + std::to_string(2 * LEAF_K) + " datasets in an HDF5 group", false;
    for (const Attribute& a : g.attributes)
      if (a.data.size() != a.type.size * elements(a.dims)) return err = "attribute " + a.name + ": size mismatch", false;
  }
  if (groups.size() > 2 * LEAF_K) return err = "more than " + std::to_string(2 * LEAF_K) + " HDF5 groups", false;
  std::vector<std::string> gnames;
  for (const Group& g : groups) gnames.push_back(g.name);
  const Children root = children_of(gnames);
  // groups in name order: the root's symbol-table node lists them that way
  std::vector<size_t> gorder(groups.size());
  for (size_t i = 0; i < groups.size(); i++)
    gorder[i] = (size_t)(std::find(gnames.begin(), gnames.end(), root.names[i]) - gnames.begin());
  std::vector<Children> kids;
  for (const Group& g : groups) {
    std::vector<std::string> dn;
    for (const Dataset& d : g.datasets) dn.push_back(d.name);
    kids.push_back(children_of(dn));
  }
  // two passes: sizes with zero addresses, then the bytes with the real ones
  struct Addr {
    uint64_t oh = 0, btree = 0, snod = 0, heap = 0;
    std::vector<uint64_t> dset_oh, data;
  };
  Addr ra;
  std::vector<Addr> ga(groups.size());
  for (size_t i = 0; i < groups.size(); i++) {
    ga[i].dset_oh.assign(groups[i].datasets.size(), 0);
    ga[i].data.assign(groups[i].datasets.size(), 0);
  }
  uint64_t eof = 0;
  Buf meta;
  auto dataset_header = [&](const Dataset& d, uint64_t data_addr, Buf& o) {
    std::vector<Msg> m(3);
    m[0].type = MSG_DATASPACE;
    put_space(m[0].body, d.dims);
    m[1].type = MSG_DATATYPE;
    put_type(m[1].body, d.type);
    m[2].type = MSG_LAYOUT;
    m[2].body.u8(3);  // version 3
    m[2].body.u8(1);  // contiguous
    m[2].body.u64(data_addr);
    m[2].body.u64(d.type.size * elements(d.dims));
    return put_header(o, m, err);
  };
  auto group_header = [&](uint64_t btree, uint64_t heap, const std::vector<Attribute>& attrs, Buf& o) {
    std::vector<Msg> m(1);
    m[0].type = MSG_SYMTAB;
    m[0].body.u64(btree);
    m[0].body.u64(heap);
    for (const Attribute& a : attrs) m.push_back(Msg{MSG_ATTRIBUTE, attribute_body(a)});
    return put_header(o, m, err);
  };
  for (int pass = 0; pass < 2; pass++) {
    meta = Buf();
    meta.zeros(96);  // superblock, filled in below
    auto place = [&](uint64_t& a) {
      meta.align8();
      a = meta.size();
    };
    std::vector<Attribute> none;
    place(ra.oh);
    if (!group_header(ra.btree, ra.heap, none, meta)) return false;
    place(ra.btree);
    put_btree(meta, root, ra.snod);
    place(ra.snod);
    std::vector<Entry> re;
    for (size_t i = 0; i < groups.size(); i++) {
      const Addr& a = ga[gorder[i]];
      re.push_back(Entry{a.oh, true, a.btree, a.heap});
    }
    put_snod(meta, root, re);
    place(ra.heap);
    put_heap(meta, root, ra.heap);
    for (size_t gi = 0; gi < groups.size(); gi++) {
      const Group& g = groups[gi];
      Addr& a = ga[gi];
      place(a.oh);
      if (!group_header(a.btree, a.heap, g.attributes, meta)) return false;
      place(a.btree);
      put_btree(meta, kids[gi], a.snod);
      if (!g.datasets.empty()) {
        place(a.snod);
        std::vector<Entry> de;
        for (const std::string& n : kids[gi].names) {
          size_t di = 0;
          while (g.datasets[di].name != n) di++;
          de.push_back(Entry{a.dset_oh[di], false, 0, 0});
        }
        put_snod(meta, kids[gi], de);
      }
      place(a.heap);
      put_heap(meta, kids[gi], a.heap);
      for (size_t di = 0; di < g.datasets.size(); di++) {
        place(a.dset_oh[di]);
        if (!dataset_header(g.datasets[di], a.data[di], meta)) return false;
      }
    }
    meta.align8();
    uint64_t at = meta.size();
    for (size_t gi = 0; gi < groups.size(); gi++)
      for (size_t di = 0; di < groups[gi].datasets.size(); di++) {
        const Dataset& d = groups[gi].datasets[di];
        ga[gi].data[di] = at;
        at = pad8(at + d.type.size * elements(d.dims));
      }
    eof = at;
  }
  // superblock version 0
  Buf sb;
  sb.raw(SIGNATURE, 8);
  sb.u8(0);  // superblock
  sb.u8(0);  // free-space storage
  sb.u8(0);  // root group symbol-table entry
  sb.u8(0);
  sb.u8(0);  // shared header messages
  sb.u8(8);  // size of offsets
  sb.u8(8);  // size of lengths
  sb.u8(0);
  sb.u16(LEAF_K);
  sb.u16(INTERNAL_K);
  sb.u32(0);  // file consistency flags
  sb.u64(0);  // base address
  sb.u64(UNDEF);  // free-space info
  sb.u64(eof);
  sb.u64(UNDEF);  // driver information block
  sb.u64(0);      // root entry: link name offset
  sb.u64(ra.oh);
  sb.u32(1);
  sb.u32(0);
  sb.u64(ra.btree);
  sb.u64(ra.heap);
  std::memcpy(meta.b.data(), sb.b.data(), 96);

  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return err = "cannot create " + path, false;
  bool ok = std::fwrite(meta.b.data(), 1, meta.size(), f) == meta.size();
  uint64_t pos = meta.size();
  static const uint8_t zero8[8] = {0};
  for (size_t gi = 0; ok && gi < groups.size(); gi++)
    for (size_t di = 0; ok && di < groups[gi].datasets.size(); di++) {
      const Dataset& d = groups[gi].datasets[di];
      const uint64_t bytes = d.type.size * elements(d.dims);
      ok = pos == ga[gi].data[di] && d.write(f);
      pos += bytes;
      if (ok && pad8(pos) != pos) {
        ok = std::fwrite(zero8, 1, pad8(pos) - pos, f) == pad8(pos) - pos;
        pos = pad8(pos);
      }
    }
  ok = ok && pos == eof;
  if (std::fclose(f) != 0) ok = false;
  if (!ok) err = "write failed: " + path;
  return ok;
}

// reader ------------------------------------------------------------------------------

Reader::~Reader() {
  if (f_) std::fclose(f_);
}

bool Reader::rd(uint64_t addr, void* dst, size_t n) {
  if (fseeko(f_, (off_t)(base_ + addr), SEEK_SET) != 0) return false;
  return std::fread(dst, 1, n, f_) == n;
}

bool Reader::open(const std::string& path, std::string& err) {
  f_ = std::fopen(path.c_str(), "rb");
  if (!f_) return err = "cannot open " + path, false;
  // the superblock sits at 0 or after a user block of 512, 1024, 2048 ... bytes
  uint8_t b[128];
  uint64_t at = 0;
  for (;; at = at ? 2 * at : 512) {
    base_ = 0;
    if (!rd(at, b, 8)) return err = path + ": no HDF5 signature", false;
    if (std::memcmp(b, SIGNATURE, 8) == 0) break;
  }
  if (!rd(at, b, 96 + 4)) return err = path + ": truncated superblock", false;
  const int ver = b[8];
  if (ver > 1) return err = path + ": superblock version " + std::to_string(ver) + " is not supported", false;
  so_ = b[13];
  sl_ = b[14];
  if (so_ != 8 || sl_ != 8) return err = path + ": only 8-byte offsets and lengths are supported", false;
  size_t p = 24 + (ver == 1 ? 4 : 0);
  base_ = get(b + p, 8);
  p += 32;                   // base, free space, end of file, driver block
  root_ = get(b + p + 8, 8);  // the root entry's object header
  return true;
}

namespace {

// a datatype message at p (n bytes available): float, 32-bit integer or compound of floats
bool parse_type(const uint8_t* p, size_t n, Type& t, size_t& used, std::string& err) {
  if (n < 8) return err = "truncated datatype", false;
  const int cls = p[0] & 15, ver = p[0] >> 4;
  const uint32_t size = (uint32_t)get(p + 4, 4);
  if (cls == 1) {
    if (p[1] & 0x41) return err = "big-endian or VAX float data", false;
    if (size != 4 && size != 8) return err = "float of " + std::to_string(size) + " bytes", false;
    t = Type{Type::FLOAT, size, {}};
    used = 8 + 12;
    return true;
  }
  if (cls == 0) {
    if ((p[1] & 1) || size != 4) return err = "integer other than 32-bit little-endian", false;
    t = Type{Type::INT32, 4, {}};
    used = 8 + 4;
    return true;
  }
  if (cls != 6) return err = "datatype class " + std::to_string(cls) + " is not supported", false;
  const int nm = (int)get(p + 1, 2);
  t = Type{Type::COMPOUND, size, {}};
  size_t q = 8;
  const int offbytes = size < 256 ? 1 : size < 65536 ? 2 : size < (1u << 24) ? 3 : 4;
  for (int i = 0; i < nm; i++) {
    const size_t len = strnlen((const char*)p + q, n - q);
    if (q + len >= n) return err = "truncated compound member name", false;
    Member m;
    m.name.assign((const char*)p + q, len);
    q += ver >= 3 ? len + 1 : ((len + 8) / 8) * 8;
    // every field read below must lie inside the message
    const size_t need = ver >= 3 ? (size_t)offbytes : (ver == 1 ? 4 + 28 : 4);
    if (q + need > n) return err = "truncated compound member " + m.name, false;
    if (ver >= 3) {
      m.offset = (uint32_t)get(p + q, offbytes);
      q += offbytes;
    } else {
      m.offset = (uint32_t)get(p + q, 4);
      q += 4;
      if (ver == 1) {
        if (p[q] != 0) return err = "compound member " + m.name + " with array dimensions", false;
        q += 28;
      }
    }
    Type mt;
    size_t mu = 0;
    if (q > n || !parse_type(p + q, n - q, mt, mu, err)) return false;
    if (mt.kind != Type::FLOAT) return err = "compound member " + m.name + " is not a float", false;
    m.fsize = (int)mt.size;
    if ((uint64_t)m.offset + (uint64_t)m.fsize > size)
      return err = "compound member " + m.name + " lies outside its record", false;
    t.members.push_back(m);
    q += mu;
  }
  used = q;
  return true;
}

bool parse_space(const uint8_t* p, size_t n, std::vector<uint64_t>& dims, std::string& err) {
  if (n < 8) return err = "truncated dataspace", false;
  const int ver = p[0], rank = p[1];
  size_t q = ver == 1 ? 8 : 4;  // version 2: scalar, simple and null spaces, no reserved bytes
  dims.clear();
  for (int i = 0; i < rank; i++, q += 8) {
    if (q + 8 > n) return err = "truncated dataspace", false;
    dims.push_back(get(p + q, 8));
  }
  return true;
}

}  // namespace

bool Reader::object(uint64_t addr, Object& o, uint64_t& btree, uint64_t& heap, std::string& err) {
  uint8_t pre[16];
  if (!rd(addr, pre, 16)) return err = "object header beyond the end of the file", false;
  if (std::memcmp(pre, "OHDR", 4) == 0) return err = "version-2 object headers are not supported", false;
  if (pre[0] != 1) return err = "unknown object header version", false;
  const int nmsgs = (int)get(pre + 2, 2);
  std::vector<std::pair<uint64_t, uint64_t>> chunks{{addr + 16, get(pre + 8, 4)}};
  int seen = 0;
  o = Object();
  btree = heap = UNDEF;
  for (size_t c = 0; c < chunks.size() && seen < nmsgs; c++) {
    std::vector<uint8_t> buf(chunks[c].second);
    if (!rd(chunks[c].first, buf.data(), buf.size())) return err = "truncated object header", false;
    size_t p = 0;
    while (p + 8 <= buf.size() && seen < nmsgs) {
      const int type = (int)get(&buf[p], 2);
      const size_t len = (size_t)get(&buf[p + 2], 2);
      const uint8_t* m = &buf[p + 8];
      if (p + 8 + len > buf.size()) return err = "object header message overruns its block", false;
      seen++;
      size_t used = 0;
      switch (type) {
        case MSG_DATASPACE:
          if (!parse_space(m, len, o.dims, err)) return false;
          break;
        case MSG_DATATYPE:
          if (!parse_type(m, len, o.type, used, err)) return false;
          o.is_dataset = true;
          break;
        case MSG_LAYOUT: {
          const int ver = m[0];
          if (ver == 3) {
            if (m[1] != 1) return err = m[1] == 2 ? "chunked storage is not supported" : "compact storage is not supported", false;
            o.data_addr = get(m + 2, 8);
            o.data_size = get(m + 10, 8);
          } else if (ver == 1 || ver == 2) {
            const int nd = m[1];
            if (m[2] != 1) return err = "non-contiguous storage is not supported", false;
            o.data_addr = get(m + 8, 8);
            o.data_size = 1;
            for (int i = 0; i < nd; i++) o.data_size *= get(m + 16 + 4 * i, 4);
          } else {
            return err = "data layout message version " + std::to_string(ver) + " is not supported", false;
          }
          break;
        }
        case MSG_FILTERS:
          return err = "filtered (compressed) data is not supported", false;
        case MSG_ATTRIBUTE: {
          const int ver = m[0];
          if (ver < 1 || ver > 3) return err = "attribute message version " + std::to_string(ver), false;
          const size_t nlen = get(m + 2, 2), tlen = get(m + 4, 2), slen = get(m + 6, 2);
          size_t q = ver == 3 ? 9 : 8;
          Attribute a;
          a.name.assign((const char*)m + q, nlen ? nlen - 1 : 0);
          q += ver == 1 ? pad8(nlen) : nlen;
          size_t tu = 0;
          if (q > len || !parse_type(m + q, len - q, a.type, tu, err)) return false;
          q += ver == 1 ? pad8(tlen) : tlen;
          if (q > len || !parse_space(m + q, len - q, a.dims, err)) return false;
          q += ver == 1 ? pad8(slen) : slen;
          const size_t bytes = a.type.size * elements(a.dims);
          if (q + bytes > len) return err = "truncated attribute " + a.name, false;
          a.data.assign(m + q, m + q + bytes);
          o.attributes.push_back(a);
          break;
        }
        case MSG_CONTINUATION:
          chunks.push_back({get(m, 8), get(m + 8, 8)});
          break;
        case MSG_SYMTAB:
          btree = get(m, 8);
          heap = get(m + 8, 8);
          o.is_group = true;
          break;
        default:
          break;
      }
      p += 8 + len;
    }
  }
  return true;
}

bool Reader::lookup(uint64_t btree, uint64_t heap, const std::string& name, uint64_t& child, std::string& err) {
  uint8_t hh[32];
  if (!rd(heap, hh, 32) || std::memcmp(hh, "HEAP", 4) != 0) return err = "bad local heap", false;
  std::vector<char> names(get(hh + 8, 8) + 1, 0);
  if (!rd(get(hh + 24, 8), names.data(), names.size() - 1)) return err = "truncated local heap", false;
  std::vector<uint64_t> todo{btree};
  while (!todo.empty()) {
    const uint64_t node = todo.back();
    todo.pop_back();
    uint8_t nh[24];
    if (!rd(node, nh, 24) || std::memcmp(nh, "TREE", 4) != 0 || nh[4] != 0) return err = "bad group B-tree node", false;
    const int level = nh[5], used = (int)get(nh + 6, 2);
    std::vector<uint8_t> kc(used * 16 + 8);
    if (!rd(node + 24, kc.data(), kc.size())) return err = "truncated B-tree node", false;
    for (int i = 0; i < used; i++) {
      const uint64_t c = get(&kc[8 + 16 * i], 8);
      if (level > 0) {
        todo.push_back(c);
        continue;
      }
      uint8_t sh[8];
      if (!rd(c, sh, 8) || std::memcmp(sh, "SNOD", 4) != 0) return err = "bad symbol-table node", false;
      const int ns = (int)get(sh + 6, 2);
      std::vector<uint8_t> ent(ns * ENTRY);
      if (!rd(c + 8, ent.data(), ent.size())) return err = "truncated symbol-table node", false;
      for (int e = 0; e < ns; e++) {
        const uint64_t off = get(&ent[e * ENTRY], 8);
        if (off < names.size() - 1 && name == &names[off]) {
          child = get(&ent[e * ENTRY + 8], 8);
          return true;
        }
      }
    }
  }
  return err = "no object named " + name, false;
}

bool Reader::find(const std::string& path, Object& out, std::string& err) {
  uint64_t cur = root_, bt, hp;
  size_t p = 0;
  while (p < path.size()) {
    while (p < path.size() && path[p] == '/') p++;
    if (p >= path.size()) break;
    const size_t q = path.find('/', p);
    const std::string part = path.substr(p, q == std::string::npos ? std::string::npos : q - p);
    Object g;
    if (!object(cur, g, bt, hp, err)) return false;
    if (!g.is_group) return err = part + ": parent is not a group", false;
    if (!lookup(bt, hp, part, cur, err)) return false;
    p = q == std::string::npos ? path.size() : q;
  }
  return object(cur, out, bt, hp, err);
}

bool Reader::read_raw(const Object& o, void* dst, std::string& err) {
  if (!o.is_dataset || o.data_addr == UNDEF) return err = "not a dataset with stored data", false;
  if (!rd(o.data_addr, dst, o.data_size)) return err = "dataset data beyond the end of the file", false;
  return true;
}

bool Reader::read_members(const Object& o, const std::vector<std::string>& names, double* dst, size_t stride,
                          std::string& err) {
  if (!o.is_dataset || o.data_addr == UNDEF) return err = "not a dataset with stored data", false;
  const size_t nm = names.size();
  std::vector<uint32_t> off(nm, 0);
  std::vector<int> fs(nm, 0);
  for (size_t k = 0; k < nm; k++) {
    if (o.type.kind == Type::FLOAT && names[k].empty()) {
      fs[k] = (int)o.type.size;
    } else {
      for (const Member& m : o.type.members)
        if (m.name == names[k]) off[k] = m.offset, fs[k] = m.fsize;
      if (!fs[k]) return err = "no member " + names[k], false;
    }
  }
  const uint64_t n = elements(o.dims), es = o.type.size;
  if (o.data_size < n * es) return err = "dataset storage smaller than its dataspace", false;
  const uint64_t per = std::max<uint64_t>(1, (64u << 20) / es);
  std::vector<uint8_t> buf;
  for (uint64_t i0 = 0; i0 < n; i0 += per) {
    const uint64_t m = std::min(per, n - i0);
    buf.resize(m * es);
    if (!rd(o.data_addr + i0 * es, buf.data(), buf.size())) return err = "truncated dataset data", false;
    for (uint64_t i = 0; i < m; i++)
      for (size_t k = 0; k < nm; k++) {
        const uint8_t* p = &buf[i * es + off[k]];
        double v;
        if (fs[k] == 8) {
          std::memcpy(&v, p, 8);
        } else {
          float x;
          std::memcpy(&x, p, 4);
          v = x;
        }
        dst[(i0 + i) * stride + k] = v;
      }
  }
  return true;
}

}  // namespace h5
