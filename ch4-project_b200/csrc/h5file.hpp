// A small HDF5 container, written from the public HDF5 file format specification
// (superblock version 0, version-1 object headers, groups as symbol tables).  No HDF5
// library is linked: the image has none.  It writes what the reference's output_h5.c
// writes through libhdf5 -- groups under the root holding contiguous datasets of IEEE
// floats or compounds of them, and attributes -- and reads the same subset back,
// including files written by libhdf5 with its default (earliest) format: superblock
// version 0/1, version-1 object headers with continuation blocks, version-1 group
// B-trees of any depth, contiguous layout (message versions 1-3), dataspace versions
// 1-2, datatype versions 1-3.  Chunked or filtered storage and version-2 object headers
// are refused by name.
#pragma once
#include <cstdint>
#include <cstdio>
#include <functional>
#include <string>
#include <utility>
#include <vector>

namespace h5 {

// IEEE little-endian float (4 or 8 bytes), 32-bit signed integer, or a compound of
// floats (member name, byte offset, float size)
struct Member {
  std::string name;
  uint32_t offset;
  int fsize;
};
struct Type {
  enum Kind { FLOAT, INT32, COMPOUND } kind = FLOAT;
  uint32_t size = 8;
  std::vector<Member> members;
  static Type f64() { return Type{FLOAT, 8, {}}; }
  static Type i32() { return Type{INT32, 4, {}}; }
  // members packed in the order given, each a float of fsize bytes
  static Type compound(const std::vector<std::string>& names, int fsize);
};

struct Attribute {
  std::string name;
  Type type;
  std::vector<uint64_t> dims;  // empty: a scalar
  std::vector<uint8_t> data;   // little-endian values
};

struct Dataset {
  std::string name;
  Type type;
  std::vector<uint64_t> dims;
  // writes exactly type.size * prod(dims) bytes at the file's current position
  std::function<bool(FILE*)> write;
};

struct Group {
  std::string name;  // a child of the root
  std::vector<Dataset> datasets;
  std::vector<Attribute> attributes;
};

// writes `path` with the given groups under "/"; false with err set on failure
bool write_file(const std::string& path, const std::vector<Group>& groups, std::string& err);

// one object found by path: a dataset (dims, type, contiguous data address) and its
// attributes
struct Object {
  bool is_dataset = false, is_group = false;
  std::vector<uint64_t> dims;
  Type type;
  uint64_t data_addr = ~0ull, data_size = 0;
  std::vector<Attribute> attributes;
};

class Reader {
 public:
  ~Reader();
  bool open(const std::string& path, std::string& err);
  // "/group/name": false with err when it does not exist or uses an unsupported form
  bool find(const std::string& path, Object& out, std::string& err);
  // the raw bytes of a dataset (data_size of them)
  bool read_raw(const Object& o, void* dst, std::string& err);
  // float members (or the float dataset itself, name "") of every element, as doubles:
  // element i, member k -> dst[i * stride + k]
  bool read_members(const Object& o, const std::vector<std::string>& names, double* dst, size_t stride,
                    std::string& err);

 private:
  FILE* f_ = nullptr;
  int so_ = 8, sl_ = 8;  // sizes of offsets and lengths
  uint64_t base_ = 0, root_ = 0;
  bool rd(uint64_t addr, void* dst, size_t n);
  bool object(uint64_t addr, Object& o, uint64_t& btree, uint64_t& heap, std::string& err);
  bool lookup(uint64_t btree, uint64_t heap, const std::string& name, uint64_t& child, std::string& err);
};

}  // namespace h5
