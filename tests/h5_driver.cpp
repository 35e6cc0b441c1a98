// Test driver for the library's HDF5 container code (ch4-project_b200/csrc/h5file.cpp):
//   h5_driver write <path>                 writes the fixed test file
//   h5_driver read <path> <dataset> [m..]  prints the dataset's values (members m.., or
//                                          the float dataset itself), one per line, %.17g
//   h5_driver attrs <path> <group>         prints each attribute's name and byte count
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "h5file.hpp"

static h5::Dataset vec(const char* name, std::vector<uint64_t> dims, const std::vector<double>* v) {
  h5::Dataset d;
  d.name = name;
  d.type = h5::Type::f64();
  d.dims = dims;
  d.write = [v](FILE* f) { return std::fwrite(v->data(), 8, v->size(), f) == v->size(); };
  return d;
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  std::string err;
  if (!std::strcmp(argv[1], "write")) {
    const int NZ = 3, NY = 4, NX = 5, n = NZ * NY * NX;
    static std::vector<double> f[12];
    h5::Group e;
    e.name = "euler";
    const char* names[12] = {"velocity_x", "velocity_y", "velocity_z", "density", "temperature", "scalar",
                             "position_x", "position_y", "position_z", "extra_a", "extra_b", "extra_c"};
    for (int d = 0; d < 12; d++) {
      f[d].resize(n);
      for (int i = 0; i < n; i++) f[d][i] = d * 1000.0 + i + 0.25;
      e.datasets.push_back(vec(names[d], {NZ, NY, NX}, &f[d]));
    }
    static std::vector<double> pop(19 * 2 * 3 * 4);
    for (size_t i = 0; i < pop.size(); i++) pop[i] = 0.5 * i - 7;
    h5::Group p;
    p.name = "population";
    h5::Dataset d;
    d.name = "velocity";
    std::vector<std::string> m;
    for (int q = 0; q < 19; q++) m.push_back("p" + std::to_string(q));
    d.type = h5::Type::compound(m, 8);
    d.dims = {2, 3, 4};
    d.write = [](FILE* fp) { return std::fwrite(pop.data(), 8, pop.size(), fp) == pop.size(); };
    p.datasets.push_back(d);
    h5::Group fg;
    fg.name = "forcing";
    h5::Attribute nk{"number of modes (nk)", h5::Type::i32(), {}, {6, 0, 0, 0}};
    h5::Attribute ph{"phi_u", h5::Type::compound({"x", "y", "z"}, 8), {6}, {}};
    for (int i = 0; i < 18; i++) {
      double v = 0.1 * i;
      const uint8_t* b = (const uint8_t*)&v;
      ph.data.insert(ph.data.end(), b, b + 8);
    }
    fg.attributes = {nk, ph};
    if (!h5::write_file(argv[2], {p, e, fg}, err)) return std::fprintf(stderr, "%s\n", err.c_str()), 1;
    return 0;
  }
  h5::Reader r;
  if (!r.open(argv[2], err)) return std::fprintf(stderr, "%s\n", err.c_str()), 1;
  h5::Object o;
  if (argc < 4 || !r.find(argv[3], o, err)) return std::fprintf(stderr, "%s\n", err.c_str()), 1;
  if (!std::strcmp(argv[1], "attrs")) {
    for (const h5::Attribute& a : o.attributes) std::printf("%s %zu\n", a.name.c_str(), a.data.size());
    return 0;
  }
  std::vector<std::string> names;
  for (int i = 4; i < argc; i++) names.push_back(argv[i]);
  if (names.empty()) names.push_back("");
  uint64_t n = 1;
  for (uint64_t x : o.dims) n *= x;
  std::vector<double> v(n * names.size());
  if (!r.read_members(o, names, v.data(), names.size(), err)) return std::fprintf(stderr, "%s\n", err.c_str()), 1;
  for (double x : v) std::printf("%.17g\n", x);
  return 0;
}
