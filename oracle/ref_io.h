// Binary record writer and option helpers shared by the reference drivers
// (oracle test infrastructure).  Record format: "BBWA0001", then per record
// u32 name length, name, u32 dtype (0 f32, 1 f64, 2 i32), u64 count, data.
// Include after the reference's fem.h (occa::memory and Eigen types).
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

namespace refio {

struct Writer {
  std::ofstream f;
  explicit Writer(const std::string &p) : f(p, std::ios::binary) {
    f.write("BBWA0001", 8);
  }
  void rec(const std::string &name, int dtype, const void *data, uint64_t count) {
    uint32_t n = (uint32_t)name.size();
    f.write((const char *)&n, 4);
    f.write(name.data(), n);
    uint32_t dt = (uint32_t)dtype;
    f.write((const char *)&dt, 4);
    f.write((const char *)&count, 8);
    size_t esz = dtype == 1 ? 8 : 4;
    f.write((const char *)data, count * esz);
  }
  void f32(const std::string &n, const occa::memory &m) {
    rec(n, 0, m.ptr(), m.bytes() / 4);
  }
  void i32(const std::string &n, const occa::memory &m) {
    rec(n, 2, m.ptr(), m.bytes() / 4);
  }
  void f64(const std::string &n, const MatrixXd &A) {  // column-major
    rec(n, 1, A.data(), (uint64_t)A.size());
  }
  void f64v(const std::string &n, const VectorXd &v) { rec(n, 1, v.data(), (uint64_t)v.size()); }
  void i32m(const std::string &n, const MatrixXi &A) { rec(n, 2, A.data(), (uint64_t)A.size()); }
  void scal(const std::string &n, double v) { rec(n, 1, &v, 1); }
};

std::string opt(int argc, char **argv, const std::string &key, const std::string &dflt) {
  for (int i = 1; i + 1 < argc; ++i)
    if (key == argv[i]) return argv[i + 1];
  return dflt;
}

std::vector<char> slurp(const std::string &p) {
  std::ifstream f(p, std::ios::binary);
  if (!f) {
    fprintf(stderr, "cannot read %s\n", p.c_str());
    exit(1);
  }
  return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

void load_into(occa::memory &m, const std::string &path) {
  std::vector<char> b = slurp(path);
  if (b.size() != m.bytes()) {
    fprintf(stderr, "%s: %zu bytes, expected %zu\n", path.c_str(), b.size(), m.bytes());
    exit(1);
  }
  m.copyFrom(b.data());
}

}  // namespace refio
