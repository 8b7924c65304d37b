// Minimal host-side stand-in for the OCCA runtime (oracle test
// infrastructure).  The reference's host code (cpp/src/WaveOKL3d.cpp and
// friends) is compiled unchanged against this header; OCCA itself is not
// available in this environment.
//
// * occa::memory   - a host buffer (the "device" is the CPU).
// * occa::kernel   - bound to an OKL kernel translated to C++ by
//                    oracle/okl2c.py and JIT-compiled with the host compiler
//                    and the kernelInfo defines, the way OCCA's OpenMP mode
//                    compiles OKL.
// * timers         - wall-clock tic/toc.
#pragma once

#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iomanip>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

union okl_arg { int i; double f; const void *p; };

namespace occa {

class memory {
 public:
  std::shared_ptr<std::vector<char> > buf;
  size_t bytes_ = 0;
  void *ptr() const { return buf ? (void *)buf->data() : nullptr; }
  size_t bytes() const { return bytes_; }
  void copyFrom(const void *src, size_t n = 0) {
    std::memcpy(ptr(), src, n ? n : bytes_);
  }
  void copyTo(void *dst, size_t n = 0) const {
    std::memcpy(dst, ptr(), n ? n : bytes_);
  }
  void free() { buf.reset(); bytes_ = 0; }
};

class kernelInfo {
 public:
  std::map<std::string, std::string> defines;
  std::vector<std::string> flags;
  template <class T>
  void addDefine(const std::string &name, const T &value) {
    std::ostringstream os;
    os.precision(17);
    os << value;
    defines[name] = os.str();
  }
  void addCompilerFlag(const std::string &f) { flags.push_back(f); }
};

class kernel {
 public:
  std::string name;
  void (*fn)(const okl_arg *) = nullptr;
  int nargs = -1;

  template <class... A>
  void operator()(const A &...a) {
    okl_arg args[sizeof...(A) + 1] = {to_arg(a)...};
    launch(args, (int)sizeof...(A));
  }

 private:
  static okl_arg to_arg(const memory &m) { okl_arg r; r.p = m.ptr(); return r; }
  static okl_arg to_arg(int v) { okl_arg r; r.i = v; return r; }
  static okl_arg to_arg(unsigned v) { okl_arg r; r.i = (int)v; return r; }
  static okl_arg to_arg(float v) { okl_arg r; r.f = v; return r; }
  static okl_arg to_arg(double v) { okl_arg r; r.f = v; return r; }
  void launch(const okl_arg *args, int n);
};

class device {
 public:
  void setup(const std::string &) {}
  std::string mode() const { return "OpenMP"; }
  void finish() {}
  memory malloc(size_t bytes, const void *src = nullptr);
  kernel buildKernelFromSource(const std::string &file, const std::string &name,
                               const kernelInfo &info);
};

void printAvailableDevices();
void initTimer(const device &);
void tic(const std::string &);
double toc(const std::string &);
double toc(const std::string &, const kernel &, double flops = 0, double bytes = 0);
void printTimer();

}  // namespace occa
