// Implementation of the OCCA stand-in declared in occa.hpp (oracle test
// infrastructure).  buildKernelFromSource() JIT-compiles the C++ that
// oracle/okl2c.py produced from the reference's OKL file, with the
// kernelInfo defines passed as -D flags, and binds the resulting entry point.
#include "occa.hpp"

#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <fstream>
#include <functional>

#ifndef OKL_REF_DIR
#define OKL_REF_DIR "."
#endif

namespace occa {

static std::string ref_dir() {
  const char *e = getenv("OKL_REF_DIR");
  return e ? std::string(e) : std::string(OKL_REF_DIR);
}

memory device::malloc(size_t bytes, const void *src) {
  memory m;
  m.buf = std::make_shared<std::vector<char> >(bytes ? bytes : 1, 0);
  m.bytes_ = bytes;
  if (src && bytes) std::memcpy(m.ptr(), src, bytes);
  return m;
}

static bool file_has(const std::string &path, const std::string &needle) {
  std::ifstream f(path);
  if (!f) return false;
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str().find(needle) != std::string::npos;
}

kernel device::buildKernelFromSource(const std::string &file, const std::string &name,
                                     const kernelInfo &info) {
  kernel k;
  k.name = name;
  std::string base = file.substr(file.find_last_of('/') + 1);
  std::string src = ref_dir() + "/okl/" + base + ".cpp";
  if (!file_has(src, "OKL_WANT_" + name + "\n")) {
    // Kernels outside the translated set (curvilinear, BB-multiply
    // experiments) are never launched on the affine WADG path.
    return k;
  }
  std::string defs;
  for (auto &d : info.defines) defs += " -D" + d.first + "=" + d.second;
  defs += " -DOKL_WANT_" + name;
  const char *cxx = getenv("OKL_CXX");
  const char *flags = getenv("OKL_CXXFLAGS");
  std::string cmd_flags = flags ? flags : "-O3 -march=native -fopenmp";
  size_t h = std::hash<std::string>()(defs + cmd_flags + src);
  std::string jit = ref_dir() + "/jit";
  mkdir(jit.c_str(), 0755);
  char hbuf[32];
  snprintf(hbuf, sizeof hbuf, "%016zx", h);
  std::string so = jit + "/" + name + "_" + hbuf + ".so";
  struct stat st;
  if (stat(so.c_str(), &st) != 0) {
    std::string tmp = so + ".tmp." + std::to_string(getpid());
    std::string cmd = std::string(cxx ? cxx : "/usr/bin/g++") + " " + cmd_flags +
                      " -fPIC -shared -w -std=c++11 -I" + ref_dir() + "/okl" + defs + " -x c++ " +
                      src + " -o " + tmp;
    if (system(cmd.c_str()) != 0 || rename(tmp.c_str(), so.c_str()) != 0) {
      fprintf(stderr, "occa shim: JIT build of %s failed:\n  %s\n", name.c_str(), cmd.c_str());
      exit(2);
    }
  }
  void *lib = dlopen(so.c_str(), RTLD_NOW | RTLD_LOCAL);
  if (!lib) {
    fprintf(stderr, "occa shim: dlopen %s: %s\n", so.c_str(), dlerror());
    exit(2);
  }
  k.fn = (void (*)(const okl_arg *))dlsym(lib, ("okl_call_" + name).c_str());
  int (*na)(void) = (int (*)(void))dlsym(lib, ("okl_nargs_" + name).c_str());
  k.nargs = na ? na() : -1;
  if (!k.fn) {
    fprintf(stderr, "occa shim: symbol okl_call_%s missing\n", name.c_str());
    exit(2);
  }
  return k;
}

void kernel::launch(const okl_arg *args, int n) {
  if (!fn) {
    fprintf(stderr, "occa shim: kernel '%s' is not available in the oracle build\n",
            name.c_str());
    exit(2);
  }
  if (nargs >= 0 && n != nargs) {
    fprintf(stderr, "occa shim: kernel '%s' expects %d arguments, got %d\n", name.c_str(),
            nargs, n);
    exit(2);
  }
  fn(args);
}

static std::map<std::string, std::chrono::steady_clock::time_point> g_tic;

void printAvailableDevices() {}
void initTimer(const device &) {}
void tic(const std::string &s) { g_tic[s] = std::chrono::steady_clock::now(); }
double toc(const std::string &s) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - g_tic[s]).count();
}
double toc(const std::string &s, const kernel &, double, double) { return toc(s); }
void printTimer() {}

}  // namespace occa
