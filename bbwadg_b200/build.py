"""Builds the in-tree native library bbwadg_b200/libbbwadg_b200.so.

CUDA sources are compiled for sm_100a only (no PTX for other targets), host
sources with the system g++; objects go to bbwadg_b200/_build and are
rebuilt when a source or header is newer.  Usage:
    python -m bbwadg_b200.build [--force] [--verbose]
"""
import concurrent.futures
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libbbwadg_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# the image exports CXX=/opt/gcc/bin/g++, a wrapper without libgomp
HOSTCXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INC = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-ccbin", HOSTCXX, "--expt-relaxed-constexpr",
                  "-Xcompiler", "-fPIC,-fopenmp,-O2", "-Xptxas", "-O3"] + INC
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unknown-pragmas"] + INC


def _headers():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, force, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest = max(os.path.getmtime(src), _headers())
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + NVFLAGS + ["-c", src, "-o", obj]
    else:
        cmd = [HOSTCXX] + CXXFLAGS + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        return obj, "%s\n%s%s" % (" ".join(cmd), p.stdout, p.stderr)
    return obj, None


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("native build failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(map(os.path.getmtime, objs)):
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", HOSTCXX, "-o", LIB] + objs + \
              ["-Xcompiler", "-fopenmp", "-lgomp", "-lcublas"]
        if verbose:
            print(" ".join(cmd), flush=True)
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s%s" % (" ".join(cmd), p.stdout, p.stderr))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
