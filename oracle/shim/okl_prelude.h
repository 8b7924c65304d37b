// Prelude for OKL kernels translated by oracle/okl2c.py (oracle test
// infrastructure).  Supplies the OKL vector types and the OpenMP outer-loop
// marker that OCCA's OpenMP backend would provide.  The p_* constants arrive
// as -D definitions from the shim's JIT step, exactly as OCCA passes the
// kernelInfo defines (cpp/src/WaveOKL3d.cpp:1618-1650).
#pragma once
#include <math.h>

#if defined(USE_DOUBLE) && USE_DOUBLE
typedef double dfloat;
#else
typedef float dfloat;
#endif

struct float4 { float x, y, z, w; };
struct double4 { double x, y, z, w; };
struct int4 { int x, y, z, w; };

#if defined(USE_DOUBLE) && USE_DOUBLE
typedef double4 dfloat4;
#else
typedef float4 dfloat4;
#endif

union okl_arg { int i; double f; const void *p; };

#ifdef _OPENMP
#define OKL_OMP_FOR _Pragma("omp parallel for schedule(static)")
#else
#define OKL_OMP_FOR
#endif
