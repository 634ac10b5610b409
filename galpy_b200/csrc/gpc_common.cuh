// galpy_b200/csrc/gpc_common.cuh
//
// Portability shims so that the force library and the per-orbit stepper state
// machines compile both as CUDA device code (the product) and as plain host
// C++ (a test-only harness under tests/ that checks the very same logic
// against the CPU oracle without a GPU).
#pragma once
#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#include <cuda_runtime.h>
#define GPC_HD __host__ __device__
#define GPC_FI __forceinline__
#else
#define GPC_HD
#define GPC_FI inline
#endif

namespace gpc {

// per-orbit status (the reference uses 0, -10 for SIGINT and, in dopr54, 1
// for a step forced at the smallest allowed size; the orbit still completes)
enum : int { E_OK = 0, E_MINSTEP = 1, E_BUDGET = 2, E_NONFINITE = 3, E_ABORT = -10 };

template <typename T>
GPC_HD GPC_FI T ldg(const T* p)
{
#if defined(__CUDA_ARCH__)
  return __ldg(p);
#else
  return *p;
#endif
}

GPC_HD GPC_FI double rsq(double x)
{
#if defined(__CUDA_ARCH__)
  return rsqrt(x);
#else
  return 1.0 / sqrt(x);
#endif
}

GPC_HD GPC_FI float rsqf(float x)
{
#if defined(__CUDA_ARCH__)
  return rsqrtf(x);
#else
  return 1.0f / sqrtf(x);
#endif
}

GPC_HD GPC_FI double dmax(double a, double b) { return (a > b) ? a : b; }
GPC_HD GPC_FI double dmin(double a, double b) { return (a < b) ? a : b; }
GPC_HD GPC_FI double csign(double x, double y) { return (y > 0.0) ? fabs(x) : -fabs(x); }
GPC_HD GPC_FI bool finite3(double a, double b, double c) { return isfinite(a + b + c); }

}  // namespace gpc
